// C ABI of libegpr.so (declared in include/egpr.h).
//
// Host-side runtime around the kernels: prepared-graph handles bound to one
// device, per-handle streams and workspaces, the solve sequence (set-up
// kernels, the CUDA-graph while-loop of sweeps, the FP64 correction sweep and
// the normalisation), the multi-graph plan cache and the keyed prepared-graph
// cache behind the drop-in egpr_pagerank_csr.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "egpr_internal.cuh"

namespace egpr {

namespace {
thread_local std::string t_last_error;
std::atomic<int64_t> g_live_graphs{0};
std::atomic<int64_t> g_live_bytes{0};
}  // namespace

int set_cuda_error(cudaError_t e, const char* what) {
    t_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM;
    return EGPR_DEVICE_ERR;
}

static int fail_arg(const char* why) {
    t_last_error = why;
    return EGPR_INVALID_ARGUMENT;
}

int arg_error(const char* why) { return fail_arg(why); }

// Loop mechanism of the sweeps: a CUDA-graph while node (default) or plain
// launches (EGPR_GRAPH_LOOP=0; profilers cannot capture kernels of conditional
// graphs).
bool graph_loop_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("EGPR_GRAPH_LOOP");
        return !(v && (v[0] == '0' || v[0] == 'n' || v[0] == 'N' || v[0] == 'f' || v[0] == 'F'));
    }();
    return on;
}

double wall_seconds() {
    using clock = std::chrono::steady_clock;
    return std::chrono::duration<double>(clock::now().time_since_epoch()).count();
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
cudaStream_t g_alloc_streams[64] = {};

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return dev;
}

// A non-blocking stream per device that orders pool allocations and frees.
cudaStream_t alloc_stream(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_alloc_streams[dev] && cudaStreamCreateWithFlags(&g_alloc_streams[dev], cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        g_alloc_streams[dev] = nullptr;
    }
    return g_alloc_streams[dev];
}
}  // namespace

cudaMemPool_t device_pool() {
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        // freed memory the pool keeps for reuse: EGPR_POOL_KEEP_MB, else a
        // quarter of the device (a scale-25 preparation frees ~17 GB of
        // scratch; mapping it again on every graph would cost ~1 s)
        const char* e = std::getenv("EGPR_POOL_KEEP_MB");
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            total_b = 32ull << 30;
        }
        const long long mb = e ? std::atoll(e) : (long long)(total_b >> 22);  // total / 4, in MiB
        unsigned long long keep = (unsigned long long)std::max(0LL, mb) << 20;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = p;
    }
    return g_pools[dev];
}

// Device buffers come from the device pool: an allocation is ordered on the
// device's allocation stream and waited for, so it is usable from any stream.
int DevBuf::alloc(size_t b) {
    release();
    if (b == 0) b = 16;
    const int d = current_device();
    cudaMemPool_t pool = device_pool();
    cudaStream_t s = alloc_stream(d);
    cudaError_t e;
    if (pool && s) {
        e = cudaMallocFromPoolAsync(&p, b, pool, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        pooled = true;
    } else {
        e = cudaMalloc(&p, b);
        pooled = false;
    }
    if (e != cudaSuccess) {
        if (p && pooled) cudaFreeAsync(p, s);
        p = nullptr;
        cudaGetLastError();
        set_cuda_error(e, "device allocation");
        return EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM;
    }
    dev = d;
    bytes = b;
    g_live_bytes += (int64_t)b;
    return EGPR_SUCC;
}

// Like cudaFree, a release first waits for the device, so no launch still in
// flight can read the buffer once the pool hands it out again.
void DevBuf::release() {
    if (p) {
        if (pooled) {
            int cur = current_device();
            if (dev >= 0 && cur != dev) cudaSetDevice(dev);
            cudaDeviceSynchronize();
            cudaFreeAsync(p, alloc_stream(dev));
            if (cur >= 0 && cur != dev) cudaSetDevice(cur);
        } else {
            cudaFree(p);
        }
        g_live_bytes -= (int64_t)bytes;
    }
    p = nullptr;
    bytes = 0;
    dev = -1;
    pooled = false;
}

int DevBuf::grow_on(size_t b, cudaStream_t s) {
    if (b == 0) b = 16;
    const int d = current_device();
    if (p && b <= bytes && dev == d) return EGPR_SUCC;
    release_on(s);
    cudaMemPool_t pool = device_pool();
    cudaError_t e;
    if (pool) {
        e = cudaMallocFromPoolAsync(&p, b, pool, s);
        pooled = true;
    } else {
        e = cudaMalloc(&p, b);
        pooled = false;
    }
    if (e != cudaSuccess) {
        p = nullptr;
        pooled = false;
        cudaGetLastError();
        set_cuda_error(e, "device allocation");
        return EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM;
    }
    dev = d;
    bytes = b;
    g_live_bytes += (int64_t)b;
    return EGPR_SUCC;
}

void DevBuf::release_on(cudaStream_t s) {
    if (p) {
        if (pooled) {
            cudaFreeAsync(p, s);  // after the work already queued on s
        } else {
            cudaStreamSynchronize(s);
            cudaFree(p);
        }
        g_live_bytes -= (int64_t)bytes;
    }
    p = nullptr;
    bytes = 0;
    dev = -1;
    pooled = false;
}

Plan::~Plan() { release(); }

void Plan::release() {
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg) cudaGraphDestroy(cg);
    cg_exec = nullptr;
    cg = nullptr;
    cond = 0;
    cg_failed = false;
    d_chunks.release();
    d_graphs.release();
    d_states.release();
    d_ndang.release();
    d_ctl.release();
    d_acc.release();
    d_span_acc.release();
    d_span_cnt.release();
    d_span_list.release();
    ngraphs = nchunks = grid = any_weighted = max_n = nspans = nacc = 0;
}

void Plan::release_on(cudaStream_t s) {
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg) cudaGraphDestroy(cg);
    cg_exec = nullptr;
    cg = nullptr;
    cond = 0;
    cg_failed = false;
    for (DevBuf* b : {&d_chunks, &d_graphs, &d_states, &d_ndang, &d_ctl, &d_acc, &d_span_acc, &d_span_cnt, &d_span_list})
        b->release_on(s);
    ngraphs = nchunks = grid = any_weighted = max_n = nspans = nacc = 0;
}

int check_device(const egpr_graph* g) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    if (dev != g->device) {
        t_last_error = "graph handle belongs to CUDA device " + std::to_string(g->device) +
                       " but device " + std::to_string(dev) + " is current";
        return EGPR_DEVICE_ERR;
    }
    return EGPR_SUCC;
}

// ---- profiler ranges ------------------------------------------------------------
// NVTX ranges around the phases of a call (prepare, solve, readback, tune), so a
// profiler's timeline shows where host time goes; free when no tool listens.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

static int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

static int64_t plain_bytes_per_iter(int64_t n, int64_t nnz, bool weighted) {
    // 4(n+1) row offsets + 4 nnz indices (+4 nnz weights) + 16 n of rank vectors.
    return 4 * (n + 1) + 4 * nnz + (weighted ? 4 * nnz : 0) + 16 * n;
}

// ---------------------------------------------------------------- solves ---

struct SolveOut {
    int32_t iterations = 0;
    int32_t converged = 0;
    double residual = 0.0;
    int32_t launches = 0;
    int32_t error = 0;
};

// Enqueues set-up, sweeps and finish for a plan on `s` (no host sync).
static int enqueue_plan(Plan& plan, double alpha, int32_t max_iter, double tol, bool personalised,
                        uint32_t flags, cudaStream_t s, int32_t* host_launches) {
    int rc;
    if ((rc = launch_init(plan, alpha, max_iter, tol, personalised, s))) return rc;
    int32_t l_loop = 0, l_fin = 0;
    if ((rc = launch_loop(plan, max_iter, s, &l_loop))) return rc;
    if ((rc = launch_finish(plan, (flags & EGPR_FLAG_NO_CORRECTION) == 0, s, &l_fin))) return rc;
    *host_launches = 3 + l_fin;  // init kernels + finish kernels; sweeps are counted on the device
    return EGPR_SUCC;
}

static int read_states(Plan& plan, int32_t idx, cudaStream_t s, SolveOut* o) {
    GraphState st;
    Ctl ctl;
    int rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(&st, plan.d_states.as<GraphState>() + idx, sizeof(st), cudaMemcpyDeviceToHost, s), "D2H state")) ||
        (rc = cuda_ok(cudaMemcpyAsync(&ctl, plan.d_ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "solve")))
        return rc;
    o->iterations = st.iter;
    o->converged = st.converged;
    o->residual = st.residual;
    o->launches = ctl.launches;
    o->error = ctl.error;
    return EGPR_SUCC;
}

// The state of a graph's last single-vector solve (binned or tile sweep).
static int read_single_state(egpr_graph* g, cudaStream_t s, SolveOut* o) {
    if (!g->bins) return read_states(g->plan, 0, s, o);
    return bins_read_state(g, s, &o->iterations, &o->converged, &o->residual, &o->launches, &o->error);
}

static void fill_stats(egpr_stats* stats, const egpr_graph* g, const SolveOut& o, double kernel_s,
                       double total_s, int32_t launches) {
    if (!stats) return;
    stats->iterations = o.iterations;
    stats->converged = o.converged;
    stats->residual = o.residual;
    stats->kernel_seconds = kernel_s;
    stats->total_seconds = total_s;
    stats->bytes_per_iter = plain_bytes_per_iter(g->n, g->nnz, g->weighted != 0);
    stats->launches = launches;
    stats->reserved = 0;
}

static void uniform_result(const egpr_graph* g, double* out, egpr_stats* stats, double t0) {
    if (out)
        for (int32_t i = 0; i < g->n; ++i) out[i] = 1.0 / g->n;
    SolveOut o;
    fill_stats(stats, g, o, 0.0, wall_seconds() - t0, 0);
}

static int upload_teleport(egpr_graph* g, const double* p, cudaStream_t s, std::vector<float>& staging) {
    double sum = 0.0;
    for (int32_t i = 0; i < g->n; ++i) {
        if (!(p[i] >= 0.0) || !std::isfinite(p[i])) return fail_arg("personalization values must be finite and >= 0");
        sum += p[i];
    }
    if (!(sum > 0.0)) return fail_arg("personalization must have a positive sum");
    staging.resize((size_t)g->n);
    for (int32_t i = 0; i < g->n; ++i) staging[(size_t)i] = (float)(p[i] / sum);
    int rc = cuda_ok(cudaMemcpyAsync(g->tele.p, staging.data(), staging.size() * sizeof(float), cudaMemcpyHostToDevice, s), "H2D teleport");
    if (rc) return rc;
    return cuda_ok(cudaStreamSynchronize(s), "H2D teleport");
}

// Seed-set teleport on the device: g->tele = 0, then 1/|S| at the seeds
// (sorted, duplicates removed, checked to lie in [0, n)).
__global__ void k_tele_seeds(float* __restrict__ tele, int32_t n, const int32_t* __restrict__ ids, int32_t count) {
    const float val = 1.0f / (float)count;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) tele[ids[i]] = val;
}

static int upload_teleport_seeds(egpr_graph* g, const int32_t* seeds, int32_t count, cudaStream_t s) {
    std::vector<int32_t> sv(seeds, seeds + count);
    std::sort(sv.begin(), sv.end());
    sv.erase(std::unique(sv.begin(), sv.end()), sv.end());
    if (sv.empty() || sv.front() < 0 || sv.back() >= g->n) return fail_arg("seed ids must lie in [0, n)");
    int rc = g->seed_ids.grow_on(sv.size() * sizeof(int32_t), s);  // the graph's own buffer, kept
    if (rc) return rc;
    rc = cuda_ok(cudaMemcpyAsync(g->seed_ids.p, sv.data(), sv.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s),
                 "H2D seeds");
    if (!rc) rc = cuda_ok(cudaMemsetAsync(g->tele.p, 0, (size_t)g->n * sizeof(float), s), "memset");
    if (!rc) {
        k_tele_seeds<<<(unsigned)std::min<size_t>((sv.size() + 255) / 256, 1024), 256, 0, s>>>(
            g->tele.as<float>(), g->n, g->seed_ids.as<int32_t>(), (int32_t)sv.size());
        rc = cuda_ok(cudaGetLastError(), "seed teleport");
    }
    if (rc) return rc;
    return cuda_ok(cudaStreamSynchronize(s), "seed teleport");  // sv is freed on return
}

// One single-vector solve; the teleport is the uniform vector, a dense host
// vector (pers) or one already on the device (tele_on_device).
static int solve_single(egpr_graph* g, double alpha, int32_t max_iter, double tol, const double* pers,
                        uint32_t flags, double* out, egpr_stats* stats, bool tele_on_device = false) {
    const double t0 = wall_seconds();
    int rc;
    if ((rc = check_device(g))) return rc;
    if (!out) return fail_arg("out_ranks is NULL");
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    if (g->nnz == 0) {
        uniform_result(g, out, stats, t0);
        return EGPR_SUCC;
    }
    cudaStream_t s = g->stream;
    std::vector<float> staging;
    if (pers && (rc = upload_teleport(g, pers, s, staging))) return rc;
    const bool personalised = pers != nullptr || tele_on_device;
    if (personalised && g->bins && (rc = bins_upload_tele(g, s))) return rc;
    int32_t host_launches = 0;
    {
        NvtxRange nv("egpr solve");
        if ((rc = cuda_ok(cudaEventRecord(g->ev0, s), "event"))) return rc;
        if (g->bins)
            rc = bins_enqueue(g, alpha, max_iter, tol, personalised, flags, s, &host_launches);
        else
            rc = enqueue_plan(g->plan, alpha, max_iter, tol, personalised, flags, s, &host_launches);
        if (rc) return rc;
        if ((rc = cuda_ok(cudaEventRecord(g->ev1, s), "event"))) return rc;
    }
    NvtxRange nv_read("egpr readback");
    if ((rc = download_d2h(out, g->out.p, (size_t)g->n * sizeof(double), s, "D2H ranks")))
        return rc;
    SolveOut o;
    if ((rc = read_single_state(g, s, &o))) return rc;
    if (o.error) {
        t_last_error = "sweep launch cap reached";
        return o.error;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    fill_stats(stats, g, o, ms * 1e-3, wall_seconds() - t0, host_launches + o.launches);
    return EGPR_SUCC;
}

// ------------------------------------------------------- multi-graph plans --
struct MultiPlan {
    std::vector<egpr_graph*> graphs;
    Plan plan;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~MultiPlan() {
        plan.release_on(stream);  // the plan's buffers serve this stream only
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

std::mutex g_multi_mu;
std::map<std::vector<egpr_graph*>, std::shared_ptr<MultiPlan>> g_multi_plans;

static void drop_multi_plans_with(egpr_graph* g) {
    std::lock_guard<std::mutex> lk(g_multi_mu);
    for (auto it = g_multi_plans.begin(); it != g_multi_plans.end();) {
        if (std::find(it->first.begin(), it->first.end(), g) != it->first.end()) it = g_multi_plans.erase(it);
        else ++it;
    }
}

static int get_multi_plan(egpr_graph* const* graphs, int32_t count, std::shared_ptr<MultiPlan>* out) {
    std::vector<egpr_graph*> key(graphs, graphs + count);
    std::lock_guard<std::mutex> lk(g_multi_mu);
    auto it = g_multi_plans.find(key);
    if (it != g_multi_plans.end()) {
        *out = it->second;
        return EGPR_SUCC;
    }
    auto mp = std::make_shared<MultiPlan>();
    mp->graphs = key;
    int rc;
    if ((rc = cuda_ok(cudaStreamCreateWithFlags(&mp->stream, cudaStreamNonBlocking), "stream")) ||
        (rc = cuda_ok(cudaEventCreate(&mp->ev0), "event")) || (rc = cuda_ok(cudaEventCreate(&mp->ev1), "event")))
        return rc;
    if ((rc = plan_build(mp->plan, graphs, count, mp->stream))) return rc;
    if (g_multi_plans.size() >= 16) g_multi_plans.erase(g_multi_plans.begin());
    g_multi_plans[key] = mp;
    *out = mp;
    return EGPR_SUCC;
}

// ------------------------------------------------------ keyed csr cache ----
struct CsrKey {
    uint64_t graph_id;
    const int32_t* V;
    const int32_t* E;
    const double* W;
    int32_t n;
    int64_t m;
    int32_t v_last;
    int32_t e_first, e_last;
    uint64_t w_first, w_last;
    int device;
    bool operator==(const CsrKey& o) const {
        return graph_id == o.graph_id && V == o.V && E == o.E && W == o.W && n == o.n && m == o.m &&
               v_last == o.v_last && e_first == o.e_first && e_last == o.e_last && w_first == o.w_first &&
               w_last == o.w_last && device == o.device;
    }
};

struct CsrEntry {
    CsrKey key;
    std::shared_ptr<egpr_graph> graph;
    int64_t bytes;
};

std::mutex g_csr_mu;
std::list<CsrEntry> g_csr_lru;  // front = most recent
int64_t g_csr_budget = 0;
int64_t g_csr_hits = 0, g_csr_misses = 0, g_csr_evictions = 0;
constexpr size_t kCsrMaxEntries = 8;

static uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof(u));
    return u;
}

}  // namespace egpr

int64_t egpr_graph::device_bytes() const {
    return (int64_t)(in_row.bytes + in_col.bytes + in_w.bytes + outw.bytes + dangling01.bytes +
                     sw_row.bytes + sw_col.bytes + sw_w.bytes + tile_bits.bytes + tile_row.bytes +
                     hub_ids.bytes + hub_slot.bytes + hubz.bytes + hubz64.bytes + plan.d_acc.bytes + plan.d_span_acc.bytes + plan.d_span_cnt.bytes +
                     plan.d_span_list.bytes +
                     scale.bytes + tele.bytes + x0.bytes + x1.bytes + z0.bytes + z1.bytes + out.bytes + z64.bytes +
                     plan.d_chunks.bytes + plan.d_graphs.bytes + plan.d_states.bytes + plan.d_ndang.bytes +
                     plan.d_ctl.bytes) + (bins ? bins->device_bytes() : 0);
}

using namespace egpr;

static void destroy_graph_object(egpr_graph* g) {
    if (!g) return;
    drop_multi_plans_with(g);
    int cur = -1;
    cudaGetDevice(&cur);
    if (g->device >= 0 && cur != g->device) cudaSetDevice(g->device);
    if (g->own_stream) cudaStreamSynchronize(g->own_stream);
    spmm_work_release(g);
    delete g->bins;
    g->bins = nullptr;
    g->plan.release();
    for (DevBuf* b : {&g->in_row, &g->in_col, &g->in_w, &g->outw, &g->dangling01, &g->sw_row,
                      &g->sw_col, &g->sw_w, &g->tile_bits, &g->tile_row,
                      &g->hub_ids, &g->hub_slot, &g->hubz, &g->hubz64, &g->scale, &g->tele, &g->seed_ids,
                      &g->x0, &g->x1, &g->z0, &g->z1, &g->out, &g->z64})
        b->release();
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->own_stream) cudaStreamDestroy(g->own_stream);
    if (cur >= 0 && cur != g->device) cudaSetDevice(cur);
    g_live_graphs -= 1;
    delete g;
}

// ---- persisted layout choices ------------------------------------------------------
// egpr_graph_autotune records its choice per GPU model and graph-shape bucket
// (log2 of n, log2 of the mean degree, weighted or not) in a small text file:
// EGPR_TUNE_CACHE names it (EGPR_TUNE_CACHE=0 turns the store off), default
// $XDG_CACHE_HOME/eggpu_b200/tuning.txt or ~/.cache/eggpu_b200/tuning.txt.  A
// graph prepared later (egpr_graph_create, and so egpr_pagerank_csr) whose
// shape falls in a recorded bucket starts with that layout, unless the layout
// is fixed through EGPR_CHUNKS_PER_WARP / EGPR_ROW_COST / EGPR_SPMM_CHUNK.
// One line per bucket: key, chunks_per_warp, row_cost, spmm_chunk, sweep ms.
namespace {
std::mutex g_tune_mu;

std::string tune_store_path() {
    const char* e = std::getenv("EGPR_TUNE_CACHE");
    if (e && e[0] == '0' && e[1] == 0) return std::string();
    if (e && e[0]) return std::string(e);
    const char* x = std::getenv("XDG_CACHE_HOME");
    const char* h = std::getenv("HOME");
    std::string dir = (x && x[0]) ? std::string(x) : (h && h[0]) ? std::string(h) + "/.cache" : std::string("/tmp");
    return dir + "/eggpu_b200/tuning.txt";
}

int floor_log2(uint64_t x) {
    int b = -1;
    while (x) {
        x >>= 1;
        ++b;
    }
    return b;
}

std::string tune_key(int dev, int32_t n, int64_t m, bool weighted) {
    static std::mutex name_mu;
    static std::map<int, std::string> names;
    std::string name;
    {
        std::lock_guard<std::mutex> lk(name_mu);
        auto it = names.find(dev);
        if (it == names.end()) {
            cudaDeviceProp pr = {};
            if (cudaGetDeviceProperties(&pr, dev) != cudaSuccess) {
                cudaGetLastError();
                std::snprintf(pr.name, sizeof(pr.name), "device%d", dev);
            }
            std::string nm(pr.name);
            for (char& c : nm)
                if (c == ' ' || c == '\t') c = '_';
            it = names.emplace(dev, nm).first;
        }
        name = it->second;
    }
    const int ln = floor_log2((uint64_t)std::max<int32_t>(n, 1));
    const int ld = floor_log2((uint64_t)std::max<int64_t>(m / std::max<int32_t>(n, 1), 1));
    return name + "|n2^" + std::to_string(ln) + "|d2^" + std::to_string(ld) + "|w" + (weighted ? "1" : "0");
}

bool tune_lookup(const std::string& key, egpr_tuning* out) {
    const std::string path = tune_store_path();
    if (path.empty()) return false;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string k;
        egpr_tuning t = {};
        if (!(ss >> k >> t.chunks_per_warp >> t.row_cost >> t.spmm_chunk >> t.sweep_ms)) continue;
        if (k == key) {
            *out = t;
            return true;
        }
    }
    return false;
}

void tune_record(const std::string& key, const egpr_tuning& t) {
    const std::string path = tune_store_path();
    if (path.empty()) return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::vector<std::string> keep;
    {
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string k;
            if ((ss >> k) && k != key) keep.push_back(line);
        }
    }
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        const std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)  // the directory chain, part by part
            if (i == dir.size() || dir[i] == '/') {
                const std::string part = dir.substr(0, i);
                if (!part.empty()) ::mkdir(part.c_str(), 0755);
            }
    }
    const std::string tmp = path + ".tmp" + std::to_string((long long)::getpid());
    {
        std::ofstream o(tmp, std::ios::trunc);
        if (!o) return;
        for (const std::string& l : keep) o << l << "\n";
        o << key << " " << t.chunks_per_warp << " " << t.row_cost << " " << t.spmm_chunk << " " << t.sweep_ms << "\n";
    }
    std::rename(tmp.c_str(), path.c_str());
}
}  // namespace

// The recorded layout of a graph of this shape, if any (before preparation).
void apply_recorded_tuning(egpr_graph* g) {
    if (std::getenv("EGPR_CHUNKS_PER_WARP") || std::getenv("EGPR_ROW_COST") || std::getenv("EGPR_SPMM_CHUNK")) return;
    egpr_tuning t = {};
    if (!tune_lookup(tune_key(g->device, g->n, g->m_input, g->weighted != 0), &t)) return;
    if (t.chunks_per_warp >= 1 && t.chunks_per_warp <= 64 && t.row_cost >= 0 && t.row_cost <= 64 &&
        t.spmm_chunk >= 64 && t.spmm_chunk <= (1 << 16) && (t.spmm_chunk % 32) == 0) {
        g->tune_cpw = t.chunks_per_warp;
        g->tune_rc = t.row_cost;
        g->tune_spmm_chunk = t.spmm_chunk;
        g->tuning_recorded = 1;
    }
}

// ---- layout tuning ----------------------------------------------------------
namespace {

bool tuning_valid(const egpr_tuning& t) {
    return t.chunks_per_warp >= 1 && t.chunks_per_warp <= 64 && t.row_cost >= 0 && t.row_cost <= 64 &&
           t.spmm_chunk >= 64 && t.spmm_chunk <= (1 << 16) && (t.spmm_chunk % 32) == 0;
}

// Rebuilds the sweep layout and the single-graph plan for the graph's current
// parameters (the inbound CSR and the hub codes stay as prepared).
int rebuild_sweep(egpr_graph* g) {
    cudaStream_t s = g->own_stream;
    int rc;
    if ((rc = cuda_ok(cudaStreamSynchronize(g->stream), "tuning")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "tuning")))
        return rc;
    drop_multi_plans_with(g);  // they hold copies of the graph's chunk table
    if ((rc = build_sweep_layout(g, sweep_resident_warps(), nullptr, s))) return rc;
    egpr_graph* self = g;
    if ((rc = plan_build(g->plan, &self, 1, s))) return rc;
    const size_t nf = ((size_t)g->n + 8) * sizeof(float);
    plan_set_l2_window(g->plan, g->z0.p, 2 * nf);
    return EGPR_SUCC;
}

// Device time of one sweep of the graph's current layout: fixed-count solves
// of S and S + L sweeps (no correction sweep), best of three, difference / L
// (the candidates differ by a few percent, about the spread of one sample).
int time_sweep(egpr_graph* g, double* ms) {
    cudaStream_t s = g->stream;
    const int32_t S = 3, L = 24;
    double best[2] = {1e30, 1e30};
    for (int rep = 0; rep < 3; ++rep)
        for (int i = 0; i < 2; ++i) {
            int32_t launches = 0;
            int rc;
            if ((rc = cuda_ok(cudaEventRecord(g->ev0, s), "event")) ||
                (rc = enqueue_plan(g->plan, 0.85, i ? S + L : S, 0.0, false, EGPR_FLAG_NO_CORRECTION, s, &launches)) ||
                (rc = cuda_ok(cudaEventRecord(g->ev1, s), "event")) ||
                (rc = cuda_ok(cudaStreamSynchronize(s), "tuning")))
                return rc;
            float t = 0.f;
            cudaEventElapsedTime(&t, g->ev0, g->ev1);
            best[i] = std::min(best[i], (double)t);
        }
    *ms = std::max(0.0, (best[1] - best[0]) / L);
    return EGPR_SUCC;
}

// Device time of one batched sweep (one panel: 32 single-vertex seed sets).
int time_spmm(egpr_graph* g, double* ms) {
    const int32_t k = 32, S = 2, L = 8;
    std::vector<int32_t> ptr(k + 1), seeds(k);
    for (int32_t j = 0; j < k; ++j) {
        ptr[(size_t)j] = j;
        seeds[(size_t)j] = (int32_t)(((int64_t)j * 2654435761LL) % g->n);
    }
    ptr[(size_t)k] = k;
    std::vector<egpr_stats> st((size_t)k);
    double best[2] = {1e30, 1e30};
    for (int rep = 0; rep < 2; ++rep)
        for (int i = 0; i < 2; ++i) {
            int rc = ppr_batch_solve(g, 0.85, i ? S + L : S, 0.0, k, nullptr, ptr.data(), seeds.data(),
                                     EGPR_FLAG_NO_CORRECTION, nullptr, st.data());
            if (rc) return rc;
            best[i] = std::min(best[i], st[0].kernel_seconds * 1e3);
        }
    *ms = std::max(0.0, (best[1] - best[0]) / L);
    return EGPR_SUCC;
}

}  // namespace

extern "C" {

const char* egpr_status_string(int status) {
    switch (status) {
        case EGPR_SUCC: return "EasyGraph GPU: success";
        case EGPR_FAILED_TO_ALLOCATE_HOST_MEM: return "EasyGraph GPU: failed to allocate host mem";
        case EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM: return "EasyGraph GPU: failed to allocate gpu mem";
        case EGPR_DEVICE_ERR: return "EasyGraph GPU: gpu error occurred";
        case EGPR_UNKNOWN_ERROR: return "EasyGraph GPU: gpu unknown error";
        case EGPR_UNSUPPORTED_GRAPH: return "EasyGraph GPU: unsupported graph type";
        case EGPR_NEGATIVE_CYCLE: return "EasyGraph GPU: negative weight cycle detected";
        case EGPR_TIMEOUT: return "EasyGraph GPU: bounded device wait timed out";
        case EGPR_INVALID_ARGUMENT: return "EasyGraph GPU: invalid argument";
        default: return "EasyGraph GPU: not a valid err_code";
    }
}

const char* egpr_last_error(void) { return egpr::t_last_error.c_str(); }

int egpr_graph_create(const int32_t* V, const int32_t* E, const double* W, int32_t n, int64_t m,
                      egpr_graph** out) {
    if (!out) return fail_arg("out is NULL");
    *out = nullptr;
    if (n < 1 || n >= INT32_MAX) return fail_arg("n must be in [1, 2^31-1)");
    if (m < 0 || m >= INT32_MAX) return fail_arg("m must be in [0, 2^31-1)");
    if (!V) return fail_arg("V is NULL");
    if (m > 0 && !E) return fail_arg("E is NULL");
    if (V[0] != 0 || (int64_t)V[n] != m) return fail_arg("CSR offsets must start at 0 and end at m");
    {
        // branch-free over blocks of 4096 (the compiler vectorises them), the
        // blocks spread over host threads for large graphs
        int bad = 0;
        const int64_t blocks = ((int64_t)n + 4095) / 4096;
#pragma omp parallel for schedule(static) reduction(| : bad) if (blocks >= 64)
        for (int64_t k = 0; k < blocks; ++k) {
            const int32_t b = (int32_t)(k * 4096), e = std::min(n, b + 4096);
            int bb = 0;
            for (int32_t i = b; i < e; ++i) bb |= V[i + 1] < V[i];
            bad |= bb;
        }
        if (bad) return fail_arg("CSR offsets must be non-decreasing");
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    egpr_graph* g = new (std::nothrow) egpr_graph();
    if (!g) return EGPR_FAILED_TO_ALLOCATE_HOST_MEM;
    g_live_graphs += 1;
    g->device = dev;
    g->n = n;
    g->m_input = m;
    g->weighted = W ? 1 : 0;
    int rc;
    if ((rc = cuda_ok(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking), "stream")) ||
        (rc = cuda_ok(cudaEventCreate(&g->ev0), "event")) || (rc = cuda_ok(cudaEventCreate(&g->ev1), "event"))) {
        destroy_graph_object(g);
        return rc;
    }
    g->stream = g->own_stream;
    g->tune_cpw = default_chunks_per_warp();
    g->tune_rc = default_row_cost();
    g->tune_spmm_chunk = default_spmm_chunk();
    apply_recorded_tuning(g);
    {
        NvtxRange r("egpr prepare");
        if ((rc = prepare_graph(g, V, E, W))) {
            destroy_graph_object(g);
            return rc;
        }
    }
    // Row arrays are read by 16-byte bulk copies that may run up to 3 elements past n.
    const size_t nf = ((size_t)n + 8) * sizeof(float), nd = (size_t)n * sizeof(double);
    if ((rc = g->scale.alloc(nf)) || (rc = g->tele.alloc(nf)) || (rc = g->x0.alloc(nf)) || (rc = g->x1.alloc(nf)) ||
        (rc = g->z0.alloc(2 * nf)) || (rc = g->out.alloc(nd)) || (rc = g->z64.alloc(nd + sizeof(double))) ||
        (rc = g->hubz.alloc(2 * (size_t)hub_stride(g->nhub) * sizeof(float))) ||
        (rc = g->hubz64.alloc(((size_t)g->nhub + 1) * sizeof(double))) ||
        // zero slots: hubz[.][nhub] and z64[n] are read by placeholder entries
        (rc = (cudaMemsetAsync(g->hubz.p, 0, g->hubz.bytes, g->own_stream) == cudaSuccess &&
               cudaMemsetAsync(g->z64.p, 0, g->z64.bytes, g->own_stream) == cudaSuccess)
                  ? EGPR_SUCC
                  : set_cuda_error(cudaGetLastError(), "memset"))) {
        destroy_graph_object(g);
        return rc;
    }
    egpr_graph* self = g;
    if ((rc = plan_build(g->plan, &self, 1, g->own_stream))) {
        destroy_graph_object(g);
        return rc;
    }
    plan_set_l2_window(g->plan, g->z0.p, 2 * nf);
    *out = g;
    return EGPR_SUCC;
}

int egpr_graph_destroy(egpr_graph* g) {
    if (!g) return EGPR_SUCC;
    {
        std::lock_guard<std::mutex> lk(g->mu);
        if (g->sessions > 0) return fail_arg("the graph has live sessions (egpr_session_destroy them first)");
    }
    destroy_graph_object(g);
    return EGPR_SUCC;
}

int egpr_graph_info_get(const egpr_graph* g, egpr_graph_info* info) {
    if (!g || !info) return fail_arg("NULL argument");
    info->n = g->n;
    info->device = g->device;
    info->m_input = g->m_input;
    info->nnz = g->nnz;
    info->weighted = g->weighted;
    info->n_dangling = g->n_dangling;
    info->device_bytes = g->device_bytes();
    info->prep_seconds = g->prep_seconds;
    return EGPR_SUCC;
}

int egpr_graph_export_inbound(const egpr_graph* gc, int32_t* in_row, int32_t* in_col, float* in_w,
                              int32_t* dangling01, double* out_weight_sum) {
    egpr_graph* g = const_cast<egpr_graph*>(gc);
    if (!g || !in_row || !dangling01 || !out_weight_sum || (g->nnz > 0 && !in_col)) return fail_arg("NULL argument");
    std::lock_guard<std::mutex> lk(g->mu);
    int rc;
    if ((rc = check_device(g))) return rc;
    cudaStream_t s = g->stream;
    if ((rc = cuda_ok(cudaMemcpyAsync(in_row, g->in_row.p, ((size_t)g->n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H")) ||
        (rc = export_in_col(g, in_col, s)) ||
        (rc = cuda_ok(cudaMemcpyAsync(dangling01, g->dangling01.p, (size_t)g->n * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H")) ||
        (rc = cuda_ok(cudaMemcpyAsync(out_weight_sum, g->outw.p, (size_t)g->n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H")))
        return rc;
    if (in_w && g->nnz > 0) {
        if (g->weighted) {
            if ((rc = cuda_ok(cudaMemcpyAsync(in_w, g->in_w.p, (size_t)g->nnz * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H")))
                return rc;
        } else {
            for (int64_t i = 0; i < g->nnz; ++i) in_w[i] = 1.0f;
        }
    }
    return cuda_ok(cudaStreamSynchronize(s), "export");
}

int egpr_graph_get_tuning(const egpr_graph* g, egpr_tuning* out) {
    if (!g || !out) return fail_arg("NULL argument");
    std::memset(out, 0, sizeof(*out));
    out->chunks_per_warp = g->tune_cpw;
    out->row_cost = g->tune_rc;
    out->spmm_chunk = g->tune_spmm_chunk;
    return EGPR_SUCC;
}

int egpr_graph_set_tuning(egpr_graph* g, const egpr_tuning* in) {
    if (!g || !in) return fail_arg("NULL argument");
    if (!tuning_valid(*in))
        return fail_arg("tuning out of range: chunks_per_warp 1..64, row_cost 0..64, spmm_chunk 64..65536 in steps of 32");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    int rc;
    if ((rc = check_device(g))) return rc;
    const bool sweep = in->chunks_per_warp != g->tune_cpw || in->row_cost != g->tune_rc;
    const bool spmm = in->spmm_chunk != g->tune_spmm_chunk;
    if (spmm && g->sessions > 0) return fail_arg("the batched solve's layout is in use by a session");
    g->tune_cpw = in->chunks_per_warp;
    g->tune_rc = in->row_cost;
    g->tune_spmm_chunk = in->spmm_chunk;
    if (spmm) {
        cudaStreamSynchronize(g->stream);
        spmm_work_release(g);  // rebuilt for the new tile by the next batched solve
    }
    if (sweep && g->nnz > 0 && (rc = rebuild_sweep(g))) return rc;
    return EGPR_SUCC;
}

int egpr_graph_autotune(egpr_graph* g, uint32_t what, egpr_tuning* out) {
    if (!g) return fail_arg("NULL graph");
    NvtxRange nv("egpr autotune");
    if (what == 0) what = EGPR_TUNE_SWEEP | EGPR_TUNE_SPMM;
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    int rc;
    if ((rc = check_device(g))) return rc;
    egpr_tuning res;
    std::memset(&res, 0, sizeof(res));
    if (g->nnz > 0 && (what & EGPR_TUNE_SWEEP)) {
        double best = 1e30;
        int32_t bc = g->tune_cpw, br = g->tune_rc;
        for (int32_t cpw : {4, 8, 16})
            for (int32_t rcost : {2, 4, 8}) {
                g->tune_cpw = cpw;
                g->tune_rc = rcost;
                double ms = 0.0;
                if ((rc = rebuild_sweep(g)) || (rc = time_sweep(g, &ms))) return rc;
                res.configs_tried += 1;
                if (ms < best) {
                    best = ms;
                    bc = cpw;
                    br = rcost;
                }
            }
        g->tune_cpw = bc;
        g->tune_rc = br;
        if ((rc = rebuild_sweep(g))) return rc;
        res.sweep_ms = best;
    }
    if (g->nnz > 0 && (what & EGPR_TUNE_SPMM) && g->sessions > 0)
        return fail_arg("the batched solve's layout is in use by a session");
    if (g->nnz > 0 && (what & EGPR_TUNE_SPMM)) {
        double best = 1e30;
        int32_t bc = g->tune_spmm_chunk;
        for (int32_t c : {512, 1024, 2048}) {
            cudaStreamSynchronize(g->stream);
            spmm_work_release(g);
            g->tune_spmm_chunk = c;
            double ms = 0.0;
            if ((rc = time_spmm(g, &ms))) return rc;
            res.configs_tried += 1;
            if (ms < best) {
                best = ms;
                bc = c;
            }
        }
        if (bc != g->tune_spmm_chunk) {
            cudaStreamSynchronize(g->stream);
            spmm_work_release(g);
            g->tune_spmm_chunk = bc;
        }
        res.spmm_sweep_ms = best;
    }
    res.chunks_per_warp = g->tune_cpw;
    res.row_cost = g->tune_rc;
    res.spmm_chunk = g->tune_spmm_chunk;
    if (g->nnz > 0) tune_record(tune_key(g->device, g->n, g->m_input, g->weighted != 0), res);
    if (out) *out = res;
    return EGPR_SUCC;
}

int egpr_graph_set_stream(egpr_graph* g, void* stream) {
    if (!g) return fail_arg("NULL graph");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    g->stream = stream ? static_cast<cudaStream_t>(stream) : g->own_stream;
    return EGPR_SUCC;
}

int egpr_pagerank(egpr_graph* g, double alpha, int32_t max_iter, double tol, const double* personalization,
                  uint32_t flags, double* out_ranks, egpr_stats* stats) {
    if (!g) return fail_arg("NULL graph");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    return solve_single(g, alpha, max_iter, tol, personalization, flags, out_ranks, stats);
}

int egpr_pagerank_enqueue(egpr_graph* g, double alpha, int32_t max_iter, double tol, uint32_t flags) {
    if (!g) return fail_arg("NULL graph");
    std::lock_guard<std::mutex> lk(g->mu);
    int rc;
    if ((rc = check_device(g))) return rc;
    // A new enqueue supersedes an uncollected one: both run in stream order
    // on the same workspace and collect reports the latest.
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    g->pending_t0 = wall_seconds();
    g->pending_launches = 0;
    if (g->nnz > 0) {
        if ((rc = cuda_ok(cudaEventRecord(g->ev0, g->stream), "event"))) return rc;
        if (g->bins)
            rc = bins_enqueue(g, alpha, max_iter, tol, false, flags, g->stream, &g->pending_launches);
        else
            rc = enqueue_plan(g->plan, alpha, max_iter, tol, false, flags, g->stream, &g->pending_launches);
        if (rc) return rc;
        if ((rc = cuda_ok(cudaEventRecord(g->ev1, g->stream), "event"))) return rc;
    }
    g->pending = true;
    return EGPR_SUCC;
}

int egpr_pagerank_collect(egpr_graph* g, double* out_ranks, egpr_stats* stats) {
    if (!g) return fail_arg("NULL graph");
    std::lock_guard<std::mutex> lk(g->mu);
    if (!g->pending) return fail_arg("no solve is pending on this graph");
    g->pending = false;
    int rc;
    if ((rc = check_device(g))) return rc;
    if (g->nnz == 0) {
        uniform_result(g, out_ranks, stats, g->pending_t0);
        return EGPR_SUCC;
    }
    cudaStream_t s = g->stream;
    if (out_ranks &&
        (rc = download_d2h(out_ranks, g->out.p, (size_t)g->n * sizeof(double), s, "D2H ranks")))
        return rc;
    SolveOut o;
    if ((rc = read_single_state(g, s, &o))) return rc;
    if (o.error) return o.error;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    fill_stats(stats, g, o, ms * 1e-3, wall_seconds() - g->pending_t0, g->pending_launches + o.launches);
    return EGPR_SUCC;
}

int egpr_pagerank_batch(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k, const double* teleport,
                        uint32_t flags, double* out, egpr_stats* stats) {
    if (!g) return fail_arg("NULL graph");
    if (k < 1 || !teleport || !out) return fail_arg("k >= 1, teleport and out are required");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    if (k < kSpmmMinColumns) {  // a few columns: single-vector solves cost less than a 32-column panel
        for (int32_t j = 0; j < k; ++j) {
            int rc = solve_single(g, alpha, max_iter, tol, teleport + (size_t)j * g->n, flags, out + (size_t)j * g->n,
                                  stats ? stats + j : nullptr);
            if (rc) return rc;
        }
        return EGPR_SUCC;
    }
    return ppr_batch_solve(g, alpha, max_iter, tol, k, teleport, nullptr, nullptr, flags, out, stats);
}

int egpr_pagerank_seeds(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k, const int32_t* seed_ptr,
                        const int32_t* seeds, uint32_t flags, double* out, egpr_stats* stats) {
    if (!g) return fail_arg("NULL graph");
    if (k < 1 || !seed_ptr || !out) return fail_arg("k >= 1, seed_ptr and out are required");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return fail_arg("a solve is pending on this graph");
    if (k < kSpmmMinColumns) {  // a few columns: single-vector solves with the seed sets uploaded sparse
        int rc;
        if ((rc = check_device(g))) return rc;
        for (int32_t j = 0; j < k; ++j) {
            const int32_t b = seed_ptr[j], e = seed_ptr[j + 1];
            if (e <= b || b < 0) return fail_arg("every seed set needs at least one seed");
            if (g->nnz > 0 && (rc = upload_teleport_seeds(g, seeds + b, e - b, g->stream))) return rc;
            if ((rc = solve_single(g, alpha, max_iter, tol, nullptr, flags, out + (size_t)j * g->n,
                                   stats ? stats + j : nullptr, true)))
                return rc;
        }
        return EGPR_SUCC;
    }
    return ppr_batch_solve(g, alpha, max_iter, tol, k, nullptr, seed_ptr, seeds, flags, out, stats);
}

int egpr_pagerank_multi(int32_t count, egpr_graph* const* graphs, double alpha, int32_t max_iter, double tol,
                        uint32_t flags, double* const* outs, egpr_stats* stats) {
    const double t0 = wall_seconds();
    if (count < 1 || !graphs || !outs) return fail_arg("count >= 1, graphs and outs are required");
    for (int32_t i = 0; i < count; ++i) {
        if (!graphs[i] || !outs[i]) return fail_arg("NULL graph or output");
        for (int32_t j = 0; j < i; ++j)
            if (graphs[j] == graphs[i]) return fail_arg("a graph appears twice in one batch");
    }
    // Lock every handle in address order.
    std::vector<egpr_graph*> order(graphs, graphs + count);
    std::sort(order.begin(), order.end());
    std::vector<std::unique_lock<std::mutex>> locks;
    for (egpr_graph* g : order) locks.emplace_back(g->mu);
    int rc;
    for (egpr_graph* g : order) {
        if ((rc = check_device(g))) return rc;
        if (g->pending) return fail_arg("a solve is pending on a graph of the batch");
    }
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    // Graphs without inbound entries are answered on the host (uniform).
    std::vector<egpr_graph*> live;
    std::vector<int32_t> live_idx;
    for (int32_t i = 0; i < count; ++i) {
        if (graphs[i]->nnz == 0) uniform_result(graphs[i], outs[i], stats ? &stats[i] : nullptr, t0);
        else {
            live.push_back(graphs[i]);
            live_idx.push_back(i);
        }
    }
    if (live.empty()) return EGPR_SUCC;
    std::shared_ptr<MultiPlan> mp;
    if ((rc = get_multi_plan(live.data(), (int32_t)live.size(), &mp))) return rc;
    cudaStream_t s = mp->stream;
    if ((rc = cuda_ok(cudaEventRecord(mp->ev0, s), "event"))) return rc;
    int32_t host_launches = 0;
    if ((rc = enqueue_plan(mp->plan, alpha, max_iter, tol, false, flags, s, &host_launches))) return rc;
    if ((rc = cuda_ok(cudaEventRecord(mp->ev1, s), "event"))) return rc;
    for (size_t i = 0; i < live.size(); ++i) {
        egpr_graph* g = live[i];
        if ((rc = download_d2h(outs[live_idx[i]], g->out.p, (size_t)g->n * sizeof(double), s, "D2H ranks")))
            return rc;
    }
    std::vector<GraphState> st(live.size());
    Ctl ctl;
    if ((rc = cuda_ok(cudaMemcpyAsync(st.data(), mp->plan.d_states.p, st.size() * sizeof(GraphState), cudaMemcpyDeviceToHost, s), "D2H states")) ||
        (rc = cuda_ok(cudaMemcpyAsync(&ctl, mp->plan.d_ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "multi solve")))
        return rc;
    if (ctl.error) return ctl.error;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, mp->ev0, mp->ev1);
    const double total = wall_seconds() - t0;
    if (stats) {
        for (size_t i = 0; i < live.size(); ++i) {
            SolveOut o;
            o.iterations = st[i].iter;
            o.converged = st[i].converged;
            o.residual = st[i].residual;
            fill_stats(&stats[live_idx[i]], live[i], o, ms * 1e-3, total, host_launches + ctl.launches);
        }
    }
    return EGPR_SUCC;
}

int egpr_pagerank_csr(const int32_t* V, int32_t len_V, const int32_t* E, int64_t len_E, const double* W,
                      uint64_t graph_id, double alpha, int32_t max_iter_num, double threshold, double* PR,
                      double* kernel_seconds) {
    if (kernel_seconds) *kernel_seconds = 0.0;
    const int32_t n = len_V - 1;
    if (n <= 0) return EGPR_SUCC;  // centrality.cpp:160-165
    if (!V || !PR || (len_E > 0 && !E)) return fail_arg("NULL argument");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    CsrKey key;
    key.graph_id = graph_id;
    key.V = V;
    key.E = E;
    key.W = W;
    key.n = n;
    key.m = len_E;
    key.v_last = V[n];
    key.e_first = len_E > 0 ? E[0] : 0;
    key.e_last = len_E > 0 ? E[len_E - 1] : 0;
    key.w_first = (W && len_E > 0) ? bits_of(W[0]) : 0;
    key.w_last = (W && len_E > 0) ? bits_of(W[len_E - 1]) : 0;
    key.device = dev;
    std::shared_ptr<egpr_graph> g;
    {
        std::lock_guard<std::mutex> lk(g_csr_mu);
        for (auto it = g_csr_lru.begin(); it != g_csr_lru.end(); ++it) {
            if (it->key == key) {
                g = it->graph;
                g_csr_lru.splice(g_csr_lru.begin(), g_csr_lru, it);
                ++g_csr_hits;
                break;
            }
        }
    }
    if (!g) {
        egpr_graph* raw = nullptr;
        int rc = egpr_graph_create(V, E, W, n, len_E, &raw);
        if (rc) return rc;
        g = std::shared_ptr<egpr_graph>(raw, [](egpr_graph* p) { egpr_graph_destroy(p); });
        std::lock_guard<std::mutex> lk(g_csr_mu);
        ++g_csr_misses;
        if (g_csr_budget <= 0) {
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            g_csr_budget = std::max<int64_t>((int64_t)fr / 4, (int64_t)256 << 20);
        }
        // Drop entries with the same id (a rebuilt CSR replaces the old one).
        for (auto it = g_csr_lru.begin(); it != g_csr_lru.end();) {
            if (it->key.graph_id == graph_id && it->key.device == dev) {
                it = g_csr_lru.erase(it);
                ++g_csr_evictions;
            } else
                ++it;
        }
        g_csr_lru.push_front(CsrEntry{key, g, raw->device_bytes()});
        int64_t used = 0;
        for (auto& en : g_csr_lru) used += en.bytes;
        while (g_csr_lru.size() > 1 && (used > g_csr_budget || g_csr_lru.size() > kCsrMaxEntries)) {
            used -= g_csr_lru.back().bytes;
            g_csr_lru.pop_back();
            ++g_csr_evictions;
        }
    }
    egpr_stats st;
    int rc = egpr_pagerank(g.get(), alpha, max_iter_num, threshold, nullptr, 0u, PR, &st);
    if (rc == EGPR_SUCC && kernel_seconds) *kernel_seconds = st.kernel_seconds;
    return rc;
}

int egpr_cache_stats_get(egpr_cache_stats* out) {
    if (!out) return fail_arg("NULL argument");
    std::lock_guard<std::mutex> lk(g_csr_mu);
    out->graphs = g_live_graphs.load();
    out->device_bytes = g_live_bytes.load();
    out->hits = g_csr_hits;
    out->misses = g_csr_misses;
    out->evictions = g_csr_evictions;
    out->budget_bytes = g_csr_budget;
    return EGPR_SUCC;
}

int egpr_cache_reset(void) {
    std::list<CsrEntry> drop;
    {
        std::lock_guard<std::mutex> lk(g_csr_mu);
        drop.swap(g_csr_lru);
        g_csr_hits = g_csr_misses = g_csr_evictions = 0;
    }
    drop.clear();
    return EGPR_SUCC;
}

int egpr_cache_set_budget(int64_t bytes) {
    std::lock_guard<std::mutex> lk(g_csr_mu);
    g_csr_budget = bytes < 0 ? 0 : bytes;
    return EGPR_SUCC;
}

}  // extern "C"
