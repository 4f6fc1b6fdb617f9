// PageRank on an inbound CSR that the caller already holds in device memory,
// without allocating anything: egpr_pagerank_device_noalloc.
//
// Who needs it: code that runs where it may not call cudaMalloc — inside a
// framework that owns all device memory through its own pool, on a serving
// thread with a fixed memory budget, or in a plug-in whose host forbids
// allocations while a request is in flight.  Such a caller brings its own
// inputs and outputs; every other buffer the solve needs lives in one
// file-scope device array of fixed size (g_scratch below).  Its size is set by
// kNoAllocMaxVertices: every GPU that loads this library holds these bytes until
// the process exits, whether or not the entry point is ever called.
//
// The solve is a compact variant of the sweep in sweep.cu with the same
// arithmetic (pagerank.py:75-139 restated as a pull): FP32 iterates, FP64
// residual, dangling mass and rank sums added as order-free fixed-point
// integers, a final FP64 sweep from x_{k-1}, then normalisation.  One warp
// works on one row at a time, which suits the graphs that fit the limit.
//
// Every call shares the one scratch array and leaves the last call's contents
// in it; each call clears what must start at zero.  Calls that overlap on the
// GPU (another host thread, or another stream) race on it and give wrong
// answers: callers serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <mutex>

#include "egpr_internal.cuh"

namespace egpr {
int arg_error(const char* why);
}

namespace {

using egpr::set_cuda_error;

constexpr int32_t kNoAllocMaxVertices = 1 << 18;  // 262,144 vertices
constexpr int kThreadsNa = 256;
constexpr unsigned kFullNa = 0xffffffffu;

// Solve state at the start of the scratch array.
struct NaState {
    unsigned long long acc[6];  // residual, dangling mass, rank sum: 2 fixed-point words each
    double alpha;
    double c1;                  // (1 - alpha) / n
    double tol_n;
    double dmass;               // alpha * dangling mass / n for the next sweep
    double dmass_prev;          // the value the last sweep used
    double residual;
    double residual64;
    double xsum;
    int32_t n;
    int32_t iter;
    int32_t max_iter;
    int32_t done;
    int32_t converged;
    int32_t ndang;
    uint32_t exited;            // blocks that left the running sweep
    int32_t pad;
    unsigned long long t_begin; // global timer (ns) when the solve's first kernel started
    unsigned long long t_end;   // global timer (ns) when its last kernel ran
};

constexpr size_t kStateBytes = 256;
static_assert(sizeof(NaState) <= kStateBytes, "state fits its slot");
// The state, then x0, x1, z0, z1 (FP32, kNoAllocMaxVertices each): 4 MiB + 256 B.
constexpr size_t kScratchBytes = kStateBytes + 4 * (size_t)kNoAllocMaxVertices * sizeof(float);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct NaView {
    NaState* st;
    float* x[2];
    float* z[2];
};

__device__ __forceinline__ NaView na_view(unsigned char* base) {
    NaView v;
    v.st = reinterpret_cast<NaState*>(base);
    float* f = reinterpret_cast<float*>(base + kStateBytes);
    v.x[0] = f;
    v.x[1] = f + kNoAllocMaxVertices;
    v.z[0] = f + 2 * (size_t)kNoAllocMaxVertices;
    v.z[1] = f + 3 * (size_t)kNoAllocMaxVertices;
    return v;
}

// Two's-complement fixed point in units of 2^-32 and 2^-64: integer adds, so
// the totals do not depend on the order in which blocks finish.
__device__ __forceinline__ void na_fx_add(unsigned long long* a, double v) {
    const double t = v * 4294967296.0;
    const double f = floor(t);
    atomicAdd(a, (unsigned long long)(long long)f);
    atomicAdd(a + 1, (unsigned long long)rint((t - f) * 4294967296.0));
}

__device__ __forceinline__ double na_fx_join(unsigned long long hi, unsigned long long lo) {
    return (double)(long long)hi * (1.0 / 4294967296.0) + (double)lo * (1.0 / 18446744073709551616.0);
}

__device__ __forceinline__ unsigned long long na_global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void k_na_reset(unsigned char* base, int32_t n, double alpha, double tol, int32_t max_iter) {
    NaState* st = na_view(base).st;
    st->t_begin = na_global_ns();
    st->t_end = 0ull;
    for (int i = 0; i < 6; ++i) st->acc[i] = 0ull;
    st->alpha = alpha;
    st->c1 = (1.0 - alpha) / (double)n;
    st->tol_n = tol * (double)n;
    st->dmass = st->dmass_prev = 0.0;
    st->residual = st->residual64 = st->xsum = 0.0;
    st->n = n;
    st->iter = 0;
    st->max_iter = max_iter;
    st->done = 0;
    st->converged = 0;
    st->ndang = 0;
    st->exited = 0u;
}

// x0 = 1/n; z0 = x0 * alpha/outw (0 for a dangling source, outw <= 1e-15,
// pagerank.py:118); count of dangling vertices.
__global__ void k_na_init(unsigned char* base, int32_t n, const double* __restrict__ outw, double alpha) {
    const NaView V = na_view(base);
    const float x0 = (float)(1.0 / (double)n);
    int32_t dang = 0;
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const double o = outw[v];
        const float sc = o <= 1e-15 ? -1.f : (float)(alpha / o);
        V.x[0][v] = x0;
        V.z[0][v] = sc >= 0.f ? x0 * sc : 0.f;
        dang += sc < 0.f ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) dang += __shfl_down_sync(kFullNa, dang, o);
    if ((threadIdx.x & 31) == 0 && dang) atomicAdd(&V.st->ndang, dang);
}

// Dangling term of the first sweep (dangling mass of x0).
__global__ void k_na_start(unsigned char* base) {
    NaState* st = na_view(base).st;
    const double x0 = (double)(float)(1.0 / (double)st->n);
    st->dmass = st->alpha * ((double)st->ndang * x0) / (double)st->n;
    st->dmass_prev = st->dmass;
}

// One sweep.  FP32 (kFinal false): x_new = sum w*z[u] + jump for every row,
// z_new, residual / dangling / rank sums; the last block out advances the
// state.  FP64 (kFinal true): the same rows from x_{k-1} with z computed in
// FP64, written unnormalised to ranks.
template <bool kFinal>
__global__ void k_na_sweep(unsigned char* base, int32_t n, int64_t nnz, const int32_t* __restrict__ in_row,
                           const int32_t* __restrict__ in_col, const float* __restrict__ in_w,
                           const double* __restrict__ outw, double* __restrict__ ranks) {
    __shared__ int32_t s_flag;
    __shared__ double red[kThreadsNa / 32][3];
    const NaView V = na_view(base);
    NaState* st = V.st;
    if (threadIdx.x == 0) s_flag = kFinal ? 0 : __ldcg(&st->done);
    __syncthreads();
    if (s_flag) return;  // converged earlier: the same answer for every block of this launch
    const int32_t iter = __ldcg(&st->iter);
    const double alpha = st->alpha;
    const float* xin = V.x[kFinal ? ((iter - 1) & 1) : (iter & 1)];
    const float* zin = V.z[iter & 1];
    float* xout = V.x[(iter & 1) ^ 1];
    float* zout = V.z[(iter & 1) ^ 1];
    const double jump = st->c1 + (kFinal ? __ldcg(&st->dmass_prev) : __ldcg(&st->dmass));
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double err = 0.0, dsum = 0.0, xsum = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib; r < n; r += warps) {
        // rows are clamped to [0, nnz] and sources to [0, n): no access outside the inputs
        int64_t b = in_row[r], e = in_row[r + 1];
        b = b < 0 ? 0 : (b > nnz ? nnz : b);
        e = e < b ? b : (e > nnz ? nnz : e);
        double acc64 = 0.0;
        float acc32 = 0.f;
        for (int64_t p = b + lane; p < e; p += 32) {
            const int32_t u = in_col[p];
            if (u < 0 || u >= n) continue;
            const float w = in_w ? in_w[p] : 1.f;
            if (kFinal) {
                const double o = outw[u];
                const double z = o <= 1e-15 ? 0.0 : alpha * (double)xin[u] / o;
                acc64 += (double)w * z;
            } else {
                acc32 += w * zin[u];
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc64 += __shfl_xor_sync(kFullNa, acc64, o);
            acc32 += __shfl_xor_sync(kFullNa, acc32, o);
        }
        if (lane == 0) {
            if (kFinal) {
                const double val = acc64 + jump;
                err += fabs(val - (double)xin[r]);
                ranks[r] = val;
                xsum += val;
            } else {
                const float xo = (float)((double)acc32 + jump);
                err += fabs((double)xo - (double)xin[r]);
                xout[r] = xo;
                const double o = outw[r];
                const float sc = o <= 1e-15 ? -1.f : (float)(alpha / o);
                zout[r] = sc >= 0.f ? xo * sc : 0.f;
                if (sc < 0.f) dsum += (double)xo;
                xsum += (double)xo;
            }
        }
    }
    if (lane == 0) {
        red[wib][0] = err;
        red[wib][1] = dsum;
        red[wib][2] = xsum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, d = 0.0, x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[w][0];
            d += red[w][1];
            x += red[w][2];
        }
        na_fx_add(&st->acc[0], a);
        na_fx_add(&st->acc[2], d);
        na_fx_add(&st->acc[4], x);
        __threadfence();
        const uint32_t prev = atomicAdd(&st->exited, 1u);
        s_flag = prev == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!s_flag || threadIdx.x != 0) return;
    // Last block out: the totals of this sweep.
    __threadfence();
    unsigned long long w[6];
    for (int i = 0; i < 6; ++i) {
        w[i] = __ldcg(&st->acc[i]);
        st->acc[i] = 0ull;
    }
    st->exited = 0u;
    const double e = na_fx_join(w[0], w[1]), d = na_fx_join(w[2], w[3]), x = na_fx_join(w[4], w[5]);
    if (kFinal) {
        st->residual64 = e;
        st->xsum = x;
    } else {
        st->residual = e;
        st->xsum = x;
        st->dmass_prev = st->dmass;
        st->dmass = alpha * d / (double)n;
        const int32_t it = iter + 1;
        st->iter = it;
        const bool conv = e < st->tol_n;
        if (conv || it >= st->max_iter) {
            st->done = 1;
            st->converged = conv ? 1 : 0;
        }
    }
    __threadfence();
}

// Final normalisation (pagerank.py:134-139); from_fp32: the last FP32 iterate.
__global__ void k_na_normalize(unsigned char* base, int32_t n, double* __restrict__ ranks, int32_t from_fp32) {
    const NaView V = na_view(base);
    const double norm = V.st->xsum;
    const float* xl = V.x[V.st->iter & 1];
    const double inv = norm > 0.0 ? 1.0 / norm : 0.0;
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const double val = from_fp32 ? (double)xl[v] : ranks[v];
        ranks[v] = norm > 0.0 ? val * inv : 1.0 / (double)n;
    }
}

// Device time stamp after every kernel of the solve (stream order): the
// solve's device time is t_end - t_begin, taken without creating events.
__global__ void k_na_stamp(unsigned char* base) { na_view(base).st->t_end = na_global_ns(); }

// Device address of g_scratch, looked up once per device with that device
// current.  In host code the name g_scratch stands for a host-side shadow, not
// for device memory, so kernels get this address instead.
std::mutex g_scratch_mu;
unsigned char* g_scratch_dev[64] = {};

int scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 64) return egpr::arg_error("egpr_pagerank_device_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) return set_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                         "cudaGetSymbolAddress (no-alloc scratch)");
        g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_dev[dev];
    return EGPR_SUCC;
}

}  // namespace

extern "C" EGPR_API int egpr_pagerank_device_noalloc(int32_t n, int64_t nnz, const int32_t* in_row,
                                                     const int32_t* in_col, const float* in_w,
                                                     const double* out_weight, double alpha, int32_t max_iter,
                                                     double tol, uint32_t flags, double* ranks, void* stream,
                                                     egpr_stats* stats) {
    using namespace egpr;
    const auto t0 = std::chrono::steady_clock::now();
    if (n <= 0) {
        if (stats) *stats = egpr_stats{};  // nothing to solve: zero sweeps, zero time
        return EGPR_SUCC;
    }
    if (n > kNoAllocMaxVertices)
        return arg_error("egpr_pagerank_device_noalloc: n exceeds the 262144-vertex limit of its fixed scratch");
    if (nnz < 0 || nnz > (int64_t)INT32_MAX) return arg_error("egpr_pagerank_device_noalloc: nnz out of range");
    if (!in_row || (nnz > 0 && !in_col) || !out_weight || !ranks)
        return arg_error("egpr_pagerank_device_noalloc: a required device pointer is NULL");
    if (!(alpha >= 0.0 && alpha < 1.0)) return arg_error("egpr_pagerank_device_noalloc: alpha must be in [0, 1)");
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    unsigned char* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool correction = !(flags & EGPR_FLAG_NO_CORRECTION);
    const int blocks_v = (int)std::min<int64_t>(((int64_t)n + kThreadsNa - 1) / kThreadsNa, 1184);
    const int blocks_r = (int)std::min<int64_t>(((int64_t)n * 32 + kThreadsNa - 1) / kThreadsNa, 1184);
    k_na_reset<<<1, 1, 0, s>>>(base, n, alpha, tol, max_iter);
    k_na_init<<<blocks_v, kThreadsNa, 0, s>>>(base, n, out_weight, alpha);
    k_na_start<<<1, 1, 0, s>>>(base);
    // Every sweep is launched; those after convergence return at once.
    for (int32_t it = 0; it < max_iter; ++it)
        k_na_sweep<false><<<blocks_r, kThreadsNa, 0, s>>>(base, n, nnz, in_row, in_col, in_w, out_weight, ranks);
    if (correction)
        k_na_sweep<true><<<blocks_r, kThreadsNa, 0, s>>>(base, n, nnz, in_row, in_col, in_w, out_weight, ranks);
    k_na_normalize<<<blocks_v, kThreadsNa, 0, s>>>(base, n, ranks, correction ? 0 : 1);
    k_na_stamp<<<1, 1, 0, s>>>(base);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_cuda_error(e, "no-alloc solve launch");
    if (stats) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return set_cuda_error(e, "no-alloc solve");
        NaState h;
        if ((e = cudaMemcpy(&h, base, sizeof(NaState), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return set_cuda_error(e, "no-alloc solve state");
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        stats->iterations = h.iter;
        stats->converged = h.converged;
        stats->residual = h.residual;
        stats->kernel_seconds = h.t_end > h.t_begin ? (double)(h.t_end - h.t_begin) * 1e-9 : 0.0;
        stats->total_seconds = secs;
        stats->bytes_per_iter = (int64_t)(n + 1) * 4 + nnz * (in_w ? 8 : 4) + (int64_t)n * 20;
        stats->launches = 5 + max_iter + (correction ? 1 : 0);
        stats->reserved = 0;
    }
    return EGPR_SUCC;
}
