// One power-iteration sweep per kernel launch, for one or many graphs.
//
// The sweep computes, for every vertex v (one "row" of the inbound CSR),
//     x_new[v] = sum_{u -> v} w_uv * z[u]  +  jump
// with z[u] = alpha * x[u] / outw[u] (0 for dangling u) and
// jump = (1-alpha)/n + alpha * (dangling mass)/n — the arithmetic of the
// reference's _pagerank_power_iteration (easygraph/functions/centrality/
// pagerank.py:112-132) evaluated as a pull — and in the same launch:
//   * the FP64 L1 residual sum |x_new - x| (pagerank.py:127-130),
//   * the FP64 dangling mass of x_new for the next sweep (pagerank.py:117-120),
//   * z_new = x_new * alpha / outw for the next sweep,
//   * the FP64 sum of x_new (final normalisation, pagerank.py:134-139),
//   * the stop decision err < tol*n (pagerank.py:131) and, through a CUDA
//     graph conditional node, whether the next sweep runs at all.
// This replaces, per iteration, the reference GPU path's cuSPARSE SpMV, cuBLAS
// Sdot, two memsets, add_base_and_reduce, scale_vec and the two host round
// trips (gpu_easygraph/functions/centrality/pagerank.cu:591-664).
//
// Work split.  A graph's rows are packed into stages of at most
// kStageMaxEntries inbound entries and kStageMaxRows rows (only a row longer
// than a stage is cut).  One persistent CTA runs per SM with three roles that
// meet at a ring of stage buffers in shared memory, each guarded by mbarriers:
//   * a producer warp claims stages from a global queue (a batch ahead) and
//     moves each stage's sources, weights, row offsets, previous ranks, scales
//     and hub slots into a free buffer with bulk copies (TMA);
//   * gatherer warps replace every source by its carried value: hubs (the
//     kHubCap largest out-degrees, encoded -(slot+1)) from the CTA's copy of
//     the hub values, staged once per launch, the rest with asynchronous 4-byte
//     copies from z (cp.async, tracked by the buffer's mbarrier), so a warp has
//     no register tied to a load in flight and many stages gather at once;
//   * two groups of eight consumer warps take alternate stages and work from
//     shared memory only: row ends are marked, each thread sums its 8 entries
//     segment by segment, a segmented scan over the group joins rows that cross
//     threads, and the rows are finished with coalesced stores.
// Rows cut between stages are finished by whichever stage arrives last, adding
// the pieces in stage order.  FP64 partial sums are reduced in a fixed order
// through groups of stages and then per graph, so every result is
// deterministic.  No CTA waits on another; every wait inside a CTA is bounded
// by the global timer and ends the launch with EGPR_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kGatherWarps = 4;
constexpr int kGroupWarps = kStageEntries / (32 * kLaneItems);  // consumer warps per group
constexpr int kConsumerGroups = 2;
constexpr int kCtaWarps = 1 + kGatherWarps + kConsumerGroups * kGroupWarps;
constexpr int kCtaThreads = 32 * kCtaWarps;
constexpr int kGatherThreads = 32 * kGatherWarps;
constexpr int kGroupThreads = 32 * kGroupWarps;
constexpr int kMaxSlots = 8;          // stage buffers at most
constexpr int kClaim = 4;             // stages claimed from the queue at a time
constexpr int kGatherLag = 2;         // stages a gatherer keeps in flight before signalling the oldest
constexpr int kSmemGraphs = 256;      // graph states mirrored in shared memory
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kCopyPiece = 32768;             // bytes per hub staging copy
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of every wait (2 s)

static_assert(kGroupWarps * 32 * kLaneItems == kStageEntries, "a group covers one stage buffer");
static_assert(kStageEntries % kGatherThreads == 0, "gatherers cover one stage buffer");
static_assert(kGatherLag >= 1 && kGatherLag < kMaxSlots, "the ring must hold the stages a gatherer keeps in flight");

struct StageInfo {
    Chunk ck;
    int32_t c;     // global stage id; -1: no more stages
    int32_t iter;  // sweeps done by the stage's graph
    int32_t pad[2];
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;  // valid in lane 0
}

// ---- PTX wrappers ------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Generic-proxy writes to a stage buffer are ordered before the next bulk copy into it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void group_sync(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kGroupThreads) : "memory");
}
// Barrier of one consumer group that also ORs a predicate over its threads.
__device__ __forceinline__ bool group_any(int id, bool pred) {
    uint32_t r;
    asm volatile(
        "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; bar.red.or.pred q, %2, %3, p; selp.u32 %0, 1, 0, q; }"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(kGroupThreads)
        : "memory");
    return r != 0;
}

// Bounded wait for the completion of phase `parity` of b.  Gives up when another
// role of the CTA has given up or after kWaitNs, and then flags the launch.
__device__ bool wait_bar(uint64_t* b, uint32_t parity, volatile int32_t* abort_flag, Ctl* ctl) {
    if (mbar_try(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try(b, parity)) return true;
        if ((i & 31u) == 0u) {
            if (*abort_flag) return false;
            if (global_ns() - t0 > kWaitNs) {
                *abort_flag = 1;
                atomicExch(&ctl->error, EGPR_TIMEOUT);
                return false;
            }
        }
    }
}

// ---- per-graph view ------------------------------------------------------------
struct SweepView {
    const float* xin;       // previous ranks (global; rows of cut spans)
    float* xout;
    float* zout;
    float* hub_out;         // hub values written for the next sweep
    const float* scale;
    const int32_t* hub_slot;
    const float* tele;
    double* out;
    double jump;            // (1-alpha)/n + dangling term (uniform teleport)
    double dmass;           // dangling term alone (personalised teleport)
    double one_minus_alpha;
    int32_t personalised;
    int32_t weighted;
};

template <bool kFinal>
__device__ SweepView make_view(const GraphDev& G, GraphState* st, int32_t iter) {
    SweepView W;
    W.one_minus_alpha = 1.0 - st->alpha;
    W.personalised = st->personalised;
    W.weighted = G.in_w != nullptr;
    W.scale = G.scale;
    W.hub_slot = G.hub_slot;
    W.tele = G.tele;
    W.out = G.out;
    if (!kFinal) {
        const int par = iter & 1;
        W.xin = G.x[par];
        W.xout = G.x[par ^ 1];
        W.zout = G.z[par ^ 1];
        W.hub_out = G.hubz[par ^ 1];
        W.dmass = ldcg(&st->dmass);
    } else {
        W.xin = G.x[(iter - 1) & 1];  // x_{k-1}: the input of the last sweep
        W.xout = nullptr;
        W.zout = nullptr;
        W.hub_out = nullptr;
        W.dmass = ldcg(&st->dmass_prev);
    }
    W.jump = st->c1 + W.dmass;
    return W;
}

// Finishes row v given its gathered sum; accumulates residual / dangling /
// rank sums.  FP32 sweep: writes x_new, z_new (and the hub copy of z_new); the
// residual compares the stored FP32 iterates, so the loop can stop once they no
// longer change even when tol*n is below FP32 resolution.  FP64 correction
// sweep: writes the FP64 result.
template <bool kFinal>
__device__ __forceinline__ void finish_row(const SweepView& W, int32_t v, double acc, float xin, float scale,
                                           int32_t hs, double& err, double& dsum, double& xsum) {
    double val;
    if (W.personalised) val = (acc + W.one_minus_alpha * (double)__ldg(W.tele + v)) + W.dmass;
    else val = acc + W.jump;
    if (!kFinal) {
        const float xo = (float)val;
        err += fabs((double)xo - (double)xin);
        W.xout[v] = xo;
        const float zo = scale >= 0.f ? xo * scale : 0.f;
        W.zout[v] = zo;
        if (hs >= 0) W.hub_out[hs] = zo;
        if (scale < 0.f) dsum += (double)xo;
        xsum += (double)xo;
    } else {
        err += fabs(val - (double)xin);
        W.out[v] = val;
        xsum += val;
    }
}

// ---- order-free FP64 sums ---------------------------------------------------------
// A value is split into two's-complement words in units of 2^-32 and of 2^-64
// (the remainder, truncated) and added with integer atomics, so the total does
// not depend on the order in which stages finish.  Partial sums here are far
// below 2^31 and there are far fewer than 2^21 terms, so no word overflows and
// both convert to double exactly.
__device__ __forceinline__ void fx_add(unsigned long long* a, double v) {
    const double t = v * 4294967296.0;  // exact
    const double f = floor(t);
    const unsigned long long hi = (unsigned long long)(long long)f;
    const unsigned long long lo = (unsigned long long)((t - f) * 4294967296.0);
    atomicAdd(a, hi);  // results unused: issued as reductions
    atomicAdd(a + 1, lo);
}

__device__ __forceinline__ double fx_join(unsigned long long hi, unsigned long long lo) {
    return (double)(long long)hi * (1.0 / 4294967296.0) + (double)lo * (1.0 / 18446744073709551616.0);
}

__device__ __forceinline__ unsigned long long ldcg_u64(const unsigned long long* p) { return __ldcg(p); }

// Accumulator slot of (graph, CTA, consumer group): each graph has acc_sub
// slots so that concurrent stages rarely add to the same address.
__device__ __forceinline__ unsigned long long* acc_slot(const SweepParams& P, int32_t gi, int32_t k) {
    return P.acc + (size_t)kAccWords * ((size_t)gi * (size_t)P.acc_sub + (size_t)(k % P.acc_sub));
}

// Stage done (lane 0 of a consumer group's first warp): the stage's sums, and
// the pieces of rows cut between stages, go to the accumulators.
__device__ __forceinline__ void stage_accumulate(const SweepParams& P, int32_t c, const Chunk& ck, int32_t k,
                                                 double err, double dsum, double xsum, double head_val,
                                                 double tail_val) {
    unsigned long long* a = acc_slot(P, ck.graph, k);
    fx_add(a, err);
    fx_add(a + 2, dsum);
    fx_add(a + 4, xsum);
    const int32_t f = ck.flags;
    if (f & kInterior) {
        fx_add(P.span_acc + 2 * ck.head_ta, tail_val);
    } else {
        if (f & kHasHead) fx_add(P.span_acc + 2 * ck.head_ta, head_val);
        if (f & kHasTail) fx_add(P.span_acc + 2 * c, tail_val);
    }
}

// End of a launch, run by the whole last CTA to leave the queue: finishes the
// rows cut between stages, then per graph turns the accumulators into the
// residual, dangling mass and rank sum, clears them, and advances the graph's
// state (pagerank.py:117-131).
template <bool kFinal>
__device__ void launch_tail(const SweepParams& P) {
    const int tid = threadIdx.x;
    for (int32_t q = tid; q < P.nspans; q += blockDim.x) {
        const int32_t ta = P.span_list[q];
        const int32_t gi = __ldg(&P.chunks[ta].graph);
        const int32_t v = __ldg(&P.chunks[ta].tail_row);
        GraphState* st = P.states + gi;
        if (!kFinal && ldcg(&st->done)) continue;
        unsigned long long* sa = P.span_acc + 2 * ta;
        const double sum = fx_join(ldcg_u64(sa), ldcg_u64(sa + 1));
        sa[0] = 0ull;
        sa[1] = 0ull;
        const SweepView W = make_view<kFinal>(P.graphs[gi], st, ldcg(&st->iter));
        double e = 0.0, d = 0.0, x = 0.0;
        finish_row<kFinal>(W, v, sum, W.xin[v], kFinal ? 0.f : W.scale[v], kFinal ? -1 : W.hub_slot[v], e, d, x);
        unsigned long long* a = acc_slot(P, gi, tid);
        fx_add(a, e);
        fx_add(a + 2, d);
        fx_add(a + 4, x);
    }
    __threadfence();
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int32_t gi = warp; gi < P.ngraphs; gi += (int32_t)(blockDim.x >> 5)) {
        GraphState* st = P.states + gi;
        if (!kFinal && ldcg(&st->done)) continue;
        unsigned long long w[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
        for (int32_t k = lane; k < P.acc_sub; k += 32) {
            unsigned long long* a = P.acc + (size_t)kAccWords * ((size_t)gi * (size_t)P.acc_sub + (size_t)k);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                w[i] += ldcg_u64(a + i);
                a[i] = 0ull;
            }
        }
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w[i] += __shfl_down_sync(kFull, w[i], o);
        if (lane == 0) {
            const double e = fx_join(w[0], w[1]), d = fx_join(w[2], w[3]), x = fx_join(w[4], w[5]);
            if (!kFinal) {
                st->residual = e;
                st->dsum = d;
                st->xsum = x;
                st->dmass_prev = st->dmass;
                st->dmass = st->alpha * d / (double)P.graphs[gi].n;
                const int32_t it = st->iter + 1;
                st->iter = it;
                const bool conv = e < st->tol_n;
                if (conv || it >= st->max_iter) {
                    st->done = 1;
                    st->converged = conv ? 1 : 0;
                    atomicSub(&P.ctl->active, 1);
                }
            } else {
                st->residual64 = e;
                st->xsum = x;
            }
        }
    }
    __threadfence();
    __syncthreads();
}

// ---- the three roles -------------------------------------------------------------
struct CtaShared {
    uint64_t bar_full[kMaxSlots];   // bulk copies of the stage landed (1 arrival + bytes)
    uint64_t bar_gath[kMaxSlots];   // gathered values in place (1 arrival per gatherer thread)
    uint64_t bar_empty[kMaxSlots];  // the consumers are done with the buffer (1 per consumer warp)
    uint64_t bar_hub;               // hub values staged
    StageInfo info[kMaxSlots];
    double red[kConsumerGroups][kGroupWarps][3];
    double scan_d[kConsumerGroups][kGroupWarps];
    float scan_f[kConsumerGroups][kGroupWarps];
    int32_t scan_flag[kConsumerGroups][kGroupWarps];
    int32_t giter[kSmemGraphs];
    int32_t gdone[kSmemGraphs];
    int32_t abort_flag;
    int32_t idle;
    int32_t last;
};

__device__ __forceinline__ Chunk shfl_chunk(const Chunk& a, int src) {
    Chunk b;
    const int32_t* pa = reinterpret_cast<const int32_t*>(&a);
    int32_t* pb = reinterpret_cast<int32_t*>(&b);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Chunk) / 4); ++i) pb[i] = __shfl_sync(kFull, pa[i], src);
    return b;
}

__device__ __forceinline__ Chunk load_chunk(const Chunk* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    Chunk c;
    int4* d = reinterpret_cast<int4*>(&c);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Chunk) / 16); ++i) d[i] = __ldg(q + i);
    return c;
}

template <bool kFinal>
__device__ void run_producer(const SweepParams& P, CtaShared& S, unsigned char* stages, float* hub_smem) {
    const int lane = threadIdx.x & 31;
    const StageLayout& L = P.lay;
    const uint32_t nslots = (uint32_t)L.slots;
    volatile int32_t* abort_flag = &S.abort_flag;
    if (L.hub_count > 0 && lane == 0) {
        const uint32_t bytes = (uint32_t)L.hub_count * (uint32_t)sizeof(float);
        const float* src = P.graphs[0].hubz[S.giter[0] & 1];
        mbar_arrive_tx(&S.bar_hub, bytes);
        for (uint32_t off = 0; off < bytes; off += kCopyPiece)
            bulk_load(reinterpret_cast<unsigned char*>(hub_smem) + off, reinterpret_cast<const unsigned char*>(src) + off,
                      min(kCopyPiece, bytes - off), &S.bar_hub);
    }
    // Claims run one batch ahead: the queue position of the next batch and its
    // stage records are in flight while the current batch is issued.
    int32_t base_next = 0, base_after = P.nchunks;
    if (lane == 0) base_next = (int32_t)atomicAdd(&P.ctl->queue, (uint32_t)kClaim);
    base_next = __shfl_sync(kFull, base_next, 0);
    if (lane == 0 && base_next < P.nchunks) base_after = (int32_t)atomicAdd(&P.ctl->queue, (uint32_t)kClaim);
    Chunk nk{};
    if (lane < kClaim && base_next + lane < P.nchunks) nk = load_chunk(P.chunks + base_next + lane);
    uint32_t q = 0;
    bool abort = false;
    // lane 0's cache of the current graph's arrays
    int32_t cg = -1, citer = -1;
    const int32_t* in_col = nullptr;
    const float* in_w = nullptr;
    const int32_t* in_row = nullptr;
    const float* xin = nullptr;
    const float* scale = nullptr;
    const int32_t* hslot = nullptr;
    while (!abort) {
        const int32_t base = base_next;
        if (base >= P.nchunks) break;
        const Chunk cur = nk;
        base_next = __shfl_sync(kFull, base_after, 0);
        if (lane == 0)
            base_after = base_next < P.nchunks ? (int32_t)atomicAdd(&P.ctl->queue, (uint32_t)kClaim) : P.nchunks;
        if (lane < kClaim && base_next + lane < P.nchunks) nk = load_chunk(P.chunks + base_next + lane);
        for (int i = 0; i < kClaim; ++i) {
            const int32_t c = base + i;
            if (c >= P.nchunks) break;
            const Chunk ck = shfl_chunk(cur, i);
            const int32_t gi = ck.graph;
            const int32_t iter = gi < kSmemGraphs ? S.giter[gi] : ldcg(&P.states[gi].iter);
            if (!kFinal && (gi < kSmemGraphs ? S.gdone[gi] : ldcg(&P.states[gi].done))) continue;
            const uint32_t slot = q % nslots, round = q / nslots;
            if (round > 0 && !wait_bar(&S.bar_empty[slot], (round - 1) & 1u, abort_flag, P.ctl)) {
                abort = true;
                break;
            }
            if (lane == 0) {
                if (gi != cg || iter != citer) {
                    const GraphDev& G = P.graphs[gi];
                    in_col = G.in_col;
                    in_w = G.in_w;
                    in_row = G.in_row;
                    xin = kFinal ? G.x[(iter - 1) & 1] : G.x[iter & 1];
                    scale = G.scale;
                    hslot = G.hub_slot;
                    cg = gi;
                    citer = iter;
                }
                StageInfo& in = S.info[slot];
                in.ck = ck;
                in.c = c;
                in.iter = iter;
                unsigned char* sp = stages + (size_t)slot * (size_t)L.slot_bytes;
                const int32_t e0 = ck.nnz_begin, e1 = ck.nnz_end;
                const int32_t eb = e0 & ~3;
                const uint32_t ebytes = e1 > e0 ? (uint32_t)(((e1 + 3) & ~3) - eb) * 4u : 0u;
                const int32_t ra = ck.sub_begin, nr = ck.sub_end - ck.sub_begin;
                const int32_t rb = ra & ~3;
                const uint32_t pbytes = nr > 0 ? (uint32_t)(((ra + nr + 1 + 3) & ~3) - rb) * 4u : 0u;
                const uint32_t xbytes = nr > 0 ? (uint32_t)(((ra + nr + 3) & ~3) - rb) * 4u : 0u;
                const uint32_t tx = ebytes * (in_w ? 2u : 1u) + pbytes + xbytes * (kFinal ? 1u : 3u);
                mbar_arrive_tx(&S.bar_full[slot], tx);
                if (ebytes) {
                    bulk_load(sp + L.off_col, in_col + eb, ebytes, &S.bar_full[slot]);
                    if (in_w) bulk_load(sp + L.off_w, in_w + eb, ebytes, &S.bar_full[slot]);
                }
                if (nr > 0) {
                    bulk_load(sp + L.off_rowptr, in_row + rb, pbytes, &S.bar_full[slot]);
                    bulk_load(sp + L.off_xin, xin + rb, xbytes, &S.bar_full[slot]);
                    if (!kFinal) {
                        bulk_load(sp + L.off_scale, scale + rb, xbytes, &S.bar_full[slot]);
                        bulk_load(sp + L.off_hslot, hslot + rb, xbytes, &S.bar_full[slot]);
                    }
                }
            }
            __syncwarp();
            ++q;
        }
    }
    // One end marker per consumer group (the gatherers stop at the first).
    for (int k = 0; k < kConsumerGroups && !abort; ++k) {
        const uint32_t slot = q % nslots, round = q / nslots;
        if (round > 0 && !wait_bar(&S.bar_empty[slot], (round - 1) & 1u, abort_flag, P.ctl)) {
            abort = true;
            break;
        }
        if (lane == 0) {
            S.info[slot].c = -1;
            mbar_arrive(&S.bar_full[slot]);
        }
        __syncwarp();
        ++q;
    }
    if (abort && lane == 0) {
        // Leave no bulk copy in flight into this CTA's shared memory.
        const uint32_t first = q > nslots ? q - nslots : 0u;
        for (uint32_t k = first; k < q; ++k) {
            const unsigned long long t0 = global_ns();
            while (!mbar_try(&S.bar_full[k % nslots], (k / nslots) & 1u) && global_ns() - t0 < kWaitNs) {
            }
        }
        if (L.hub_count > 0) {
            const unsigned long long t0 = global_ns();
            while (!mbar_try(&S.bar_hub, 0u) && global_ns() - t0 < kWaitNs) {
            }
        }
    }
}

template <bool kFinal>
__device__ void run_gatherer(const SweepParams& P, CtaShared& S, unsigned char* stages, const float* hub_smem) {
    constexpr int kPer = kStageEntries / kGatherThreads;  // entries per gatherer thread and stage
    const int j = threadIdx.x - 32;                       // 0 .. kGatherThreads-1
    const StageLayout& L = P.lay;
    const uint32_t nslots = (uint32_t)L.slots;
    volatile int32_t* abort_flag = &S.abort_flag;
    bool ok = L.hub_count > 0 ? wait_bar(&S.bar_hub, 0u, abort_flag, P.ctl) : true;
    int32_t cg = -1, citer = -1;
    const float* zsrc = nullptr;
    const float* hub_g = nullptr;
    const double* z64 = nullptr;
    const int32_t* hub_ids = nullptr;
    uint32_t q = 0;
    for (; ok; ++q) {
        const uint32_t slot = q % nslots, round = q / nslots;
        if (!wait_bar(&S.bar_full[slot], round & 1u, abort_flag, P.ctl)) break;
        const StageInfo& in = S.info[slot];
        if (in.c < 0) break;
        const int32_t gi = in.ck.graph, iter = in.iter;
        if (gi != cg || iter != citer) {
            const GraphDev& G = P.graphs[gi];
            zsrc = G.z[iter & 1];
            hub_g = G.hubz[iter & 1];
            z64 = G.z64;
            hub_ids = G.hub_ids;
            cg = gi;
            citer = iter;
        }
        unsigned char* sp = stages + (size_t)slot * (size_t)L.slot_bytes;
        int32_t* col = reinterpret_cast<int32_t*>(sp + L.off_col);
        double* v64 = reinterpret_cast<double*>(sp + L.off_val64);
        const int32_t eb = in.ck.nnz_begin & ~3;
        const int32_t lo = in.ck.nnz_begin - eb, hi = in.ck.nnz_end - eb;
        // Consecutive threads take consecutive entries: conflict-free shared
        // memory on both the source read and the value write.
        int32_t cv[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) cv[i] = col[j + i * kGatherThreads];
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int k = j + i * kGatherThreads;
            if (k < lo || k >= hi) continue;
            const int32_t s = cv[i];
            if (!kFinal) {
                if (s >= 0) {
                    cp_async4(col + k, zsrc + s);
                } else {
                    const int32_t h = -s - 1;
                    if (h < L.hub_count) reinterpret_cast<float*>(col)[k] = hub_smem[h];
                    else cp_async4(col + k, hub_g + h);
                }
            } else {
                const int32_t idx = s >= 0 ? s : __ldg(hub_ids + (-s - 1));
                cp_async8(v64 + k, z64 + idx);
            }
        }
        cp_async_commit();
        // Stage q - kGatherLag has landed: hand it to the consumers.
        if (q >= (uint32_t)kGatherLag) {
            cp_async_wait_group<kGatherLag>();
            mbar_arrive(&S.bar_gath[(q - kGatherLag) % nslots]);
        }
    }
    cp_async_wait_all();
    for (uint32_t p = q > (uint32_t)kGatherLag ? q - kGatherLag : 0u; p < q; ++p) mbar_arrive(&S.bar_gath[p % nslots]);
}

template <typename Real>
__device__ __forceinline__ void scan_store(CtaShared& S, int g, int w, Real v);
template <>
__device__ __forceinline__ void scan_store<float>(CtaShared& S, int g, int w, float v) { S.scan_f[g][w] = v; }
template <>
__device__ __forceinline__ void scan_store<double>(CtaShared& S, int g, int w, double v) { S.scan_d[g][w] = v; }
template <typename Real>
__device__ __forceinline__ Real scan_load(const CtaShared& S, int g, int w);
template <>
__device__ __forceinline__ float scan_load<float>(const CtaShared& S, int g, int w) { return S.scan_f[g][w]; }
template <>
__device__ __forceinline__ double scan_load<double>(const CtaShared& S, int g, int w) { return S.scan_d[g][w]; }

template <typename Real>
__device__ void run_consumer(const SweepParams& P, CtaShared& S, unsigned char* stages) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int gt = threadIdx.x - 32 * (1 + kGatherWarps);
    const int g = gt / kGroupThreads, t = gt % kGroupThreads;
    const int w = t >> 5, lane = t & 31;
    const int bar_id = 1 + g;
    const StageLayout& L = P.lay;
    const uint32_t nslots = (uint32_t)L.slots;
    volatile int32_t* abort_flag = &S.abort_flag;
    int32_t cg = -1, citer = -1;
    SweepView W{};
    const int k0 = kLaneItems * t;
    for (uint32_t q = (uint32_t)g;; q += kConsumerGroups) {
        const uint32_t slot = q % nslots, round = q / nslots;
        const bool ok = wait_bar(&S.bar_full[slot], round & 1u, abort_flag, P.ctl);
        StageInfo in;
        in.c = -1;
        if (ok) in = S.info[slot];
        if (group_any(bar_id, !ok || in.c < 0)) break;
        if (in.ck.graph != cg || in.iter != citer) {
            cg = in.ck.graph;
            citer = in.iter;
            W = make_view<kFinal>(P.graphs[cg], P.states + cg, citer);
        }
        unsigned char* sp = stages + (size_t)slot * (size_t)L.slot_bytes;
        const int32_t e0 = in.ck.nnz_begin, e1 = in.ck.nnz_end;
        const int32_t eb = e0 & ~3, lo = e0 - eb, hi = e1 - eb;
        const int32_t ra = in.ck.sub_begin, nr = in.ck.sub_end - in.ck.sub_begin, ro = ra & 3;
        const int32_t* rowp = reinterpret_cast<const int32_t*>(sp + L.off_rowptr) + ro;
        uint8_t* mark = sp + L.off_mark;
        // 1. mark the last entry of every row that ends in this stage
        for (int j = t; j < nr; j += kGroupThreads) {
            const int32_t rs = rowp[j], re = rowp[j + 1];
            if (re <= e1 && re > max(rs, e0)) mark[re - 1 - eb] = 1;
        }
        const bool ok2 = wait_bar(&S.bar_gath[slot], round & 1u, abort_flag, P.ctl);
        if (group_any(bar_id, !ok2)) break;
        // 2. per-thread segmented sums over entries k0 .. k0+7; row sums are
        //    written in place at the row's last entry
        Real* rsum = kFinal ? reinterpret_cast<Real*>(sp + L.off_val64) : reinterpret_cast<Real*>(sp + L.off_col);
        Real v[kLaneItems];
        if (!kFinal) {
            const float4 a = *reinterpret_cast<const float4*>(sp + L.off_col + 4 * k0);
            const float4 b = *reinterpret_cast<const float4*>(sp + L.off_col + 4 * k0 + 16);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
            v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
#pragma unroll
            for (int u = 0; u < kLaneItems; u += 2) {
                const double2 d = *reinterpret_cast<const double2*>(sp + L.off_val64 + 8 * (k0 + u));
                v[u] = (Real)d.x;
                v[u + 1] = (Real)d.y;
            }
        }
        if (W.weighted) {
            const float4 a = *reinterpret_cast<const float4*>(sp + L.off_w + 4 * k0);
            const float4 b = *reinterpret_cast<const float4*>(sp + L.off_w + 4 * k0 + 16);
            v[0] *= (Real)a.x; v[1] *= (Real)a.y; v[2] *= (Real)a.z; v[3] *= (Real)a.w;
            v[4] *= (Real)b.x; v[5] *= (Real)b.y; v[6] *= (Real)b.z; v[7] *= (Real)b.w;
        }
        const uint2 mk = *reinterpret_cast<const uint2*>(mark + k0);
        Real acc = Real(0), head_part = Real(0);
        int first = -1;
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            const int k = k0 + u;
            if (k >= lo && k < hi) acc += v[u];
            const uint32_t m = ((u < 4 ? mk.x : mk.y) >> (8 * (u & 3))) & 1u;
            if (m) {
                if (first < 0) {
                    first = u;
                    head_part = acc;
                } else {
                    rsum[k] = acc;
                }
                acc = Real(0);
            }
        }
        // 3. segmented scan over the group: (open sum, has a row end)
        Real sa = acc;
        int fa = first >= 0 ? 1 : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Real us = __shfl_up_sync(kFull, sa, o);
            const int uf = __shfl_up_sync(kFull, fa, o);
            if (lane >= o) {
                if (!fa) sa += us;
                fa |= uf;
            }
        }
        Real ex = __shfl_up_sync(kFull, sa, 1);
        int exf = __shfl_up_sync(kFull, fa, 1);
        if (lane == 0) {
            ex = Real(0);
            exf = 0;
        }
        if (lane == 31) {
            scan_store<Real>(S, g, w, sa);
            S.scan_flag[g][w] = fa;
        }
        group_sync(bar_id);
        Real cw = Real(0);
        if (!exf) {
            for (int w2 = w - 1; w2 >= 0; --w2) {
                cw += scan_load<Real>(S, g, w2);
                if (S.scan_flag[g][w2]) break;
            }
        }
        Real tail_val = Real(0);  // the row still open at the end of the stage
        if (t == 0) {
            for (int w2 = kGroupWarps - 1; w2 >= 0; --w2) {
                tail_val += scan_load<Real>(S, g, w2);
                if (S.scan_flag[g][w2]) break;
            }
        }
        if (first >= 0) rsum[k0 + first] = (exf ? ex : cw + ex) + head_part;
        group_sync(bar_id);
        // 4. finish the rows of the stage (not its head row begun in an earlier
        //    stage, nor its tail row that continues)
        const int32_t flags = in.ck.flags;
        const int j_lo = (flags & kHasHead) ? 1 : 0;
        const int j_hi = nr - ((flags & kHasTail) ? 1 : 0);
        const float* xin_s = reinterpret_cast<const float*>(sp + L.off_xin) + ro;
        const float* sc_s = reinterpret_cast<const float*>(sp + L.off_scale) + ro;
        const int32_t* hs_s = reinterpret_cast<const int32_t*>(sp + L.off_hslot) + ro;
        double err = 0.0, dsum = 0.0, xsum = 0.0;
        for (int j = j_lo + t; j < j_hi; j += kGroupThreads) {
            const int32_t rs = rowp[j], re = rowp[j + 1];
            const Real sum = re > rs ? rsum[re - 1 - eb] : Real(0);
            finish_row<kFinal>(W, ra + j, (double)sum, xin_s[j], kFinal ? 0.f : sc_s[j], kFinal ? -1 : hs_s[j], err,
                               dsum, xsum);
        }
        Real head_val = Real(0);
        if (t == 0 && (flags & kHasHead) && !(flags & kInterior)) head_val = rsum[rowp[1] - 1 - eb];
        *reinterpret_cast<uint2*>(mark + k0) = make_uint2(0u, 0u);
        err = warp_sum(err);
        dsum = warp_sum(dsum);
        xsum = warp_sum(xsum);
        if (lane == 0) {
            S.red[g][w][0] = err;
            S.red[g][w][1] = dsum;
            S.red[g][w][2] = xsum;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.bar_empty[slot]);
        group_sync(bar_id);
        if (w == 0) {
            double e = 0.0, d = 0.0, x = 0.0;
            if (lane < kGroupWarps) {
                e = S.red[g][lane][0];
                d = S.red[g][lane][1];
                x = S.red[g][lane][2];
            }
            e = warp_sum(e);
            d = warp_sum(d);
            x = warp_sum(x);
            if (lane == 0)
                stage_accumulate(P, in.c, in.ck, 2 * (int32_t)blockIdx.x + g, e, d, x, (double)head_val,
                                 (double)tail_val);
        }
    }
}

template <typename Real>
__global__ void __launch_bounds__(kCtaThreads, 1) k_sweep(SweepParams P) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(16) CtaShared S;
    float* hub_smem = reinterpret_cast<float*>(smem);
    unsigned char* stages = smem + P.lay.hub_bytes;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        S.abort_flag = 0;
        S.idle = (!kFinal && ldcg(&P.ctl->active) <= 0) ? 1 : 0;  // one reading for the whole CTA
        for (int i = 0; i < P.lay.slots; ++i) {
            mbar_init(&S.bar_full[i], 1);
            mbar_init(&S.bar_gath[i], kGatherThreads);
            mbar_init(&S.bar_empty[i], kGroupWarps);
        }
        mbar_init(&S.bar_hub, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < min(P.ngraphs, kSmemGraphs); i += kCtaThreads) {
        S.giter[i] = ldcg(&P.states[i].iter);
        S.gdone[i] = ldcg(&P.states[i].done);
    }
    for (int i = threadIdx.x; i < P.lay.slots * (kStageEntries / 16); i += kCtaThreads) {
        const int slot = i / (kStageEntries / 16), piece = i % (kStageEntries / 16);
        *reinterpret_cast<uint4*>(stages + (size_t)slot * P.lay.slot_bytes + P.lay.off_mark + 16 * piece) =
            make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    if (!S.idle) {
        if (warp == 0) run_producer<kFinal>(P, S, stages, hub_smem);
        else if (warp <= kGatherWarps) run_gatherer<kFinal>(P, S, stages, hub_smem);
        else run_consumer<Real>(P, S, stages);
    }
    __threadfence();  // this CTA's accumulator updates before its exit is counted
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        S.last = prev == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!S.last) return;
    // Last CTA out: every stage of this launch is done.
    __threadfence();
    launch_tail<kFinal>(P);
    if (threadIdx.x == 0) {
        P.ctl->queue = 0u;
        P.ctl->exited = 0u;
        if (!kFinal) {
            const int32_t launches = P.ctl->launches + 1;
            P.ctl->launches = launches;
            const int32_t active = ldcg(&P.ctl->active);
            const bool more = active > 0 && launches < P.ctl->cap && P.ctl->error == 0;
            if (active > 0 && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
            if (P.use_cond) cudaGraphSetConditional(P.cond, more ? 1u : 0u);
        }
        __threadfence();
    }
}

// ---- per-solve set-up and finishing kernels --------------------------------

// scale = alpha / outw (FP32), -1 marks a dangling vertex (outw <= 1e-15,
// pagerank.py:118); x0 = 1/n; z0 = x0 * scale; hub copy of z0.
__global__ void k_init_vertices(const GraphDev* graphs, int32_t count, double alpha) {
    const int32_t gi = blockIdx.y;
    if (gi >= count) return;
    const GraphDev G = graphs[gi];
    const float x0 = (float)(1.0 / (double)G.n);
    float* scale = const_cast<float*>(G.scale);
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < G.n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const double o = G.outw[v];
        const float sc = o <= 1e-15 ? -1.f : (float)(alpha / o);
        scale[v] = sc;
        G.x[0][v] = x0;
        const float z = sc >= 0.f ? x0 * sc : 0.f;
        G.z[0][v] = z;
        const int32_t hs = G.hub_slot[v];
        if (hs >= 0) G.hubz[0][hs] = z;
    }
}

__global__ void k_init_states(GraphState* states, const GraphDev* graphs, const int32_t* ndang,
                              int32_t count, double alpha, double tol, int32_t max_iter,
                              int32_t personalised) {
    const int32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= count) return;
    const int32_t n = graphs[gi].n;
    const double x0 = (double)(float)(1.0 / (double)n);
    GraphState s;
    s.alpha = alpha;
    s.c1 = (1.0 - alpha) / (double)n;
    s.tol_n = tol * (double)n;
    s.dsum = (double)ndang[gi] * x0;
    s.dmass = alpha * s.dsum / (double)n;
    s.dmass_prev = s.dmass;
    s.residual = 0.0;
    s.residual64 = 0.0;
    s.xsum = 0.0;
    s.iter = 0;
    s.max_iter = max_iter;
    s.done = 0;
    s.converged = 0;
    s.arrive = 0u;
    s.personalised = personalised;
    states[gi] = s;
}

__global__ void k_init_ctl(Ctl* ctl, int32_t active, int32_t cap) {
    Ctl c;
    c.queue = 0u;
    c.exited = 0u;
    c.active = active;
    c.launches = 0;
    c.cap = cap;
    c.error = 0;
    *ctl = c;
}

// FP64 carried values of x_{k-1} for the correction sweep.
__global__ void k_prep_z64(const GraphDev* graphs, const GraphState* states, int32_t count) {
    const int32_t gi = blockIdx.y;
    if (gi >= count) return;
    const GraphDev G = graphs[gi];
    const GraphState* st = states + gi;
    const float* xp = G.x[(st->iter - 1) & 1];
    const double alpha = st->alpha;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < G.n;
         u += (int64_t)gridDim.x * blockDim.x) {
        const double o = G.outw[u];
        G.z64[u] = o <= 1e-15 ? 0.0 : alpha * (double)xp[u] / o;
    }
}

// Final normalisation (pagerank.py:134-139).  from_fp32: ranks come from the
// last FP32 sweep; otherwise the correction sweep wrote G.out already.
__global__ void k_normalize(const GraphDev* graphs, const GraphState* states, int32_t count,
                            int32_t from_fp32) {
    const int32_t gi = blockIdx.y;
    if (gi >= count) return;
    const GraphDev G = graphs[gi];
    const GraphState* st = states + gi;
    const double norm = st->xsum;
    const float* xl = G.x[st->iter & 1];
    const double inv = norm > 0.0 ? 1.0 / norm : 0.0;
    const double uni = 1.0 / (double)G.n;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < G.n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const double val = from_fp32 ? (double)xl[v] : G.out[v];
        G.out[v] = norm > 0.0 ? val * inv : uni;
    }
}

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

int env_int(const char* name, int dflt, int lo, int hi) {
    const char* e = std::getenv(name);
    if (!e) return dflt;
    const int x = std::atoi(e);
    return x >= lo && x <= hi ? x : dflt;
}

// Dynamic shared memory a sweep launch may use on the current device (and the
// kernel's opt-in to it).
int smem_budget(int mode) {
    static int cache[2][64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int& c = cache[mode ? 1 : 0][dev];
    if (c > 0) return c;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa = {};
    if (mode == 0) cudaFuncGetAttributes(&fa, k_sweep<float>);
    else cudaFuncGetAttributes(&fa, k_sweep<double>);
    cudaGetLastError();
    if (optin <= 0) optin = 232448;
    const int b = optin - (int)fa.sharedSizeBytes - 1024;
    if (mode == 0) cudaFuncSetAttribute(k_sweep<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    else cudaFuncSetAttribute(k_sweep<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaGetLastError();
    c = b;
    return c;
}

// Stage buffer layout and ring depth.  FP32 sweeps of one graph stage up to
// kHubCap hub values; the ring keeps EGPR_SLOTS buffers (default 4) and the hub
// copy takes what is left.
StageLayout make_layout(int mode, bool weighted, int32_t nhub) {
    StageLayout L = {};
    int off = 0;
    auto take = [&](int bytes) {
        const int o = off;
        off += (bytes + 127) & ~127;
        return o;
    };
    L.off_col = take(kStageEntries * 4);
    L.off_val64 = mode ? take(kStageEntries * 8) : 0;
    L.off_w = weighted ? take(kStageEntries * 4) : 0;
    L.off_mark = take(kStageEntries);
    L.off_rowptr = take(kStageRows * 4);
    L.off_xin = take(kStageRows * 4);
    L.off_scale = mode ? 0 : take(kStageRows * 4);
    L.off_hslot = mode ? 0 : take(kStageRows * 4);
    L.slot_bytes = off;
    const int budget = smem_budget(mode);
    // A gatherer signals stage q only after issuing stage q + kGatherLag, so the
    // ring holds at least kGatherLag + 1 buffers.
    const int min_slots = kGatherLag + 1;
    const int max_slots = std::max(min_slots, std::min(kMaxSlots, budget / L.slot_bytes));
    L.slots = std::max(min_slots, std::min(max_slots, env_int("EGPR_SLOTS", mode == 0 && nhub > 0 ? 4 : max_slots,
                                                                 2, kMaxSlots)));
    int32_t hubs = 0;
    if (mode == 0 && nhub > 0) {
        const int left = budget - L.slots * L.slot_bytes;
        hubs = std::min<int32_t>(nhub, std::max(0, left) / 4) & ~31;
        hubs = std::min<int32_t>(hubs, env_int("EGPR_HUB_SMEM", kHubCap, 0, kHubCap) & ~31);
    }
    L.hub_count = hubs;
    L.hub_bytes = (hubs * 4 + 127) & ~127;
    L.dyn_bytes = L.hub_bytes + L.slots * L.slot_bytes;
    return L;
}

SweepParams make_params(Plan& plan, int mode, int use_cond) {
    SweepParams P;
    P.chunks = plan.d_chunks.as<Chunk>();
    P.nchunks = plan.nchunks;
    P.mode = mode;
    P.graphs = plan.d_graphs.as<GraphDev>();
    P.states = plan.d_states.as<GraphState>();
    P.acc = plan.d_acc.as<unsigned long long>();
    P.span_acc = plan.d_span_acc.as<unsigned long long>();
    P.acc_sub = plan.nacc / std::max(1, plan.ngraphs);
    P.span_list = plan.d_span_list.as<int32_t>();
    P.nspans = plan.nspans;
    P.ctl = plan.d_ctl.as<Ctl>();
    P.cond = plan.cond;
    P.use_cond = use_cond;
    P.ngraphs = plan.ngraphs;
    P.lay = make_layout(mode, plan.any_weighted != 0, plan.ngraphs == 1 ? plan.hub_count : 0);
    return P;
}

int vertex_grid(int32_t max_n) {
    int64_t b = ((int64_t)max_n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

// Loop mechanism: a CUDA-graph while node (default) or plain launches
// (EGPR_GRAPH_LOOP=0; profilers cannot capture kernels of conditional graphs).
bool graph_loop_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("EGPR_GRAPH_LOOP");
        return !(v && (v[0] == '0' || v[0] == 'n' || v[0] == 'N' || v[0] == 'f' || v[0] == 'F'));
    }();
    return on;
}

cudaLaunchAttributeValue l2_window(const Plan& plan) {
    cudaLaunchAttributeValue v = {};
    v.accessPolicyWindow.base_ptr = plan.l2_base;
    v.accessPolicyWindow.num_bytes = plan.l2_bytes;
    v.accessPolicyWindow.hitRatio = plan.l2_hit_ratio;
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    return v;
}

}  // namespace

// One persistent CTA per SM.
int sweep_grid() {
    static int cache[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cache[dev] > 0) return cache[dev];
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    cache[dev] = std::max(1, sms);
    return cache[dev];
}

// The FP32 carried values z (both buffers, contiguous) are gathered once per
// inbound entry every sweep.  While they fit, a persisting L2 access-policy
// window keeps them resident against the streamed CSR (EGPR_L2_WINDOW=0
// disables it).  The persisting carve-out is a limit of this process's CUDA
// context and ends with it.
void plan_set_l2_window(Plan& plan, void* base, size_t bytes) {
    plan.l2_base = nullptr;
    plan.l2_bytes = 0;
    plan.l2_hit_ratio = 0.f;
    const char* env = std::getenv("EGPR_L2_WINDOW");
    if (env && env[0] == '0') return;
    int dev = 0, max_persist = 0, max_window = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
    cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev);
    if (max_persist <= 0 || max_window <= 0 || !base || bytes == 0) return;
    size_t limit = 0;
    cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize);
    if (limit < (size_t)max_persist &&
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    const size_t win = std::min(bytes, (size_t)max_window);
    plan.l2_base = base;
    plan.l2_bytes = win;
    plan.l2_hit_ratio = (float)std::min(1.0, (double)max_persist / (double)win);
}

GraphDev graph_dev_view(const egpr_graph* g) {
    GraphDev d;
    d.in_row = g->in_row.as<int32_t>();
    d.in_col = g->in_col.as<int32_t>();
    d.in_w = g->weighted ? g->in_w.as<float>() : nullptr;
    d.outw = g->outw.as<double>();
    d.scale = g->scale.as<float>();
    d.tele = g->tele.as<float>();
    d.x[0] = g->x0.as<float>();
    d.x[1] = g->x1.as<float>();
    d.z[0] = g->z0.as<float>();
    d.z[1] = g->z0.as<float>() + g->n;  // one allocation: both buffers under one L2 window
    d.out = g->out.as<double>();
    d.z64 = g->z64.as<double>();
    d.hub_ids = g->hub_ids.as<int32_t>();
    d.hub_slot = g->hub_slot.as<int32_t>();
    d.hubz[0] = g->hubz.as<float>();
    d.hubz[1] = g->hubz.as<float>() + std::max(g->nhub, 4);
    d.nhub = g->nhub;
    d.n = g->n;
    d.chunk_begin = d.chunk_end = 0;
    d.span_begin = d.span_end = 0;
    return d;
}

int plan_build(Plan& plan, egpr_graph* const* graphs, int32_t count, cudaStream_t stream) {
    plan.release();
    std::vector<Chunk> all;
    std::vector<int32_t> spans;
    std::vector<GraphDev> views((size_t)count);
    std::vector<int32_t> ndang((size_t)count);
    int32_t max_n = 0, any_w = 0;
    for (int32_t gi = 0; gi < count; ++gi) {
        const egpr_graph* g = graphs[gi];
        const int32_t off = (int32_t)all.size();
        GraphDev v = graph_dev_view(g);
        v.chunk_begin = off;
        v.span_begin = (int32_t)spans.size();
        for (const Chunk& c0 : g->plan.h_chunks) {
            Chunk c = c0;
            c.graph = gi;
            if (c.head_ta >= 0) c.head_ta += off;
            if (c.tail_tb >= 0) c.tail_tb += off;
            all.push_back(c);
        }
        for (int32_t sp : g->plan.h_spans) spans.push_back(sp + off);
        v.chunk_end = (int32_t)all.size();
        v.span_end = (int32_t)spans.size();
        views[(size_t)gi] = v;
        ndang[(size_t)gi] = g->n_dangling_solve;
        max_n = std::max(max_n, g->n);
        if (g->weighted) any_w = 1;
    }
    plan.ngraphs = count;
    plan.nchunks = (int32_t)all.size();
    plan.nspans = (int32_t)spans.size();
    plan.max_n = max_n;
    plan.any_weighted = any_w;
    plan.hub_count = count == 1 ? graphs[0]->nhub : 0;
    plan.grid = std::max(1, std::min(plan.nchunks, sweep_grid()));
    // accumulator slots: up to one per (CTA, consumer group) for each graph
    const int32_t per_graph = std::max(1, std::min(2 * plan.grid, 8192 / std::max(1, count)));
    plan.nacc = per_graph * count;
    plan.h_chunks_all = all;
    if (spans.empty()) spans.push_back(0);
    int rc;
    if ((rc = plan.d_chunks.alloc(all.size() * sizeof(Chunk))) ||
        (rc = plan.d_graphs.alloc(views.size() * sizeof(GraphDev))) ||
        (rc = plan.d_states.alloc((size_t)count * sizeof(GraphState))) ||
        (rc = plan.d_ndang.alloc((size_t)count * sizeof(int32_t))) ||
        (rc = plan.d_acc.alloc((size_t)plan.nacc * kAccWords * sizeof(unsigned long long))) ||
        (rc = plan.d_span_acc.alloc(all.size() * 2 * sizeof(unsigned long long))) ||
        (rc = plan.d_span_list.alloc(spans.size() * sizeof(int32_t))) || (rc = plan.d_ctl.alloc(sizeof(Ctl))))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(plan.d_chunks.p, all.data(), all.size() * sizeof(Chunk), cudaMemcpyHostToDevice, stream), "H2D chunks")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_graphs.p, views.data(), views.size() * sizeof(GraphDev), cudaMemcpyHostToDevice, stream), "H2D graph table")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_ndang.p, ndang.data(), ndang.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream), "H2D counts")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_span_list.p, spans.data(), spans.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream), "H2D spans")) ||
        (rc = cuda_ok(cudaStreamSynchronize(stream), "plan upload")))
        return rc;
    return EGPR_SUCC;
}

int plan_capture_loop(Plan& plan, cudaStream_t stream) {
    (void)stream;
    if (plan.cg_exec) return EGPR_SUCC;
    if (plan.cg_failed) return EGPR_DEVICE_ERR;
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t ex = nullptr;
    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t cnode = nullptr, knode = nullptr;
    cudaGraphNodeParams cp = {};
    cudaKernelNodeParams kp = {};
    SweepParams P;
    void* args[1];
    cudaError_t e = cudaGraphCreate(&cg, 0);
    if (e != cudaSuccess) goto fail;
    e = cudaGraphConditionalHandleCreate(&h, cg, 1u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) goto fail;
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&cnode, cg, nullptr, 0, &cp);
    if (e != cudaSuccess) goto fail;
    plan.cond = h;
    P = make_params(plan, 0, 1);
    args[0] = &P;
    kp.func = (void*)k_sweep<float>;
    kp.gridDim = dim3((unsigned)plan.grid);
    kp.blockDim = dim3(kCtaThreads);
    kp.sharedMemBytes = (unsigned)P.lay.dyn_bytes;
    kp.kernelParams = args;
    e = cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp);
    if (e != cudaSuccess) goto fail;
    if (plan.l2_bytes > 0) {
        cudaLaunchAttributeValue v = l2_window(plan);
        if (cudaGraphKernelNodeSetAttribute(knode, cudaLaunchAttributeAccessPolicyWindow, &v) != cudaSuccess)
            cudaGetLastError();  // the window is a hint; run without it
    }
    e = cudaGraphInstantiate(&ex, cg, 0);
    if (e != cudaSuccess) goto fail;
    plan.cg = cg;
    plan.cg_exec = ex;
    return EGPR_SUCC;
fail:
    cudaGetLastError();
    if (cg) cudaGraphDestroy(cg);
    plan.cond = 0;
    plan.cg_failed = true;
    return EGPR_DEVICE_ERR;
}

int launch_init(Plan& plan, double alpha, int32_t max_iter, double tol, bool personalised,
                cudaStream_t stream) {
    dim3 grid((unsigned)vertex_grid(plan.max_n), (unsigned)plan.ngraphs);
    k_init_vertices<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.ngraphs, alpha);
    k_init_states<<<(plan.ngraphs + 127) / 128, 128, 0, stream>>>(plan.d_states.as<GraphState>(),
                                                                 plan.d_graphs.as<GraphDev>(),
                                                                 plan.d_ndang.as<int32_t>(), plan.ngraphs,
                                                                 alpha, tol, max_iter, personalised ? 1 : 0);
    k_init_ctl<<<1, 1, 0, stream>>>(plan.d_ctl.as<Ctl>(), plan.ngraphs, max_iter + 1);
    cudaMemsetAsync(plan.d_acc.p, 0, plan.d_acc.bytes, stream);
    cudaMemsetAsync(plan.d_span_acc.p, 0, plan.d_span_acc.bytes, stream);
    return cuda_ok(cudaGetLastError(), "init launch");
}

int launch_loop(Plan& plan, int32_t max_iter, cudaStream_t stream, int32_t* launches) {
    *launches = 0;
    if (graph_loop_enabled() && plan_capture_loop(plan, stream) == EGPR_SUCC) {
        int rc = cuda_ok(cudaGraphLaunch(plan.cg_exec, stream), "graph launch");
        *launches = -1;  // counted on the device (Ctl::launches)
        return rc;
    }
    // Plain launches; a sweep with no active graph returns at once.
    SweepParams P = make_params(plan, 0, 0);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)plan.grid);
    cfg.blockDim = dim3(kCtaThreads);
    cfg.dynamicSmemBytes = (size_t)P.lay.dyn_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    if (plan.l2_bytes > 0) {
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[0].val = l2_window(plan);
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    for (int32_t it = 0; it < max_iter; ++it) {
        cudaError_t e = cudaLaunchKernelEx(&cfg, k_sweep<float>, P);
        if (e != cudaSuccess) return cuda_ok(e, "sweep launch");
    }
    *launches = -1;
    return cuda_ok(cudaGetLastError(), "sweep launch");
}

int launch_finish(Plan& plan, bool correction, cudaStream_t stream, int32_t* launches) {
    dim3 grid((unsigned)vertex_grid(plan.max_n), (unsigned)plan.ngraphs);
    int32_t l = 0;
    if (correction) {
        k_prep_z64<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                                  plan.ngraphs);
        // The loop's last CTA left the queue reset; the control block keeps the sweep count.
        SweepParams P = make_params(plan, 1, 0);
        k_sweep<double><<<plan.grid, kCtaThreads, (size_t)P.lay.dyn_bytes, stream>>>(P);
        l += 2;
    }
    k_normalize<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                               plan.ngraphs, correction ? 0 : 1);
    l += 1;
    *launches = l;
    return cuda_ok(cudaGetLastError(), "finish launch");
}

}  // namespace egpr
