// The binned single-graph sweep: one power-iteration sweep per launch over
// the renumbered inbound CSR built by build_bin_layout (prep.cu).
//
// Per row v (a destination), as in the tile sweep (sweep.cu) and the
// reference's power iteration (easygraph/functions/centrality/pagerank.py:
// 112-132) evaluated as a pull:
//     x_new[v] = sum_{u -> v} w_uv * z[u] + jump,   z[u] = alpha * x[u] / outw[u]
// plus, in the same launch, the FP64 L1 residual, the FP64 dangling mass and
// rank sum, z_new, and the stop decision err < tol * n, which drives the CUDA
// graph's while node.  This replaces the reference GPU path's cuSPARSE SpMV,
// cuBLAS Sdot, add_base_and_reduce, scale_vec and two host round trips per
// sweep (gpu_easygraph/functions/centrality/pagerank.cu:591-664).
//
// Work split (the layout sorts rows by length inside two blocks, so each
// class is a contiguous row range):
//   * pieces of long rows, one warp each, eight gathers in flight per lane;
//     a row cut into several pieces is finished by the last piece to arrive
//     (pieces add exact fixed-point sums: the order does not matter);
//   * groups of rows of one length class, G lanes per row (G = 1..32, a power
//     of two, four to eight entries per lane), four gathers in flight per lane;
//   * rows without inbound entries (teleport and dangling terms only).
// Items of all three kinds are interleaved in one queue, so that warps bound
// by gather throughput and warps bound by latency share the SMs.  Carried
// values of the hub block (the sources of largest out-degree, renumbered to
// [0, hubs)) are staged into shared memory once per launch by a TMA bulk
// copy; a gather of source s < hubs reads shared memory, any other source
// reads z from L2/HBM.
//
// Sums.  Every lane keeps FP64 sums of the residual, the dangling mass and the
// rank sum over the rows it finishes in an item; at the end of the item the
// warp adds them in a fixed order and turns them into fixed-point integers
// (units of 2^-32 and 2^-64), added with integer atomics.  The totals are
// therefore exact sums of per-item values and independent of which warp ran
// which item: results are bit-identical from run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "egpr_internal.cuh"

namespace egpr {

BinLayout::~BinLayout() {
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg) cudaGraphDestroy(cg);
    for (DevBuf* b : {&perm, &inv, &row, &col, &w, &outw, &items, &scale, &tele, &x, &z, &z64, &out64, &states, &ctl,
                      &acc, &span_acc, &span_cnt})
        b->release();
}

namespace {

constexpr int kBinWarps = 32;  // warps per CTA, one CTA per SM
constexpr int kBinCta = 32 * kBinWarps;
constexpr unsigned kAllLanes = 0xffffffffu;
constexpr uint32_t kBinCopyPiece = 32768;                 // bytes per hub staging copy
constexpr unsigned long long kBinWaitNs = 2000000000ull;  // bound of the staging wait (2 s)
constexpr int32_t kEmptyRowsPerItem = 1024;
constexpr int kHubPad = 4;  // floats of zero in front of the staged hub values

struct BinParams {
    const BinItem* items;
    int32_t nitems;
    int32_t n;
    int32_t hubs;         // hub values staged in shared memory ([0, hubs)); 0: every gather reads global memory
    const int32_t* row;
    const int32_t* col;
    const float* w;       // NULL: unit weights
    const float* scale;   // alpha / outw (FP32), -1 for a dangling vertex
    const float* tele;    // personalisation (renumbered)
    float* x[2];          // ranks, double-buffered
    float* z[2];          // carried values, double-buffered
    const double* z64;    // FP64 sweep: carried values of x_{k-1}
    double* out64;        // FP64 sweep: its result (renumbered, unnormalised)
    GraphState* st;
    Ctl* ctl;
    unsigned long long* acc;  // kAccWords words per slot
    int32_t acc_slots;
    unsigned long long* span_acc;  // 2 words per span
    uint32_t* span_cnt;
    cudaGraphConditionalHandle cond;
    int32_t use_cond;
};

// ---- PTX wrappers -----------------------------------------------------------
__device__ __forceinline__ uint32_t bsmem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bmbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bsmem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void bmbar_arrive_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bsmem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bmbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(bsmem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bbulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     bsmem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(bsmem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ unsigned long long bglobal_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- order-free FP64 sums (two's-complement fixed point, 2^-32 and 2^-64) ----
__device__ __forceinline__ void bfx_add(unsigned long long* a, double v) {
    const double t = v * 4294967296.0;  // exact
    const double f = floor(t);
    atomicAdd(a, (unsigned long long)(long long)f);
    atomicAdd(a + 1, (unsigned long long)rint((t - f) * 4294967296.0));
}
__device__ __forceinline__ double bfx_join(unsigned long long hi, unsigned long long lo) {
    return (double)(long long)hi * (1.0 / 4294967296.0) + (double)lo * (1.0 / 18446744073709551616.0);
}

// What every lane needs of the solve's state in this launch.
struct BinView {
    const float* xin;    // previous ranks (FP64 sweep: x_{k-1})
    float* xout;
    float* zout;
    const float* zin;    // carried values gathered by this sweep
    double jump;         // (1-alpha)/n + dangling term (uniform teleport)
    double dmass;        // dangling term alone (personalised teleport)
    double oma;          // 1 - alpha
    int32_t personalised;
};

struct LaneAcc {
    double err = 0.0, dsum = 0.0, xsum = 0.0;
};

// Finishes row r given its gathered sum.
template <bool kFinal>
__device__ __forceinline__ void bin_finish(const BinParams& P, const BinView& V, int32_t r, double sum, float xin,
                                           float sc, LaneAcc& A) {
    const double val = V.personalised ? (sum + V.oma * (double)__ldg(P.tele + r)) + V.dmass : sum + V.jump;
    if (!kFinal) {
        const float xo = (float)val;
        A.err += fabs((double)xo - (double)xin);
        V.xout[r] = xo;
        V.zout[r] = sc >= 0.f ? xo * sc : 0.f;
        if (sc < 0.f) A.dsum += (double)xo;
        A.xsum += (double)xo;
    } else {
        A.err += fabs(val - (double)xin);
        P.out64[r] = val;
        A.xsum += val;
    }
}

template <typename Real>
__device__ __forceinline__ Real bin_gather(const BinParams& P, const BinView& V, const float* hub, int32_t s) {
    if constexpr (std::is_same<Real, double>::value) {
        return __ldg(P.z64 + s);
    } else {
        return s < P.hubs ? hub[s] : __ldg(V.zin + s);
    }
}

template <typename Real>
__device__ __forceinline__ Real bin_entry(const BinParams& P, const BinView& V, const float* hub, int32_t p) {
    const Real g = bin_gather<Real>(P, V, hub, __ldg(P.col + p));
    return P.w ? g * (Real)__ldg(P.w + p) : g;
}

// The warp's FP64 lane sums of an item, added to its accumulator slot.
__device__ __forceinline__ void bin_flush(const BinParams& P, LaneAcc& A) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        A.err += __shfl_xor_sync(kAllLanes, A.err, o);
        A.dsum += __shfl_xor_sync(kAllLanes, A.dsum, o);
        A.xsum += __shfl_xor_sync(kAllLanes, A.xsum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        const int32_t slot = (int32_t)((blockIdx.x * kBinWarps + (threadIdx.x >> 5)) % (uint32_t)P.acc_slots);
        unsigned long long* a = P.acc + (size_t)kAccWords * (size_t)slot;
        if (A.err != 0.0) bfx_add(a, A.err);
        if (A.dsum != 0.0) bfx_add(a + 2, A.dsum);
        if (A.xsum != 0.0) bfx_add(a + 4, A.xsum);
    }
    A = LaneAcc();
}

// A piece of a long row: one warp, eight gathers in flight per lane.
template <typename Real>
__device__ void bin_piece(const BinParams& P, const BinView& V, const float* hub, const BinItem& it, LaneAcc& A) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31;
    Real acc = Real(0);
    for (int32_t p = it.e0 + lane; p < it.e1; p += 8 * 32) {
        Real v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int32_t q = p + 32 * u;
            v[u] = q < it.e1 ? bin_entry<Real>(P, V, hub, q) : Real(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += v[u];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kAllLanes, acc, o);
    if (lane != 0) return;
    const int32_t r = it.r0;
    double sum = (double)acc;
    if (it.span >= 0) {
        unsigned long long* sa = P.span_acc + 2 * (size_t)it.span;
        bfx_add(sa, sum);
        __threadfence();
        const uint32_t prev = atomicAdd(P.span_cnt + it.span, 1u);
        if (prev != (uint32_t)(it.parts - 1)) return;  // another piece finishes the row
        __threadfence();
        sum = bfx_join(__ldcg(sa), __ldcg(sa + 1));
        sa[0] = 0ull;
        sa[1] = 0ull;
        P.span_cnt[it.span] = 0u;
    }
    bin_finish<kFinal>(P, V, r, sum, V.xin[r], kFinal ? 0.f : __ldg(P.scale + r), A);
}

// Rows [r0, r1) of one length class, G lanes per row.
template <typename Real>
__device__ void bin_group(const BinParams& P, const BinView& V, const float* hub, const BinItem& it, LaneAcc& A) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31;
    const int G = it.parts;  // 1, 2, 4, 8, 16 or 32
    const int lg = 31 - __clz(G);
    const int sub = lane & (G - 1), grp = lane >> lg, groups = 32 >> lg;
    for (int32_t rb = it.r0; rb < it.r1; rb += groups) {
        const int32_t r = rb + grp;
        const bool valid = r < it.r1;
        int32_t b = 0, e = 0;
        float xin = 0.f, sc = 0.f;
        if (valid) {
            b = __ldg(P.row + r);
            e = __ldg(P.row + r + 1);
            if (sub == 0) {
                xin = V.xin[r];
                if (!kFinal) sc = __ldg(P.scale + r);
            }
        }
        Real acc = Real(0);
        for (int32_t p = b + sub; p < e; p += 4 * G) {
            Real v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int32_t q = p + G * u;
                v[u] = q < e ? bin_entry<Real>(P, V, hub, q) : Real(0);
            }
            acc += (v[0] + v[1]) + (v[2] + v[3]);
        }
        for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(kAllLanes, acc, o);
        if (valid && sub == 0) bin_finish<kFinal>(P, V, r, (double)acc, xin, sc, A);
    }
}

// Rows [r0, r1) without inbound entries.
template <typename Real>
__device__ void bin_empty(const BinParams& P, const BinView& V, const BinItem& it, LaneAcc& A) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    for (int32_t r = it.r0 + (int32_t)(threadIdx.x & 31); r < it.r1; r += 32)
        bin_finish<kFinal>(P, V, r, 0.0, V.xin[r], kFinal ? 0.f : __ldg(P.scale + r), A);
}

__device__ __forceinline__ BinItem load_item(const BinItem* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    const int4 a = __ldg(q), b = __ldg(q + 1);
    BinItem it;
    it.kind = a.x;
    it.r0 = a.y;
    it.r1 = a.z;
    it.e0 = a.w;
    it.e1 = b.x;
    it.span = b.y;
    it.parts = b.z;
    it.pad = b.w;
    return it;
}

// End of a launch, run by the last CTA to leave the queue: the accumulators
// become the residual, dangling mass and rank sum (pagerank.py:117-131).
template <bool kFinal>
__device__ void bin_tail(const BinParams& P) {
    const int lane = threadIdx.x & 31;
    __threadfence();
    if (threadIdx.x < 32) {
        unsigned long long wsum[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
        for (int32_t k = lane; k < P.acc_slots; k += 32) {
            unsigned long long* a = P.acc + (size_t)kAccWords * (size_t)k;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                wsum[i] += __ldcg(a + i);
                a[i] = 0ull;
            }
        }
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) wsum[i] += __shfl_down_sync(kAllLanes, wsum[i], o);
        if (lane == 0) {
            GraphState* st = P.st;
            const double e = bfx_join(wsum[0], wsum[1]), d = bfx_join(wsum[2], wsum[3]), x = bfx_join(wsum[4], wsum[5]);
            if (!kFinal) {
                st->residual = e;
                st->dsum = d;
                st->xsum = x;
                st->dmass_prev = st->dmass;
                st->dmass = st->alpha * d / (double)P.n;
                const int32_t itn = st->iter + 1;
                st->iter = itn;
                const bool conv = e < st->tol_n;
                if (conv || itn >= st->max_iter) {
                    st->done = 1;
                    st->converged = conv ? 1 : 0;
                    P.ctl->active = 0;
                }
                const int32_t launches = P.ctl->launches + 1;
                P.ctl->launches = launches;
                const bool more = !st->done && launches < P.ctl->cap && P.ctl->error == 0;
                if (!st->done && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
                if (P.use_cond) cudaGraphSetConditional(P.cond, more ? 1u : 0u);
            } else {
                st->residual64 = e;
                st->xsum = x;
            }
            P.ctl->queue = 0u;
            P.ctl->exited = 0u;
            __threadfence();
        }
    }
}

template <typename Real>
__global__ void __launch_bounds__(kBinCta, 1) k_bsweep(BinParams P) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    extern __shared__ __align__(128) float hub_s[];  // kHubPad zeros, then the staged hub values
    __shared__ __align__(8) uint64_t bar_hub;
    __shared__ int32_t s_idle, s_abort, s_last;
    const float* hub = hub_s + kHubPad;
    if (threadIdx.x == 0) {
        s_abort = 0;
        s_last = 0;
        s_idle = (!kFinal && __ldcg(&P.st->done)) ? 1 : 0;  // one reading for the whole CTA
        if (!s_idle && P.hubs > 0) {
            bmbar_init(&bar_hub, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            const uint32_t bytes = (uint32_t)P.hubs * (uint32_t)sizeof(float);
            const float* src = P.z[__ldcg(&P.st->iter) & 1];
            bmbar_arrive_tx(&bar_hub, bytes);
            for (uint32_t off = 0; off < bytes; off += kBinCopyPiece)
                bbulk_load(reinterpret_cast<unsigned char*>(hub_s + kHubPad) + off,
                           reinterpret_cast<const unsigned char*>(src) + off, min(kBinCopyPiece, bytes - off), &bar_hub);
        }
    }
    if (threadIdx.x < kHubPad) hub_s[threadIdx.x] = 0.f;
    __syncthreads();
    if (!s_idle && P.hubs > 0) {
        bool ok = bmbar_try(&bar_hub, 0u);
        if (!ok) {
            const unsigned long long t0 = bglobal_ns();
            while (!(ok = bmbar_try(&bar_hub, 0u)) && bglobal_ns() - t0 < kBinWaitNs) {
            }
        }
        if (!ok) atomicExch(&s_abort, 1);
        __syncthreads();
        if (s_abort && threadIdx.x == 0) {
            atomicExch(&P.ctl->error, EGPR_TIMEOUT);
            const unsigned long long t0 = bglobal_ns();  // leave no copy in flight into shared memory
            while (!bmbar_try(&bar_hub, 0u) && bglobal_ns() - t0 < kBinWaitNs) {
            }
        }
    }
    if (!s_idle && !s_abort) {
        const GraphState* st = P.st;
        const int32_t iter = __ldcg(&st->iter);
        BinView V;
        V.oma = 1.0 - st->alpha;
        V.personalised = st->personalised;
        if (!kFinal) {
            const int par = iter & 1;
            V.xin = P.x[par];
            V.xout = P.x[par ^ 1];
            V.zout = P.z[par ^ 1];
            V.zin = P.z[par];
            V.dmass = __ldcg(&st->dmass);
        } else {
            V.xin = P.x[(iter - 1) & 1];  // x_{k-1}: the input of the last sweep
            V.xout = nullptr;
            V.zout = nullptr;
            V.zin = nullptr;
            V.dmass = __ldcg(&st->dmass_prev);
        }
        V.jump = st->c1 + V.dmass;
        const int lane = threadIdx.x & 31;
        LaneAcc A;
        uint32_t claim = 0;
        if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
        int32_t c = (int32_t)__shfl_sync(kAllLanes, claim, 0);
        if (c < P.nitems) {
            if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
            BinItem it = load_item(P.items + c);
            for (;;) {
                const int32_t cn = (int32_t)__shfl_sync(kAllLanes, claim, 0);
                const bool have = cn < P.nitems;
                BinItem nx;
                if (have) {
                    nx = load_item(P.items + cn);
                    if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
                }
                if (it.kind == kBinPiece) bin_piece<Real>(P, V, hub, it, A);
                else if (it.kind == kBinGroup) bin_group<Real>(P, V, hub, it, A);
                else bin_empty<Real>(P, V, it, A);
                __syncwarp();
                bin_flush(P, A);
                if (!have) break;
                it = nx;
            }
        }
    }
    __threadfence();  // this CTA's sums before its exit is counted
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        s_last = prev == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (!kFinal && s_idle) {  // converged before this launch: nothing to add, just stop the loop
        if (threadIdx.x == 0) {
            P.ctl->queue = 0u;
            P.ctl->exited = 0u;
            if (P.use_cond) cudaGraphSetConditional(P.cond, 0u);
            __threadfence();
        }
        return;
    }
    bin_tail<kFinal>(P);
}

// ---- per-solve set-up and finishing kernels --------------------------------
// scale = alpha / outw (FP32), -1 for a dangling vertex (outw <= 1e-15,
// pagerank.py:118); x0 = 1/n; z0 = x0 * scale; the teleport renumbered.
__global__ void k_bins_init(const double* __restrict__ outw, int32_t n, double alpha, float* __restrict__ scale,
                            float* __restrict__ x0, float* __restrict__ z0) {
    const float x = (float)(1.0 / (double)n);
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const double o = outw[v];
        const float sc = o <= 1e-15 ? -1.f : (float)(alpha / o);
        scale[v] = sc;
        x0[v] = x;
        z0[v] = sc >= 0.f ? x * sc : 0.f;
    }
}

__global__ void k_bins_state(GraphState* st, Ctl* ctl, int32_t n, int32_t ndang, double alpha, double tol,
                             int32_t max_iter, int32_t personalised) {
    const double x0 = (double)(float)(1.0 / (double)n);
    GraphState s;
    s.alpha = alpha;
    s.c1 = (1.0 - alpha) / (double)n;
    s.tol_n = tol * (double)n;
    s.dsum = (double)ndang * x0;
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
    *st = s;
    Ctl c;
    c.queue = 0u;
    c.exited = 0u;
    c.active = 1;
    c.launches = 0;
    c.cap = max_iter + 1;
    c.error = 0;
    *ctl = c;
}

__global__ void k_bins_tele(const float* __restrict__ tele, const int32_t* __restrict__ inv, int32_t n,
                            float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = tele[inv[i]];
}

// FP64 carried values of x_{k-1} for the correction sweep.
__global__ void k_bins_z64(const double* __restrict__ outw, const GraphState* st, const float* x0, const float* x1,
                           int32_t n, double* __restrict__ z64) {
    const float* xp = ((st->iter - 1) & 1) ? x1 : x0;
    const double alpha = st->alpha;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const double o = outw[u];
        z64[u] = o <= 1e-15 ? 0.0 : alpha * (double)xp[u] / o;
    }
}

// Final normalisation (pagerank.py:134-139) back into the original vertex
// order: out[v] = result[perm[v]] / sum.
__global__ void k_bins_normalize(const GraphState* st, const float* x0, const float* x1,
                                 const double* __restrict__ out64, const int32_t* __restrict__ perm, int32_t n,
                                 int32_t from_fp32, double* __restrict__ out) {
    const double norm = st->xsum;
    const float* xl = (st->iter & 1) ? x1 : x0;
    const double inv = norm > 0.0 ? 1.0 / norm : 0.0;
    const double uni = 1.0 / (double)n;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = perm[v];
        const double val = from_fp32 ? (double)xl[i] : out64[i];
        out[v] = norm > 0.0 ? val * inv : uni;
    }
}

int bcuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

// Floats (doubles) per buffer of a double-buffered vector: n plus a zero tail
// of at least 16, rounded up to 32 so that the second buffer starts on a
// 128-byte boundary (the hub staging copy reads it with TMA, which needs
// 16-byte aligned sources).
size_t bin_stride(int32_t n) { return ((size_t)n + 16 + 31) & ~(size_t)31; }

int bin_grid_for(int64_t work) {
    int64_t g = (work + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 8));
}

// Dynamic shared memory of a launch: the zero pad and the staged hub values.
size_t bin_smem(int32_t hubs) { return ((size_t)kHubPad + (size_t)hubs) * sizeof(float); }

// The kernels' opt-in to the device's shared-memory limit, once per device.
int bin_smem_optin(int mode) {
    static std::atomic<int> cache[2][64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::atomic<int>& c = cache[mode ? 1 : 0][dev];
    const int have = c.load(std::memory_order_acquire);
    if (have > 0) return have;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa = {};
    if (mode == 0) cudaFuncGetAttributes(&fa, k_bsweep<float>);
    else cudaFuncGetAttributes(&fa, k_bsweep<double>);
    cudaGetLastError();
    if (optin <= 0) optin = 232448;
    const int b = optin - (int)fa.sharedSizeBytes - 1024;
    if (mode == 0) cudaFuncSetAttribute(k_bsweep<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    else cudaFuncSetAttribute(k_bsweep<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaGetLastError();
    c.store(b, std::memory_order_release);
    return b;
}

BinParams bin_params(egpr_graph* g, int mode, int use_cond) {
    BinLayout* B = g->bins;
    BinParams P;
    P.items = B->items.as<BinItem>();
    P.nitems = B->nitems;
    P.n = B->n;
    P.hubs = mode == 0 ? B->hubs : 0;
    P.row = B->row.as<int32_t>();
    P.col = B->col.as<int32_t>();
    P.w = g->weighted ? B->w.as<float>() : nullptr;
    P.scale = B->scale.as<float>();
    P.tele = B->tele.as<float>();
    const size_t stride = bin_stride(B->n);
    P.x[0] = B->x.as<float>();
    P.x[1] = B->x.as<float>() + stride;
    P.z[0] = B->z.as<float>();
    P.z[1] = B->z.as<float>() + stride;
    P.z64 = B->z64.as<double>();
    P.out64 = B->out64.as<double>();
    P.st = B->states.as<GraphState>();
    P.ctl = B->ctl.as<Ctl>();
    P.acc = B->acc.as<unsigned long long>();
    P.acc_slots = B->acc_slots;
    P.span_acc = B->span_acc.as<unsigned long long>();
    P.span_cnt = B->span_cnt.as<uint32_t>();
    P.cond = B->cond;
    P.use_cond = use_cond;
    bin_smem_optin(mode);
    return P;
}

int bins_capture_loop(egpr_graph* g) {
    BinLayout* B = g->bins;
    if (B->cg_exec) return EGPR_SUCC;
    if (B->cg_failed) return EGPR_DEVICE_ERR;
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t ex = nullptr;
    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t cnode = nullptr, knode = nullptr;
    cudaGraphNodeParams cp = {};
    cudaKernelNodeParams kp = {};
    BinParams P;
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
    B->cond = h;
    P = bin_params(g, 0, 1);
    args[0] = &P;
    kp.func = (void*)k_bsweep<float>;
    kp.gridDim = dim3((unsigned)B->grid);
    kp.blockDim = dim3(kBinCta);
    kp.sharedMemBytes = (unsigned)bin_smem(P.hubs);
    kp.kernelParams = args;
    e = cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp);
    if (e != cudaSuccess) goto fail;
    e = cudaGraphInstantiate(&ex, cg, 0);
    if (e != cudaSuccess) goto fail;
    B->cg = cg;
    B->cg_exec = ex;
    return EGPR_SUCC;
fail:
    cudaGetLastError();
    if (cg) cudaGraphDestroy(cg);
    B->cond = 0;
    B->cg_failed = true;
    return EGPR_DEVICE_ERR;
}

__global__ void k_bin_bounds(const int32_t* __restrict__ row, int32_t a, int32_t b, const int32_t* __restrict__ thr,
                             int32_t nthr, int32_t* __restrict__ out) {
    // rows [a, b) have non-increasing lengths: the first row shorter than thr[k]
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nthr) return;
    int32_t lo = a, hi = b;
    while (lo < hi) {
        const int32_t mid = lo + ((hi - lo) >> 1);
        if (row[mid + 1] - row[mid] >= thr[k]) lo = mid + 1;
        else hi = mid;
    }
    out[k] = lo;
}

// Lanes per row for rows of about `len` entries: four to eight entries per lane.
int32_t lanes_for(int64_t len) {
    int32_t G = 1;
    while (G < 32 && (int64_t)G * 8 <= len) G <<= 1;
    return G;
}

}  // namespace

// The binned layout is built only on request (EGPR_BINS=1): measured on
// B200 it runs 2.5-3x slower than the tile sweep (R-MAT scale 22: 0.64 against
// 0.22 ms per sweep; scale 25 weighted: 6.6 against 2.6 ms), latency-bound on
// the dependent loads of each row group (row offsets, then sources, then
// gathers), where the tile sweep loads a tile's sources one tile ahead.
bool bins_wanted(int32_t n, int64_t nnz) {
    const char* e = std::getenv("EGPR_BINS");
    return e && e[0] == '1' && n > 0 && nnz > 0;
}

int32_t bin_hub_cap() {
    // the kernel's shared-memory room, at most 208 KB, which leaves L1 at
    // least 48 KB of the SM's 256 KB
    const int room = std::min(bin_smem_optin(0), 208 * 1024);
    return std::max<int32_t>(0, room / (int)sizeof(float) - kHubPad) & ~3;
}

// The work queue: class boundaries from the renumbered row offsets, then
// items of every class, interleaved.
int bins_build_items(egpr_graph* g, cudaStream_t s) {
    BinLayout* B = g->bins;
    const int32_t n = B->n;
    const int32_t piece = std::max<int32_t>(256, B->piece);
    // length thresholds, descending: pieces, then G = 32, 16, 8, 4, 2, 1, then empty rows
    std::vector<int32_t> thr = {piece, 256, 128, 64, 32, 16, 8, 1};
    const int32_t nthr = (int32_t)thr.size();
    const int32_t runs[2][2] = {{0, B->hubs}, {B->hubs, n}};
    int32_t *d_thr = nullptr, *d_out = nullptr;
    int rc = bcuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&d_thr), nthr * sizeof(int32_t), s), "cudaMallocAsync");
    if (!rc) rc = bcuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&d_out), 2 * nthr * sizeof(int32_t), s), "cudaMallocAsync");
    if (!rc) rc = bcuda_ok(cudaMemcpyAsync(d_thr, thr.data(), nthr * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D");
    for (int k = 0; k < 2 && !rc; ++k)
        k_bin_bounds<<<1, 32, 0, s>>>(B->row.as<int32_t>(), runs[k][0], runs[k][1], d_thr, nthr, d_out + k * nthr);
    std::vector<int32_t> bnd(2 * (size_t)nthr);
    if (!rc) rc = bcuda_ok(cudaMemcpyAsync(bnd.data(), d_out, bnd.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                           "D2H bounds");
    if (!rc) rc = bcuda_ok(cudaStreamSynchronize(s), "bounds");
    if (d_thr) cudaFreeAsync(d_thr, s);
    if (d_out) cudaFreeAsync(d_out, s);
    if (rc) return rc;
    // row offsets of every row of the long classes and of each class boundary
    std::vector<BinItem> pieces, groups, empties;
    int32_t nspans = 0;
    for (int k = 0; k < 2; ++k) {
        const int32_t a = runs[k][0], b = runs[k][1];
        if (b <= a) continue;
        const int32_t* c = bnd.data() + k * nthr;  // c[j]: first row of the run shorter than thr[j]
        // long rows [a, c[0]): pieces
        const int32_t nlong = c[0] - a;
        std::vector<int32_t> off((size_t)nlong + 1);
        if ((rc = bcuda_ok(cudaMemcpy(off.data(), B->row.as<int32_t>() + a, off.size() * sizeof(int32_t),
                                      cudaMemcpyDeviceToHost), "D2H rows")))
            return rc;
        for (int32_t i = 0; i < nlong; ++i) {
            const int64_t len = (int64_t)off[(size_t)i + 1] - off[(size_t)i];
            const int32_t parts = (int32_t)((len + piece - 1) / piece);
            const int32_t span = parts > 1 ? nspans++ : -1;
            for (int32_t j = 0; j < parts; ++j) {
                BinItem it = {};
                it.kind = kBinPiece;
                it.r0 = a + i;
                it.r1 = a + i + 1;
                it.e0 = (int32_t)(off[(size_t)i] + len * j / parts);
                it.e1 = (int32_t)(off[(size_t)i] + len * (j + 1) / parts);
                it.span = span;
                it.parts = parts;
                pieces.push_back(it);
            }
        }
        // classes [c[j-1], c[j]) for j = 1..nthr-1 (lengths in [thr[j], thr[j-1])), then empty rows
        int32_t offs[16];
        for (int j = 0; j < nthr; ++j) {
            if ((rc = bcuda_ok(cudaMemcpy(&offs[j], B->row.as<int32_t>() + c[j], sizeof(int32_t),
                                          cudaMemcpyDeviceToHost), "D2H rows")))
                return rc;
        }
        for (int j = 1; j < nthr; ++j) {
            const int32_t r0 = c[j - 1], r1 = c[j];
            if (r1 <= r0) continue;
            const int64_t entries = (int64_t)offs[j] - offs[j - 1];
            const int64_t avg = std::max<int64_t>(1, entries / (r1 - r0));
            const int32_t G = lanes_for(avg);
            const int32_t per_pass = 32 / G;
            // about group_entries entries, and at most 8 passes of the warp over
            // its rows (each pass waits on a chain of dependent loads)
            int64_t rows = std::max<int64_t>(per_pass, (int64_t)B->group_entries / avg);
            rows = std::min<int64_t>((rows + per_pass - 1) / per_pass * per_pass, 8 * (int64_t)per_pass);
            for (int64_t r = r0; r < r1; r += rows) {
                BinItem it = {};
                it.kind = kBinGroup;
                it.r0 = (int32_t)r;
                it.r1 = (int32_t)std::min<int64_t>(r1, r + rows);
                it.span = -1;
                it.parts = G;
                groups.push_back(it);
            }
        }
        for (int64_t r = c[nthr - 1]; r < b; r += kEmptyRowsPerItem) {
            BinItem it = {};
            it.kind = kBinEmpty;
            it.r0 = (int32_t)r;
            it.r1 = (int32_t)std::min<int64_t>(b, r + kEmptyRowsPerItem);
            it.span = -1;
            empties.push_back(it);
        }
    }
    // interleave: item i of a list of length L goes to position (i + 0.5) / L
    std::vector<std::pair<double, BinItem>> all;
    all.reserve(pieces.size() + groups.size() + empties.size());
    for (auto* lst : {&pieces, &groups, &empties})
        for (size_t i = 0; i < lst->size(); ++i) all.emplace_back(((double)i + 0.5) / (double)lst->size(), (*lst)[i]);
    std::stable_sort(all.begin(), all.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    std::vector<BinItem> items;
    items.reserve(all.size());
    for (auto& p : all) items.push_back(p.second);
    if (items.empty()) {  // keep a valid table
        BinItem it = {};
        it.kind = kBinEmpty;
        it.span = -1;
        items.push_back(it);
    }
    B->nitems = (int32_t)items.size();
    B->nspans = nspans;
    B->items.release();
    if ((rc = B->items.alloc(items.size() * sizeof(BinItem)))) return rc;
    if ((rc = bcuda_ok(cudaMemcpyAsync(B->items.p, items.data(), items.size() * sizeof(BinItem), cudaMemcpyHostToDevice, s),
                       "H2D items")) ||
        (rc = bcuda_ok(cudaStreamSynchronize(s), "items")))
        return rc;
    B->span_acc.release();
    B->span_cnt.release();
    const size_t ns = (size_t)std::max(1, nspans);
    if ((rc = B->span_acc.alloc(ns * 2 * sizeof(unsigned long long))) ||
        (rc = B->span_cnt.alloc(ns * sizeof(uint32_t))) ||
        (rc = bcuda_ok(cudaMemsetAsync(B->span_acc.p, 0, B->span_acc.bytes, s), "memset")) ||
        (rc = bcuda_ok(cudaMemsetAsync(B->span_cnt.p, 0, B->span_cnt.bytes, s), "memset")) ||
        (rc = bcuda_ok(cudaStreamSynchronize(s), "memset")))
        return rc;
    // CTAs: one per 32768 inbound entries, at most one per SM
    B->grid = std::max(1, std::min(B->nitems, work_grid(B->nnz, sweep_grid())));
    if (B->cg_exec) cudaGraphExecDestroy(B->cg_exec);
    if (B->cg) cudaGraphDestroy(B->cg);
    B->cg_exec = nullptr;
    B->cg = nullptr;
    B->cg_failed = false;
    return EGPR_SUCC;
}

int bins_alloc_solve(egpr_graph* g, cudaStream_t s) {
    BinLayout* B = g->bins;
    const size_t stride = bin_stride(B->n);
    int rc;
    B->acc_slots = 512;
    if ((rc = B->scale.alloc(stride * sizeof(float))) || (rc = B->tele.alloc(stride * sizeof(float))) ||
        (rc = B->x.alloc(2 * stride * sizeof(float))) || (rc = B->z.alloc(2 * stride * sizeof(float))) ||
        (rc = B->z64.alloc(stride * sizeof(double))) || (rc = B->out64.alloc(stride * sizeof(double))) ||
        (rc = B->states.alloc(sizeof(GraphState))) || (rc = B->ctl.alloc(sizeof(Ctl))) ||
        (rc = B->acc.alloc((size_t)B->acc_slots * kAccWords * sizeof(unsigned long long))))
        return rc;
    if ((rc = bcuda_ok(cudaMemsetAsync(B->acc.p, 0, B->acc.bytes, s), "memset")) ||
        (rc = bcuda_ok(cudaMemsetAsync(B->z.p, 0, B->z.bytes, s), "memset")) ||
        (rc = bcuda_ok(cudaMemsetAsync(B->x.p, 0, B->x.bytes, s), "memset")))
        return rc;
    return EGPR_SUCC;
}

int bins_upload_tele(egpr_graph* g, cudaStream_t s) {
    BinLayout* B = g->bins;
    k_bins_tele<<<bin_grid_for(B->n), kThreads, 0, s>>>(g->tele.as<float>(), B->inv.as<int32_t>(), B->n,
                                                        B->tele.as<float>());
    return bcuda_ok(cudaGetLastError(), "teleport renumbering");
}

int bins_enqueue(egpr_graph* g, double alpha, int32_t max_iter, double tol, bool personalised, uint32_t flags,
                 cudaStream_t s, int32_t* host_launches) {
    BinLayout* B = g->bins;
    const int32_t n = B->n;
    const int gv = bin_grid_for(n);
    const size_t stride = bin_stride(n);
    float* x0 = B->x.as<float>();
    float* z0 = B->z.as<float>();
    k_bins_init<<<gv, kThreads, 0, s>>>(B->outw.as<double>(), n, alpha, B->scale.as<float>(), x0, z0);
    k_bins_state<<<1, 1, 0, s>>>(B->states.as<GraphState>(), B->ctl.as<Ctl>(), n, g->n_dangling_solve, alpha, tol,
                                 max_iter, personalised ? 1 : 0);
    int rc = bcuda_ok(cudaGetLastError(), "binned set-up");
    if (rc) return rc;
    int32_t launches = 2;
    if (graph_loop_enabled() && bins_capture_loop(g) == EGPR_SUCC) {
        if ((rc = bcuda_ok(cudaGraphLaunch(B->cg_exec, s), "graph launch"))) return rc;
    } else {
        BinParams P = bin_params(g, 0, 0);
        for (int32_t it = 0; it < max_iter; ++it)
            k_bsweep<float><<<B->grid, kBinCta, bin_smem(P.hubs), s>>>(P);
        if ((rc = bcuda_ok(cudaGetLastError(), "binned sweep"))) return rc;
    }
    const bool correction = (flags & EGPR_FLAG_NO_CORRECTION) == 0;
    const float* x1 = x0 + stride;
    if (correction) {
        k_bins_z64<<<gv, kThreads, 0, s>>>(B->outw.as<double>(), B->states.as<GraphState>(), x0, x1, n,
                                           B->z64.as<double>());
        BinParams P = bin_params(g, 1, 0);
        k_bsweep<double><<<B->grid, kBinCta, bin_smem(0), s>>>(P);
        launches += 2;
    }
    k_bins_normalize<<<gv, kThreads, 0, s>>>(B->states.as<GraphState>(), x0, x1, B->out64.as<double>(),
                                             B->perm.as<int32_t>(), n, correction ? 0 : 1, g->out.as<double>());
    launches += 1;
    *host_launches = launches;
    return bcuda_ok(cudaGetLastError(), "binned finish");
}

int bins_read_state(egpr_graph* g, cudaStream_t s, int32_t* iterations, int32_t* converged, double* residual,
                    int32_t* launches, int32_t* error) {
    BinLayout* B = g->bins;
    GraphState st;
    Ctl ctl;
    int rc;
    if ((rc = bcuda_ok(cudaMemcpyAsync(&st, B->states.p, sizeof(st), cudaMemcpyDeviceToHost, s), "D2H state")) ||
        (rc = bcuda_ok(cudaMemcpyAsync(&ctl, B->ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
        (rc = bcuda_ok(cudaStreamSynchronize(s), "solve")))
        return rc;
    *iterations = st.iter;
    *converged = st.converged;
    *residual = st.residual;
    *launches = ctl.launches;
    *error = ctl.error;
    return EGPR_SUCC;
}

}  // namespace egpr
