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
// Work split (merge path): items = row ends + entries, cut into sub-tiles of
// kSubItems; a persistent CTA pulls chunks (runs of sub-tiles) from a queue.
// Inside a sub-tile the entries' products are staged in shared memory with
// coalesced loads, every thread walks kItemsPerThread consecutive items, and
// rows split between threads are fixed up from the threads' carries.  Rows
// split between chunks are combined by whichever chunk finishes last, in chunk
// order.  FP64 per-chunk partials are reduced by the last chunk of each graph
// in a fixed order, so every result is deterministic.  Nothing ever waits on
// another CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kWarps = kThreads / 32;

template <typename Real>
struct SweepSmem {
    Real prod[kSubItems];
    int32_t rowend[kSubItems + 1];
    Real rowval[kSubItems];
    Real carry_val[kThreads];
    int32_t carry_row[kThreads];
    Real wlast_val[kWarps];
    Real wcarry[kWarps];
    int32_t wlast_row[kWarps];
    int32_t wfirst_row[kWarps];
    double red[3][kWarps];
    Real sub_carry;
    Real head_val;
    int32_t head_pending;
    int32_t tile;
    int32_t is_last;
};

// Block-wide inclusive segmented scan of (row, value) pairs in thread order,
// rows non-decreasing: returns, for this thread, the sum of the values of the
// threads from the start of its row's run up to itself.  Leaves every
// thread's row and scanned value in S.carry_row / S.carry_val.  Fixed
// combination order, so the result is deterministic.
template <typename Real>
__device__ __forceinline__ Real segmented_scan(SweepSmem<Real>& S, int32_t row, Real v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Real up = __shfl_up_sync(0xffffffffu, v, o);
        const int32_t rup = __shfl_up_sync(0xffffffffu, row, o);
        if (lane >= o && rup == row) v += up;
    }
    const int32_t wfirst = __shfl_sync(0xffffffffu, row, 0);
    if (lane == 31) {
        S.wlast_row[warp] = row;
        S.wlast_val[warp] = v;
        S.wfirst_row[warp] = wfirst;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Real prefix = Real(0);
        for (int w = 0; w < kWarps; ++w) {
            const Real cin = (w > 0 && S.wfirst_row[w] == S.wlast_row[w - 1]) ? prefix : Real(0);
            S.wcarry[w] = cin;
            prefix = S.wlast_val[w] + (S.wlast_row[w] == S.wfirst_row[w] ? cin : Real(0));
        }
    }
    __syncthreads();
    if (row == wfirst) v += S.wcarry[warp];
    S.carry_row[threadIdx.x] = row;
    S.carry_val[threadIdx.x] = v;
    __syncthreads();
    return v;
}

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

// Block-wide sum of three FP64 values in a fixed order; result valid in thread 0.
template <typename Real>
__device__ __forceinline__ void block_sum3(SweepSmem<Real>& S, double& a, double& b, double& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        S.red[0][warp] = a;
        S.red[1][warp] = b;
        S.red[2][warp] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = 0.0; b = 0.0; c = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            a += S.red[0][w];
            b += S.red[1][w];
            c += S.red[2][w];
        }
    }
    __syncthreads();
}

// Per-launch view of one graph, read at the start of each chunk.
struct SweepView {
    const float* xin;     // previous ranks
    const float* zsrc32;  // carried values (FP32 sweep)
    float* xout;
    float* zout;
    double jump;          // (1-alpha)/n + dangling term (uniform teleport)
    double dmass;         // dangling term alone (personalised teleport)
    double one_minus_alpha;
    int32_t personalised;
};

// Row data the epilogue needs, loaded ahead of time.
constexpr int kRowPre = 2;
struct RowPre {
    float xin;
    float scale;
    float tele;
};

__device__ __forceinline__ void load_row(const GraphDev& G, const SweepView& W, int32_t v, RowPre& p) {
    p.xin = W.xin[v];
    p.scale = G.scale[v];
    p.tele = W.personalised ? G.tele[v] : 0.f;
}

template <typename Real>
__device__ __forceinline__ void finish_row_pre(const GraphDev& G, const SweepView& W, int32_t v, double acc,
                                               const RowPre& p, double& err, double& dsum, double& xsum) {
    double val;
    if (W.personalised) val = (acc + W.one_minus_alpha * (double)p.tele) + W.dmass;
    else val = acc + W.jump;
    const double prev = (double)p.xin;
    if constexpr (std::is_same<Real, float>::value) {
        const float xo = (float)val;
        err += fabs((double)xo - prev);
        W.xout[v] = xo;
        W.zout[v] = p.scale >= 0.f ? xo * p.scale : 0.f;
        if (p.scale < 0.f) dsum += (double)xo;
        xsum += (double)xo;
    } else {
        err += fabs(val - prev);
        G.out[v] = val;
        xsum += val;
    }
}

// Finishes row v given its gathered sum; accumulates residual / dangling /
// rank sums.  FP32 sweep: writes x_new and z_new.  FP64 correction sweep:
// writes the FP64 result.
template <typename Real>
__device__ __forceinline__ void finish_row(const GraphDev& G, const SweepView& W, int32_t v, double acc,
                                           double& err, double& dsum, double& xsum) {
    double val;
    if (W.personalised) val = (acc + W.one_minus_alpha * (double)G.tele[v]) + W.dmass;
    else val = acc + W.jump;
    const double prev = (double)W.xin[v];
    if constexpr (std::is_same<Real, float>::value) {
        // The residual compares the stored FP32 iterates, so the loop can stop
        // once they no longer change even when tol*n is below FP32 resolution.
        const float xo = (float)val;
        err += fabs((double)xo - prev);
        W.xout[v] = xo;
        const float sc = G.scale[v];
        W.zout[v] = sc >= 0.f ? xo * sc : 0.f;
        if (sc < 0.f) dsum += (double)xo;
        xsum += (double)xo;
    } else {
        err += fabs(val - prev);
        G.out[v] = val;
        xsum += val;
    }
}

template <typename Real>
__device__ void span_arrive(const SweepParams& P, const GraphDev& G, const SweepView& W, int32_t ta,
                            int32_t participants) {
    const uint32_t prev = atomicAdd(&P.span_cnt[ta], 1u);
    if (prev != (uint32_t)(participants - 1)) return;
    // Last participant: combine the pieces in chunk order and finish the row.
    __threadfence();
    const Chunk cta = P.chunks[ta];
    const int32_t tb = cta.tail_tb;
    double sum = ldcg(&P.piece[2 * ta + 1]);
    for (int32_t q = ta + 1; q < tb; ++q) sum += ldcg(&P.piece[2 * q + 1]);
    sum += ldcg(&P.piece[2 * tb]);
    P.span_cnt[ta] = 0u;
    double e = 0.0, d = 0.0, x = 0.0;
    finish_row<Real>(G, W, cta.tail_row, sum, e, d, x);
    P.span_part[3 * ta] = e;
    P.span_part[3 * ta + 1] = d;
    P.span_part[3 * ta + 2] = x;
    __threadfence();
}

template <typename Real>
__device__ void graph_reduce(const SweepParams& P, SweepSmem<Real>& S, const GraphDev& G, GraphState* st) {
    __threadfence();
    double e = 0.0, d = 0.0, x = 0.0;
    for (int32_t q = G.chunk_begin + (int32_t)threadIdx.x; q < G.chunk_end; q += kThreads) {
        e += ldcg(&P.chunk_part[3 * q]) + ldcg(&P.span_part[3 * q]);
        d += ldcg(&P.chunk_part[3 * q + 1]) + ldcg(&P.span_part[3 * q + 1]);
        x += ldcg(&P.chunk_part[3 * q + 2]) + ldcg(&P.span_part[3 * q + 2]);
        P.span_part[3 * q] = 0.0;
        P.span_part[3 * q + 1] = 0.0;
        P.span_part[3 * q + 2] = 0.0;
    }
    block_sum3(S, e, d, x);
    if (threadIdx.x == 0) {
        if constexpr (std::is_same<Real, float>::value) {
            st->residual = e;
            st->dsum = d;
            st->xsum = x;
            st->dmass_prev = st->dmass;
            st->dmass = st->alpha * d / (double)G.n;
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
        st->arrive = 0u;
        __threadfence();
    }
}

template <typename Real>
__device__ void process_chunk(const SweepParams& P, int32_t c, SweepSmem<Real>& S) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int tid = threadIdx.x;
    const Chunk ck = P.chunks[c];
    const GraphDev& G = P.graphs[ck.graph];
    GraphState* st = P.states + ck.graph;
    const int32_t iter = ldcg(&st->iter);
    if (!kFinal && ldcg(&st->done)) return;  // frozen graph (uniform across the CTA)

    SweepView W;
    const double alpha = st->alpha;
    W.one_minus_alpha = 1.0 - alpha;
    W.personalised = st->personalised;
    if (!kFinal) {
        const int par = iter & 1;
        W.xin = G.x[par];
        W.zsrc32 = G.z[par];
        W.xout = G.x[par ^ 1];
        W.zout = G.z[par ^ 1];
        W.dmass = ldcg(&st->dmass);
    } else {
        const int par = (iter - 1) & 1;  // x_{k-1}: the input of the last sweep
        W.xin = G.x[par];
        W.zsrc32 = nullptr;
        W.xout = nullptr;
        W.zout = nullptr;
        W.dmass = ldcg(&st->dmass_prev);
    }
    W.jump = st->c1 + W.dmass;
    const Real* __restrict__ gsrc;
    if constexpr (kFinal) gsrc = G.z64;
    else gsrc = W.zsrc32;
    const int32_t* __restrict__ in_row = G.in_row;
    const int32_t* __restrict__ in_col = G.in_col;
    const float* __restrict__ in_w = G.in_w;

    double err = 0.0, dsum = 0.0, xsum = 0.0;
    if (tid == 0) {
        S.sub_carry = Real(0);
        S.head_val = Real(0);
        S.head_pending = (ck.flags & kHasHead) ? 1 : 0;
    }
    // Software pipeline: the column indices of sub-tile s+1 are loaded while
    // sub-tile s is gathered and reduced, and each sub-tile's row data (x, scale)
    // is loaded together with its gathers, so a sub-tile waits on about one
    // memory round trip.
    int2 a = G.sub_coord[ck.sub_begin];
    int2 b = G.sub_coord[ck.sub_begin + 1];
    int32_t col[kItemsPerThread];
#pragma unroll
    for (int u = 0; u < kItemsPerThread; ++u) {
        const int32_t i = tid + u * kThreads;
        col[u] = i < b.y - a.y ? __ldcs(in_col + a.y + i) : -1;
    }
    for (int32_t sidx = ck.sub_begin; sidx < ck.sub_end; ++sidx) {
        const int32_t ra = a.x, ka = a.y;
        const int32_t nnz_sub = b.y - a.y;
        const int32_t nrows = b.x - a.x;
        const bool has_next = sidx + 1 < ck.sub_end;
        const int2 bn = has_next ? G.sub_coord[sidx + 2] : b;
        // Phase 1: gathers of this sub-tile, next sub-tile's indices, row data.
        Real val[kItemsPerThread];
#pragma unroll
        for (int u = 0; u < kItemsPerThread; ++u) val[u] = col[u] >= 0 ? gsrc[col[u]] : Real(0);
        float wv[kItemsPerThread];
        if (in_w) {
#pragma unroll
            for (int u = 0; u < kItemsPerThread; ++u) {
                const int32_t i = tid + u * kThreads;
                wv[u] = i < nnz_sub ? __ldcs(in_w + ka + i) : 0.f;
            }
        }
        const int32_t nnz_next = bn.y - b.y;
#pragma unroll
        for (int u = 0; u < kItemsPerThread; ++u) {
            const int32_t i = tid + u * kThreads;
            col[u] = (has_next && i < nnz_next) ? __ldcs(in_col + b.y + i) : -1;
        }
        RowPre pre[kRowPre];
#pragma unroll
        for (int q = 0; q < kRowPre; ++q) {
            const int32_t r = tid + q * kThreads;
            if (r < nrows) load_row(G, W, ra + r, pre[q]);
        }
        for (int32_t i = tid; i < nrows; i += kThreads) S.rowend[i] = in_row[ra + i + 1] - ka;
#pragma unroll
        for (int u = 0; u < kItemsPerThread; ++u) {
            const int32_t i = tid + u * kThreads;
            if (i < nnz_sub) S.prod[i] = in_w ? val[u] * (Real)wv[u] : val[u];
        }
        __syncthreads();
        // Phase 2: each thread walks its items of the merge path.
        const int32_t total = nrows + nnz_sub;
        const int32_t diag = min(tid * kItemsPerThread, total);
        const int32_t dend = min(diag + kItemsPerThread, total);
        int32_t lo = max(diag - nnz_sub, 0), hi = min(diag, nrows);
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (S.rowend[mid] <= diag - mid - 1) lo = mid + 1;
            else hi = mid;
        }
        int32_t i = lo, j = diag - lo;
        Real acc = Real(0);
        int32_t first = -1;
        for (int32_t d = diag; d < dend; ++d) {
            if (i < nrows && j >= S.rowend[i]) {
                S.rowval[i] = acc;
                if (first < 0) first = i;
                acc = Real(0);
                ++i;
            } else {
                acc += S.prod[j];
                ++j;
            }
        }
        // Phase 2b: each thread's carry (the partial sum of the row it stopped
        // in) is added to the row's completion by a segmented inclusive scan
        // over threads keyed by row (rows never decrease along the path).  The
        // carry from the previous sub-tile belongs to local row 0: it joins
        // thread 0's carry, or thread 0's first row if thread 0 completed it.
        const Real cin = S.sub_carry;
        Real seg = acc;
        if (tid == 0 && first != 0) seg += cin;
        seg = segmented_scan(S, i, seg);
        if (first >= 0) {
            Real v = S.rowval[first];
            if (tid == 0) v += cin;  // first == 0 here: thread 0 starts in row 0
            else if (S.carry_row[tid - 1] == first) v += S.carry_val[tid - 1];
            S.rowval[first] = v;
        }
        __syncthreads();
        if (tid == kThreads - 1) S.sub_carry = seg;  // the last thread always stops in row nrows
        // Phase 3: finish the rows that ended in this sub-tile (coalesced).
#pragma unroll
        for (int q = 0; q < kRowPre; ++q) {
            const int32_t r = tid + q * kThreads;
            if (r < nrows) {
                const Real racc = S.rowval[r];
                if (r == 0 && S.head_pending) S.head_val = racc;  // the chunk's head row: finished through its span
                else finish_row_pre<Real>(G, W, ra + r, (double)racc, pre[q], err, dsum, xsum);
            }
        }
        for (int32_t r = tid + kRowPre * kThreads; r < nrows; r += kThreads) {
            RowPre rp;
            load_row(G, W, ra + r, rp);
            finish_row_pre<Real>(G, W, ra + r, (double)S.rowval[r], rp, err, dsum, xsum);
        }
        if (tid == 0 && nrows > 0) S.head_pending = 0;
        a = b;
        b = bn;
    }
    __syncthreads();
    block_sum3(S, err, dsum, xsum);
    if (tid == 0) {
        P.chunk_part[3 * c] = err;
        P.chunk_part[3 * c + 1] = dsum;
        P.chunk_part[3 * c + 2] = xsum;
        const int32_t f = ck.flags;
        if ((f & kHasHead) && !(f & kInterior)) P.piece[2 * c] = (double)S.head_val;
        if (f & kHasTail) P.piece[2 * c + 1] = (double)S.sub_carry;
        __threadfence();
        if (f & kInterior) {
            span_arrive<Real>(P, G, W, ck.head_ta, ck.tail_tb - ck.head_ta + 1);
        } else {
            if (f & kHasHead) span_arrive<Real>(P, G, W, ck.head_ta, c - ck.head_ta + 1);
            if (f & kHasTail) span_arrive<Real>(P, G, W, c, ck.tail_tb - c + 1);
        }
        __threadfence();
        const uint32_t prev = atomicAdd(&st->arrive, 1u);
        S.is_last = (prev == (uint32_t)(G.chunk_end - G.chunk_begin - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (S.is_last) graph_reduce<Real>(P, S, G, st);
    __syncthreads();
}

template <typename Real>
__global__ void __launch_bounds__(kThreads, 3) k_sweep(SweepParams P) {
    __shared__ SweepSmem<Real> S;
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const bool idle = !kFinal && ldcg(&P.ctl->active) <= 0;
    if (!idle) {
        for (;;) {
            if (threadIdx.x == 0) S.tile = (int32_t)atomicAdd(&P.ctl->queue, 1u);
            __syncthreads();
            const int32_t c = S.tile;
            __syncthreads();
            if (c >= P.nchunks) break;
            process_chunk<Real>(P, c, S);
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        if (prev == gridDim.x - 1) {
            // Last CTA out: every chunk of this launch is done.
            P.ctl->queue = 0u;
            P.ctl->exited = 0u;
            if (!kFinal) {
                const int32_t launches = P.ctl->launches + 1;
                P.ctl->launches = launches;
                const int32_t active = ldcg(&P.ctl->active);
                const bool more = active > 0 && launches < P.ctl->cap;
                if (active > 0 && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
                if (P.use_cond) cudaGraphSetConditional(P.cond, more ? 1u : 0u);
            }
            __threadfence();
        }
    }
}

// ---- per-solve set-up and finishing kernels --------------------------------

// scale = alpha / outw (FP32), -1 marks a dangling vertex (outw <= 1e-15,
// pagerank.py:118); x0 = 1/n; z0 = x0 * scale.
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
        G.z[0][v] = sc >= 0.f ? x0 * sc : 0.f;
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

int g_grid_cache[2][64] = {};

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

SweepParams make_params(Plan& plan, int mode, int use_cond) {
    SweepParams P;
    P.chunks = plan.d_chunks.as<Chunk>();
    P.nchunks = plan.nchunks;
    P.mode = mode;
    P.graphs = plan.d_graphs.as<GraphDev>();
    P.states = plan.d_states.as<GraphState>();
    P.chunk_part = plan.d_chunk_part.as<double>();
    P.piece = plan.d_piece.as<double>();
    P.span_cnt = plan.d_span_cnt.as<uint32_t>();
    P.span_part = plan.d_span_part.as<double>();
    P.ctl = plan.d_ctl.as<Ctl>();
    P.cond = plan.cond;
    P.use_cond = use_cond;
    return P;
}

int vertex_grid(int32_t max_n) {
    int64_t b = ((int64_t)max_n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

}  // namespace

int sweep_occupancy_grid(int mode) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int& cached = g_grid_cache[mode ? 1 : 0][dev];
    if (cached > 0) return cached;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (mode == 0)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<float>, kThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<double>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    cached = sms * per_sm;
    return cached;
}

GraphDev graph_dev_view(const egpr_graph* g) {
    GraphDev d;
    d.in_row = g->in_row.as<int32_t>();
    d.in_col = g->in_col.as<int32_t>();
    d.in_w = g->weighted ? g->in_w.as<float>() : nullptr;
    d.sub_coord = g->sub_coord.as<int2>();
    d.outw = g->outw.as<double>();
    d.scale = g->scale.as<float>();
    d.tele = g->tele.as<float>();
    d.x[0] = g->x0.as<float>();
    d.x[1] = g->x1.as<float>();
    d.z[0] = g->z0.as<float>();
    d.z[1] = g->z1.as<float>();
    d.out = g->out.as<double>();
    d.z64 = g->z64.as<double>();
    d.n = g->n;
    d.chunk_begin = 0;
    d.chunk_end = 0;
    d.pad = 0;
    return d;
}

int plan_build(Plan& plan, egpr_graph* const* graphs, int32_t count, cudaStream_t stream) {
    plan.release();
    std::vector<Chunk> all;
    std::vector<GraphDev> views((size_t)count);
    std::vector<int32_t> ndang((size_t)count);
    int32_t max_n = 0;
    for (int32_t gi = 0; gi < count; ++gi) {
        const egpr_graph* g = graphs[gi];
        const int32_t off = (int32_t)all.size();
        GraphDev v = graph_dev_view(g);
        v.chunk_begin = off;
        for (const Chunk& c0 : g->plan.h_chunks) {
            Chunk c = c0;
            c.graph = gi;
            if (c.head_ta >= 0) c.head_ta += off;
            if (c.tail_tb >= 0) c.tail_tb += off;
            all.push_back(c);
        }
        v.chunk_end = (int32_t)all.size();
        views[(size_t)gi] = v;
        ndang[(size_t)gi] = g->n_dangling_solve;
        max_n = std::max(max_n, g->n);
    }
    plan.ngraphs = count;
    plan.nchunks = (int32_t)all.size();
    plan.max_n = max_n;
    plan.grid = std::max(1, std::min(plan.nchunks, sweep_occupancy_grid(0)));
    plan.grid_final = std::max(1, std::min(plan.nchunks, sweep_occupancy_grid(1)));
    plan.h_chunks_all = all;
    int rc;
    if ((rc = plan.d_chunks.alloc(all.size() * sizeof(Chunk))) ||
        (rc = plan.d_graphs.alloc(views.size() * sizeof(GraphDev))) ||
        (rc = plan.d_states.alloc((size_t)count * sizeof(GraphState))) ||
        (rc = plan.d_ndang.alloc((size_t)count * sizeof(int32_t))) ||
        (rc = plan.d_chunk_part.alloc(all.size() * 3 * sizeof(double))) ||
        (rc = plan.d_piece.alloc(all.size() * 2 * sizeof(double))) ||
        (rc = plan.d_span_cnt.alloc(all.size() * sizeof(uint32_t))) ||
        (rc = plan.d_span_part.alloc(all.size() * 3 * sizeof(double))) ||
        (rc = plan.d_ctl.alloc(sizeof(Ctl))))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(plan.d_chunks.p, all.data(), all.size() * sizeof(Chunk), cudaMemcpyHostToDevice, stream), "H2D chunks")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_graphs.p, views.data(), views.size() * sizeof(GraphDev), cudaMemcpyHostToDevice, stream), "H2D graph table")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_ndang.p, ndang.data(), ndang.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream), "H2D counts")) ||
        (rc = cuda_ok(cudaMemsetAsync(plan.d_span_cnt.p, 0, all.size() * sizeof(uint32_t), stream), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(plan.d_span_part.p, 0, all.size() * 3 * sizeof(double), stream), "memset")) ||
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
    kp.blockDim = dim3(kThreads);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    e = cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp);
    if (e != cudaSuccess) goto fail;
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
    return cuda_ok(cudaGetLastError(), "init launch");
}

int launch_loop(Plan& plan, int32_t max_iter, cudaStream_t stream, int32_t* launches) {
    *launches = 0;
    if (plan_capture_loop(plan, stream) == EGPR_SUCC) {
        int rc = cuda_ok(cudaGraphLaunch(plan.cg_exec, stream), "graph launch");
        *launches = -1;  // counted on the device (Ctl::launches)
        return rc;
    }
    // Fallback: plain launches; a sweep with no active graph returns at once.
    SweepParams P = make_params(plan, 0, 0);
    for (int32_t it = 0; it < max_iter; ++it)
        k_sweep<float><<<plan.grid, kThreads, 0, stream>>>(P);
    *launches = -1;
    return cuda_ok(cudaGetLastError(), "sweep launch");
}

int launch_finish(Plan& plan, bool correction, cudaStream_t stream, int32_t* launches) {
    dim3 grid((unsigned)vertex_grid(plan.max_n), (unsigned)plan.ngraphs);
    int32_t l = 0;
    if (correction) {
        k_prep_z64<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                                  plan.ngraphs);
        k_init_ctl<<<1, 1, 0, stream>>>(plan.d_ctl.as<Ctl>(), plan.ngraphs, 1);
        SweepParams P = make_params(plan, 1, 0);
        k_sweep<double><<<plan.grid_final, kThreads, 0, stream>>>(P);
        l += 3;
    }
    k_normalize<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                               plan.ngraphs, correction ? 0 : 1);
    l += 1;
    *launches = l;
    return cuda_ok(cudaGetLastError(), "finish launch");
}

}  // namespace egpr
