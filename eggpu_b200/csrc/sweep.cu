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
// Work split (merge path, one warp per tile): the items of a graph's merge
// path (one per row end, one per inbound entry) are cut into chunks of whole
// rows, and chunks into warp tiles of kTileItems items.  Every warp is an
// independent worker: it pulls chunks from a queue and, per tile, stages the
// entries' products in its own shared memory with coalesced loads, lets each
// lane walk kLaneItems consecutive items, joins rows split between lanes with
// a shuffle segmented scan, and finishes the tile's rows with coalesced
// stores.  No block-wide barrier exists, so the SM always has independent
// warps to issue from.  Only rows longer than a chunk are cut between chunks;
// the last chunk of such a row to finish combines its pieces in chunk order.
// FP64 partial sums are reduced in a fixed order through groups of chunks and
// then per graph, so every result is deterministic.  Nothing waits on another
// warp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kCtaWarps = 4;                 // independent warps per CTA
constexpr int kCtaThreads = 32 * kCtaWarps;
constexpr int kRowPre = 1;                   // row-data loads issued with the gathers (x 32 rows)
constexpr int kMinCtasPerSm = 8;             // 32 warps per SM: registers capped at 64
constexpr unsigned kFull = 0xffffffffu;

template <typename Real>
struct WarpSmem {
    Real prod[kTileItems];
    int32_t rowend[kTileItems + 1];
    Real rowval[kTileItems];
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;  // valid in lane 0
}

// Per-chunk view of one graph.
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

// Finishes row v given its gathered sum; accumulates residual / dangling /
// rank sums.  FP32 sweep: writes x_new and z_new; the residual compares the
// stored FP32 iterates, so the loop can stop once they no longer change even
// when tol*n is below FP32 resolution.  FP64 correction sweep: writes the FP64
// result.
template <typename Real>
__device__ __forceinline__ void finish_row(const GraphDev& G, const SweepView& W, int32_t v, double acc,
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

// Span arrival (lane 0 only).  The last participant adds the pieces in chunk
// order and finishes the row; its contribution goes to the span's own slot.
template <typename Real>
__device__ void span_arrive(const SweepParams& P, const GraphDev& G, const SweepView& W, int32_t ta,
                            int32_t participants) {
    const uint32_t prev = atomicAdd(&P.span_cnt[ta], 1u);
    if (prev != (uint32_t)(participants - 1)) return;
    __threadfence();
    const Chunk cta = P.chunks[ta];
    const int32_t tb = cta.tail_tb;
    double sum = ldcg(&P.piece[2 * ta + 1]);
    for (int32_t q = ta + 1; q < tb; ++q) sum += ldcg(&P.piece[2 * q + 1]);
    sum += ldcg(&P.piece[2 * tb]);
    P.span_cnt[ta] = 0u;
    RowPre rp;
    load_row(G, W, cta.tail_row, rp);
    double e = 0.0, d = 0.0, x = 0.0;
    finish_row<Real>(G, W, cta.tail_row, sum, rp, e, d, x);
    P.span_part[3 * ta] = e;
    P.span_part[3 * ta + 1] = d;
    P.span_part[3 * ta + 2] = x;
    __threadfence();
}

// The last group of a graph (whole warp): reduce the graph's group partials
// and span slots in a fixed order and advance the graph's state.
template <typename Real>
__device__ void graph_reduce(const SweepParams& P, const GraphDev& G, GraphState* st) {
    const int lane = threadIdx.x & 31;
    __threadfence();
    double e = 0.0, d = 0.0, x = 0.0;
    for (int32_t q = G.group_begin + lane; q < G.group_end; q += 32) {
        e += ldcg(&P.group_part[3 * q]);
        d += ldcg(&P.group_part[3 * q + 1]);
        x += ldcg(&P.group_part[3 * q + 2]);
    }
    for (int32_t q = G.span_begin + lane; q < G.span_end; q += 32) {
        const int32_t ta = P.span_list[q];
        e += ldcg(&P.span_part[3 * ta]);
        d += ldcg(&P.span_part[3 * ta + 1]);
        x += ldcg(&P.span_part[3 * ta + 2]);
        P.span_part[3 * ta] = 0.0;
        P.span_part[3 * ta + 1] = 0.0;
        P.span_part[3 * ta + 2] = 0.0;
    }
    e = warp_sum(e);
    d = warp_sum(d);
    x = warp_sum(x);
    if (lane == 0) {
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
    __syncwarp();
}

// Chunk done (whole warp): chunk partials, spans, group and graph arrival.
template <typename Real>
__device__ void chunk_finish(const SweepParams& P, int32_t c, const Chunk& ck, const GraphDev& G,
                             const SweepView& W, GraphState* st, double err, double dsum, double xsum,
                             double head_val, double tail_val) {
    const int lane = threadIdx.x & 31;
    err = warp_sum(err);
    dsum = warp_sum(dsum);
    xsum = warp_sum(xsum);
    int32_t last_group = 0;
    if (lane == 0) {
        P.chunk_part[3 * c] = err;
        P.chunk_part[3 * c + 1] = dsum;
        P.chunk_part[3 * c + 2] = xsum;
        const int32_t f = ck.flags;
        if ((f & kHasHead) && !(f & kInterior)) P.piece[2 * c] = head_val;
        if (f & kHasTail) P.piece[2 * c + 1] = tail_val;
        __threadfence();
        if (f & kInterior) {
            span_arrive<Real>(P, G, W, ck.head_ta, ck.tail_tb - ck.head_ta + 1);
        } else {
            if (f & kHasHead) span_arrive<Real>(P, G, W, ck.head_ta, c - ck.head_ta + 1);
            if (f & kHasTail) span_arrive<Real>(P, G, W, c, ck.tail_tb - c + 1);
        }
        __threadfence();
        const Group gr = P.groups[ck.group];
        const uint32_t prev = atomicAdd(&P.group_cnt[ck.group], 1u);
        last_group = prev == (uint32_t)(gr.chunk_end - gr.chunk_begin - 1) ? 1 : 0;
    }
    last_group = __shfl_sync(kFull, last_group, 0);
    if (!last_group) return;
    // Last chunk of its group: fixed-order reduction of the group's chunks.
    __threadfence();
    const Group gr = P.groups[ck.group];
    double e = 0.0, d = 0.0, x = 0.0;
    for (int32_t q = gr.chunk_begin + lane; q < gr.chunk_end; q += 32) {
        e += ldcg(&P.chunk_part[3 * q]);
        d += ldcg(&P.chunk_part[3 * q + 1]);
        x += ldcg(&P.chunk_part[3 * q + 2]);
    }
    e = warp_sum(e);
    d = warp_sum(d);
    x = warp_sum(x);
    int32_t last_graph = 0;
    if (lane == 0) {
        P.group_part[3 * ck.group] = e;
        P.group_part[3 * ck.group + 1] = d;
        P.group_part[3 * ck.group + 2] = x;
        P.group_cnt[ck.group] = 0u;
        __threadfence();
        const uint32_t prev = atomicAdd(&st->arrive, 1u);
        last_graph = prev == (uint32_t)(G.group_end - G.group_begin - 1) ? 1 : 0;
    }
    last_graph = __shfl_sync(kFull, last_graph, 0);
    if (last_graph) graph_reduce<Real>(P, G, st);
}

template <typename Real>
__device__ void process_chunk(const SweepParams& P, int32_t c, WarpSmem<Real>& S) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31;
    const Chunk ck = P.chunks[c];
    const GraphDev& G = P.graphs[ck.graph];
    GraphState* st = P.states + ck.graph;
    const int32_t iter = ldcg(&st->iter);
    if (!kFinal && ldcg(&st->done)) return;  // frozen graph (same answer for the whole warp)

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
    const int2* __restrict__ coord = G.sub_coord;

    double err = 0.0, dsum = 0.0, xsum = 0.0;
    Real carry = Real(0);  // partial of the row in progress from the previous tile
    Real head_val = Real(0);
    bool head_pending = (ck.flags & kHasHead) != 0;

    // Software pipeline: tile t+1's indices load while tile t is reduced.
    int2 a = coord[ck.sub_begin];
    int2 b = coord[ck.sub_begin + 1];
    int32_t col[kLaneItems];
#pragma unroll
    for (int u = 0; u < kLaneItems; ++u) {
        const int32_t i = lane + 32 * u;
        col[u] = i < b.y - a.y ? __ldcs(in_col + a.y + i) : -1;
    }
    for (int32_t sidx = ck.sub_begin; sidx < ck.sub_end; ++sidx) {
        const int32_t ra = a.x, ka = a.y;
        const int32_t nnz_sub = b.y - a.y;
        const int32_t nrows = b.x - a.x;
        const bool has_next = sidx + 1 < ck.sub_end;
        const int2 bn = has_next ? coord[sidx + 2] : b;
        // Phase 1: gathers of this tile, next tile's indices, row data.
        Real val[kLaneItems];
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) val[u] = col[u] >= 0 ? gsrc[col[u]] : Real(0);
        if (in_w) {
#pragma unroll
            for (int u = 0; u < kLaneItems; ++u) {
                const int32_t i = lane + 32 * u;
                if (i < nnz_sub) val[u] *= (Real)__ldcs(in_w + ka + i);
            }
        }
        const int32_t nnz_next = bn.y - b.y;
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            const int32_t i = lane + 32 * u;
            col[u] = (has_next && i < nnz_next) ? __ldcs(in_col + b.y + i) : -1;
        }
        RowPre pre[kRowPre];
#pragma unroll
        for (int q = 0; q < kRowPre; ++q) {
            const int32_t r = lane + 32 * q;
            if (r < nrows) load_row(G, W, ra + r, pre[q]);
        }
        for (int32_t i = lane; i < nrows; i += 32) S.rowend[i] = in_row[ra + i + 1] - ka;
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            const int32_t i = lane + 32 * u;
            if (i < nnz_sub) S.prod[i] = val[u];
        }
        __syncwarp();
        // Phase 2: each lane walks kLaneItems consecutive items of the merge path.
        const int32_t total = nrows + nnz_sub;
        const int32_t diag = min(lane * kLaneItems, total);
        const int32_t dend = min(diag + kLaneItems, total);
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
        // Phase 2b: segmented inclusive scan of the lanes' carries keyed by the
        // row they stopped in (rows never decrease across lanes).  The carry
        // from the previous tile belongs to local row 0: it joins lane 0's carry,
        // or lane 0's first row if lane 0 completed row 0.
        Real seg = acc;
        if (lane == 0 && first != 0) seg += carry;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Real up = __shfl_up_sync(kFull, seg, o);
            const int32_t rup = __shfl_up_sync(kFull, i, o);
            if (lane >= o && rup == i) seg += up;
        }
        const Real prev_seg = __shfl_up_sync(kFull, seg, 1);
        const int32_t prev_row = __shfl_up_sync(kFull, i, 1);
        if (first >= 0) {
            Real v = S.rowval[first];
            if (lane == 0) v += carry;  // first == 0 here: lane 0 starts in row 0
            else if (prev_row == first) v += prev_seg;
            S.rowval[first] = v;
        }
        carry = __shfl_sync(kFull, seg, 31);  // lane 31 always stops in row nrows
        __syncwarp();
        // Phase 3: finish the rows that ended in this tile (coalesced).
#pragma unroll
        for (int q = 0; q < kRowPre; ++q) {
            const int32_t r = lane + 32 * q;
            if (r < nrows) {
                const Real racc = S.rowval[r];
                if (r == 0 && head_pending) head_val = racc;  // finished through its span
                else finish_row<Real>(G, W, ra + r, (double)racc, pre[q], err, dsum, xsum);
            }
        }
        for (int32_t r = lane + 32 * kRowPre; r < nrows; r += 32) {
            RowPre rp;
            load_row(G, W, ra + r, rp);
            finish_row<Real>(G, W, ra + r, (double)S.rowval[r], rp, err, dsum, xsum);
        }
        head_val = __shfl_sync(kFull, head_val, 0);
        if (nrows > 0) head_pending = false;
        __syncwarp();
        a = b;
        b = bn;
    }
    chunk_finish<Real>(P, c, ck, G, W, st, err, dsum, xsum, (double)head_val, (double)carry);
}

template <typename Real>
__global__ void __launch_bounds__(kCtaThreads, kMinCtasPerSm) k_sweep(SweepParams P) {
    __shared__ WarpSmem<Real> smem[kCtaWarps];
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem<Real>& S = smem[warp];
    const bool idle = !kFinal && ldcg(&P.ctl->active) <= 0;
    if (!idle) {
        for (;;) {
            int32_t c = 0;
            if (lane == 0) c = (int32_t)atomicAdd(&P.ctl->queue, 1u);
            c = __shfl_sync(kFull, c, 0);
            if (c >= P.nchunks) break;
            process_chunk<Real>(P, c, S);
        }
    }
    if (lane == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        if (prev == (uint32_t)(P.total_warps - 1)) {
            // Last warp out: every chunk of this launch is done.
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

int g_cta_cache[2][64] = {};

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
    P.groups = plan.d_groups.as<Group>();
    P.group_cnt = plan.d_group_cnt.as<uint32_t>();
    P.group_part = plan.d_group_part.as<double>();
    P.span_list = plan.d_span_list.as<int32_t>();
    P.ctl = plan.d_ctl.as<Ctl>();
    P.cond = plan.cond;
    P.use_cond = use_cond;
    P.total_warps = (mode ? plan.grid_final : plan.grid) * kCtaWarps;
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

// Resident CTAs of a sweep kernel on the current device.
int sweep_ctas(int mode) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int& cached = g_cta_cache[mode ? 1 : 0][dev];
    if (cached > 0) return cached;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (mode == 0)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<float>, kCtaThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<double>, kCtaThreads, 0);
    if (per_sm < 1) per_sm = 1;
    cached = sms * per_sm;
    return cached;
}

}  // namespace

int sweep_resident_warps() { return sweep_ctas(0) * kCtaWarps; }

int sweep_occupancy_grid(int mode) { return sweep_ctas(mode); }

int chunks_per_warp() {
    static const int v = [] {
        const char* e = std::getenv("EGPR_CHUNKS_PER_WARP");
        const int x = e ? std::atoi(e) : 4;
        return x >= 1 && x <= 64 ? x : 4;
    }();
    return v;
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
    d.sub_coord = g->tile_coord.as<int2>();
    d.outw = g->outw.as<double>();
    d.scale = g->scale.as<float>();
    d.tele = g->tele.as<float>();
    d.x[0] = g->x0.as<float>();
    d.x[1] = g->x1.as<float>();
    d.z[0] = g->z0.as<float>();
    d.z[1] = g->z0.as<float>() + g->n;  // one allocation: both buffers under one L2 window
    d.out = g->out.as<double>();
    d.z64 = g->z64.as<double>();
    d.n = g->n;
    d.chunk_begin = d.chunk_end = 0;
    d.group_begin = d.group_end = 0;
    d.span_begin = d.span_end = 0;
    d.pad = 0;
    return d;
}

int plan_build(Plan& plan, egpr_graph* const* graphs, int32_t count, cudaStream_t stream) {
    plan.release();
    std::vector<Chunk> all;
    std::vector<Group> groups;
    std::vector<int32_t> spans;
    std::vector<GraphDev> views((size_t)count);
    std::vector<int32_t> ndang((size_t)count);
    int32_t max_n = 0;
    for (int32_t gi = 0; gi < count; ++gi) {
        const egpr_graph* g = graphs[gi];
        const int32_t off = (int32_t)all.size();
        const int32_t goff = (int32_t)groups.size();
        GraphDev v = graph_dev_view(g);
        v.chunk_begin = off;
        v.group_begin = goff;
        v.span_begin = (int32_t)spans.size();
        for (const Chunk& c0 : g->plan.h_chunks) {
            Chunk c = c0;
            c.graph = gi;
            if (c.head_ta >= 0) c.head_ta += off;
            if (c.tail_tb >= 0) c.tail_tb += off;
            c.group += goff;
            all.push_back(c);
        }
        for (const Group& g0 : g->plan.h_groups)
            groups.push_back(Group{g0.chunk_begin + off, g0.chunk_end + off, gi, 0});
        for (int32_t sp : g->plan.h_spans) spans.push_back(sp + off);
        v.chunk_end = (int32_t)all.size();
        v.group_end = (int32_t)groups.size();
        v.span_end = (int32_t)spans.size();
        views[(size_t)gi] = v;
        ndang[(size_t)gi] = g->n_dangling_solve;
        max_n = std::max(max_n, g->n);
    }
    plan.ngraphs = count;
    plan.nchunks = (int32_t)all.size();
    plan.ngroups = (int32_t)groups.size();
    plan.max_n = max_n;
    const int32_t chunk_ctas = std::max(1, (plan.nchunks + kCtaWarps - 1) / kCtaWarps);
    plan.grid = std::max(1, std::min(chunk_ctas, sweep_ctas(0)));
    plan.grid_final = std::max(1, std::min(chunk_ctas, sweep_ctas(1)));
    plan.h_chunks_all = all;
    if (spans.empty()) spans.push_back(0);
    int rc;
    if ((rc = plan.d_chunks.alloc(all.size() * sizeof(Chunk))) ||
        (rc = plan.d_graphs.alloc(views.size() * sizeof(GraphDev))) ||
        (rc = plan.d_states.alloc((size_t)count * sizeof(GraphState))) ||
        (rc = plan.d_ndang.alloc((size_t)count * sizeof(int32_t))) ||
        (rc = plan.d_chunk_part.alloc(all.size() * 3 * sizeof(double))) ||
        (rc = plan.d_piece.alloc(all.size() * 2 * sizeof(double))) ||
        (rc = plan.d_span_cnt.alloc(all.size() * sizeof(uint32_t))) ||
        (rc = plan.d_span_part.alloc(all.size() * 3 * sizeof(double))) ||
        (rc = plan.d_groups.alloc(groups.size() * sizeof(Group))) ||
        (rc = plan.d_group_cnt.alloc(groups.size() * sizeof(uint32_t))) ||
        (rc = plan.d_group_part.alloc(groups.size() * 3 * sizeof(double))) ||
        (rc = plan.d_span_list.alloc(spans.size() * sizeof(int32_t))) || (rc = plan.d_ctl.alloc(sizeof(Ctl))))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(plan.d_chunks.p, all.data(), all.size() * sizeof(Chunk), cudaMemcpyHostToDevice, stream), "H2D chunks")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_graphs.p, views.data(), views.size() * sizeof(GraphDev), cudaMemcpyHostToDevice, stream), "H2D graph table")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_ndang.p, ndang.data(), ndang.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream), "H2D counts")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_groups.p, groups.data(), groups.size() * sizeof(Group), cudaMemcpyHostToDevice, stream), "H2D groups")) ||
        (rc = cuda_ok(cudaMemcpyAsync(plan.d_span_list.p, spans.data(), spans.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream), "H2D spans")) ||
        (rc = cuda_ok(cudaMemsetAsync(plan.d_span_cnt.p, 0, all.size() * sizeof(uint32_t), stream), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(plan.d_span_part.p, 0, all.size() * 3 * sizeof(double), stream), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(plan.d_group_cnt.p, 0, groups.size() * sizeof(uint32_t), stream), "memset")) ||
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
    kp.sharedMemBytes = 0;
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
        // The loop's last warp left the queue reset; the control block keeps the sweep count.
        SweepParams P = make_params(plan, 1, 0);
        k_sweep<double><<<plan.grid_final, kCtaThreads, 0, stream>>>(P);
        l += 2;
    }
    k_normalize<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                               plan.ngraphs, correction ? 0 : 1);
    l += 1;
    *launches = l;
    return cuda_ok(cudaGetLastError(), "finish launch");
}

}  // namespace egpr
