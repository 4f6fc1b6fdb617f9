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
// Work split.  A graph's rows are cut into chunks of whole rows (only rows
// longer than a chunk are cut, into "spans"), chunks into warp tiles of
// kTileItems inbound entries starting on 8-entry boundaries.  One persistent
// CTA of 32 independent warps runs per SM; warps pull chunks from a queue.
// Per tile a warp
//   1. loads its 256 entries' sources with two 16-byte loads per lane (lane l
//      owns entries 8l..8l+7) and gathers their carried values: sources among
//      the graph's hubs (the kHubCap largest out-degrees, encoded as -(slot+1))
//      read the CTA's shared-memory copy of the hub values, staged once per
//      launch by a TMA bulk copy; the rest read z from L2/HBM;
//   2. marks the last entry of every row finished in the tile in a 256-bit
//      mask (row ends come from in_row) and lists those rows in order; rows
//      without entries are finished on the spot;
//   3. sums each lane's 8 products segment by segment and joins rows that
//      cross lanes with one shuffle segmented scan; a row still open at the
//      tile's end carries into the next tile;
//   4. finishes the listed rows (coalesced).
// Rows cut between chunks are finished by whichever chunk arrives last, adding
// the pieces in chunk order.  FP64 partial sums are reduced in a fixed order
// through groups of chunks and then per graph, so every result is
// deterministic.  Nothing waits on another warp; the only wait is on the TMA
// copy, and it is bounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kCtaWarps = 32;                 // independent warps per CTA, one CTA per SM
constexpr int kCtaThreads = 32 * kCtaWarps;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kCopyPiece = 32768;        // bytes per bulk copy instruction
constexpr long long kWaitLimit = 1ll << 26;   // bounded wait on the hub staging copy

template <typename Real>
struct WarpScratch {
    uint32_t flags[kTileItems / 32];
    int32_t list[kTileItems];
    Real rowval[kTileItems];
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;  // valid in lane 0
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Per-chunk view of one graph.
struct SweepView {
    const float* xin;     // previous ranks
    const float* zsrc32;  // carried values (FP32 sweep)
    float* xout;
    float* zout;
    const float* hub_in;  // hub values read by this sweep (global copy)
    float* hub_out;       // hub values written for the next sweep
    double jump;          // (1-alpha)/n + dangling term (uniform teleport)
    double dmass;         // dangling term alone (personalised teleport)
    double one_minus_alpha;
    int32_t personalised;
};

// Finishes row v given its gathered sum; accumulates residual / dangling /
// rank sums.  FP32 sweep: writes x_new, z_new (and the hub copy of z_new); the
// residual compares the stored FP32 iterates, so the loop can stop once they no
// longer change even when tol*n is below FP32 resolution.  FP64 correction
// sweep: writes the FP64 result.
template <typename Real>
__device__ __forceinline__ void finish_row(const GraphDev& G, const SweepView& W, int32_t v, double acc,
                                           double& err, double& dsum, double& xsum) {
    const float xin = W.xin[v];
    const float scale = G.scale[v];
    double val;
    if (W.personalised) val = (acc + W.one_minus_alpha * (double)G.tele[v]) + W.dmass;
    else val = acc + W.jump;
    const double prev = (double)xin;
    if constexpr (std::is_same<Real, float>::value) {
        const float xo = (float)val;
        err += fabs((double)xo - prev);
        W.xout[v] = xo;
        const float zo = scale >= 0.f ? xo * scale : 0.f;
        W.zout[v] = zo;
        const int32_t hs = G.hub_slot[v];
        if (hs >= 0) W.hub_out[hs] = zo;
        if (scale < 0.f) dsum += (double)xo;
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
    double e = 0.0, d = 0.0, x = 0.0;
    finish_row<Real>(G, W, cta.tail_row, sum, e, d, x);
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
__device__ void process_chunk(const SweepParams& P, int32_t c, WarpScratch<Real>& S, const float* hub_smem) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
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
        W.hub_in = G.hubz[par];
        W.hub_out = G.hubz[par ^ 1];
        W.dmass = ldcg(&st->dmass);
    } else {
        const int par = (iter - 1) & 1;  // x_{k-1}: the input of the last sweep
        W.xin = G.x[par];
        W.zsrc32 = nullptr;
        W.xout = nullptr;
        W.zout = nullptr;
        W.hub_in = nullptr;
        W.hub_out = nullptr;
        W.dmass = ldcg(&st->dmass_prev);
    }
    W.jump = st->c1 + W.dmass;
    const float* __restrict__ hub = hub_smem ? hub_smem : W.hub_in;
    const int32_t* __restrict__ in_row = G.in_row;
    const int4* __restrict__ col4 = reinterpret_cast<const int4*>(G.in_col);
    const float4* __restrict__ w4 = reinterpret_cast<const float4*>(G.in_w);
    const int2* __restrict__ coord = G.sub_coord;

    double err = 0.0, dsum = 0.0, xsum = 0.0;
    Real carry = Real(0);  // partial of the row still open at the end of the previous tile
    Real head_val = Real(0);
    bool head_pending = (ck.flags & kHasHead) != 0;

    int2 tc = coord[ck.sub_begin];
    int4 ca = __ldcs(col4 + (tc.x >> 2) + 2 * lane);
    int4 cb = __ldcs(col4 + (tc.x >> 2) + 2 * lane + 1);
    for (int32_t t = ck.sub_begin; t < ck.sub_end; ++t) {
        const int32_t T = tc.x, fa = tc.y;
        const bool has_next = t + 1 < ck.sub_end;
        const int2 tn = has_next ? coord[t + 1] : make_int2(T, ck.row_end);
        const int32_t fb = tn.y;
        const int32_t lo = max(T, ck.nnz_begin), hi = min(T + kTileItems, ck.nnz_end);
        // 1. gathers of this tile's entries
        const int32_t cc[kLaneItems] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
        const int32_t p0 = T + kLaneItems * lane;
        Real v[kLaneItems];
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            const int32_t p = p0 + u;
            const int32_t cu = cc[u];
            Real x = Real(0);
            if (p >= lo && p < hi) {
                if constexpr (kFinal) x = G.z64[cu >= 0 ? cu : G.hub_ids[-cu - 1]];
                else x = cu >= 0 ? W.zsrc32[cu] : hub[-cu - 1];
            }
            v[u] = x;
        }
        if (w4) {
            const float4 wa = __ldcs(w4 + (T >> 2) + 2 * lane);
            const float4 wb = __ldcs(w4 + (T >> 2) + 2 * lane + 1);
            const float ww[kLaneItems] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
            for (int u = 0; u < kLaneItems; ++u) v[u] *= (Real)ww[u];
        }
        if (has_next) {
            ca = __ldcs(col4 + (tn.x >> 2) + 2 * lane);
            cb = __ldcs(col4 + (tn.x >> 2) + 2 * lane + 1);
        }
        // 2. rows finished in this tile: end marks for rows with entries, the
        //    rest finished on the spot
        if (lane < kTileItems / 32) S.flags[lane] = 0u;
        __syncwarp();
        int32_t nlist = 0;
        for (int32_t r0 = fa; r0 < fb; r0 += 32) {
            const int32_t r = r0 + lane;
            const bool in = r < fb;
            const int32_t s = in ? in_row[r] : 0;
            int32_t e = __shfl_down_sync(kFull, s, 1);
            if (lane == 31 && in) e = in_row[r + 1];
            if (in && r + 1 == fb && lane != 31) e = in_row[r + 1];
            const bool ne = in && e > s;
            const unsigned bal = __ballot_sync(kFull, ne);
            if (ne) {
                S.list[nlist + __popc(bal & lt_mask)] = r;
                const int32_t bit = e - 1 - T;  // in [0, kTileItems) by construction of the tiles
                if ((unsigned)bit < (unsigned)kTileItems) atomicOr(&S.flags[bit >> 5], 1u << (bit & 31));
            } else if (in) {
                finish_row<Real>(G, W, r, 0.0, err, dsum, xsum);
            }
            nlist += __popc(bal);
        }
        __syncwarp();
        // 3. per-lane segmented sums, then lanes joined by a segmented scan
        const uint32_t fw = S.flags[lane >> 2];
        const int sh = (lane & 3) * 8;
        const uint32_t mybits = (fw >> sh) & 0xffu;
        int32_t k = __popc(fw & ((1u << sh) - 1u));
        for (int w = 0; w < (lane >> 2); ++w) k += __popc(S.flags[w]);
        Real acc = Real(0), head_part = Real(0);
        int32_t first_close = -1;
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            acc += v[u];
            if ((mybits >> u) & 1u) {
                if (first_close < 0) {
                    first_close = k;
                    head_part = acc;
                } else {
                    S.rowval[k] = acc;
                }
                acc = Real(0);
                ++k;
            }
        }
        bool f = first_close >= 0;
        Real seg = acc;
        if (lane == 0 && !f) seg += carry;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Real up = __shfl_up_sync(kFull, seg, o);
            const bool fup = __shfl_up_sync(kFull, (int)f, o) != 0;
            if (lane >= o) {
                if (!f) seg += up;
                f = f || fup;
            }
        }
        const Real prev_seg = __shfl_up_sync(kFull, seg, 1);
        if (first_close >= 0) S.rowval[first_close] = head_part + (lane == 0 ? carry : prev_seg);
        carry = __shfl_sync(kFull, seg, 31);
        __syncwarp();
        // 4. finish the listed rows; the chunk's head row (cut before the chunk)
        //    is the chunk's first listed row and becomes its span piece instead
        int32_t jstart = 0;
        if (head_pending && nlist > 0) {
            head_val = S.rowval[0];
            head_pending = false;
            jstart = 1;
        }
        for (int32_t j = jstart + lane; j < nlist; j += 32)
            finish_row<Real>(G, W, S.list[j], (double)S.rowval[j], err, dsum, xsum);
        __syncwarp();
        tc = tn;
    }
    chunk_finish<Real>(P, c, ck, G, W, st, err, dsum, xsum, (double)head_val, (double)carry);
}

template <typename Real>
__global__ void __launch_bounds__(kCtaThreads, 1) k_sweep(SweepParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ int32_t s_abort;
    __shared__ int32_t s_idle;
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool stage = !kFinal && P.hub_smem;
    const float* hub_smem = stage ? reinterpret_cast<const float*>(smem) : nullptr;
    const size_t hub_bytes = stage ? (size_t)kHubCap * sizeof(float) : 0;
    WarpScratch<Real>& S = reinterpret_cast<WarpScratch<Real>*>(smem + hub_bytes)[warp];
    if (threadIdx.x == 0) {
        s_abort = 0;
        s_idle = (!kFinal && ldcg(&P.ctl->active) <= 0) ? 1 : 0;  // one reading for the whole CTA
    }
    __syncthreads();
    bool idle = s_idle != 0;
    if (stage && !idle) {
        // Stage graph 0's hub values for this launch's parity.  A CTA that reads
        // the next parity can only do so after every chunk was taken, so it gets
        // no work.
        const GraphDev& G = P.graphs[0];
        const uint32_t bytes = (uint32_t)G.nhub * (uint32_t)sizeof(float);
        if (threadIdx.x == 0 && bytes > 0) {
            const float* src = G.hubz[ldcg(&P.states[0].iter) & 1];
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(bytes)
                         : "memory");
            for (uint32_t off = 0; off < bytes; off += kCopyPiece) {
                const uint32_t piece = min(kCopyPiece, bytes - off);
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_u32(smem + off)),
                    "l"(reinterpret_cast<const unsigned char*>(src) + off), "r"(piece), "r"(smem_u32(&mbar))
                    : "memory");
            }
        }
        __syncthreads();
        if (bytes > 0) {
            uint32_t ok = 0;
            for (long long i = 0; i < kWaitLimit && !ok; ++i) {
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                    : "=r"(ok)
                    : "r"(smem_u32(&mbar))
                    : "memory");
            }
            if (!ok) atomicExch(&s_abort, 1);
        }
        __syncthreads();
        if (s_abort) {
            if (threadIdx.x == 0) atomicExch(&P.ctl->error, EGPR_TIMEOUT);
            idle = true;
        }
    }
    if (!idle) {
        for (;;) {
            int32_t c = 0;
            if (lane == 0) c = (int32_t)atomicAdd(&P.ctl->queue, 1u);
            c = __shfl_sync(kFull, c, 0);
            if (c >= P.nchunks) break;
            process_chunk<Real>(P, c, S, hub_smem);
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
                const bool more = active > 0 && launches < P.ctl->cap && P.ctl->error == 0;
                if (active > 0 && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
                if (P.use_cond) cudaGraphSetConditional(P.cond, more ? 1u : 0u);
            }
            __threadfence();
        }
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

int g_cta_cache[2][64] = {};

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

size_t sweep_smem_bytes(int mode, bool hub) {
    if (mode == 0) return (hub ? (size_t)kHubCap * sizeof(float) : 0) + kCtaWarps * sizeof(WarpScratch<float>);
    return kCtaWarps * sizeof(WarpScratch<double>);
}

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
    P.hub_smem = (mode == 0 && plan.ngraphs == 1) ? 1 : 0;
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

// Resident CTAs of a sweep kernel on the current device (dynamic shared memory
// sized for the hub cache).
int sweep_ctas(int mode) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int& cached = g_cta_cache[mode ? 1 : 0][dev];
    if (cached > 0) return cached;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (mode == 0) {
        cudaFuncSetAttribute(k_sweep<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep_smem_bytes(0, true));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<float>, kCtaThreads, sweep_smem_bytes(0, true));
    } else {
        cudaFuncSetAttribute(k_sweep<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep_smem_bytes(1, false));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<double>, kCtaThreads,
                                                      sweep_smem_bytes(1, false));
    }
    cudaGetLastError();
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
    d.hub_ids = g->hub_ids.as<int32_t>();
    d.hub_slot = g->hub_slot.as<int32_t>();
    d.hubz[0] = g->hubz.as<float>();
    d.hubz[1] = g->hubz.as<float>() + std::max(g->nhub, 4);
    d.nhub = g->nhub;
    d.n = g->n;
    d.chunk_begin = d.chunk_end = 0;
    d.group_begin = d.group_end = 0;
    d.span_begin = d.span_end = 0;
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
    kp.sharedMemBytes = (unsigned)sweep_smem_bytes(0, P.hub_smem != 0);
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
    cfg.dynamicSmemBytes = sweep_smem_bytes(0, P.hub_smem != 0);
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
        k_sweep<double><<<plan.grid_final, kCtaThreads, sweep_smem_bytes(1, false), stream>>>(P);
        l += 2;
    }
    k_normalize<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                               plan.ngraphs, correction ? 0 : 1);
    l += 1;
    *launches = l;
    return cuda_ok(cudaGetLastError(), "finish launch");
}

}  // namespace egpr
