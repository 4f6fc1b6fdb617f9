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
// Work split.  The sweep reads its own copy of the inbound CSR in which every
// row ends on an entry of its own (an empty row holds one placeholder entry
// whose carried value is 0).  Rows are packed into chunks (only a row longer
// than a chunk is cut); a chunk is walked in warp tiles of kTileItems entries,
// lane l owning entries 8l..8l+7.  For every tile the layout holds a 256-bit
// mask of the entries that end a row and the row the first of them ends, so
// the k-th mark of a tile ends row tile_row + k.  One persistent CTA per SM
// runs independent warps that pull chunks from a queue; per tile a warp
//   1. gathers the carried values of its 256 entries: hubs (the largest
//      out-degrees, encoded -(slot+1)) from the CTA's shared-memory copy of
//      the hub values, staged once per launch by a TMA bulk copy; the rest
//      from z in L2/HBM.  The next tile's sources and mask are already loaded,
//      and the previous ranks, scales and hub slots of the tile's rows are
//      requested before the gathers return;
//   2. sums each lane's entries segment by segment and joins the segments
//      that cross lanes with a five-step shuffle scan bounded by the marked
//      lanes; a row still open at the tile's end carries into the next tile;
//   3. finishes the tile's rows with coalesced stores.
// FP64 sums (residual, dangling mass, rank sum) are added as fixed-point
// integers, so their total does not depend on the order in which chunks
// finish; rows cut between chunks are finished by the last CTA to leave the
// launch, which also advances every graph's state.  No warp waits on another;
// the only wait is on the hub staging copy, and it is bounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <type_traits>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kCtaWarps = 24;         // independent warps per CTA, one CTA per SM
constexpr int kCtaThreads = 32 * kCtaWarps;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kCopyPiece = 32768;                 // bytes per hub staging copy
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of the staging wait (2 s)

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long ldcg_u64(const unsigned long long* p) { return __ldcg(p); }

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
// Shared-memory load by 32-bit shared address (read-only data of the launch).
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float x;
    asm("ld.shared.f32 %0, [%1];" : "=f"(x) : "r"(a));
    return x;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- per-graph view ------------------------------------------------------------
struct SweepView {
    const float* xin;       // previous ranks
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
};

template <bool kFinal>
__device__ SweepView make_view(const GraphDev& G, GraphState* st, int32_t iter) {
    SweepView W;
    W.one_minus_alpha = 1.0 - st->alpha;
    W.personalised = st->personalised;
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
template <bool kFinal, typename Acc>
__device__ __forceinline__ void finish_row(const SweepView& W, int32_t v, double acc, float xin, float scale,
                                           int32_t hs, Acc& err, Acc& dsum, double& xsum) {
    double val;
    if (W.personalised) val = (acc + W.one_minus_alpha * (double)__ldg(W.tele + v)) + W.dmass;
    else val = acc + W.jump;
    if (!kFinal) {
        const float xo = (float)val;
        err += (Acc)fabsf(xo - xin);
        W.xout[v] = xo;
        const float zo = scale >= 0.f ? xo * scale : 0.f;
        W.zout[v] = zo;
        if (hs >= 0) W.hub_out[hs] = zo;
        if (scale < 0.f) dsum += (Acc)xo;
        xsum += (double)xo;
    } else {
        err += (Acc)fabs(val - (double)xin);
        W.out[v] = val;
        xsum += val;
    }
}

// ---- order-free FP64 sums ---------------------------------------------------------
// A value is split into two's-complement words in units of 2^-32 and of 2^-64
// (the remainder, rounded) and added with integer atomics, so the total does
// not depend on the order in which chunks finish.  Partial sums here are far
// below 2^31 and there are far fewer than 2^20 terms per word, so no word
// overflows and both convert to double exactly.
__device__ __forceinline__ void fx_add(unsigned long long* a, double v) {
    const double t = v * 4294967296.0;  // exact
    const double f = floor(t);
    const unsigned long long hi = (unsigned long long)(long long)f;
    const unsigned long long lo = (unsigned long long)rint((t - f) * 4294967296.0);
    atomicAdd(a, hi);  // results unused: issued as reductions
    atomicAdd(a + 1, lo);
}

__device__ __forceinline__ double fx_join(unsigned long long hi, unsigned long long lo) {
    return (double)(long long)hi * (1.0 / 4294967296.0) + (double)lo * (1.0 / 18446744073709551616.0);
}

// Accumulator slot of (graph, k): each graph has acc_sub slots so that
// concurrent chunks rarely add to the same address.
__device__ __forceinline__ unsigned long long* acc_slot(const SweepParams& P, int32_t gi, int32_t k) {
    return P.acc + (size_t)kAccWords * ((size_t)gi * (size_t)P.acc_sub + (size_t)(k % P.acc_sub));
}

// A piece of a row cut between chunks has been added to the span's
// accumulator (lane 0).  The last of the span's chunks to arrive finishes the
// row; the sum is exact fixed point, so it does not matter which one that is.
template <bool kFinal>
__device__ void span_arrive(const SweepParams& P, const SweepView& W, int32_t ta, int32_t parts, int32_t slot) {
    __threadfence();
    const uint32_t prev = atomicAdd(&P.span_cnt[ta], 1u);
    if (prev != (uint32_t)(parts - 1)) return;
    __threadfence();
    unsigned long long* sa = P.span_acc + 2 * ta;
    const double sum = fx_join(ldcg_u64(sa), ldcg_u64(sa + 1));
    sa[0] = 0ull;
    sa[1] = 0ull;
    P.span_cnt[ta] = 0u;
    const int32_t v = __ldg(&P.chunks[ta].tail_row);
    double e = 0.0, d = 0.0, x = 0.0;
    finish_row<kFinal, double>(W, v, sum, W.xin[v], kFinal ? 0.f : W.scale[v], kFinal ? -1 : W.hub_slot[v], e, d, x);
    unsigned long long* a = acc_slot(P, __ldg(&P.chunks[ta].graph), slot);
    fx_add(a, e);
    fx_add(a + 2, d);
    fx_add(a + 4, x);
}

// End of a launch, run by the whole last CTA to leave the queue: per graph,
// turns the accumulators into the residual, dangling mass and rank sum, clears
// them, and advances the graph's state (pagerank.py:117-131).
template <bool kFinal>
__device__ void launch_tail(const SweepParams& P) {
    const int tid = threadIdx.x;
    __threadfence();
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int32_t gi = warp; gi < P.ngraphs; gi += (int32_t)(blockDim.x >> 5)) {
        GraphState* st = P.states + gi;
        if (!kFinal && ldcg(&st->done)) continue;
        // all of a lane's loads first (they are independent), then the clears
        unsigned long long w[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
        for (int32_t k0 = 0; k0 < P.acc_sub; k0 += 64) {
            unsigned long long* a = P.acc + (size_t)kAccWords * ((size_t)gi * (size_t)P.acc_sub + (size_t)(k0 + lane));
            unsigned long long* b = a + (size_t)kAccWords * 32;
            const bool ha = k0 + lane < P.acc_sub, hb = k0 + 32 + lane < P.acc_sub;
            unsigned long long ra[6], rb[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                ra[i] = ha ? ldcg_u64(a + i) : 0ull;
                rb[i] = hb ? ldcg_u64(b + i) : 0ull;
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                w[i] += ra[i] + rb[i];
                if (ha) a[i] = 0ull;
                if (hb) b[i] = 0ull;
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

// ---- the sweep kernel ---------------------------------------------------------------
// What a warp needs of the graph it works on; kept in shared memory so that the
// tile loop keeps its registers for data in flight.
struct WarpCtx {
    SweepView W;
    const int32_t* cols;
    const float* w;
    const uint32_t* tile_bits;
    const int32_t* tile_row;
    const float* zsrc;      // carried values read by this sweep
    const float* hub_g;     // their hub copy (global)
    const double* z64;
    const double* hubz64;    // the hubs' FP64 carried values (correction sweep)
    const int32_t* hub_ids;
    int32_t graph;
    int32_t iter;
    int32_t done;           // the graph had converged before this launch
    int32_t hub_slots;      // hub codes of the graph: slots 0 .. nhub (the zero slot)
};

__device__ __forceinline__ Chunk load_chunk(const Chunk* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    Chunk c;
    int4* d = reinterpret_cast<int4*>(&c);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Chunk) / 16); ++i) d[i] = __ldg(q + i);
    return c;
}

// Sources, mark bits, marks of the lanes below, and first-mark row of warp
// tile t (entries T .. T+255).
__device__ __forceinline__ void fetch_tile(const int32_t* cols, const uint32_t* tile_bits, const int32_t* tile_row,
                                           int32_t t, int32_t T, int lane, int4& ca, int4& cb, uint32_t& bits,
                                           uint32_t& below, int32_t& row) {
    const int4* c4 = reinterpret_cast<const int4*>(cols) + (T >> 2) + 2 * lane;
    ca = __ldcs(c4);
    cb = __ldcs(c4 + 1);
    const uint32_t* tw = tile_bits + (size_t)t * kTileWords + (lane >> 2);
    const int sh = 8 * (lane & 3);
    bits = (__ldcs(tw) >> sh) & 0xffu;
    below = (__ldcs(tw + 8) >> sh) & 0xffu;
    row = __ldcs(tile_row + t);
}

template <typename Real>
__device__ void process_chunk(const SweepParams& P, int32_t c, const Chunk& ck, const WarpCtx& X,
                              const float* hub_s, int32_t hub_count, Real* scr) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    // per-lane sums of the chunk (residual, dangling mass, rank sum) are FP64
    // in both sweeps: they decide the stop rule and the mass carried into the
    // next sweep
    using Acc = double;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int32_t kb = ck.nnz_begin, ke = ck.nnz_end, T0 = kb & ~7;
    const int32_t fl = ck.flags;
    bool head_pending = (fl & kHasHead) && !(fl & kInterior);
    double head_val = 0.0;
    Acc err = Acc(0), dsum = Acc(0);
    double xsum = 0.0;
    Real carry = Real(0);  // the row still open at the end of the previous tile
    // this chunk's pointers, held in registers
    const int32_t* cols = X.cols;
    const uint32_t* tbits = X.tile_bits;
    const int32_t* trows = X.tile_row;
    const float* zsrc = X.zsrc;
    const float* hub_g = X.hub_g;
    const bool hubs_local = hub_count >= X.hub_slots;       // every hub code reads shared memory
    const uint32_t hub_m4 = smem_u32(hub_s) - 4u;           // shared address of hub slot -1
    int4 ca, cb;
    uint32_t bits, below;
    int32_t row;
    fetch_tile(cols, tbits, trows, ck.tile_begin, T0, lane, ca, cb, bits, below, row);
    for (int32_t t = ck.tile_begin; t < ck.tile_end; ++t) {
        const int32_t T = T0 + (t - ck.tile_begin) * kTileItems;
        const int32_t cc[kLaneItems] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
        const uint32_t mb = bits;
        const int32_t pre = (int32_t)below;
        const int32_t r0 = row;
        if (t + 1 < ck.tile_end) fetch_tile(cols, tbits, trows, t + 1, T + kTileItems, lane, ca, cb, bits, below, row);
        // 1. gathers of this tile's entries (only a chunk's first and last
        //    tiles hold entries of other chunks)
        const int32_t p0 = T + kLaneItems * lane;
        Real v[kLaneItems];
        // One load per entry: z from global memory, a hub from the CTA's shared
        // copy (predicated pair); a graph whose hubs are not all staged reads
        // the rest of them from its global hub copy.
        auto carried = [&](int32_t s) -> Real {
            if (kFinal) return s >= 0 ? X.z64[s] : X.hubz64[-s - 1];
            float x;
            if (hubs_local) {
                if (s >= 0) x = __ldg(zsrc + s);
                else x = lds_f32(hub_m4 - 4u * (uint32_t)s);
            } else {
                const int32_t h = -s - 1;
                x = s >= 0 ? __ldg(zsrc + s) : (h < hub_count ? lds_f32(hub_m4 - 4u * (uint32_t)s) : hub_g[h]);
            }
            return (Real)x;
        };
        if (T >= kb && T + kTileItems <= ke) {
#pragma unroll
            for (int u = 0; u < kLaneItems; ++u) v[u] = carried(cc[u]);
        } else {
#pragma unroll
            for (int u = 0; u < kLaneItems; ++u) {
                const int32_t p = p0 + u;
                v[u] = (p >= kb && p < ke) ? carried(cc[u]) : Real(0);
            }
        }
        if (X.w) {
            const float4* w4 = reinterpret_cast<const float4*>(X.w) + (T >> 2) + 2 * lane;
            const float4 wa = __ldcs(w4), wb = __ldcs(w4 + 1);
            v[0] *= (Real)wa.x; v[1] *= (Real)wa.y; v[2] *= (Real)wa.z; v[3] *= (Real)wa.w;
            v[4] *= (Real)wb.x; v[5] *= (Real)wb.y; v[6] *= (Real)wb.z; v[7] *= (Real)wb.w;
        }
        // 2. marks of the tile (pre: marks of the lanes below, from the tile table)
        const int32_t nm = __shfl_sync(kFull, pre + __popc(mb), 31);
        if (nm == 0) {
            // No row ends in this tile (inside a long row): its entries all join
            // the open row.
            Real part = v[0];
#pragma unroll
            for (int u = 1; u < kLaneItems; ++u) part += v[u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
            carry = carry + part;
            continue;
        }
        // the rows this lane finishes first: request their data now
        float xin0 = 0.f, sc0 = 0.f;
        int32_t hs0 = -1;
        if (lane < nm) {
            const int32_t v0 = r0 + lane;
            xin0 = X.W.xin[v0];
            if (!kFinal) {
                sc0 = X.W.scale[v0];
                hs0 = X.W.hub_slot[v0];
            }
        }
        // 3. per-lane segment sums; row values by mark ordinal
        Real acc = Real(0), head_part = Real(0);
        int first = -1, k = pre;
#pragma unroll
        for (int u = 0; u < kLaneItems; ++u) {
            acc += v[u];
            if ((mb >> u) & 1u) {
                if (first < 0) {
                    first = u;
                    head_part = acc;
                } else {
                    scr[k] = acc;
                }
                ++k;
                acc = Real(0);
            }
        }
        if (lane == 0) {
            if (first >= 0) head_part = carry + head_part;
            else acc = carry + acc;
        }
        // 4. segmented inclusive scan of the open sums; a lane's segment starts
        //    at the nearest marked lane at or below it
        const unsigned mm = __ballot_sync(kFull, first >= 0);
        const unsigned le = mm & (lt | (1u << lane));
        const int sl = le ? 31 - __clz(le) : 0;
        Real S = acc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Real up = __shfl_up_sync(kFull, S, o);
            if (lane - o >= sl) S += up;
        }
        const Real below = __shfl_up_sync(kFull, S, 1);
        if (first >= 0) scr[pre] = lane == 0 ? head_part : below + head_part;
        carry = __shfl_sync(kFull, S, 31);
        __syncwarp();
        // 5. finish the tile's rows; the chunk's first mark ends its head row
        //    (cut before the chunk), whose piece goes to the span instead
        if (lane < nm) {
            const Real val = scr[lane];
            if (head_pending && lane == 0) head_val = (double)val;
            else finish_row<kFinal>(X.W, r0 + lane, (double)val, xin0, sc0, hs0, err, dsum, xsum);
        }
        for (int32_t j = lane + 32; j < nm; j += 32) {  // tiles that end more than 32 rows
            const int32_t v0 = r0 + j;
            finish_row<kFinal>(X.W, v0, (double)scr[j], X.W.xin[v0], kFinal ? 0.f : X.W.scale[v0],
                               kFinal ? -1 : X.W.hub_slot[v0], err, dsum, xsum);
        }
        if (nm > 0) head_pending = false;
        __syncwarp();
    }
    const double err64 = warp_sum((double)err);
    const double dsum64 = warp_sum((double)dsum);
    xsum = warp_sum(xsum);
    if (lane == 0) {
        unsigned long long* a = acc_slot(P, ck.graph, (int32_t)(blockIdx.x * kCtaWarps + (threadIdx.x >> 5)));
        fx_add(a, err64);
        fx_add(a + 2, dsum64);
        fx_add(a + 4, xsum);
        const int32_t slot = (int32_t)(blockIdx.x * kCtaWarps + (threadIdx.x >> 5));
        if (fl & kInterior) {
            fx_add(P.span_acc + 2 * ck.head_ta, (double)carry);
            span_arrive<kFinal>(P, X.W, ck.head_ta, ck.pad, slot);
        } else {
            if (fl & kHasHead) {
                fx_add(P.span_acc + 2 * ck.head_ta, head_val);
                span_arrive<kFinal>(P, X.W, ck.head_ta, ck.pad, slot);
            }
            if (fl & kHasTail) {
                fx_add(P.span_acc + 2 * c, (double)carry);
                span_arrive<kFinal>(P, X.W, c, ck.pad2, slot);
            }
        }
    }
}

template <typename Real>
__global__ void __launch_bounds__(kCtaThreads, 1) k_sweep(SweepParams P) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_hub;
    __shared__ WarpCtx ctx[kCtaWarps];
    __shared__ int32_t s_idle, s_abort, s_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t hub_count = kFinal ? 0 : P.hub_count;
    const size_t hub_bytes = ((size_t)hub_count * sizeof(float) + 127) & ~(size_t)127;
    float* hub_s = reinterpret_cast<float*>(smem);
    Real* scr = reinterpret_cast<Real*>(smem + hub_bytes) + (size_t)warp * kTileItems;
    if (threadIdx.x == 0) {
        s_abort = 0;
        s_last = 0;
        s_idle = (!kFinal && ldcg(&P.ctl->active) <= 0) ? 1 : 0;  // one reading for the whole CTA
        if (!s_idle && hub_count > 0) {
            // Stage graph 0's hub values for this launch's parity.  A CTA that
            // reads the next parity can only do so after every chunk was taken,
            // so it gets no work.
            mbar_init(&bar_hub, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            const uint32_t bytes = (uint32_t)hub_count * (uint32_t)sizeof(float);
            const float* src = P.graphs[0].hubz[ldcg(&P.states[0].iter) & 1];
            mbar_arrive_tx(&bar_hub, bytes);
            for (uint32_t off = 0; off < bytes; off += kCopyPiece)
                bulk_load(reinterpret_cast<unsigned char*>(hub_s) + off, reinterpret_cast<const unsigned char*>(src) + off,
                          min(kCopyPiece, bytes - off), &bar_hub);
        }
    }
    __syncthreads();
    if (!s_idle && hub_count > 0) {
        bool ok = mbar_try(&bar_hub, 0u);
        if (!ok) {
            const unsigned long long t0 = global_ns();
            while (!(ok = mbar_try(&bar_hub, 0u)) && global_ns() - t0 < kWaitNs) {
            }
        }
        if (!ok) atomicExch(&s_abort, 1);
        __syncthreads();
        if (s_abort && threadIdx.x == 0) {
            atomicExch(&P.ctl->error, EGPR_TIMEOUT);
            // leave no copy in flight into this CTA's shared memory
            const unsigned long long t0 = global_ns();
            while (!mbar_try(&bar_hub, 0u) && global_ns() - t0 < kWaitNs) {
            }
        }
    }
    if (!s_idle && !s_abort) {
        // Each warp keeps one claim and one chunk record ahead of the chunk it
        // works on; the record is only read once the chunk is done.
        WarpCtx& X = ctx[warp];
        if (lane == 0) X.graph = -1;
        __syncwarp();
        uint32_t claim = 0;
        if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
        int32_t c = (int32_t)__shfl_sync(kFull, claim, 0);
        if (c < P.nchunks) {
            if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
            Chunk ck = load_chunk(P.chunks + c);
            for (;;) {
                if (ck.graph != X.graph) {
                    const int32_t gi = ck.graph;
                    GraphState* st = P.states + gi;
                    const int32_t iter = ldcg(&st->iter);
                    const int32_t done = kFinal ? 0 : ldcg(&st->done);
                    __syncwarp();
                    if (lane == 0) {
                        const GraphDev& G = P.graphs[gi];
                        X.W = make_view<kFinal>(G, st, iter);
                        X.cols = G.cols;
                        X.w = G.w;
                        X.tile_bits = G.tile_bits;
                        X.tile_row = G.tile_row;
                        X.zsrc = G.z[iter & 1];
                        X.hub_g = G.hubz[iter & 1];
                        X.z64 = G.z64;
                        X.hubz64 = G.hubz64;
                        X.hub_ids = G.hub_ids;
                        X.hub_slots = G.nhub + 1;
                        X.graph = gi;
                        X.iter = iter;
                        X.done = done;
                    }
                    __syncwarp();
                }
                // the next chunk: its claim was issued one chunk ago
                const int32_t cn = (int32_t)__shfl_sync(kFull, claim, 0);
                const bool have = cn < P.nchunks;
                Chunk nk;
                if (have) {
                    nk = load_chunk(P.chunks + cn);
                    if (lane == 0) claim = atomicAdd(&P.ctl->queue, 1u);
                }
                if (!X.done) process_chunk<Real>(P, c, ck, X, hub_s, hub_count, scr);  // else: frozen graph
                if (!have) break;
                c = cn;
                ck = nk;
            }
        }
    }
    __threadfence();  // this CTA's accumulator updates before its exit is counted
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        s_last = prev == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    // Last CTA out: every chunk of this launch is done.
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
    // the hubs' copy, by slot (the same value, so a hub entry reads one word
    // instead of its slot's id and then the value); slot nhub is the zero slot
    for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h <= G.nhub;
         h += (int64_t)gridDim.x * blockDim.x) {
        double z = 0.0;
        if (h < G.nhub) {
            const int32_t u = G.hub_ids[h];
            const double o = G.outw[u];
            z = o <= 1e-15 ? 0.0 : alpha * (double)xp[u] / o;
        }
        G.hubz64[h] = z;
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

// Dynamic shared memory of a sweep launch: the staged hub values (FP32 sweeps of
// one graph) and one tile of row values per warp.  The kernel opts in to the
// device's limit once per device.
int smem_optin(int mode) {
    static std::atomic<int> cache[2][64];  // per device; host threads may race to fill it with the same value
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::atomic<int>& c = cache[mode ? 1 : 0][dev];
    const int have = c.load(std::memory_order_acquire);
    if (have > 0) return have;
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
    c.store(b, std::memory_order_release);
    return b;
}

size_t scratch_bytes(int mode) { return (size_t)kCtaWarps * kTileItems * (mode ? sizeof(double) : sizeof(float)); }

size_t dyn_smem(int mode, int32_t hub_count) {
    return (((size_t)hub_count * sizeof(float) + 127) & ~(size_t)127) + scratch_bytes(mode);
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
    P.span_cnt = plan.d_span_cnt.as<uint32_t>();
    P.acc_sub = plan.nacc / std::max(1, plan.ngraphs);
    P.span_list = plan.d_span_list.as<int32_t>();
    P.nspans = plan.nspans;
    P.ctl = plan.d_ctl.as<Ctl>();
    P.cond = plan.cond;
    P.use_cond = use_cond;
    P.ngraphs = plan.ngraphs;
    smem_optin(mode);  // the kernel's opt-in to more than 48 KB of dynamic shared memory
    int32_t hubs = 0;
    if (mode == 0 && plan.ngraphs == 1) {
        // all hub slots (the zero slot included) while they fit, and no more than
        // EGPR_HUB_SMEM values (tuning)
        const size_t room = (size_t)smem_optin(0) - scratch_bytes(0);
        hubs = std::min<int32_t>(plan.hub_count, (int32_t)(room / sizeof(float)) & ~31);
        hubs = std::min<int32_t>(hubs, env_int("EGPR_HUB_SMEM", kHubCap, 0, kHubCap) & ~31);
    }
    P.hub_count = hubs;
    return P;
}

int vertex_grid(int32_t max_n) {
    int64_t b = ((int64_t)max_n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
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

int32_t hub_stride(int32_t nhub) { return (nhub + 1 + 31) & ~31; }

int sweep_resident_warps() { return sweep_grid() * kCtaWarps; }

// CTAs for a persistent launch over `entries` inbound entries: one per
// EGPR_CTA_ENTRIES entries (default 32768), at most `full`.  A small graph
// then holds a few SMs instead of all of them, so solves of other graphs on
// other streams run beside it (0: always the full grid).
int work_grid(int64_t entries, int full) {
    static const int64_t per = [] {
        const char* e = std::getenv("EGPR_CTA_ENTRIES");
        const long long x = e ? std::atoll(e) : 32768;
        return (int64_t)(x >= 0 ? x : 32768);
    }();
    if (per == 0) return std::max(1, full);
    const int64_t want = (entries + per - 1) / per;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, full));
}

// One persistent CTA per SM.
int sweep_grid() {
    static std::atomic<int> cache[64];  // per device; host threads may race to fill it with the same value
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    const int have = cache[dev].load(std::memory_order_acquire);
    if (have > 0) return have;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    const int grid = std::max(1, sms);
    cache[dev].store(grid, std::memory_order_release);
    return grid;
}

// The FP32 carried values z (both buffers, contiguous) are gathered once per
// inbound entry every sweep.  A persisting L2 access-policy window over them
// (EGPR_L2_WINDOW=1) is off by default: on B200 the lines it holds persisting
// take L2 from ordinary caching, and the sweep measured faster without it
// (R-MAT scale 25 weighted: 2.06 ms per sweep against 2.28 ms; scale 22:
// 0.228 against 0.233 ms).  The persisting carve-out is a limit of this
// process's CUDA context and ends with it.
void plan_set_l2_window(Plan& plan, void* base, size_t bytes) {
    plan.l2_base = nullptr;
    plan.l2_bytes = 0;
    plan.l2_hit_ratio = 0.f;
    const char* env = std::getenv("EGPR_L2_WINDOW");
    if (!env || env[0] != '1') return;
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
    d.cols = g->sw_col.as<int32_t>();
    d.w = g->weighted ? g->sw_w.as<float>() : nullptr;
    d.tile_bits = g->tile_bits.as<uint32_t>();
    d.tile_row = g->tile_row.as<int32_t>();
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
    d.hubz[1] = g->hubz.as<float>() + hub_stride(g->nhub);
    d.hubz64 = g->hubz64.as<double>();
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
    plan.hub_count = count == 1 ? hub_stride(graphs[0]->nhub) : 0;
    int64_t entries = 0;
    for (int32_t gi = 0; gi < count; ++gi) entries += graphs[gi]->sw_nnz;
    plan.grid = std::max(1, std::min(plan.nchunks, work_grid(entries, sweep_grid())));
    // accumulator slots: 64 per graph (few for the launch's last CTA to read,
    // enough that concurrent chunks rarely add to the same address), fewer
    // for many graphs
    const int32_t per_graph = std::max(1, std::min(64, 8192 / std::max(1, count)));
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
        (rc = plan.d_span_cnt.alloc(all.size() * sizeof(uint32_t))) ||
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
    kp.sharedMemBytes = (unsigned)dyn_smem(0, P.hub_count);
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
    cudaMemsetAsync(plan.d_span_cnt.p, 0, plan.d_span_cnt.bytes, stream);
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
    cfg.dynamicSmemBytes = dyn_smem(0, P.hub_count);
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
        k_sweep<double><<<plan.grid, kCtaThreads, dyn_smem(1, 0), stream>>>(P);
        l += 2;
    }
    k_normalize<<<grid, kThreads, 0, stream>>>(plan.d_graphs.as<GraphDev>(), plan.d_states.as<GraphState>(),
                                               plan.ngraphs, correction ? 0 : 1);
    l += 1;
    *launches = l;
    return cuda_ok(cudaGetLastError(), "finish launch");
}

}  // namespace egpr
