// Batched personalised PageRank: k teleport vectors per graph, one CSR x dense
// SpMM per sweep.
//
// Maths per column j (the reference's power iteration, easygraph/functions/
// centrality/pagerank.py:112-139, with the (1-alpha)/n teleport term replaced
// by (1-alpha) * p_j[v]; dangling mass stays uniform):
//     X_new[v][j] = alpha * sum_{u -> v} X[u][j] * w_uv / outw[u]
//                 + (1-alpha) * p_j[v] + alpha * D_j / n
// Column j stops on its own L1 rule err_j < tol*n and keeps its own count.
//
// Layout, built once per graph and kept with it:
//   * the entry stream: the inbound CSR in row order with one placeholder in
//     every empty row (the sweep's padded CSR), padded with placeholders to a
//     whole number of chunks.  Per entry the source vertex, with bit 31 set on
//     the last entry of each row (placeholders read the all-zero row n), and
//     the coefficient w / outw[source] in FP32 and in FP64 (0 for placeholders
//     and for sources whose out-weight is at most 1e-15);
//   * chunks of C consecutive entries (C a multiple of 32).  A row cut by a
//     chunk boundary is a span: each chunk it touches stores its piece, and the
//     last of them to arrive adds the pieces in chunk order and finishes the row
//     (deterministic, no waiting);
//   * iterates panel-major, [panel][n + 1][32] FP32: 32 columns per panel, so
//     one source row of a panel is one 128-byte line; row n stays zero.
//
// Sweep (one launch): warps claim (panel, chunk) units from a queue in
// panel-major order, so all SMs gather from one 128 MB-class panel at a time.
// A warp reads 32 entries with one coalesced load; its half-warps take the
// even and the odd entries, each lane gathering two columns with one 8-byte
// load (two source rows per warp instruction).  Row sums go to a per-warp
// buffer in shared memory; the rows a batch finishes are then written in one
// pass (previous iterate, teleport, dangling term), with their loads issued
// together.  Column sums (residual and dangling mass; the FP64 sweep's rank
// sum) are converted to fixed point per chunk and added with integer atomics,
// so their value does not depend on which warp ran which chunk.
//
// Batches of fewer than kSpmmMinColumns columns do not come here: the entry
// points run them as single-vector solves (a panel costs about seven sweeps).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kLanes = 32;          // columns per panel
constexpr int kSpWarps = 28;        // warps per CTA of the FP32 sweep (one CTA per SM)
constexpr int kSpWarps64 = 16;      // of the FP64 sweep (its row buffers are twice as large)
template <bool kF64>
__host__ __device__ constexpr int sp_threads() { return 32 * (kF64 ? kSpWarps64 : kSpWarps); }
constexpr int kMaxPanels = 16;      // panels of one device solve (larger batches run in groups)
constexpr int kAccQ = 4;            // fixed-point words per column and panel
constexpr int32_t kRowEnd = (int32_t)0x80000000u;  // entry: last of its row
constexpr uint32_t kDangBit = 0x80000000u;         // row meta: dangling vertex

struct SpChunk {
    int32_t e0, e1;   // entries [e0, e1)
    int32_t r0;       // the row of entry e0 (the chunk's first row end finishes it)
    int32_t flags;    // kHasHead / kHasTail / kInterior
    int32_t hkey;     // head (or interior) span: its first chunk
    int32_t hparts;   // chunks of that span
    int32_t tparts;   // tail span (first chunk = this one): chunks of it
    int32_t trow;     // the row of entry e1 - 1
};

struct ColState {
    double dmass;
    double dmass_prev;
    double residual;
    double residual64;
    double xsum;
    double dsum;
    int32_t iter;      // sweeps of the column's panel when the column last advanced (parity of its iterate)
    int32_t done;
    int32_t converged;
    int32_t active;    // column < k (a session: the slot holds a request)
    int32_t base;      // panel sweeps before the column joined (its own sweeps are iter - base)
    int32_t max_iter;  // the column's sweep limit
};

struct SpmmParams {
    const SpChunk* chunks;
    int32_t nchunks;
    int32_t npanels;
    int32_t n;
    int32_t tele_ld;          // floats per teleport row (npanels * 32)
    int32_t max_iter;
    const int32_t* src;       // entry stream: source | row-end bit
    const float* coef32;
    const double* coef64;
    const uint32_t* meta;     // per vertex: dangling bit | teleport row + 1 (0: none)
    const float* tele;        // teleport rows: p_j[v] for the vertices that have one
    float* X[2];              // iterates, panel-major [panel][n + 1][32]
    double* out64;            // FP64 result, same layout
    ColState* cols;
    double alpha;
    double tol_n;
    float alpha_hi, alpha_lo;  // alpha = alpha_hi + alpha_lo (FP32 sweep)
    float oma_hi, oma_lo;      // 1 - alpha, likewise
    void* parts;              // [panel][chunk][2][32] pieces of cut rows (Real)
    uint32_t* span_cnt;       // [panel][chunk] arrivals per span (reset by the last)
    unsigned long long* gacc; // [panel][kAccQ][32] fixed-point column sums
    Ctl* ctl;
    int32_t step_cap;         // session steps: stop after this many sweeps without an error (0: none)
};

template <bool kF64>
using RealT = typename std::conditional<kF64, double, float>::type;

template <typename Real>
struct V2 {
    Real x, y;
};

template <bool kF64>
struct SpSmem {
    RealT<kF64> rows[kF64 ? kSpWarps64 : kSpWarps][32][kLanes];  // row sums of the batch in flight, per warp
    unsigned long long acc[kMaxPanels][kAccQ][kLanes];
    int32_t idle;
};

__device__ __forceinline__ size_t pc_index(int32_t p, int32_t c, int32_t nchunks) {
    return (size_t)p * (size_t)nchunks + (size_t)c;
}

// Fixed point.  FP32 sweep: one word in units of 2^-40 per quantity (a chunk's
// per-column sums are below 2^10, their totals below 2^23).  FP64 sweep: two
// words, units of 2^-32 and of 2^-64 (the remainder, rounded), as the
// single-vector sweep keeps them.
__device__ __forceinline__ unsigned long long fx40(double v) {
    return (unsigned long long)__double2ll_rn(v * 1099511627776.0);
}
__device__ __forceinline__ double fx40_join(unsigned long long w) {
    return (double)(long long)w * (1.0 / 1099511627776.0);
}
__device__ __forceinline__ void fx64_split(double v, unsigned long long& hi, unsigned long long& lo) {
    const double t = v * 4294967296.0;  // exact
    const double f = floor(t);
    hi = (unsigned long long)(long long)f;
    lo = (unsigned long long)rint((t - f) * 4294967296.0);
}
__device__ __forceinline__ double fx64_join(unsigned long long hi, unsigned long long lo) {
    return (double)(long long)hi * (1.0 / 4294967296.0) + (double)lo * (1.0 / 18446744073709551616.0);
}

// Adds a lane's two columns of (err, dsum) (FP32 sweep) or (err, xsum) (FP64
// sweep) to the CTA's accumulators of
// panel p (lanes of the lower half-warp; each holds columns c2, c2 + 1).
template <bool kF64>
__device__ __forceinline__ void acc_add(SpSmem<kF64>& S, int32_t p, int c2, double e0, double e1, double d0,
                                        double d1, double x0, double x1) {
    unsigned long long* a = &S.acc[p][0][0];
    if (!kF64) {
        if (e0 != 0.0) atomicAdd(a + 0 * kLanes + c2, fx40(e0));
        if (e1 != 0.0) atomicAdd(a + 0 * kLanes + c2 + 1, fx40(e1));
        if (d0 != 0.0) atomicAdd(a + 1 * kLanes + c2, fx40(d0));
        if (d1 != 0.0) atomicAdd(a + 1 * kLanes + c2 + 1, fx40(d1));
    } else {
        unsigned long long h, l;
        fx64_split(e0, h, l);
        atomicAdd(a + 0 * kLanes + c2, h);
        atomicAdd(a + 1 * kLanes + c2, l);
        fx64_split(e1, h, l);
        atomicAdd(a + 0 * kLanes + c2 + 1, h);
        atomicAdd(a + 1 * kLanes + c2 + 1, l);
        fx64_split(x0, h, l);
        atomicAdd(a + 2 * kLanes + c2, h);
        atomicAdd(a + 3 * kLanes + c2, l);
        fx64_split(x1, h, l);
        atomicAdd(a + 2 * kLanes + c2 + 1, h);
        atomicAdd(a + 3 * kLanes + c2 + 1, l);
    }
}

// What a lane needs of the panel its warp works on.  The lane holds columns
// c2 and c2 + 1 (c2 = 2 * (lane % 16)); both half-warps hold the same columns.
template <bool kF64>
struct Lane {
    const float* xa;  // gathered iterate of column c2 (panel base); FP32 sweep: of both columns
    const float* xb;  // FP64 sweep: of column c2 + 1
    float* xout;      // FP32 sweep: the next iterate (panel base)
    double* out64;    // FP64 sweep: the result (panel base)
    double dm0, dm1;  // FP64 sweep: dangling term of the two columns
    float df0, df1;   // FP32 sweep: the same in FP32
    int32_t p;
    bool live0, live1;
    bool all;         // every column of the panel takes part
    bool same;        // FP64 sweep: every column's x_{k-1} is in the same buffer (xa)
};

// Reads the lane's two column states for panel p; skip = no column of the
// panel takes part in this sweep.
template <bool kF64>
__device__ Lane<kF64> make_lane(const SpmmParams& P, int32_t p, bool& skip) {
    const int lane = threadIdx.x & 31, c2 = 2 * (lane & 15);
    const ColState* cs = P.cols + (size_t)p * kLanes + c2;
    const int32_t a0 = __ldcg(&cs[0].active), a1 = __ldcg(&cs[1].active);
    const int32_t d0 = __ldcg(&cs[0].done), d1 = __ldcg(&cs[1].done);
    const int32_t i0 = __ldcg(&cs[0].iter), i1 = __ldcg(&cs[1].iter);
    const size_t pbase = (size_t)p * ((size_t)P.n + 1) * kLanes;
    Lane<kF64> L;
    L.p = p;
    L.xout = nullptr;
    L.out64 = nullptr;
    L.dm0 = L.dm1 = 0.0;
    L.df0 = L.df1 = 0.f;
    L.same = true;
    if (!kF64) {
        L.live0 = a0 && !d0;
        L.live1 = a1 && !d1;
        const unsigned lm = __ballot_sync(kAll, L.live0 || L.live1);
        skip = lm == 0u;
        L.all = __all_sync(kAll, L.live0 && L.live1);
        // live columns of a panel have taken the same number of sweeps
        const int32_t it = __shfl_sync(kAll, L.live0 ? i0 : i1, lm ? __ffs(lm) - 1 : 0);
        const int par = it & 1;
        L.xa = P.X[par] + pbase;
        L.xb = L.xa;
        L.xout = P.X[par ^ 1] + pbase;
        L.df0 = (float)__ldcg(&cs[0].dmass);
        L.df1 = (float)__ldcg(&cs[1].dmass);
    } else {
        // each column's x_{k-1}, recomputed to x_k in FP64
        L.live0 = a0 != 0;
        L.live1 = a1 != 0;
        skip = __ballot_sync(kAll, L.live0 || L.live1) == 0u;
        L.all = __all_sync(kAll, L.live0 && L.live1);
        const int par0 = (i0 - 1) & 1, par1 = (i1 - 1) & 1;
        const unsigned odd = __ballot_sync(kAll, (L.live0 && par0) || (L.live1 && par1));
        const unsigned even = __ballot_sync(kAll, (L.live0 && !par0) || (L.live1 && !par1));
        L.same = odd == 0u || even == 0u;
        if (L.same) {
            L.xa = P.X[odd ? 1 : 0] + pbase;
            L.xb = L.xa;
        } else {
            L.xa = P.X[par0] + pbase;
            L.xb = P.X[par1] + pbase;
        }
        L.out64 = P.out64 + pbase;
        L.dm0 = __ldcg(&cs[0].dmass_prev);
        L.dm1 = __ldcg(&cs[1].dmass_prev);
    }
    return L;
}

// Per-lane sums of a chunk for its two columns; each chunk's sums are then
// added as fixed point.  The dangling mass is kept in FP64 even in the FP32
// sweep: many rows carry exactly the same value (every vertex without inbound
// entries holds the teleport and dangling terms only), and an FP32 running sum
// of equal terms rounds the same way at every step, a bias of about 1e-6
// relative that the dangling term would feed back into every row.  The FP32
// sweep keeps no rank sum (the result is normalised from an exact sum).
template <bool kF64>
struct LaneSums {
    RealT<kF64> e0 = 0, e1 = 0;  // residual (steers the stop rule)
    double d0 = 0.0, d1 = 0.0;   // FP32 sweep: dangling mass
    double x0 = 0.0, x1 = 0.0;   // FP64 sweep: rank sum
};

// One finished row v of the lane's two columns: rs = sum of the inbound
// terms without alpha, pa/pb = previous value of the columns, mt = row meta.
// FP32 sweep: alpha and 1 - alpha enter as FP32 pairs (high + low part), since
// alpha rounded to FP32 would move the fixed point by about its rounding
// error / (1 - alpha)^2 in L1.
template <bool kF64>
__device__ __forceinline__ void row_out(const SpmmParams& P, const Lane<kF64>& L, int c2, int32_t v,
                                        RealT<kF64> rsx, RealT<kF64> rsy, RealT<kF64> pa, RealT<kF64> pb,
                                        uint32_t mt, LaneSums<kF64>& A) {
    const uint32_t t = mt & ~kDangBit;
    const size_t off = (size_t)v * kLanes + c2;
    if constexpr (!kF64) {
        float bx = L.df0, by = L.df1;
        if (t) {  // a teleport row (seed vertices only)
            const float2 tl = __ldg(
                reinterpret_cast<const float2*>(P.tele + (size_t)(t - 1) * (size_t)P.tele_ld + L.p * kLanes + c2));
            bx = fmaf(P.oma_hi, tl.x, fmaf(P.oma_lo, tl.x, bx));
            by = fmaf(P.oma_hi, tl.y, fmaf(P.oma_lo, tl.y, by));
        }
        const float vx = fmaf(P.alpha_hi, rsx, fmaf(P.alpha_lo, rsx, bx));
        const float vy = fmaf(P.alpha_hi, rsy, fmaf(P.alpha_lo, rsy, by));
        float* o = L.xout + off;
        const bool dang = (mt & kDangBit) != 0u;
        if (L.all) {
            __stcs(reinterpret_cast<float2*>(o), make_float2(vx, vy));
            A.e0 += fabsf(vx - pa);
            A.e1 += fabsf(vy - pb);
            if (dang) {
                A.d0 += (double)vx;
                A.d1 += (double)vy;
            }
        } else {
            if (L.live0) {
                __stcs(o, vx);
                A.e0 += fabsf(vx - pa);
                if (dang) A.d0 += (double)vx;
            }
            if (L.live1) {
                __stcs(o + 1, vy);
                A.e1 += fabsf(vy - pb);
                if (dang) A.d1 += (double)vy;
            }
        }
    } else {
        const double alpha = P.alpha, oma = 1.0 - P.alpha;
        double tx = 0.0, ty = 0.0;
        if (t) {
            const float2 tl = __ldg(
                reinterpret_cast<const float2*>(P.tele + (size_t)(t - 1) * (size_t)P.tele_ld + L.p * kLanes + c2));
            tx = (double)tl.x;
            ty = (double)tl.y;
        }
        const double vx = fma(alpha, rsx, fma(oma, tx, L.dm0));
        const double vy = fma(alpha, rsy, fma(oma, ty, L.dm1));
        double* o = L.out64 + off;
        if (L.live0 && L.live1) {
            *reinterpret_cast<double2*>(o) = make_double2(vx, vy);
        } else {
            if (L.live0) o[0] = vx;
            if (L.live1) o[1] = vy;
        }
        if (L.live0) {
            A.e0 += fabs(vx - pa);
            A.x0 += vx;
        }
        if (L.live1) {
            A.e1 += fabs(vy - pb);
            A.x1 += vy;
        }
    }
}

template <bool kF64>
__device__ __forceinline__ RealT<kF64>* part_ptr(const SpmmParams& P, int32_t p, int32_t c, int slot) {
    return reinterpret_cast<RealT<kF64>*>(P.parts) + (pc_index(p, c, P.nchunks) * 2 + (size_t)slot) * kLanes;
}

template <bool kF64>
__device__ __forceinline__ V2<RealT<kF64>> load_part(const SpmmParams& P, int32_t p, int32_t c, int slot, int c2) {
    const RealT<kF64>* q = part_ptr<kF64>(P, p, c, slot) + c2;
    V2<RealT<kF64>> r;
    if (!kF64) {
        const float2 v = __ldcg(reinterpret_cast<const float2*>(q));
        r.x = v.x;
        r.y = v.y;
    } else {
        const double2 v = __ldcg(reinterpret_cast<const double2*>(q));
        r.x = v.x;
        r.y = v.y;
    }
    return r;
}

template <bool kF64>
__device__ __forceinline__ void store_part(const SpmmParams& P, int32_t p, int32_t c, int slot, int c2,
                                           RealT<kF64> x, RealT<kF64> y) {
    RealT<kF64>* q = part_ptr<kF64>(P, p, c, slot) + c2;
    q[0] = x;
    q[1] = y;
}

// The previous value of the lane's two columns at row v.
template <bool kF64>
__device__ __forceinline__ void prev_of(const Lane<kF64>& L, int c2, int32_t v, RealT<kF64>& a, RealT<kF64>& b) {
    const size_t off = (size_t)v * kLanes + c2;
    if (!kF64) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(L.xa + off));
        a = q.x;
        b = q.y;
    } else if (L.same) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(L.xa + off));
        a = (double)q.x;
        b = (double)q.y;
    } else {
        a = (double)__ldg(L.xa + off);
        b = (double)__ldg(L.xb + off + 1);
    }
}

// A chunk's piece of span `key` (spanning `parts` chunks) is stored.  The last
// of the span's chunks to arrive adds the pieces in chunk order (the first
// chunk's tail piece, whole chunks, the last chunk's head piece) and finishes
// the row; its column sums are added on their own, so the totals do not depend
// on which chunk that was.
template <bool kF64>
__device__ void span_arrive(const SpmmParams& P, SpSmem<kF64>& S, const Lane<kF64>& L, int32_t p, int32_t key,
                            int32_t parts) {
    using Real = RealT<kF64>;
    const int lane = threadIdx.x & 31, g = lane >> 4, c2 = 2 * (lane & 15);
    uint32_t prev = 0;
    if (lane == 0) prev = atomicAdd(&P.span_cnt[pc_index(p, key, P.nchunks)], 1u);
    prev = __shfl_sync(kAll, prev, 0);
    if (prev != (uint32_t)(parts - 1)) return;
    __threadfence();
    if (lane == 0) P.span_cnt[pc_index(p, key, P.nchunks)] = 0u;
    if (g != 0) return;
    const int32_t cb = key + parts - 1;
    V2<Real> s = load_part<kF64>(P, p, key, 1, c2);
    for (int32_t q = key + 1; q < cb; ++q) {
        const V2<Real> t = load_part<kF64>(P, p, q, 0, c2);
        s.x += t.x;
        s.y += t.y;
    }
    {
        const V2<Real> t = load_part<kF64>(P, p, cb, 0, c2);
        s.x += t.x;
        s.y += t.y;
    }
    const int32_t v = __ldg(&P.chunks[key].trow);
    Real pa, pb;
    prev_of<kF64>(L, c2, v, pa, pb);
    LaneSums<kF64> A;
    row_out<kF64>(P, L, c2, v, s.x, s.y, pa, pb, __ldg(P.meta + v), A);
    acc_add<kF64>(S, p, c2, (double)A.e0, (double)A.e1, A.d0, A.d1, A.x0, A.x1);
}

// One (panel, chunk) unit.
template <bool kF64>
__device__ void process_unit(const SpmmParams& P, SpSmem<kF64>& S, int32_t p, int32_t c, const Lane<kF64>& L) {
    using Real = RealT<kF64>;
    using Coef = RealT<kF64>;  // FP32 coefficients for the FP32 sweep, FP64 ones for the FP64 sweep
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 4, c2 = 2 * (lane & 15);
    SpChunk ck;
    {
        const int4* q = reinterpret_cast<const int4*>(P.chunks + c);
        const int4 a = __ldg(q), b = __ldg(q + 1);
        ck.e0 = a.x; ck.e1 = a.y; ck.r0 = a.z; ck.flags = a.w;
        ck.hkey = b.x; ck.hparts = b.y; ck.tparts = b.z; ck.trow = b.w;
    }
    Real(*rows)[kLanes] = S.rows[warp];
    const int32_t* __restrict__ src = P.src;
    const Coef* __restrict__ coef = kF64 ? reinterpret_cast<const Coef*>(P.coef64)
                                         : reinterpret_cast<const Coef*>(P.coef32);
    const float* __restrict__ xa = L.xa;
    const float* __restrict__ xb = L.xb;
    using Acc = Real;
    Acc ax = Acc(0), ay = Acc(0);  // this half-warp's part of the open row
    LaneSums<kF64> A;
    int32_t rb = ck.r0;  // the row the next row end finishes
    bool head_pending = (ck.flags & kHasHead) && !(ck.flags & kInterior);
    int32_t ent = __ldcs(src + ck.e0 + lane);
    Coef cf = __ldcs(coef + ck.e0 + lane);
    for (int32_t b = ck.e0; b < ck.e1; b += 32) {
        const int32_t ec = ent;
        const Coef cc = cf;
        if (b + 32 < ck.e1) {
            ent = __ldcs(src + b + 32 + lane);
            cf = __ldcs(coef + b + 32 + lane);
        }
        const uint32_t m = __ballot_sync(kAll, ec < 0);
        const int nr = __popc(m);
        uint32_t mt = 0u;  // meta of the batch's rows, lane k: row rb + k
        if (lane < nr) mt = __ldg(P.meta + rb + lane);
        int ord = 0;
        auto emit = [&](Acc tx, Acc ty) {
            const Acc sx = tx + __shfl_xor_sync(kAll, tx, 16);
            const Acc sy = ty + __shfl_xor_sync(kAll, ty, 16);
            if (g == 0) *reinterpret_cast<V2<Real>*>(&rows[ord][c2]) = V2<Real>{(Real)sx, (Real)sy};
            ++ord;
        };
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            Real gx[8], gy[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const int32_t u = __shfl_sync(kAll, ec, 16 * h + 2 * s + g) & 0x7fffffff;
                const size_t off = (size_t)u * kLanes + c2;
                if (!kF64 || L.same) {
                    const float2 v = __ldg(reinterpret_cast<const float2*>(xa + off));
                    gx[s] = (Real)v.x;
                    gy[s] = (Real)v.y;
                } else {
                    gx[s] = (Real)__ldg(xa + off);
                    gy[s] = (Real)__ldg(xb + off + 1);
                }
            }
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const Coef q = __shfl_sync(kAll, cc, 16 * h + 2 * s + g);
                const uint32_t mp = (m >> (16 * h + 2 * s)) & 3u;  // row ends at the even / odd entry
                if (mp == 0u) {
                    ax = fma((Acc)q, (Acc)gx[s], ax);
                    ay = fma((Acc)q, (Acc)gy[s], ay);
                } else {
                    const Acc px = (Acc)q * (Acc)gx[s], py = (Acc)q * (Acc)gy[s];
                    if (mp & 1u) {
                        emit(g == 0 ? ax + px : ax, g == 0 ? ay + py : ay);
                        ax = g == 0 ? Acc(0) : px;
                        ay = g == 0 ? Acc(0) : py;
                    } else {
                        ax += px;
                        ay += py;
                    }
                    if (mp & 2u) {
                        emit(ax, ay);
                        ax = Acc(0);
                        ay = Acc(0);
                    }
                }
            }
        }
        if (nr == 0) continue;
        __syncwarp();
        int k0 = 0;
        if (head_pending) {  // the chunk's first row end finishes a row cut before it: its piece
            if (g == 0) store_part<kF64>(P, p, c, 0, c2, rows[0][c2], rows[0][c2 + 1]);
            head_pending = false;
            k0 = 1;
        }
        // the batch's rows: half-warp g takes rows k0 + g, k0 + g + 2, ...
        // four rows per half-warp at a time (their loads issued together) while
        // eight or more remain, then one at a time: the cost follows the row count
        int kk = k0;
        for (; kk + 8 <= nr; kk += 8) {
            Real pa[4], pb[4];
            uint32_t mr[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k = kk + 2 * i + g;
                mr[i] = __shfl_sync(kAll, mt, k);
                prev_of<kF64>(L, c2, rb + k, pa[i], pb[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k = kk + 2 * i + g;
                row_out<kF64>(P, L, c2, rb + k, rows[k][c2], rows[k][c2 + 1], pa[i], pb[i], mr[i], A);
            }
        }
        for (; kk < nr; kk += 2) {
            const int k = kk + g;
            const uint32_t m1 = __shfl_sync(kAll, mt, k & 31);
            if (k < nr) {
                Real pa, pb;
                prev_of<kF64>(L, c2, rb + k, pa, pb);
                row_out<kF64>(P, L, c2, rb + k, rows[k][c2], rows[k][c2 + 1], pa, pb, m1, A);
            }
        }
        rb += nr;
        __syncwarp();
    }
    // the row still open at the end of the chunk: the chunk's piece of a span
    const int32_t f = ck.flags;
    if (f & kHasTail) {
        const Acc tx = ax + __shfl_xor_sync(kAll, ax, 16);
        const Acc ty = ay + __shfl_xor_sync(kAll, ay, 16);
        if (g == 0) store_part<kF64>(P, p, c, (f & kInterior) ? 0 : 1, c2, (Real)tx, (Real)ty);
    }
    // the chunk's column sums (both half-warps, fixed order)
    {
        const double e0 = (double)A.e0 + (double)__shfl_xor_sync(kAll, A.e0, 16);
        const double e1 = (double)A.e1 + (double)__shfl_xor_sync(kAll, A.e1, 16);
        double d0 = 0.0, d1 = 0.0, x0 = 0.0, x1 = 0.0;
        if (!kF64) {
            d0 = A.d0 + __shfl_xor_sync(kAll, A.d0, 16);
            d1 = A.d1 + __shfl_xor_sync(kAll, A.d1, 16);
        } else {
            x0 = A.x0 + __shfl_xor_sync(kAll, A.x0, 16);
            x1 = A.x1 + __shfl_xor_sync(kAll, A.x1, 16);
        }
        if (g == 0) acc_add<kF64>(S, p, c2, e0, e1, d0, d1, x0, x1);
    }
    if (f & (kHasHead | kHasTail)) {
        __threadfence();  // the pieces before the arrivals
        __syncwarp();
        if (f & kInterior) {
            span_arrive<kF64>(P, S, L, p, ck.hkey, ck.hparts);
        } else {
            if (f & kHasHead) span_arrive<kF64>(P, S, L, p, ck.hkey, ck.hparts);
            if (f & kHasTail) span_arrive<kF64>(P, S, L, p, c, ck.tparts);
        }
    }
}

// The sweep: persistent CTAs, warps claiming units; the last CTA to finish
// turns the column sums into the column states (pagerank.py:117-131 per
// column) and decides whether the CUDA-graph loop runs another sweep.
template <bool kF64>
__global__ void __launch_bounds__(sp_threads<kF64>(), 1)
k_spmm(const SpmmParams* __restrict__ Pd, cudaGraphConditionalHandle cond, int32_t use_cond) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SpSmem<kF64>& S = *reinterpret_cast<SpSmem<kF64>*>(smem_raw);
    __shared__ SpmmParams P;
    __shared__ int32_t s_last;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        P = *Pd;
        S.idle = (!kF64 && __ldcg(&Pd->ctl->active) <= 0) ? 1 : 0;
    }
    __syncthreads();
    const int32_t nacc = P.npanels * kAccQ * kLanes;
    unsigned long long* sacc = &S.acc[0][0][0];
    for (int32_t i = tid; i < nacc; i += sp_threads<kF64>()) sacc[i] = 0ull;
    __syncthreads();
    if (!S.idle) {
        const int32_t units = P.npanels * P.nchunks;
        int32_t u = 0;
        if (lane == 0) u = (int32_t)atomicAdd(&P.ctl->queue, 1u);
        u = __shfl_sync(kAll, u, 0);
        int32_t cur = -1;
        bool skip = true;
        Lane<kF64> L;
        while (u < units) {
            int32_t next = 0;
            if (lane == 0) next = (int32_t)atomicAdd(&P.ctl->queue, 1u);  // claimed one ahead
            const int32_t p = u / P.nchunks, c = u - p * P.nchunks;
            if (p != cur) {
                L = make_lane<kF64>(P, p, skip);
                cur = p;
            }
            if (!skip) process_unit<kF64>(P, S, p, c, L);
            u = __shfl_sync(kAll, next, 0);
        }
    }
    __syncthreads();
    for (int32_t i = tid; i < nacc; i += sp_threads<kF64>()) {
        const unsigned long long w = sacc[i];
        if (w) atomicAdd(P.gacc + i, w);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(&P.ctl->exited, 1u) == gridDim.x - 1 ? 1 : 0;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int32_t j = tid; j < P.npanels * kLanes; j += sp_threads<kF64>()) {
        const int32_t p = j / kLanes, col = j - p * kLanes;
        unsigned long long w[kAccQ];
#pragma unroll
        for (int q = 0; q < kAccQ; ++q) {
            unsigned long long* a = P.gacc + ((size_t)p * kAccQ + q) * kLanes + col;
            w[q] = __ldcg(a);
            *a = 0ull;
        }
        ColState* cs = P.cols + j;
        if (!kF64) {
            if (cs->active && !cs->done) {
                const double e = fx40_join(w[0]), d = fx40_join(w[1]);
                cs->residual = e;
                cs->dsum = d;
                cs->dmass_prev = cs->dmass;
                cs->dmass = P.alpha * d / (double)P.n;
                const int32_t it = cs->iter + 1;
                cs->iter = it;
                const bool conv = e < P.tol_n;
                if (conv || it - cs->base >= cs->max_iter) {
                    cs->done = 1;
                    cs->converged = conv ? 1 : 0;
                    atomicSub(&P.ctl->active, 1);
                }
            }
        } else if (cs->active) {
            cs->residual64 = fx64_join(w[0], w[1]);
            cs->xsum = fx64_join(w[2], w[3]);
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        P.ctl->queue = 0u;
        P.ctl->exited = 0u;
        if (!kF64) {
            const int32_t launches = P.ctl->launches + 1;
            P.ctl->launches = launches;
            const int32_t active = __ldcg(&P.ctl->active);
            const bool more = active > 0 && launches < P.ctl->cap && (P.step_cap == 0 || launches < P.step_cap);
            if (active > 0 && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
            if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
        }
        __threadfence();
    }
}

// ---- layout ------------------------------------------------------------------------
// Entry stream from the sweep's padded CSR: resolved sources and coefficients;
// entries past the last one are placeholders.
__global__ void k_sp_entries(const int32_t* __restrict__ sw_col, const float* __restrict__ sw_w, int64_t sw_nnz,
                             int64_t epad, const int32_t* __restrict__ hub_ids, int32_t nhub,
                             const double* __restrict__ outw, int32_t n, int32_t* __restrict__ src,
                             float* __restrict__ c32, double* __restrict__ c64) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < epad; e += (int64_t)gridDim.x * blockDim.x) {
        int32_t s = n;
        double cf = 0.0;
        if (e < sw_nnz) {
            const int32_t code = sw_col[e];
            if (code != -(nhub + 1)) {  // not a placeholder
                s = code >= 0 ? code : hub_ids[-code - 1];
                const double o = outw[s];
                const double w = sw_w ? (double)sw_w[e] : 1.0;
                cf = o <= 1e-15 ? 0.0 : w / o;
            } else {
                s = n;
            }
        }
        src[e] = s;
        c32[e] = (float)cf;
        c64[e] = cf;
    }
}

// Bit 31 on the last entry of every row.
__global__ void k_sp_marks(const int32_t* __restrict__ sw_row, int32_t n, int32_t* __restrict__ src) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int32_t e = sw_row[r + 1] - 1;
        src[e] |= kRowEnd;
    }
}

// The row of entry e (every row has at least one entry): the largest r < n
// with sw_row[r] <= e.
__device__ __forceinline__ int32_t row_of(const int32_t* __restrict__ sw_row, int32_t n, int32_t e) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (sw_row[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_sp_chunks(const int32_t* __restrict__ sw_row, int32_t n, int32_t sw_nnz, int32_t C, int32_t nch,
                            SpChunk* __restrict__ out) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    SpChunk k;
    k.e0 = c * C;
    k.e1 = k.e0 + C;
    const int32_t last = min(k.e1, sw_nnz) - 1;  // last real entry of the chunk
    k.r0 = row_of(sw_row, n, k.e0);
    const int32_t rl = row_of(sw_row, n, last);
    const bool head = sw_row[k.r0] < k.e0;
    const bool tail = sw_row[rl + 1] > k.e1;
    k.flags = (head ? kHasHead : 0) | (tail ? kHasTail : 0) | ((head && tail && k.r0 == rl) ? kInterior : 0);
    k.hkey = -1;
    k.hparts = 0;
    k.tparts = 0;
    if (head) {
        k.hkey = sw_row[k.r0] / C;
        k.hparts = ((k.flags & kInterior) ? (sw_row[k.r0 + 1] - 1) / C : c) - k.hkey + 1;
    }
    if (tail && !(k.flags & kInterior)) k.tparts = (sw_row[rl + 1] - 1) / C - c + 1;
    k.trow = rl;
    out[c] = k;
}

// ---- per solve -----------------------------------------------------------------------
// Row meta: dangling bit (out-weight <= 1e-15, pagerank.py:106-108).
__global__ void k_sp_meta(const double* __restrict__ outw, int32_t n, uint32_t* __restrict__ meta) {
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        meta[v] = outw[v] <= 1e-15 ? kDangBit : 0u;
}

// Teleport rows of the seed vertices.
__global__ void k_sp_tele_rows(const int32_t* __restrict__ tv, int32_t nt, uint32_t* __restrict__ meta) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nt) meta[tv[t]] |= (uint32_t)(t + 1);
}

// Teleport rows row0 .. row0 + nt - 1 of a session, for vertices tv[0 .. nt).
__global__ void k_sp_tele_rows_at(const int32_t* __restrict__ tv, int32_t nt, int32_t row0,
                                  uint32_t* __restrict__ meta) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nt) meta[tv[t]] |= (uint32_t)(row0 + t + 1);
}

// Teleport entry writes of a session: tele[at[i]] = val[i] (distinct at).
__global__ void k_sp_tele_write(float* __restrict__ tele, const uint64_t* __restrict__ at,
                                const float* __restrict__ val, int64_t count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) tele[at[i]] = val[i];
}

// X0 = 1/n on live columns, 0 on padding columns and on row n of both
// iterates (grid.y = panel, 16-byte stores); column states.
__global__ void k_sp_init(float* X0, float* X1, ColState* cols, int32_t n, int32_t npanels, int32_t k, double alpha,
                          int32_t ndang, int32_t max_iter) {
    const float x0 = (float)(1.0 / (double)n);
    const int32_t p = blockIdx.y;
    const int64_t quads = ((int64_t)n + 1) * (kLanes / 4);
    float4* a = reinterpret_cast<float4*>(X0 + (size_t)p * ((size_t)n + 1) * kLanes);
    float4* b = reinterpret_cast<float4*>(X1 + (size_t)p * ((size_t)n + 1) * kLanes);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = p * kLanes + 4 * (int32_t)(q & 7);  // first column of the quad
        if ((q >> 3) == n) {
            a[q] = make_float4(0.f, 0.f, 0.f, 0.f);
            b[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            a[q] = make_float4(c < k ? x0 : 0.f, c + 1 < k ? x0 : 0.f, c + 2 < k ? x0 : 0.f, c + 3 < k ? x0 : 0.f);
        }
    }
    const int32_t j = p * kLanes + (int32_t)threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < kLanes) {
        ColState cs;
        cs.dsum = (double)ndang * (double)x0;
        cs.dmass = alpha * cs.dsum / (double)n;
        cs.dmass_prev = cs.dmass;
        cs.residual = 0.0;
        cs.residual64 = 0.0;
        cs.xsum = 0.0;
        cs.iter = 0;
        cs.active = j < k ? 1 : 0;
        cs.done = j < k ? 0 : 1;
        cs.converged = 0;
        cs.base = 0;
        cs.max_iter = max_iter;
        cols[j] = cs;
    }
}

// A session's newly admitted columns start at x0 = 1/n in the iterate their
// panel reads next (X[panel sweeps & 1]); row n stays zero.  Per listed panel
// pn[i]: the bit mask of its new columns and their buffer (all of a panel's
// new columns share its sweep count).  A warp writes one 128-byte row of a
// panel, masked, so the writes are whole lines instead of one sector per value.
__global__ void k_sp_init_cols(float* X0, float* X1, int32_t n, const int32_t* __restrict__ pn,
                               const uint32_t* __restrict__ mask, const int32_t* __restrict__ par, int32_t count) {
    const float x0 = (float)(1.0 / (double)n);
    const int64_t per = (int64_t)n * kLanes;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)count * per;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = (int32_t)(t / per);
        const int64_t r = t - (int64_t)i * per;  // row * 32 + column
        if ((mask[i] >> (r & (kLanes - 1))) & 1u)
            (par[i] ? X1 : X0)[(size_t)pn[i] * ((size_t)n + 1) * kLanes + (size_t)r] = x0;
    }
}

// Rank sum of each column's final FP32 iterate (runs when the FP64 correction
// sweep, which sums its own result, is switched off): FP64 partial sums per
// warp, added as two-word fixed point so the total is independent of order.
__global__ void k_sp_colsum(const float* __restrict__ X0, const float* __restrict__ X1,
                            const ColState* __restrict__ cols, int32_t n, unsigned long long* __restrict__ words) {
    const int32_t p = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const ColState& cs = cols[p * kLanes + lane];
    const float* x = ((cs.iter & 1) ? X1 : X0) + (size_t)p * ((size_t)n + 1) * kLanes;
    double sum = 0.0;
    for (int64_t v = (int64_t)blockIdx.x * nw + warp; v < n; v += (int64_t)gridDim.x * nw)
        sum += (double)x[(size_t)v * kLanes + lane];
    unsigned long long h, l;
    fx64_split(sum, h, l);
    atomicAdd(words + ((size_t)p * 2) * kLanes + lane, h);
    atomicAdd(words + ((size_t)p * 2 + 1) * kLanes + lane, l);
}

__global__ void k_sp_colsum_set(ColState* __restrict__ cols, const unsigned long long* __restrict__ words,
                                int32_t npanels) {
    const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= npanels * kLanes) return;
    const int32_t p = j / kLanes, lane = j - p * kLanes;
    cols[j].xsum = fx64_join(words[((size_t)p * 2) * kLanes + lane], words[((size_t)p * 2 + 1) * kLanes + lane]);
}

// out[j*n + v] = final iterate / its sum (panel-major FP64 or FP32 source),
// transposed through shared memory 128 vertices at a time so that both sides
// are coalesced.
constexpr int kNormRows = 128;
__global__ void __launch_bounds__(256) k_sp_normalize(const double* __restrict__ out64, const float* X0, const float* X1,
                                                      const ColState* __restrict__ cols, int32_t n, int32_t k,
                                                      int32_t from_fp32, double* __restrict__ out,
                                                      const int32_t* __restrict__ out_row) {
    __shared__ double tile[kNormRows][kLanes + 1];
    const int32_t p = blockIdx.y;
    const int32_t v0 = blockIdx.x * kNormRows;
    const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
    const int32_t col = p * kLanes + lane;
    const ColState cs = cols[col];
    const float* xl = ((cs.iter & 1) ? X1 : X0) + (size_t)p * ((size_t)n + 1) * kLanes;
    const double* ol = out64 + (size_t)p * ((size_t)n + 1) * kLanes;
    const double inv = cs.xsum > 0.0 ? 1.0 / cs.xsum : 0.0;
    const double uni = 1.0 / (double)n;
    for (int r = row; r < kNormRows; r += (int)(blockDim.x >> 5)) {
        const int32_t v = v0 + r;
        double val = 0.0;
        if (v < n) {
            const size_t off = (size_t)v * kLanes + lane;
            const double raw = from_fp32 ? (double)xl[off] : ol[off];
            val = cs.xsum > 0.0 ? raw * inv : uni;
        }
        tile[r][lane] = val;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kLanes * kNormRows; idx += blockDim.x) {
        const int jj = idx / kNormRows, i = idx - jj * kNormRows;
        const int32_t j = p * kLanes + jj, v = v0 + i;
        if (j >= k || v >= n) continue;
        const int32_t r = out_row ? out_row[j] : j;  // a session writes only the columns it collects
        if (r >= 0) out[(size_t)r * n + v] = tile[i][jj];
    }
}

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

size_t smem_bytes(bool f64) { return f64 ? sizeof(SpSmem<true>) : sizeof(SpSmem<false>); }

int spmm_grid(bool f64) {
    static std::atomic<int> cached[2][64];  // per device; host threads may race to fill it with the same value
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::atomic<int>& c = cached[f64 ? 1 : 0][dev];
    const int have = c.load(std::memory_order_acquire);
    if (have > 0) return have;
    int sms = 148, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (f64) {
        cudaFuncSetAttribute(k_spmm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(true));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_spmm<true>, sp_threads<true>(), smem_bytes(true));
    } else {
        cudaFuncSetAttribute(k_spmm<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(false));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_spmm<false>, sp_threads<false>(), smem_bytes(false));
    }
    const int grid = sms * std::max(per, 1);
    c.store(grid, std::memory_order_release);
    return grid;
}

}  // namespace

// Default entries per chunk (a multiple of 32).
int32_t default_spmm_chunk() {
    static const int32_t v = [] {
        const char* e = std::getenv("EGPR_SPMM_CHUNK");
        const int x = e ? std::atoi(e) : 1024;
        return (x >= 64 && x <= (1 << 16)) ? (x & ~31) : 1024;
    }();
    return v;
}

// Per-graph SpMM workspace: the layout (entry stream and chunks, built on the
// first batched solve) and the solve buffers, grown to the largest group of
// panels solved so far.
struct SpmmWork {
    int32_t C = 0;
    int32_t nchunks = 0;
    int64_t epad = 0;
    DevBuf src, c32, c64, chunks;
    int32_t cap_panels = 0;
    DevBuf X0, X1, out64, cols, parts, span_cnt, gacc, colsum, ctl, meta, params, out, tele, tele_v;
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t cg_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    int cg_grid = 0;
    bool cg_failed = false;
    ~SpmmWork() {
        if (cg_exec) cudaGraphExecDestroy(cg_exec);
        if (cg) cudaGraphDestroy(cg);
        for (DevBuf* b : buffers()) b->release();
    }
    // Frees the buffers in the order of stream s (no wait for the device, so
    // other graphs' solves on other streams keep running).
    void release_on(cudaStream_t s) {
        for (DevBuf* b : buffers()) b->release_on(s);
    }
    std::array<DevBuf*, 18> buffers() {
        return {&src, &c32, &c64, &chunks, &X0, &X1, &out64, &cols, &parts, &span_cnt, &gacc, &colsum, &ctl,
                &meta, &params, &out, &tele, &tele_v};
    }
};

void spmm_work_release(egpr_graph* g) {
    delete g->spmm;
    g->spmm = nullptr;
}

namespace {

int grid_1d(int64_t work) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 32));
}

int build_spmm_layout(egpr_graph* g, SpmmWork& w, cudaStream_t s) {
    const int32_t n = g->n;
    const int32_t C = std::max(64, g->tune_spmm_chunk & ~31);
    if (g->sw_nnz <= 0 || g->sw_nnz > (int64_t)INT32_MAX - 2 * C) return arg_error("graph too large for the batched solve");
    const int32_t nch = (int32_t)((g->sw_nnz + C - 1) / C);
    const int64_t epad = (int64_t)nch * C;
    int rc;
    if ((rc = w.src.grow_on((size_t)epad * sizeof(int32_t), s)) || (rc = w.c32.grow_on((size_t)epad * sizeof(float), s)) ||
        (rc = w.c64.grow_on((size_t)epad * sizeof(double), s)) || (rc = w.chunks.grow_on((size_t)nch * sizeof(SpChunk), s)))
        return rc;
    k_sp_entries<<<grid_1d(epad), 256, 0, s>>>(g->sw_col.as<int32_t>(), g->weighted ? g->sw_w.as<float>() : nullptr,
                                               g->sw_nnz, epad, g->hub_ids.as<int32_t>(), g->nhub,
                                               g->outw.as<double>(), n, w.src.as<int32_t>(), w.c32.as<float>(),
                                               w.c64.as<double>());
    k_sp_marks<<<grid_1d(n), 256, 0, s>>>(g->sw_row.as<int32_t>(), n, w.src.as<int32_t>());
    k_sp_chunks<<<(nch + 255) / 256, 256, 0, s>>>(g->sw_row.as<int32_t>(), n, (int32_t)g->sw_nnz, C, nch,
                                                  w.chunks.as<SpChunk>());
    if ((rc = cuda_ok(cudaGetLastError(), "SpMM layout"))) return rc;
    w.C = C;
    w.nchunks = nch;
    w.epad = epad;
    return EGPR_SUCC;
}

int ensure_capacity(egpr_graph* g, SpmmWork& w, int32_t npanels, cudaStream_t s) {
    if (w.cap_panels >= npanels) return EGPR_SUCC;
    const int32_t n = g->n;
    const size_t xs = (size_t)npanels * ((size_t)n + 1) * kLanes;
    const size_t units = (size_t)npanels * w.nchunks;
    int rc;
    if ((rc = w.X0.grow_on(xs * sizeof(float), s)) || (rc = w.X1.grow_on(xs * sizeof(float), s)) ||
        (rc = w.out64.grow_on(xs * sizeof(double), s)) ||
        (rc = w.cols.grow_on((size_t)npanels * kLanes * sizeof(ColState), s)) ||
        (rc = w.parts.grow_on(units * 2 * kLanes * sizeof(double), s)) ||
        (rc = w.span_cnt.grow_on(units * sizeof(uint32_t), s)) ||
        (rc = w.gacc.grow_on((size_t)npanels * kAccQ * kLanes * sizeof(unsigned long long), s)) ||
        (rc = w.colsum.grow_on((size_t)npanels * 2 * kLanes * sizeof(unsigned long long), s)) ||
        (rc = w.ctl.grow_on(sizeof(Ctl), s)) || (rc = w.params.grow_on(sizeof(SpmmParams), s)) ||
        (rc = w.meta.grow_on(((size_t)n + 1) * sizeof(uint32_t), s)))
        return rc;
    if ((rc = cuda_ok(cudaMemsetAsync(w.X1.p, 0, xs * sizeof(float), s), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(w.span_cnt.p, 0, units * sizeof(uint32_t), s), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(w.gacc.p, 0, (size_t)npanels * kAccQ * kLanes * sizeof(unsigned long long), s),
                      "memset")))
        return rc;
    // the loop graph holds the parameter block's address
    if (w.cg_exec) cudaGraphExecDestroy(w.cg_exec);
    if (w.cg) cudaGraphDestroy(w.cg);
    w.cg_exec = nullptr;
    w.cg = nullptr;
    w.cg_failed = false;
    w.cap_panels = npanels;
    return EGPR_SUCC;
}

// The sweep loop as a CUDA-graph while node whose body is one k_spmm launch.
void build_loop_graph(SpmmWork& w, int grid) {
    if (w.cg_exec && w.cg_grid != grid) {  // built for another launch size
        cudaGraphExecDestroy(w.cg_exec);
        cudaGraphDestroy(w.cg);
        w.cg_exec = nullptr;
        w.cg = nullptr;
    }
    if (w.cg_exec || w.cg_failed) return;
    const SpmmParams* Pd = w.params.as<SpmmParams>();
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t ex = nullptr;
    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t cnode = nullptr, knode = nullptr;
    cudaGraphNodeParams cp = {};
    bool ok = cudaGraphCreate(&cg, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&h, cg, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&cnode, cg, nullptr, 0, &cp) == cudaSuccess;
    }
    if (ok) {
        int32_t one = 1;
        void* args[3] = {(void*)&Pd, (void*)&h, (void*)&one};
        cudaKernelNodeParams kp = {};
        kp.func = (void*)k_spmm<false>;
        kp.gridDim = dim3((unsigned)grid);
        kp.blockDim = dim3(sp_threads<false>());
        kp.sharedMemBytes = (unsigned)smem_bytes(false);
        kp.kernelParams = args;
        ok = cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp) == cudaSuccess &&
             cudaGraphInstantiate(&ex, cg, 0) == cudaSuccess;
    }
    if (ok) {
        w.cg = cg;
        w.cg_exec = ex;
        w.cond = h;
        w.cg_grid = grid;
    } else {
        cudaGetLastError();
        if (cg) cudaGraphDestroy(cg);
        w.cg_failed = true;
    }
}

using ColEntries = std::vector<std::pair<int32_t, float>>;

// One device solve over columns [j0, j0 + kg) (kg <= kMaxPanels * 32).
int solve_group(egpr_graph* g, SpmmWork& w, double alpha, int32_t max_iter, double tol, int32_t j0, int32_t kg,
                const std::vector<ColEntries>& per_col, uint32_t flags, double* out, egpr_stats* stats) {
    const double t0 = wall_seconds();
    const int32_t n = g->n;
    cudaStream_t s = g->stream;
    const int32_t npanels = (kg + kLanes - 1) / kLanes;
    int rc;
    if ((rc = ensure_capacity(g, w, npanels, s))) return rc;
    // teleport rows: one per vertex that has a teleport entry in the group
    const int32_t ld = npanels * kLanes;
    std::vector<int32_t> tidx((size_t)n, -1), tv;
    for (int32_t jj = 0; jj < kg; ++jj)
        for (const auto& pr : per_col[(size_t)(j0 + jj)])
            if (tidx[(size_t)pr.first] < 0) {
                tidx[(size_t)pr.first] = (int32_t)tv.size();
                tv.push_back(pr.first);
            }
    const int32_t nt = (int32_t)tv.size();
    std::vector<float> tt((size_t)std::max(nt, 1) * ld, 0.f);
    for (int32_t jj = 0; jj < kg; ++jj)
        for (const auto& pr : per_col[(size_t)(j0 + jj)]) tt[(size_t)tidx[(size_t)pr.first] * ld + jj] = pr.second;
    if ((rc = w.tele.grow_on(tt.size() * sizeof(float), s)) ||
        (rc = w.tele_v.grow_on((size_t)std::max(nt, 1) * sizeof(int32_t), s)) ||
        (rc = w.out.grow_on((size_t)kg * n * sizeof(double), s)))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(w.tele.p, tt.data(), tt.size() * sizeof(float), cudaMemcpyHostToDevice, s),
                      "H2D teleport")) ||
        (nt > 0 && (rc = cuda_ok(cudaMemcpyAsync(w.tele_v.p, tv.data(), (size_t)nt * sizeof(int32_t),
                                                 cudaMemcpyHostToDevice, s), "H2D teleport"))))
        return rc;

    SpmmParams P;
    std::memset(&P, 0, sizeof(P));
    P.chunks = w.chunks.as<SpChunk>();
    P.nchunks = w.nchunks;
    P.npanels = npanels;
    P.n = n;
    P.tele_ld = ld;
    P.max_iter = max_iter;
    P.src = w.src.as<int32_t>();
    P.coef32 = w.c32.as<float>();
    P.coef64 = w.c64.as<double>();
    P.meta = w.meta.as<uint32_t>();
    P.tele = w.tele.as<float>();
    P.X[0] = w.X0.as<float>();
    P.X[1] = w.X1.as<float>();
    P.out64 = w.out64.as<double>();
    P.cols = w.cols.as<ColState>();
    P.alpha = alpha;
    P.alpha_hi = (float)alpha;
    P.alpha_lo = (float)(alpha - (double)P.alpha_hi);
    P.oma_hi = (float)(1.0 - alpha);
    P.oma_lo = (float)((1.0 - alpha) - (double)P.oma_hi);
    P.tol_n = tol * (double)n;
    P.parts = w.parts.p;
    P.span_cnt = w.span_cnt.as<uint32_t>();
    P.gacc = w.gacc.as<unsigned long long>();
    P.ctl = w.ctl.as<Ctl>();
    Ctl c{};
    c.active = kg;
    c.cap = max_iter + 1;
    if ((rc = cuda_ok(cudaMemcpyAsync(w.params.p, &P, sizeof(P), cudaMemcpyHostToDevice, s), "H2D params")) ||
        (rc = cuda_ok(cudaMemcpyAsync(w.ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, s), "H2D ctl")))
        return rc;
    const SpmmParams* Pd = w.params.as<SpmmParams>();
    // the SpMM does about four times the work of a single-vector sweep per entry and panel
    const int64_t work = 4 * (int64_t)npanels * w.epad;
    const int grid = work_grid(work, spmm_grid(false));
    const int grid64 = work_grid(work, spmm_grid(true));
    if ((rc = cuda_ok(cudaEventRecord(g->ev0, s), "event"))) return rc;
    k_sp_meta<<<grid_1d(n), 256, 0, s>>>(g->outw.as<double>(), n, w.meta.as<uint32_t>());
    if (nt > 0) k_sp_tele_rows<<<(nt + 255) / 256, 256, 0, s>>>(w.tele_v.as<int32_t>(), nt, w.meta.as<uint32_t>());
    k_sp_init<<<dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n + 1) * 8 / 256 + 1, 148 * 8)),
                     (unsigned)npanels), 256, 0, s>>>(
        w.X0.as<float>(), w.X1.as<float>(), w.cols.as<ColState>(), n, npanels, kg, alpha, g->n_dangling_solve, max_iter);
    int32_t launches = nt > 0 ? 3 : 2;
    if (graph_loop_enabled()) build_loop_graph(w, grid);
    if (w.cg_exec && graph_loop_enabled()) {
        if ((rc = cuda_ok(cudaGraphLaunch(w.cg_exec, s), "graph launch"))) return rc;
    } else {
        for (int32_t it = 0; it < max_iter; ++it) k_spmm<false><<<grid, sp_threads<false>(), smem_bytes(false), s>>>(Pd, 0, 0);
        if ((rc = cuda_ok(cudaGetLastError(), "spmm launch"))) return rc;
    }
    const bool correction = (flags & EGPR_FLAG_NO_CORRECTION) == 0;
    if (correction) {
        k_spmm<true><<<grid64, sp_threads<true>(), smem_bytes(true), s>>>(Pd, 0, 0);
        launches += 1;
    }
    if (!correction) {
        if ((rc = cuda_ok(cudaMemsetAsync(w.colsum.p, 0, (size_t)npanels * 2 * kLanes * sizeof(unsigned long long), s),
                          "memset")))
            return rc;
        k_sp_colsum<<<dim3(148, (unsigned)npanels), 256, 0, s>>>(w.X0.as<float>(), w.X1.as<float>(),
                                                                 w.cols.as<ColState>(), n,
                                                                 w.colsum.as<unsigned long long>());
        k_sp_colsum_set<<<(npanels * kLanes + 255) / 256, 256, 0, s>>>(w.cols.as<ColState>(),
                                                                       w.colsum.as<unsigned long long>(), npanels);
        launches += 2;
    }
    {
        dim3 gr((unsigned)((n + kNormRows - 1) / kNormRows), (unsigned)npanels);
        k_sp_normalize<<<gr, 256, 0, s>>>(w.out64.as<double>(), w.X0.as<float>(), w.X1.as<float>(),
                                          w.cols.as<ColState>(), n, kg, correction ? 0 : 1, w.out.as<double>(),
                                          nullptr);
        launches += 1;
    }
    if ((rc = cuda_ok(cudaGetLastError(), "spmm finish"))) return rc;
    if ((rc = cuda_ok(cudaEventRecord(g->ev1, s), "event"))) return rc;
    // out == NULL: device timing only (the tuner)
    if (out && (rc = download_d2h(out, w.out.p, (size_t)kg * n * sizeof(double), s, "D2H ranks"))) return rc;
    std::vector<ColState> hc((size_t)npanels * kLanes);
    Ctl ctl;
    if ((rc = cuda_ok(cudaMemcpyAsync(hc.data(), w.cols.p, hc.size() * sizeof(ColState), cudaMemcpyDeviceToHost, s),
                      "D2H cols")) ||
        (rc = cuda_ok(cudaMemcpyAsync(&ctl, w.ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "batch solve")))
        return rc;
    if (ctl.error) return ctl.error;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    if (stats) {
        // compulsory bytes of one sweep: per panel the entry stream, the
        // previous and the next iterate, and the row meta
        const int64_t bytes = (int64_t)npanels * (w.epad * 8 + 2 * ((int64_t)n + 1) * kLanes * 4 + 4 * (int64_t)n);
        for (int32_t jj = 0; jj < kg; ++jj) {
            egpr_stats& st = stats[jj];
            st.iterations = hc[(size_t)jj].iter;
            st.converged = hc[(size_t)jj].converged;
            st.residual = hc[(size_t)jj].residual;
            st.kernel_seconds = ms * 1e-3;
            st.total_seconds = wall_seconds() - t0;
            st.bytes_per_iter = bytes;
            st.launches = launches + ctl.launches;
            st.reserved = 0;
        }
    }
    return EGPR_SUCC;
}

}  // namespace

int ppr_batch_solve(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k,
                    const double* teleport_dense, const int32_t* seed_ptr, const int32_t* seeds, uint32_t flags,
                    double* out, egpr_stats* stats) {
    const double t0 = wall_seconds();
    int rc;
    if ((rc = check_device(g))) return rc;
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    const int32_t n = g->n;
    // teleport entries per column: (vertex, probability)
    std::vector<ColEntries> per_col((size_t)k);
    for (int32_t j = 0; j < k; ++j) {
        auto& ent = per_col[(size_t)j];
        if (teleport_dense) {
            const double* pj = teleport_dense + (size_t)j * n;
            double sum = 0.0;
            for (int32_t v = 0; v < n; ++v) {
                if (!(pj[v] >= 0.0) || !std::isfinite(pj[v])) return EGPR_INVALID_ARGUMENT;
                sum += pj[v];
            }
            if (!(sum > 0.0)) return EGPR_INVALID_ARGUMENT;
            for (int32_t v = 0; v < n; ++v)
                if (pj[v] > 0.0) ent.emplace_back(v, (float)(pj[v] / sum));
        } else {
            const int32_t b = seed_ptr[j], e = seed_ptr[j + 1];
            if (e <= b || b < 0) return EGPR_INVALID_ARGUMENT;
            std::vector<int32_t> sv(seeds + b, seeds + e);
            std::sort(sv.begin(), sv.end());
            sv.erase(std::unique(sv.begin(), sv.end()), sv.end());
            if (sv.front() < 0 || sv.back() >= n) return EGPR_INVALID_ARGUMENT;
            const float val = (float)(1.0 / (double)sv.size());
            for (int32_t v : sv) ent.emplace_back(v, val);
        }
    }
    if (g->nnz == 0) {  // pagerank.py:96-98: no edges -> uniform
        if (out)
            for (size_t i = 0; i < (size_t)k * n; ++i) out[i] = 1.0 / n;
        if (stats)
            for (int32_t j = 0; j < k; ++j) {
                std::memset(&stats[j], 0, sizeof(egpr_stats));
                stats[j].total_seconds = wall_seconds() - t0;
            }
        return EGPR_SUCC;
    }
    if (!g->spmm) g->spmm = new SpmmWork();
    SpmmWork& w = *g->spmm;
    cudaStream_t s = g->stream;
    if (!w.C && (rc = build_spmm_layout(g, w, s))) return rc;
    // device solves of up to kMaxPanels panels each
    constexpr int32_t kGroup = kMaxPanels * kLanes;
    for (int32_t j0 = 0; j0 < k; j0 += kGroup) {
        const int32_t kg = std::min(kGroup, k - j0);
        if ((rc = solve_group(g, w, alpha, max_iter, tol, j0, kg, per_col, flags, out ? out + (size_t)j0 * n : nullptr,
                              stats ? stats + j0 : nullptr)))
            return rc;
    }
    if (stats && k > kGroup) {  // the whole batch's device time in every column
        double ks = 0.0;
        for (int32_t j0 = 0; j0 < k; j0 += kGroup) ks += stats[j0].kernel_seconds;
        for (int32_t j = 0; j < k; ++j) {
            stats[j].kernel_seconds = ks;
            stats[j].total_seconds = wall_seconds() - t0;
        }
    }
    return EGPR_SUCC;
}


// ---- continuous batching: a session of column slots ------------------------
// No counterpart in the reference.  A session keeps one batched solve of a
// graph running: requests join it in free column slots between steps of a
// few sweeps, each column keeps its own stop rule and sweep count, and a
// finished column is collected (FP64 correction sweep, normalisation, D2H)
// and its slot freed while the others keep sweeping.  Live columns of a
// 32-column panel share the parity of their iterate buffers, so a column that
// joins a panel starts at the panel's sweep count and counts its own sweeps
// from there (ColState::base).
namespace {
constexpr uint8_t kSlotFree = 0, kSlotRunning = 1, kSlotDone = 2;

struct SessionState {
    egpr_graph* g = nullptr;
    SpmmWork w;                       // solve buffers; the entry stream is the graph's (g->spmm)
    double alpha = 0.85, tol = 0.0;
    int32_t slots = 0, npanels = 0;
    std::vector<ColState> cols;       // host mirror of the column states
    std::vector<int32_t> panel_sweeps;
    std::vector<uint8_t> state;
    std::vector<std::vector<int32_t>> rows_of;  // per slot: its teleport rows
    std::vector<double> started, device_s;      // per slot: admission time, device time while live
    std::unordered_map<int32_t, int32_t> row_of_vertex;
    std::vector<int32_t> row_vertex;  // teleport row -> vertex
    // teleport matrix (rows x npanels * 32) on the device only: admissions and
    // collections queue entry writes (last write wins), applied by a scatter
    // before the next step
    std::unordered_map<uint64_t, float> tele_writes;
    int32_t tele_cap_rows = 0;        // rows the device teleport buffer holds
    int32_t rows_on_device = 0;       // rows whose meta bits are set
    bool tele_dirty = false;
    // what the device holds: the column states equal the host mirror unless
    // an admission or a collection changed them since; the parameter block is
    // that of params_cap (-1: stale)
    bool cols_dirty = true;
    int32_t params_cap = -1;
    DevBuf out_row, tele_upd;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~SessionState() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        // stream-ordered frees: closing a session does not wait for the
        // solves of other graphs running on other streams
        if (g) {
            w.release_on(g->stream);
            out_row.release_on(g->stream);
            tele_upd.release_on(g->stream);
        }
        out_row.release();
    }
};

int session_params(SessionState& S, int32_t step_cap, cudaStream_t s) {
    if (S.params_cap == step_cap) return EGPR_SUCC;  // the device already holds this block
    egpr_graph* g = S.g;
    SpmmWork& base = *g->spmm;
    SpmmWork& w = S.w;
    SpmmParams P;
    std::memset(&P, 0, sizeof(P));
    P.chunks = base.chunks.as<SpChunk>();
    P.nchunks = base.nchunks;
    P.npanels = S.npanels;
    P.n = g->n;
    P.tele_ld = S.npanels * kLanes;
    P.max_iter = 1 << 30;
    P.src = base.src.as<int32_t>();
    P.coef32 = base.c32.as<float>();
    P.coef64 = base.c64.as<double>();
    P.meta = w.meta.as<uint32_t>();
    P.tele = w.tele.as<float>();
    P.X[0] = w.X0.as<float>();
    P.X[1] = w.X1.as<float>();
    P.out64 = w.out64.as<double>();
    P.cols = w.cols.as<ColState>();
    P.alpha = S.alpha;
    P.alpha_hi = (float)S.alpha;
    P.alpha_lo = (float)(S.alpha - (double)P.alpha_hi);
    P.oma_hi = (float)(1.0 - S.alpha);
    P.oma_lo = (float)((1.0 - S.alpha) - (double)P.oma_hi);
    P.tol_n = S.tol * (double)g->n;
    P.parts = w.parts.p;
    P.span_cnt = w.span_cnt.as<uint32_t>();
    P.gacc = w.gacc.as<unsigned long long>();
    P.ctl = w.ctl.as<Ctl>();
    P.step_cap = step_cap;
    const int rc = cuda_ok(cudaMemcpyAsync(w.params.p, &P, sizeof(P), cudaMemcpyHostToDevice, s), "H2D params");
    S.params_cap = rc ? -1 : step_cap;
    return rc;
}

int session_upload(SessionState& S, int32_t active, cudaStream_t s) {
    SpmmWork& w = S.w;
    int rc;
    if (S.tele_dirty) {
        const int32_t nrows = (int32_t)S.row_vertex.size();
        const size_t ld = (size_t)S.npanels * kLanes;
        if (nrows > S.tele_cap_rows) {  // grow: zeroed, the old rows copied over
            const int32_t cap = std::max(nrows, std::max(2 * S.tele_cap_rows, 256));
            DevBuf nb;
            if ((rc = nb.grow_on((size_t)cap * ld * sizeof(float), s))) return rc;
            if ((rc = cuda_ok(cudaMemsetAsync(nb.p, 0, (size_t)cap * ld * sizeof(float), s), "memset")) ||
                (S.tele_cap_rows > 0 &&
                 (rc = cuda_ok(cudaMemcpyAsync(nb.p, w.tele.p, (size_t)S.tele_cap_rows * ld * sizeof(float),
                                               cudaMemcpyDeviceToDevice, s), "D2D teleport")))) {
                nb.release_on(s);
                return rc;
            }
            w.tele.release_on(s);
            w.tele = nb;
            S.tele_cap_rows = cap;
            S.params_cap = -1;  // the parameter block holds the teleport buffer's address
        }
        const size_t nw = S.tele_writes.size();
        if (nw > 0) {
            std::vector<uint64_t> at;
            std::vector<float> val;
            at.reserve(nw);
            val.reserve(nw);
            for (const auto& kv : S.tele_writes) {
                at.push_back(kv.first);
                val.push_back(kv.second);
            }
            if ((rc = S.tele_upd.grow_on(nw * (sizeof(uint64_t) + sizeof(float)), s)) ||
                (rc = cuda_ok(cudaMemcpyAsync(S.tele_upd.p, at.data(), nw * sizeof(uint64_t), cudaMemcpyHostToDevice, s),
                              "H2D teleport writes")) ||
                (rc = cuda_ok(cudaMemcpyAsync(S.tele_upd.as<uint64_t>() + nw, val.data(), nw * sizeof(float),
                                              cudaMemcpyHostToDevice, s), "H2D teleport writes")))
                return rc;
            k_sp_tele_write<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(
                w.tele.as<float>(), S.tele_upd.as<uint64_t>(),
                reinterpret_cast<const float*>(S.tele_upd.as<uint64_t>() + nw), (int64_t)nw);
            // the host arrays may go: pageable copies return once their data is staged
            S.tele_writes.clear();
        }
        if (nrows > S.rows_on_device) {
            const int32_t nt = nrows - S.rows_on_device;
            if ((rc = w.tele_v.grow_on((size_t)nt * sizeof(int32_t), s)) ||
                (rc = cuda_ok(cudaMemcpyAsync(w.tele_v.p, S.row_vertex.data() + S.rows_on_device,
                                              (size_t)nt * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D rows")))
                return rc;
            k_sp_tele_rows_at<<<(nt + 255) / 256, 256, 0, s>>>(w.tele_v.as<int32_t>(), nt, S.rows_on_device,
                                                               w.meta.as<uint32_t>());
            S.rows_on_device = nrows;
        }
        S.tele_dirty = false;
    }
    Ctl c{};
    c.active = active;
    c.cap = 1 << 30;
    if (S.cols_dirty) {
        if ((rc = cuda_ok(cudaMemcpyAsync(w.cols.p, S.cols.data(), S.cols.size() * sizeof(ColState),
                                          cudaMemcpyHostToDevice, s), "H2D cols")))
            return rc;
        S.cols_dirty = false;
    }
    return cuda_ok(cudaMemcpyAsync(w.ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, s), "H2D ctl");
}

int session_create(egpr_graph* g, double alpha, double tol, int32_t slots, SessionState** out) {
    *out = nullptr;
    int rc;
    if ((rc = check_device(g))) return rc;
    if (g->nnz <= 0) return arg_error("a session needs a graph with inbound entries");
    if (!(alpha >= 0.0 && alpha < 1.0)) return arg_error("alpha must be in [0, 1)");
    if (slots < 1 || slots > kMaxPanels * kLanes) return arg_error("slots must be in [1, 512]");
    cudaStream_t s = g->stream;
    if (!g->spmm) g->spmm = new SpmmWork();
    if (!g->spmm->C && (rc = build_spmm_layout(g, *g->spmm, s))) return rc;
    SessionState* S = new SessionState();
    S->g = g;
    S->alpha = alpha;
    S->tol = tol > 0.0 ? tol : 0.0;
    S->npanels = (slots + kLanes - 1) / kLanes;
    S->slots = S->npanels * kLanes;
    S->w.C = g->spmm->C;
    S->w.nchunks = g->spmm->nchunks;
    S->w.epad = g->spmm->epad;
    if ((rc = ensure_capacity(g, S->w, S->npanels, s)) ||
        (rc = cuda_ok(cudaMemsetAsync(S->w.X0.p, 0, S->w.X0.bytes, s), "memset")) ||
        (rc = S->out_row.alloc((size_t)S->slots * sizeof(int32_t))) ||
        (rc = cuda_ok(cudaEventCreate(&S->e0), "event")) || (rc = cuda_ok(cudaEventCreate(&S->e1), "event"))) {
        delete S;
        return rc;
    }
    k_sp_meta<<<grid_1d(g->n), 256, 0, s>>>(g->outw.as<double>(), g->n, S->w.meta.as<uint32_t>());
    ColState free_col;
    std::memset(&free_col, 0, sizeof(free_col));
    free_col.done = 1;
    S->cols.assign((size_t)S->slots, free_col);
    S->panel_sweeps.assign((size_t)S->npanels, 0);
    S->state.assign((size_t)S->slots, kSlotFree);
    S->rows_of.assign((size_t)S->slots, {});
    S->started.assign((size_t)S->slots, 0.0);
    S->device_s.assign((size_t)S->slots, 0.0);
    if ((rc = cuda_ok(cudaStreamSynchronize(s), "session"))) {
        delete S;
        return rc;
    }
    *out = S;
    return EGPR_SUCC;
}

int session_admit(SessionState& S, int32_t count, const int32_t* seed_ptr, const int32_t* seeds, int32_t max_iter,
                  int32_t* slots_out) {
    egpr_graph* g = S.g;
    const int32_t n = g->n;
    if (max_iter < 1) max_iter = 1;
    std::vector<int32_t> free_slots;
    for (int32_t j = 0; j < S.slots && (int32_t)free_slots.size() < count; ++j)
        if (S.state[(size_t)j] == kSlotFree) free_slots.push_back(j);
    if ((int32_t)free_slots.size() < count) return arg_error("not enough free slots in the session");
    std::vector<std::vector<int32_t>> sets((size_t)count);
    for (int32_t i = 0; i < count; ++i) {
        const int32_t b = seed_ptr[i], e = seed_ptr[i + 1];
        if (e <= b || b < 0) return arg_error("every request needs at least one seed");
        std::vector<int32_t> sv(seeds + b, seeds + e);
        std::sort(sv.begin(), sv.end());
        sv.erase(std::unique(sv.begin(), sv.end()), sv.end());
        if (sv.front() < 0 || sv.back() >= n) return arg_error("seed ids must lie in [0, n)");
        sets[(size_t)i] = std::move(sv);
    }
    const int32_t ld = S.npanels * kLanes;
    std::vector<uint32_t> panel_mask((size_t)S.npanels, 0u);
    std::vector<int32_t> panel_par((size_t)S.npanels, 0);
    const double x0 = (double)(float)(1.0 / (double)n);
    const double t0 = wall_seconds();
    for (int32_t i = 0; i < count; ++i) {
        const int32_t j = free_slots[(size_t)i], p = j / kLanes;
        const float val = (float)(1.0 / (double)sets[(size_t)i].size());
        for (int32_t v : sets[(size_t)i]) {
            auto it = S.row_of_vertex.find(v);
            int32_t r;
            if (it == S.row_of_vertex.end()) {
                r = (int32_t)S.row_vertex.size();
                S.row_of_vertex.emplace(v, r);
                S.row_vertex.push_back(v);
            } else {
                r = it->second;
            }
            S.tele_writes[(uint64_t)r * (uint64_t)ld + (uint64_t)j] = val;
            S.rows_of[(size_t)j].push_back(r);
        }
        // the panel's sweep count: that of its live columns, if any
        ColState& cs = S.cols[(size_t)j];
        std::memset(&cs, 0, sizeof(cs));
        const int32_t base = S.panel_sweeps[(size_t)p];
        cs.dsum = (double)g->n_dangling_solve * x0;
        cs.dmass = S.alpha * cs.dsum / (double)n;
        cs.dmass_prev = cs.dmass;
        cs.iter = base;
        cs.base = base;
        cs.max_iter = max_iter;
        cs.active = 1;
        cs.done = 0;
        S.state[(size_t)j] = kSlotRunning;
        S.started[(size_t)j] = t0;
        S.device_s[(size_t)j] = 0.0;
        panel_mask[(size_t)p] |= 1u << (j - p * kLanes);
        panel_par[(size_t)p] = base & 1;  // every new column of the panel starts at its sweep count
        slots_out[i] = j;
    }
    S.tele_dirty = true;
    S.cols_dirty = true;
    // the new columns' start vectors (stream order: before the next step)
    cudaStream_t s = g->stream;
    int rc;
    std::vector<int32_t> lst;  // panel, mask, buffer of each panel with new columns
    for (int32_t p = 0; p < S.npanels; ++p)
        if (panel_mask[(size_t)p]) lst.push_back(p);
    const size_t cn = lst.size();
    for (size_t i = 0; i < cn; ++i) lst.push_back((int32_t)panel_mask[(size_t)lst[i]]);
    for (size_t i = 0; i < cn; ++i) lst.push_back(panel_par[(size_t)lst[i]]);
    if ((rc = S.w.colsum.grow_on(lst.size() * sizeof(int32_t), s)) ||
        (rc = cuda_ok(cudaMemcpyAsync(S.w.colsum.p, lst.data(), lst.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                      s), "H2D columns")))
        return rc;
    const int32_t* dl = S.w.colsum.as<int32_t>();
    k_sp_init_cols<<<grid_1d((int64_t)cn * n * kLanes), 256, 0, s>>>(
        S.w.X0.as<float>(), S.w.X1.as<float>(), n, dl, reinterpret_cast<const uint32_t*>(dl + cn), dl + 2 * cn,
        (int32_t)cn);
    if ((rc = cuda_ok(cudaGetLastError(), "session admit"))) return rc;
    // the colsum buffer is reused by the next call: the copies must be done
    return cuda_ok(cudaStreamSynchronize(s), "session admit");
}

int session_step(SessionState& S, int32_t sweeps, int32_t* done_slots, int32_t* ndone) {
    egpr_graph* g = S.g;
    cudaStream_t s = g->stream;
    *ndone = 0;
    int32_t live = 0;
    for (int32_t j = 0; j < S.slots; ++j) live += S.state[(size_t)j] == kSlotRunning ? 1 : 0;
    int rc;
    if (live > 0 && sweeps > 0) {
        if ((rc = session_upload(S, live, s)) || (rc = session_params(S, sweeps, s))) return rc;
        const int64_t work = 4 * (int64_t)S.npanels * S.w.epad;
        const int grid = work_grid(work, spmm_grid(false));
        if ((rc = cuda_ok(cudaEventRecord(S.e0, s), "event"))) return rc;
        const SpmmParams* Pd = S.w.params.as<SpmmParams>();
        if (graph_loop_enabled()) build_loop_graph(S.w, grid);
        if (S.w.cg_exec && graph_loop_enabled()) {
            if ((rc = cuda_ok(cudaGraphLaunch(S.w.cg_exec, s), "graph launch"))) return rc;
        } else {
            for (int32_t it = 0; it < sweeps; ++it)
                k_spmm<false><<<grid, sp_threads<false>(), smem_bytes(false), s>>>(Pd, 0, 0);
            if ((rc = cuda_ok(cudaGetLastError(), "spmm launch"))) return rc;
        }
        if ((rc = cuda_ok(cudaEventRecord(S.e1, s), "event"))) return rc;
        Ctl ctl;
        if ((rc = cuda_ok(cudaMemcpyAsync(S.cols.data(), S.w.cols.p, S.cols.size() * sizeof(ColState),
                                          cudaMemcpyDeviceToHost, s), "D2H cols")) ||
            (rc = cuda_ok(cudaMemcpyAsync(&ctl, S.w.ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
            (rc = cuda_ok(cudaStreamSynchronize(s), "session step")))
            return rc;
        if (ctl.error) return ctl.error;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, S.e0, S.e1);
        for (int32_t j = 0; j < S.slots; ++j)
            if (S.state[(size_t)j] == kSlotRunning) {
                S.device_s[(size_t)j] += ms * 1e-3;
                if (S.cols[(size_t)j].done) S.state[(size_t)j] = kSlotDone;
            }
        // A panel's sweep count (the parity of its iterate buffers) is that of
        // its columns still running: one that stopped inside the step holds
        // an older count, and a column admitted next would start in the wrong
        // buffer.  A panel with no running column keeps its count.
        for (int32_t j = 0; j < S.slots; ++j)
            if (S.state[(size_t)j] == kSlotRunning) S.panel_sweeps[(size_t)(j / kLanes)] = S.cols[(size_t)j].iter;
    }
    for (int32_t j = 0; j < S.slots; ++j)
        if (S.state[(size_t)j] == kSlotDone) done_slots[(*ndone)++] = j;
    return EGPR_SUCC;
}

int session_collect(SessionState& S, int32_t count, const int32_t* slots, uint32_t flags, double* out,
                    egpr_stats* stats) {
    egpr_graph* g = S.g;
    const int32_t n = g->n;
    cudaStream_t s = g->stream;
    for (int32_t i = 0; i < count; ++i)
        if (slots[i] < 0 || slots[i] >= S.slots || S.state[(size_t)slots[i]] != kSlotDone)
            return arg_error("only finished slots can be collected");
    // the FP64 correction and the normalisation see only the collected columns
    std::vector<ColState> view = S.cols;
    std::vector<int32_t> out_row((size_t)S.slots, -1);
    for (ColState& c : view) c.active = 0;
    for (int32_t i = 0; i < count; ++i) {
        view[(size_t)slots[i]].active = 1;
        out_row[(size_t)slots[i]] = i;
    }
    int rc;
    const bool correction = (flags & EGPR_FLAG_NO_CORRECTION) == 0;
    if ((rc = S.w.out.grow_on((size_t)count * n * sizeof(double), s)) ||
        (rc = cuda_ok(cudaMemcpyAsync(S.w.cols.p, view.data(), view.size() * sizeof(ColState), cudaMemcpyHostToDevice, s),
                      "H2D cols")) ||
        (rc = cuda_ok(cudaMemcpyAsync(S.out_row.p, out_row.data(), out_row.size() * sizeof(int32_t),
                                      cudaMemcpyHostToDevice, s), "H2D rows")) ||
        (rc = session_params(S, 0, s)))
        return rc;
    if ((rc = cuda_ok(cudaEventRecord(S.e0, s), "event"))) return rc;
    const int64_t work = 4 * (int64_t)S.npanels * S.w.epad;
    const SpmmParams* Pd = S.w.params.as<SpmmParams>();
    if (correction) {
        k_spmm<true><<<work_grid(work, spmm_grid(true)), sp_threads<true>(), smem_bytes(true), s>>>(Pd, 0, 0);
    } else {
        if ((rc = cuda_ok(cudaMemsetAsync(S.w.colsum.p, 0, (size_t)S.npanels * 2 * kLanes * sizeof(unsigned long long),
                                          s), "memset")))
            return rc;
        k_sp_colsum<<<dim3(148, (unsigned)S.npanels), 256, 0, s>>>(S.w.X0.as<float>(), S.w.X1.as<float>(),
                                                                   S.w.cols.as<ColState>(), n,
                                                                   S.w.colsum.as<unsigned long long>());
        k_sp_colsum_set<<<(S.npanels * kLanes + 255) / 256, 256, 0, s>>>(S.w.cols.as<ColState>(),
                                                                         S.w.colsum.as<unsigned long long>(),
                                                                         S.npanels);
    }
    dim3 gr((unsigned)((n + kNormRows - 1) / kNormRows), (unsigned)S.npanels);
    k_sp_normalize<<<gr, 256, 0, s>>>(S.w.out64.as<double>(), S.w.X0.as<float>(), S.w.X1.as<float>(),
                                      S.w.cols.as<ColState>(), n, S.slots, correction ? 0 : 1, S.w.out.as<double>(),
                                      S.out_row.as<int32_t>());
    if ((rc = cuda_ok(cudaGetLastError(), "session collect"))) return rc;
    if ((rc = cuda_ok(cudaEventRecord(S.e1, s), "event"))) return rc;
    if (out && (rc = download_d2h(out, S.w.out.p, (size_t)count * n * sizeof(double), s, "D2H ranks")))
        return rc;
    if ((rc = cuda_ok(cudaStreamSynchronize(s), "session collect"))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S.e0, S.e1);
    const int32_t ld = S.npanels * kLanes;
    const double now = wall_seconds();
    for (int32_t i = 0; i < count; ++i) {
        const int32_t j = slots[i];
        const ColState& c = S.cols[(size_t)j];
        if (stats) {
            egpr_stats& st = stats[i];
            std::memset(&st, 0, sizeof(st));
            st.iterations = c.iter - c.base;
            st.converged = c.converged;
            st.residual = c.residual;
            st.kernel_seconds = S.device_s[(size_t)j] + ms * 1e-3;
            st.total_seconds = now - S.started[(size_t)j];
            st.bytes_per_iter = (int64_t)S.npanels * (S.w.epad * 8 + 2 * ((int64_t)n + 1) * kLanes * 4 + 4 * (int64_t)n);
        }
        // free the slot: its teleport entries go, its state is a free column again
        for (int32_t r : S.rows_of[(size_t)j]) S.tele_writes[(uint64_t)r * (uint64_t)ld + (uint64_t)j] = 0.f;
        S.rows_of[(size_t)j].clear();
        std::memset(&S.cols[(size_t)j], 0, sizeof(ColState));
        S.cols[(size_t)j].done = 1;
        S.state[(size_t)j] = kSlotFree;
    }
    S.tele_dirty = true;
    S.cols_dirty = true;  // the device holds the collection's view of the states
    return EGPR_SUCC;
}

}  // namespace

}  // namespace egpr


// ---- C ABI of the sessions ---------------------------------------------------
extern "C" {

struct egpr_session {
    egpr::SessionState* st;
};

int egpr_session_create(egpr_graph* g, double alpha, double tol, int32_t slots, egpr_session** out) {
    using namespace egpr;
    if (!g || !out) return arg_error("NULL argument");
    *out = nullptr;
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pending) return arg_error("a solve is pending on this graph");
    SessionState* S = nullptr;
    int rc = session_create(g, alpha, tol, slots, &S);
    if (rc) return rc;
    egpr_session* h = new (std::nothrow) egpr_session{S};
    if (!h) {
        delete S;
        return EGPR_FAILED_TO_ALLOCATE_HOST_MEM;
    }
    g->sessions += 1;
    *out = h;
    return EGPR_SUCC;
}

int egpr_session_admit(egpr_session* h, int32_t count, const int32_t* seed_ptr, const int32_t* seeds,
                       int32_t max_iter, int32_t* slots_out) {
    using namespace egpr;
    if (!h || !h->st) return arg_error("NULL session");
    if (count < 0 || (count > 0 && (!seed_ptr || !seeds || !slots_out))) return arg_error("NULL argument");
    if (count == 0) return EGPR_SUCC;
    SessionState& S = *h->st;
    std::lock_guard<std::mutex> lk(S.g->mu);
    int rc;
    if ((rc = check_device(S.g))) return rc;
    return session_admit(S, count, seed_ptr, seeds, max_iter, slots_out);
}

int egpr_session_step(egpr_session* h, int32_t sweeps, int32_t* done_slots, int32_t* ndone) {
    using namespace egpr;
    if (!h || !h->st) return arg_error("NULL session");
    if (!done_slots || !ndone) return arg_error("NULL argument");
    SessionState& S = *h->st;
    std::lock_guard<std::mutex> lk(S.g->mu);
    int rc;
    if ((rc = check_device(S.g))) return rc;
    return session_step(S, sweeps, done_slots, ndone);
}

int egpr_session_collect(egpr_session* h, int32_t count, const int32_t* slots, uint32_t flags, double* out,
                         egpr_stats* stats) {
    using namespace egpr;
    if (!h || !h->st) return arg_error("NULL session");
    if (count < 0 || (count > 0 && !slots)) return arg_error("NULL argument");
    if (count == 0) return EGPR_SUCC;
    SessionState& S = *h->st;
    std::lock_guard<std::mutex> lk(S.g->mu);
    int rc;
    if ((rc = check_device(S.g))) return rc;
    return session_collect(S, count, slots, flags, out, stats);
}

int egpr_session_info(const egpr_session* h, int32_t* slots, int32_t* running, int32_t* done) {
    using namespace egpr;
    if (!h || !h->st || !slots || !running || !done) return arg_error("NULL argument");
    const SessionState& S = *h->st;
    *slots = S.slots;
    *running = 0;
    *done = 0;
    for (uint8_t st : S.state) {
        *running += st == kSlotRunning ? 1 : 0;
        *done += st == kSlotDone ? 1 : 0;
    }
    return EGPR_SUCC;
}

int egpr_session_destroy(egpr_session* h) {
    using namespace egpr;
    if (!h) return EGPR_SUCC;
    if (h->st) {
        egpr_graph* g = h->st->g;
        std::lock_guard<std::mutex> lk(g->mu);
        cudaStreamSynchronize(g->stream);
        delete h->st;
        g->sessions -= 1;
    }
    delete h;
    return EGPR_SUCC;
}

}  // extern "C"
