// Device-side graph preparation.
//
// Replaces the reference's single-threaded host pass build_inbound_from_csr
// (gpu_easygraph/functions/centrality/pagerank.cu:286-347) and its H2D of the
// result (:472-518) with GPU kernels over the uploaded out-edge CSR:
//
//   k_out_weight_exact  FP64 out-weight sum per source after sanitising each
//                    weight, bit-identical to the sequential sum in row order
//                    (pagerank.cu:301-316): four lanes per source (a warp for
//                    sources of more than 64 entries, 4096-entry segments on
//                    several warps for more than 16384) where the sum is
//                    provably order-free, one thread per source otherwise
//   k_in_degree      in-degree histogram over valid endpoints (:315)
//   exclusive scan   in_row (:319-320)
//   radix sort       stable LSD sort of the entries by destination: entries of
//                    one destination keep ascending entry order, i.e. the
//                    ascending-source order of the reference's sequential
//                    scatter (:328-346); the sorted pairs carry each entry's
//                    source and, when weighted, its FP32 weight, so the sorted
//                    values are in_col and in_w
//   k_dangling       dangling mask outw <= 0 (:323-326) and the counts used by
//                    the solver
//
// The results are bit-identical to build_inbound_from_csr for in_row, in_col,
// the dangling mask and the FP64 out-weight sums.  The engine stores raw
// (sanitised) FP32 weights instead of the alpha-scaled in_val, so a prepared
// graph does not depend on alpha.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kScanPerThread = 8;
constexpr int kScanTile = kThreads * kScanPerThread;
constexpr int kSortPerLane = 16;
constexpr int kWarps = kThreads / 32;
constexpr int kSortTile = kThreads * kSortPerLane;

// ---------------------------------------------------------------- scan -----
// Exclusive scan of uint32 values, tile by tile; tile totals go to tile_sums.
__global__ void __launch_bounds__(kThreads)
k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t len,
             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t s[kScanTile];
    __shared__ uint32_t warp_tot[kWarps];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < kScanPerThread; ++i) {
        int64_t idx = base + tid + (int64_t)i * kThreads;
        s[tid + i * kThreads] = idx < len ? in[idx] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanPerThread];
    uint32_t run = 0;
#pragma unroll
    for (int i = 0; i < kScanPerThread; ++i) {
        v[i] = run;
        run += s[tid * kScanPerThread + i];
    }
    // inclusive warp scan of the thread totals
    const int lane = tid & 31, warp = tid >> 5;
    uint32_t inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t warp_off = 0, block_tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        if (w < warp) warp_off += warp_tot[w];
        block_tot += warp_tot[w];
    }
    const uint32_t excl = warp_off + inc - run;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanPerThread; ++i) s[tid * kScanPerThread + i] = v[i] + excl;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanPerThread; ++i) {
        int64_t idx = base + tid + (int64_t)i * kThreads;
        if (idx < len) out[idx] = s[tid + i * kThreads];
    }
    if (tid == 0 && tile_sums) tile_sums[blockIdx.x] = block_tot;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, int64_t len, const uint32_t* __restrict__ tile_off) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < len) out[i] += tile_off[i / kScanTile];
}

// -------------------------------------------------------------- radix ------
// LSD radix sort of (key, value) pairs with digits of kBits bits (8 in use):
// a key of B bits takes ceil(B / kBits) passes.
template <int kBits>
__global__ void __launch_bounds__(kThreads)
k_radix_hist(const uint32_t* __restrict__ keys, int64_t len, int shift, int64_t ntiles,
             uint32_t* __restrict__ hist) {
    constexpr int kD = 1 << kBits;
    __shared__ uint32_t h[kD];
    for (int d = threadIdx.x; d < kD; d += kThreads) h[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kThreads) {
        int64_t idx = base + i;
        if (idx < len) atomicAdd(&h[(keys[idx] >> shift) & (kD - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kD; d += kThreads) hist[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

// Stable scatter: within a tile, warp w owns items [w*32*kSortPerLane, ...) in
// order; inside a warp, rounds of 32 consecutive items rank equal digits by
// lane order.  Global order = tile order (digit-major scanned histogram),
// then warp order, then item order.  keys_out may be NULL (last pass: only
// the values are needed).  kTwo: a second value array moves with the first.
template <int kBits, bool kTwo>
__global__ void __launch_bounds__(kThreads)
k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int64_t len,
                int shift, int64_t ntiles, const uint32_t* __restrict__ offsets,
                const uint32_t* __restrict__ vals2_in, uint32_t* __restrict__ vals2_out) {
    constexpr int kD = 1 << kBits;
    extern __shared__ uint32_t radix_smem[];
    uint32_t (*warp_hist)[kD] = reinterpret_cast<uint32_t (*)[kD]>(radix_smem);  // [kWarps][kD]
    uint32_t* tile_off = radix_smem + kWarps * kD;                               // [kD]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kWarps * kD; i += kThreads) radix_smem[i] = 0;
    for (int d = tid; d < kD; d += kThreads) tile_off[d] = offsets[(int64_t)d * ntiles + blockIdx.x];
    __syncthreads();
    const int64_t wbase = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * 32 * kSortPerLane;
    uint32_t key[kSortPerLane], val[kSortPerLane], val2[kTwo ? kSortPerLane : 1], rank[kSortPerLane];
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSortPerLane; ++r) {
        const int64_t idx = wbase + (int64_t)r * 32 + lane;
        const bool valid = idx < len;
        key[r] = valid ? keys_in[idx] : 0u;
        val[r] = valid ? vals_in[idx] : 0u;
        if (kTwo) val2[r] = valid ? vals2_in[idx] : 0u;
        const uint32_t d = (key[r] >> shift) & (kD - 1);
        const uint32_t tag = valid ? d : (uint32_t)(kD + lane);
        const uint32_t peers = __match_any_sync(0xffffffffu, tag);
        const uint32_t before = valid ? warp_hist[warp][d] : 0u;
        __syncwarp();
        if (valid && (peers & lt_mask) == 0u) warp_hist[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    // per digit: the warps' prefix, and the tile's count (then its start in the tile)
    uint32_t* dstart = tile_off + kD;  // [kD]
    for (int d = tid; d < kD; d += kThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            uint32_t c = warp_hist[w][d];
            warp_hist[w][d] = run;
            run += c;
        }
        dstart[d] = run;
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the kD counts, one warp
        uint32_t carry = 0;
        for (int d0 = 0; d0 < kD; d0 += 32) {
            const uint32_t c = dstart[d0 + lane];
            uint32_t x = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            dstart[d0 + lane] = carry + x - c;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
    __syncthreads();
    // the tile in digit order in shared memory (same order as before: digit,
    // then warp, then item), then each digit's run written out contiguously
    uint32_t* skey = dstart + kD;          // [kSortTile]
    uint32_t* sval = skey + kSortTile;     // [kSortTile]
    uint32_t* sval2 = sval + kSortTile;    // [kSortTile] (kTwo)
#pragma unroll
    for (int r = 0; r < kSortPerLane; ++r) {
        const int64_t idx = wbase + (int64_t)r * 32 + lane;
        if (idx < len) {
            const uint32_t d = (key[r] >> shift) & (kD - 1);
            const uint32_t lpos = dstart[d] + warp_hist[warp][d] + rank[r];
            skey[lpos] = key[r];
            sval[lpos] = val[r];
            if (kTwo) sval2[lpos] = val2[r];
        }
    }
    __syncthreads();
    const int64_t tbase = (int64_t)blockIdx.x * kSortTile;
    const int nvalid = (int)(len - tbase < (int64_t)kSortTile ? len - tbase : (int64_t)kSortTile);
    for (int i = tid; i < nvalid; i += kThreads) {
        const uint32_t k = skey[i];
        const uint32_t d = (k >> shift) & (kD - 1);
        const uint32_t dst = tile_off[d] + ((uint32_t)i - dstart[d]);
        if (keys_out) keys_out[dst] = k;
        vals_out[dst] = sval[i];
        if (kTwo) vals2_out[dst] = sval2[i];
    }
}

// -------------------------------------------------------------- graph ------
__device__ __forceinline__ double sanitize_w(double w) {
    return (!isfinite(w) || w < 0.0) ? 0.0 : w;
}

// Exponent of the lowest set bit of a finite w > 0: w = M * 2^q with M odd.
__device__ __forceinline__ int lsb_exponent(double w) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(w);
    const int ef = (int)((b >> 52) & 0x7ffull);
    unsigned long long m = b & 0xfffffffffffffull;
    int e = -1074;  // subnormal: w = m * 2^-1074
    if (ef != 0) {
        m |= 1ull << 52;
        e = ef - 1075;
    }
    return e + __ffsll((long long)m) - 1;
}

// FP64 out-weight sums, one warp per source, bit-identical to the sequential
// sum in entry order (pagerank.cu:301-316) without summing sequentially.
// Sanitised weights are >= 0; let 2^q be the lowest set bit among a row's
// nonzero weights.  Every partial sum, in any order, is then a multiple of
// 2^q no larger than the row's total T, so when T < 2^(q+53) every partial sum
// is an exact double and the lanes' sums and the shuffle tree give T, which
// is also what the sequential loop gives.  The computed sum s is within a few
// ulps of T, so s < 2^(q+52) proves T < 2^(q+53).  A row that fails the test
// (weights of very different scales) is listed and summed sequentially by
// k_out_weight_serial.  Weights drawn as FP32 values, as in the synthetic
// workloads, always pass.
// One source's sums over G lanes (lanes sub = 0..G-1 of a G-lane group).
template <int G>
__device__ __forceinline__ void out_weight_row(const int32_t* __restrict__ E, const double* __restrict__ W,
                                               int32_t n, int32_t b, int32_t e, int sub, double& s, int32_t& c,
                                               int& q) {
    s = 0.0;
    c = 0;
    q = 4096;  // no nonzero weight yet
    for (int32_t p = b + sub; p < e; p += G) {
        const int32_t v = E[p];
        if (v >= 0 && v < n) {
            const double w = W ? sanitize_w(W[p]) : 1.0;  // unit weights: q = 0, every sum exact
            s += w;
            ++c;
            if (w > 0.0) q = min(q, lsb_exponent(w));
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
        q = min(q, __shfl_xor_sync(0xffffffffu, q, o));
    }
}

// The sum s of a source's weights is its sequential sum when every partial sum
// is provably exact (see above); otherwise the source is listed for the
// sequential kernel.
__device__ __forceinline__ void out_weight_store(int64_t u, double s, int32_t c, int q, double* __restrict__ outw,
                                                 uint32_t* __restrict__ hub_key, uint32_t* __restrict__ hub_val,
                                                 int32_t* __restrict__ serial_rows,
                                                 uint32_t* __restrict__ serial_count) {
    bool exact;
    if (q == 4096) exact = true;             // only zero weights: the sum is 0
    else if (q + 52 >= 1024) exact = false;  // 2^(q+52) would overflow: sum sequentially
    else exact = s < ldexp(1.0, q + 52);
    if (exact) outw[u] = s;
    else serial_rows[atomicAdd(serial_count, 1u)] = (int32_t)u;
    // hub ranking: descending out-degree, ascending id (stable sort of ~count)
    hub_key[u] = ~(uint32_t)c;
    hub_val[u] = (uint32_t)u;
}

constexpr int32_t kOutWeightShort = 64;  // sources with more entries are summed by a whole warp
// Sources with more than kOutWeightHuge entries are summed in segments of
// kOutWeightSeg entries by several warps; each segment's sums go into the
// source's accumulator and the last segment to arrive finishes the source.
// A segment's sum is one of the source's partial sums, so the exactness test
// above covers the segments and their FP64 atomic adds, in any order.
constexpr int32_t kOutWeightHuge = 16384;
constexpr int32_t kOutWeightSeg = 4096;

struct HugeAcc {
    double s;          // sum of the segments' sums
    int32_t c;         // valid entries
    int32_t q;         // lowest set bit exponent of the nonzero weights
    uint32_t arrived;  // segments added so far
    int32_t pad;
};

struct OutSegs {
    int4* seg;           // (source, segment, accumulator, segments of the source)
    uint32_t* seg_count;
    HugeAcc* acc;
    uint32_t* acc_count;
};

// Lists the segments of source u (called by one thread for a huge source).
__device__ __forceinline__ void list_segments(const OutSegs& H, int32_t u, int32_t len) {
    const int32_t nseg = (len + kOutWeightSeg - 1) / kOutWeightSeg;
    const uint32_t h = atomicAdd(H.acc_count, 1u);
    H.acc[h].s = 0.0;
    H.acc[h].c = 0;
    H.acc[h].q = 4096;
    H.acc[h].arrived = 0u;
    const uint32_t s0 = atomicAdd(H.seg_count, (uint32_t)nseg);
    for (int32_t j = 0; j < nseg; ++j) H.seg[s0 + (uint32_t)j] = make_int4(u, j, (int32_t)h, nseg);
}

// Sources [r0, r1), four lanes each; a source with more than kOutWeightShort
// entries is listed for k_out_weight_long instead.
__global__ void k_out_weight_exact(const int32_t* __restrict__ V, const int32_t* __restrict__ E,
                                   const double* __restrict__ W, int32_t n, int32_t r0, int32_t r1,
                                   double* __restrict__ outw, uint32_t* __restrict__ hub_key,
                                   uint32_t* __restrict__ hub_val, int32_t* __restrict__ serial_rows,
                                   uint32_t* __restrict__ serial_count, int32_t* __restrict__ long_rows,
                                   uint32_t* __restrict__ long_count, OutSegs H) {
    constexpr int G = 4;
    const int lane = threadIdx.x & 31, sub = lane & (G - 1), grp = lane / G;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ub = r0 + warp * (32 / G); ub < r1; ub += nwarps * (32 / G)) {
        const int64_t u = ub + grp;
        int32_t b = 0, e = 0;
        if (u < r1) {
            b = V[u];
            e = V[u + 1];
            if (e - b > kOutWeightShort) {
                if (sub == 0) {
                    if (e - b > kOutWeightHuge) list_segments(H, (int32_t)u, e - b);
                    else long_rows[atomicAdd(long_count, 1u)] = (int32_t)u;
                }
                e = b;  // the group still takes part in the shuffles
            }
        }
        double s;
        int32_t c;
        int q;
        out_weight_row<G>(E, W, n, b, e, sub, s, c, q);
        if (u < r1 && sub == 0 && V[u + 1] - V[u] <= kOutWeightShort)
            out_weight_store(u, s, c, q, outw, hub_key, hub_val, serial_rows, serial_count);
    }
}

// The long sources listed by k_out_weight_exact, one warp each, then the
// segments of the huge ones (weighted or not).
__global__ void k_out_weight_long(const int32_t* __restrict__ V, const int32_t* __restrict__ E,
                                  const double* __restrict__ W, int32_t n, const int32_t* __restrict__ long_rows,
                                  const uint32_t* __restrict__ long_count, double* __restrict__ outw,
                                  uint32_t* __restrict__ hub_key, uint32_t* __restrict__ hub_val,
                                  int32_t* __restrict__ serial_rows, uint32_t* __restrict__ serial_count,
                                  OutSegs H) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = long_count ? *long_count : 0u;
    for (int64_t i = warp; i < (int64_t)k; i += nwarps) {
        const int32_t u = long_rows[i];
        double s;
        int32_t c;
        int q;
        out_weight_row<32>(E, W, n, V[u], V[u + 1], lane, s, c, q);
        if (lane == 0) out_weight_store(u, s, c, q, outw, hub_key, hub_val, serial_rows, serial_count);
    }
    // segments of the huge sources: the last segment of a source to arrive finishes it
    const uint32_t ns = *H.seg_count;
    for (int64_t i = warp; i < (int64_t)ns; i += nwarps) {
        const int4 sg = H.seg[i];
        const int32_t u = sg.x, b = V[u] + sg.y * kOutWeightSeg, e = min(V[u + 1], b + kOutWeightSeg);
        double s;
        int32_t c;
        int q;
        out_weight_row<32>(E, W, n, b, e, lane, s, c, q);
        if (lane == 0) {
            HugeAcc& A = H.acc[sg.z];
            if (s != 0.0) atomicAdd(&A.s, s);
            atomicAdd(&A.c, c);
            atomicMin(&A.q, q);
            __threadfence();
            if (atomicAdd(&A.arrived, 1u) == (uint32_t)(sg.w - 1)) {
                __threadfence();
                const double ts = __ldcg(&A.s);
                const int32_t tc = __ldcg(&A.c);
                const int tq = __ldcg(&A.q);
                if (W) {
                    out_weight_store(u, ts, tc, tq, outw, hub_key, hub_val, serial_rows, serial_count);
                } else {  // unit weights: the count
                    outw[u] = (double)tc;
                    hub_key[u] = ~(uint32_t)tc;
                    hub_val[u] = (uint32_t)u;
                }
            }
        }
    }
}

// The rows k_out_weight_exact could not prove order-free: summed in entry
// order, one thread per row, exactly as pagerank.cu:301-316 does.
__global__ void k_out_weight_serial(const int32_t* __restrict__ V, const int32_t* __restrict__ E,
                                    const double* __restrict__ W, int32_t n, const int32_t* __restrict__ rows,
                                    const uint32_t* __restrict__ count, double* __restrict__ outw) {
    const uint32_t k = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const int32_t u = rows[i];
        double s = 0.0;
        for (int32_t p = V[u]; p < V[u + 1]; ++p) {
            const int32_t v = E[p];
            if (v >= 0 && v < n) s += sanitize_w(W[p]);
        }
        outw[u] = s;
    }
}

// Unit weights: the out-weight sum is the count of valid entries, exact in any
// order, so one warp counts a row.
__global__ void k_out_degree(const int32_t* __restrict__ V, const int32_t* __restrict__ E, int32_t n, int32_t r0,
                             int32_t r1, double* __restrict__ outw, uint32_t* __restrict__ hub_key,
                             uint32_t* __restrict__ hub_val, OutSegs H) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = r0 + warp; u < r1; u += nwarps) {
        const int32_t b = V[u], e = V[u + 1];
        if (e - b > kOutWeightHuge) {  // counted in segments by k_out_weight_long
            if (lane == 0) list_segments(H, (int32_t)u, e - b);
            continue;
        }
        int32_t c = 0;
        for (int32_t p = b + lane; p < e; p += 32) {
            const int32_t v = E[p];
            c += (v >= 0 && v < n) ? 1 : 0;
        }
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) {
            outw[u] = (double)c;
            hub_key[u] = ~(uint32_t)c;
            hub_val[u] = (uint32_t)u;
        }
    }
}

__global__ void k_hub_slots(const uint32_t* __restrict__ ranked, int32_t nhub, int32_t* __restrict__ hub_ids,
                            int32_t* __restrict__ hub_slot) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nhub; s += gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)ranked[s];
        hub_ids[s] = v;
        hub_slot[v] = s;
    }
}

// Inbound entries from a hub store -(slot + 1).
__global__ void k_encode_hubs(int32_t* __restrict__ in_col, int64_t nnz, const int32_t* __restrict__ hub_slot) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = hub_slot[in_col[i]];
        if (s >= 0) in_col[i] = -(s + 1);
    }
}

__global__ void k_decode_hubs(const int32_t* __restrict__ in_col, int64_t nnz, const int32_t* __restrict__ hub_ids,
                              int32_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = in_col[i];
        out[i] = c < 0 ? hub_ids[-c - 1] : c;
    }
}

// In-degree histogram and the sort keys: destination, or n for an entry whose
// destination is outside [0, n) (those sort last and are dropped).
__global__ void k_in_degree_keys(const int32_t* __restrict__ E, int64_t p0, int64_t p1, int32_t n,
                                 uint32_t* __restrict__ indeg, uint32_t* __restrict__ keys) {
    for (int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < p1;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = E[p];
        const bool ok = v >= 0 && v < n;
        if (ok) atomicAdd(&indeg[v], 1u);
        keys[p] = ok ? (uint32_t)v : (uint32_t)n;
    }
}

// Source id of every entry: one warp per row writes its range.
__global__ void k_expand_src(const int32_t* __restrict__ V, int32_t n, int32_t* __restrict__ src) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        const int32_t b = V[u], e = V[u + 1];
        for (int32_t p = b + lane; p < e; p += 32) src[p] = (int32_t)u;
    }
}

// FP32 bits of each entry's sanitised weight (the stored in_w), for entries [p0, p1).
__global__ void k_weight_bits(const double* __restrict__ W, int64_t p0, int64_t p1, uint32_t* __restrict__ out) {
    for (int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < p1;
         p += (int64_t)gridDim.x * blockDim.x)
        out[p] = __float_as_uint((float)sanitize_w(W[p]));
}

__global__ void k_dangling(const double* __restrict__ outw, int32_t n, int32_t* __restrict__ mask,
                           unsigned long long* __restrict__ counts) {
    __shared__ unsigned long long c0, c1;
    if (threadIdx.x == 0) { c0 = 0; c1 = 0; }
    __syncthreads();
    unsigned long long a = 0, b = 0;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
         u += (int64_t)gridDim.x * blockDim.x) {
        const double w = outw[u];
        const int d = w <= 0.0 ? 1 : 0;
        mask[u] = d;
        a += d;
        b += (w <= 1e-15) ? 1 : 0;
    }
    atomicAdd(&c0, a);
    atomicAdd(&c1, b);
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&counts[0], c0);
        atomicAdd(&counts[1], c1);
    }
}

// Merge-path coordinate of diagonal d over (row ends = in_row[1..n], entries).
__device__ __forceinline__ int2 merge_search(const int32_t* __restrict__ in_row, int32_t n,
                                             int64_t nnz, int64_t d) {
    int64_t lo = d - nnz > 0 ? d - nnz : 0;
    int64_t hi = d < n ? d : n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)in_row[mid + 1] <= d - mid - 1) lo = mid + 1;
        else hi = mid;
    }
    return make_int2((int32_t)lo, (int32_t)(d - lo));
}

inline int grid_for(int64_t work, int per_block = kThreads) {
    int64_t g = (work + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

// Stream-ordered scratch of the preparation comes from the library's device
// pool (device_pool), which keeps freed memory for the next preparation.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
    cudaMemPool_t pool = device_pool();
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}

struct TmpAlloc {
    cudaStream_t s;
    std::vector<void*> ptrs;
    explicit TmpAlloc(cudaStream_t st) : s(st) {}
    ~TmpAlloc() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
    template <typename T>
    T* get(size_t count, int* rc) {
        void* p = nullptr;
        cudaError_t e = scratch_alloc(&p, std::max<size_t>(count, 1) * sizeof(T), s);
        if (e != cudaSuccess) {
            set_cuda_error(e, "cudaMallocAsync (preparation scratch)");
            *rc = EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM;
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

template <int kBits, bool kTwo>
int radix_pass(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t len, int shift,
               bool last, int64_t ntiles, uint32_t* hist, cudaStream_t s, const uint32_t* v2in, uint32_t* v2out) {
    constexpr int kD = 1 << kBits;
    // warp histograms, tile offsets, digit starts, and the tile's keys and values
    const size_t smem = ((size_t)(kWarps + 2) * kD + (kTwo ? 3 : 2) * (size_t)kSortTile) * sizeof(uint32_t);
    // The shared-memory opt-in is a per-device attribute of the function: made
    // once per device (bit d of the mask; devices past 63 repeat it, which is
    // harmless).  Atomic: several host threads prepare graphs at once.
    static std::atomic<uint64_t> attr_devices{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (!bit || !(attr_devices.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(k_radix_scatter<kBits, kTwo>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_devices.fetch_or(bit, std::memory_order_release);
    }
    k_radix_hist<kBits><<<(unsigned)ntiles, kThreads, 0, s>>>(kin, len, shift, ntiles, hist);
    int rc = exclusive_scan_u32(hist, hist, ntiles * kD, s);
    if (rc) return rc;
    k_radix_scatter<kBits, kTwo><<<(unsigned)ntiles, kThreads, smem, s>>>(kin, vin, last ? nullptr : kout, vout, len,
                                                                          shift, ntiles, hist, v2in, v2out);
    return EGPR_SUCC;
}

// Sorts (keys, vals) by the low `bits` bits of the keys, stable.  After the
// call the values are in the buffer *result_in_alt names; the keys are sorted
// alongside except in the last pass, which writes values only.
int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                     int64_t len, int bits, cudaStream_t s, TmpAlloc& tmp, bool* result_in_alt,
                     bool keys_needed = true, uint32_t* vals2 = nullptr, uint32_t* vals2_alt = nullptr) {
    *result_in_alt = false;
    if (len <= 1 || bits <= 0) return EGPR_SUCC;
    int rc = EGPR_SUCC;
    // 8-bit digits: with 4096-item tiles a digit's run averages 16 items, so
    // the runs written out are 64-byte pieces (11-bit digits, one pass fewer,
    // leave 2-item runs and were slower in total).  Where one or two 9-bit
    // digits save a whole pass (25-bit keys: 9 + 8 + 8 instead of 8 + 8 + 8 + 1)
    // they are used: 8-item runs, one pass of the data fewer.
    int passes = (bits + 7) / 8;
    int nine = 0;  // leading passes of 9-bit digits
    if (passes > 1 && bits <= 9 * (passes - 1)) {
        passes -= 1;
        nine = bits - 8 * passes;
    }
    const int64_t ntiles = (len + kSortTile - 1) / kSortTile;
    uint32_t* hist = tmp.get<uint32_t>((size_t)ntiles << (nine ? 9 : 8), &rc);
    if (!hist) return rc;
    uint32_t *kin = keys, *vin = vals, *kout = keys_alt, *vout = vals_alt, *v2in = vals2, *v2out = vals2_alt;
    int shift = 0;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1 && !keys_needed;
        if (p < nine)
            rc = vals2 ? radix_pass<9, true>(kin, vin, kout, vout, len, shift, last, ntiles, hist, s, v2in, v2out)
                       : radix_pass<9, false>(kin, vin, kout, vout, len, shift, last, ntiles, hist, s, nullptr, nullptr);
        else
            rc = vals2 ? radix_pass<8, true>(kin, vin, kout, vout, len, shift, last, ntiles, hist, s, v2in, v2out)
                       : radix_pass<8, false>(kin, vin, kout, vout, len, shift, last, ntiles, hist, s, nullptr, nullptr);
        shift += p < nine ? 9 : 8;
        if (rc) return rc;
        std::swap(kin, kout);
        std::swap(vin, vout);
        std::swap(v2in, v2out);
    }
    *result_in_alt = (vin == vals_alt);
    return cuda_ok(cudaGetLastError(), "radix sort");
}

}  // namespace

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t len, cudaStream_t s) {
    if (len <= 0) return EGPR_SUCC;
    const int64_t ntiles = (len + kScanTile - 1) / kScanTile;
    if (ntiles == 1) {
        k_scan_tiles<<<1, kThreads, 0, s>>>(in, out, len, nullptr);
        return cuda_ok(cudaGetLastError(), "scan");
    }
    uint32_t* sums = nullptr;
    cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&sums), (size_t)ntiles * sizeof(uint32_t), s);
    if (e != cudaSuccess) {
        set_cuda_error(e, "cudaMallocAsync (scan)");
        return EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM;
    }
    k_scan_tiles<<<(unsigned)ntiles, kThreads, 0, s>>>(in, out, len, sums);
    int rc = exclusive_scan_u32(sums, sums, ntiles, s);
    if (rc == EGPR_SUCC) {
        k_scan_add<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(out, len, sums);
        rc = cuda_ok(cudaGetLastError(), "scan add");
    }
    cudaFreeAsync(sums, s);
    return rc;
}

// The sweep's copy of the inbound CSR: every row keeps its entries (hub-encoded,
// in the order of in_col) and a row without entries gets one placeholder entry
// that reads a carried value of 0 (hub slot nhub).  One warp per row.
__global__ void k_build_sweep_cols(const int32_t* __restrict__ in_row, const int32_t* __restrict__ in_col,
                                   const float* __restrict__ in_w, int32_t n, const int32_t* __restrict__ sw_row,
                                   int32_t* __restrict__ sw_col, float* __restrict__ sw_w, int32_t zero_code) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n; r += nwarps) {
        const int32_t b = in_row[r], e = in_row[r + 1], o = sw_row[r];
        if (e == b) {
            if (lane == 0) {
                sw_col[o] = zero_code;
                if (sw_w) sw_w[o] = 0.f;
            }
            continue;
        }
        for (int32_t p = lane; p < e - b; p += 32) {
            sw_col[o + p] = in_col[b + p];
            if (sw_w) sw_w[o + p] = in_w[b + p];
        }
    }
}

// max(1, length of row r); 0 for the closing slot r = n.
__global__ void k_row_len1(const int32_t* __restrict__ in_row, int32_t n, uint32_t* __restrict__ out) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = r < n ? (uint32_t)max(1, in_row[r + 1] - in_row[r]) : 0u;
}

// sw_row[n+1 .. n+7] = sw_row[n] (bulk reads of row data may run past n).
__global__ void k_pad_tail(int32_t* sw_row, int32_t n) {
    if (threadIdx.x > 0 && threadIdx.x < 8) sw_row[(int64_t)n + threadIdx.x] = sw_row[n];
}

// For the ideal boundary d = i * cap: the row r whose cost range holds d
// (cost of the start of row r = sw_row[r] + R * r), the offset of d into the
// row's entries, the row's start and its length.
__global__ void k_chunk_cuts(const int32_t* __restrict__ sw_row, int32_t n, int64_t R, int64_t cap, int32_t ideal,
                             int4* __restrict__ out) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= ideal; i += gridDim.x * blockDim.x) {
        const int64_t d = (int64_t)i * cap;
        int32_t lo = 0, hi = n - 1;  // largest r with sw_row[r] + R*r <= d
        while (lo < hi) {
            const int32_t mid = lo + ((hi - lo + 1) >> 1);
            if ((int64_t)sw_row[mid] + R * mid <= d) lo = mid;
            else hi = mid - 1;
        }
        const int64_t off = d - ((int64_t)sw_row[lo] + R * lo);
        const int32_t len = sw_row[lo + 1] - sw_row[lo];
        out[i] = make_int4(lo, (int32_t)(off < (int64_t)len ? off : (int64_t)len), sw_row[lo], len);
    }
}

// Every row ends on an entry; mark it in the tile of the chunk that holds it.
__global__ void k_tile_marks(const int32_t* __restrict__ sw_row, int32_t n, const int32_t* __restrict__ cstart,
                             const int32_t* __restrict__ ctile, int32_t nch, uint32_t* __restrict__ bits,
                             int32_t* __restrict__ trow) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int32_t p = sw_row[r + 1] - 1;
        int32_t lo = 0, hi = nch - 1;  // last chunk starting at or before p
        while (lo < hi) {
            const int32_t mid = lo + ((hi - lo + 1) >> 1);
            if (cstart[mid] <= p) lo = mid;
            else hi = mid - 1;
        }
        const int32_t q = p - (cstart[lo] & ~7);
        const int32_t t = ctile[lo] + q / kTileItems, i = q % kTileItems;
        atomicOr(&bits[(size_t)t * kTileWords + (i >> 5)], 1u << (i & 31));
        atomicMin(&trow[t], r);
    }
}

// Per lane of every tile: the marks of the lanes below it (one byte per lane).
__global__ void k_tile_offsets(uint32_t* __restrict__ bits, int64_t ntiles) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < ntiles; t += nwarps) {
        uint32_t* w = bits + (size_t)t * kTileWords;
        const uint32_t mine = __popc((w[lane >> 2] >> (8 * (lane & 3))) & 0xffu);
        uint32_t incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t up = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += up;
        }
        const uint32_t below = incl - mine;
        uint32_t word = below;
        word |= __shfl_down_sync(0xffffffffu, below, 1) << 8;
        word |= __shfl_down_sync(0xffffffffu, below, 2) << 16;
        word |= __shfl_down_sync(0xffffffffu, below, 3) << 24;
        if ((lane & 3) == 0) w[8 + (lane >> 2)] = word;
    }
}

// Entry i (destination dst[i]) of the inbound CSR to its place in the sweep's copy.
__global__ void k_sweep_cols_by_entry(const uint32_t* __restrict__ dst, const int32_t* __restrict__ in_row,
                                      const int32_t* __restrict__ in_col, const float* __restrict__ in_w, int64_t nnz,
                                      const int32_t* __restrict__ sw_row, int32_t* __restrict__ sw_col,
                                      float* __restrict__ sw_w) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = dst[i];
        const int64_t o = i + (int64_t)(sw_row[r] - in_row[r]);
        sw_col[o] = in_col[i];
        if (sw_w) sw_w[o] = in_w[i];
    }
}

// The placeholder entry of every empty row.
__global__ void k_sweep_placeholders(const int32_t* __restrict__ in_row, int32_t n, const int32_t* __restrict__ sw_row,
                                     int32_t* __restrict__ sw_col, float* __restrict__ sw_w, int32_t zero_code) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        if (in_row[r + 1] == in_row[r]) {
            sw_col[sw_row[r]] = zero_code;
            if (sw_w) sw_w[sw_row[r]] = 0.f;
        }
    }
}

// Defaults of a graph's layout parameters (egpr_graph_set_tuning and
// egpr_graph_autotune change them per graph).
int default_chunks_per_warp() {
    static const int v = [] {
        const char* e = std::getenv("EGPR_CHUNKS_PER_WARP");  // queue granularity
        const int x = e ? std::atoi(e) : 8;
        return x >= 1 && x <= 64 ? x : 8;
    }();
    return v;
}

// Cost of finishing one row, in entries (a row costs its entries plus this).
int default_row_cost() {
    static const int v = [] {
        const char* e = std::getenv("EGPR_ROW_COST");
        const int x = e ? std::atoi(e) : 4;
        return x >= 0 && x <= 64 ? x : 4;
    }();
    return v;
}

// The sweep's work layout, built on the device (the host only sees the chunk
// boundaries):
//   * sw_row / sw_col / sw_w: the inbound CSR with a placeholder entry in every
//     empty row, so that every row ends on an entry of its own;
//   * chunks: boundaries at multiples of a cost cap along the rows, where a
//     row costs its entries plus the graph's row cost; a boundary moves back to the
//     start of its row unless that row began before the previous boundary (a
//     row longer than a chunk), which is then cut (a span: its chunks add
//     pieces to the span's accumulator and the sweep finishes the row when the
//     launch ends); every cut leaves at least one entry on each side;
//   * warp tiles: chunk c covers tiles of kTileItems entries from
//     (start & ~7); per tile a 256-bit mask of the entries that end a row, per
//     lane the number of marks in the lanes below it, and the first row a mark
//     of the tile ends (the k-th mark of a tile ends row tile_row + k, since
//     every row has an entry).
// Chunks are stored costliest first, which is their queue order.
// The layout's tables (row offsets, chunks, tile masks, span links), which
// need in_row only; the entries follow in build_sweep_entries.
int build_sweep_tables(egpr_graph* g, int32_t resident_warps, cudaStream_t s) {
    const int32_t n = g->n;
    TmpAlloc tmp(s);
    int rc = EGPR_SUCC;
    // placeholder offsets: sw_row = exclusive scan of max(1, row length)
    uint32_t* len1 = tmp.get<uint32_t>((size_t)n + 1, &rc);
    if (rc || (rc = g->sw_row.alloc(((size_t)n + 8) * sizeof(int32_t)))) return rc;
    k_row_len1<<<grid_for((int64_t)n + 1), kThreads, 0, s>>>(g->in_row.as<int32_t>(), n, len1);
    if ((rc = exclusive_scan_u32(len1, reinterpret_cast<uint32_t*>(g->sw_row.as<int32_t>()), (int64_t)n + 1, s))) return rc;
    k_pad_tail<<<1, 32, 0, s>>>(g->sw_row.as<int32_t>(), n);
    uint32_t nnz_u = 0;
    if ((rc = cuda_ok(cudaMemcpyAsync(&nnz_u, g->sw_row.as<int32_t>() + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "D2H sweep entries")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "sweep layout")))
        return rc;
    if ((int64_t)nnz_u > (int64_t)INT32_MAX - 4096) return EGPR_UNSUPPORTED_GRAPH;
    const int32_t nnz = (int32_t)nnz_u;
    g->sw_nnz = nnz;
    // chunk boundaries at ideal costs d_i = i * cap
    const int64_t R = g->tune_rc;
    const int64_t warps = std::max(1, resident_warps);
    const int64_t total = (int64_t)nnz + R * (int64_t)n;
    const int64_t cpw = std::max(1, g->tune_cpw);
    int64_t cap = (total + warps * cpw - 1) / (warps * cpw);
    cap = std::min<int64_t>(std::max<int64_t>(kTileItems + R + 1, cap), 1 << 24);
    const int64_t ideal = std::max<int64_t>(1, (total + cap - 1) / cap);
    int4* d_cut = tmp.get<int4>((size_t)ideal + 1, &rc);
    if (rc) return rc;
    k_chunk_cuts<<<grid_for(ideal + 1), kThreads, 0, s>>>(g->sw_row.as<int32_t>(), n, R, cap, (int32_t)ideal, d_cut);
    std::vector<int4> cut((size_t)ideal + 1);
    if ((rc = cuda_ok(cudaMemcpyAsync(cut.data(), d_cut, cut.size() * sizeof(int4), cudaMemcpyDeviceToHost, s), "D2H chunk cuts")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "sweep layout")))
        return rc;
    struct B {
        int32_t r, k, rs;  // boundary: row, entry, start of that row
    };
    std::vector<B> bs;
    bs.push_back(B{0, 0, 0});
    for (int64_t i = 1; i < ideal; ++i) {
        const int4 c = cut[(size_t)i];  // (row, offset into the row, row start, row length)
        const B& p = bs.back();
        if (c.z > p.k) {
            bs.push_back(B{c.x, c.z, c.z});  // the row's start
        } else if (c.w >= 2) {
            const int32_t k = c.z + std::min(std::max(c.y, 1), c.w - 1);  // a cut inside a long row
            if (c.x == p.r && k > p.k) bs.push_back(B{c.x, k, c.z});
        }
    }
    bs.push_back(B{n, nnz, nnz});
    const int32_t nch = (int32_t)bs.size() - 1;
    std::vector<Chunk>& ch = g->plan.h_chunks;
    ch.assign((size_t)nch, Chunk{});
    std::vector<int32_t> cstart((size_t)nch), ctile((size_t)nch);
    int64_t ntiles = 0;
    for (int32_t c = 0; c < nch; ++c) {
        const B& a = bs[(size_t)c];
        const B& b = bs[(size_t)c + 1];
        const int32_t t0 = a.k & ~7;
        const int32_t nt = std::max<int32_t>(1, (b.k - t0 + kTileItems - 1) / kTileItems);
        Chunk& k = ch[(size_t)c];
        const bool head = a.r < n && a.k > a.rs;
        const bool tail = b.r < n && b.k > b.rs;
        int32_t f = 0;
        if (head) f |= kHasHead;
        if (tail) f |= kHasTail;
        if (head && tail && a.r == b.r) f |= kInterior;
        k.flags = f;
        k.tile_begin = (int32_t)ntiles;
        k.tile_end = (int32_t)(ntiles + nt);
        k.nnz_begin = a.k;
        k.nnz_end = b.k;
        k.row_end = b.r;
        k.pad = (int32_t)std::min<int64_t>((int64_t)(b.k - a.k) + R * (int64_t)(b.r - a.r + 1), INT32_MAX);  // cost
        k.graph = 0;
        k.tail_row = tail ? b.r : -1;
        k.head_ta = -1;
        k.tail_tb = -1;
        k.pad2 = 0;
        cstart[(size_t)c] = a.k;
        ctile[(size_t)c] = (int32_t)ntiles;
        ntiles += nt;
    }
    if (ntiles > INT32_MAX / 2) return EGPR_UNSUPPORTED_GRAPH;
    g->ntiles = (int32_t)ntiles;
    // tile tables: marks by row ends, then per-lane offsets
    int32_t* d_cstart = tmp.get<int32_t>((size_t)nch, &rc);
    int32_t* d_ctile = tmp.get<int32_t>((size_t)nch, &rc);
    if (rc || (rc = g->tile_bits.alloc((size_t)ntiles * kTileWords * sizeof(uint32_t))) ||
        (rc = g->tile_row.alloc((size_t)ntiles * sizeof(int32_t))))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(d_cstart, cstart.data(), (size_t)nch * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D chunk starts")) ||
        (rc = cuda_ok(cudaMemcpyAsync(d_ctile, ctile.data(), (size_t)nch * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D chunk tiles")) ||
        (rc = cuda_ok(cudaMemsetAsync(g->tile_bits.p, 0, g->tile_bits.bytes, s), "memset")) ||
        (rc = cuda_ok(cudaMemsetAsync(g->tile_row.p, 0x7f, g->tile_row.bytes, s), "memset")))
        return rc;
    k_tile_marks<<<grid_for(n), kThreads, 0, s>>>(g->sw_row.as<int32_t>(), n, d_cstart, d_ctile, nch,
                                                   g->tile_bits.as<uint32_t>(), g->tile_row.as<int32_t>());
    k_tile_offsets<<<grid_for(ntiles * 32), kThreads, 0, s>>>(g->tile_bits.as<uint32_t>(), ntiles);
    // span links (row order), then the queue order: costliest chunks first
    g->plan.h_spans.clear();
    for (int32_t c = 0; c < nch; ++c) {
        Chunk& k = ch[(size_t)c];
        if (k.flags & kHasHead) k.head_ta = (ch[(size_t)c - 1].flags & kInterior) ? ch[(size_t)c - 1].head_ta : c - 1;
        if ((k.flags & kHasTail) && !(k.flags & kInterior)) g->plan.h_spans.push_back(c);
    }
    for (int32_t c = nch - 1; c >= 0; --c) {
        Chunk& k = ch[(size_t)c];
        if (k.flags & kHasTail) k.tail_tb = (ch[(size_t)c + 1].flags & kInterior) ? ch[(size_t)c + 1].tail_tb : c + 1;
    }
    {
        // chunks of the span each chunk adds to (its head row's, its tail row's),
        // counted before the renumbering
        std::vector<int32_t> hparts((size_t)nch, 0), tparts((size_t)nch, 0);
        for (int32_t c = 0; c < nch; ++c) {
            const Chunk& k = ch[(size_t)c];
            if (k.flags & kInterior) hparts[(size_t)c] = k.tail_tb - k.head_ta + 1;
            else if (k.flags & kHasHead) hparts[(size_t)c] = c - k.head_ta + 1;
            if ((k.flags & kHasTail) && !(k.flags & kInterior)) tparts[(size_t)c] = k.tail_tb - c + 1;
        }
        // costliest first: a stable counting sort over 4096 cost classes (the
        // order only needs to be roughly by cost, and a comparison sort of the
        // ~28K records costs milliseconds of host time)
        std::vector<int32_t> perm((size_t)nch), pos_of((size_t)nch);
        {
            int64_t cmax = 1;
            for (int32_t c = 0; c < nch; ++c) cmax = std::max<int64_t>(cmax, ch[(size_t)c].pad);
            constexpr int kClasses = 4096;
            std::vector<int32_t> start(kClasses + 1, 0);
            auto cls = [&](int32_t c) {
                return kClasses - 1 - (int32_t)(((int64_t)ch[(size_t)c].pad * (kClasses - 1)) / cmax);
            };
            for (int32_t c = 0; c < nch; ++c) start[(size_t)cls(c) + 1] += 1;
            for (int i = 0; i < kClasses; ++i) start[(size_t)i + 1] += start[(size_t)i];
            for (int32_t c = 0; c < nch; ++c) perm[(size_t)start[(size_t)cls(c)]++] = c;
        }
        for (int32_t i = 0; i < nch; ++i) pos_of[(size_t)perm[(size_t)i]] = i;
        std::vector<Chunk> sorted((size_t)nch);
        for (int32_t i = 0; i < nch; ++i) {
            Chunk k = ch[(size_t)perm[(size_t)i]];
            if (k.head_ta >= 0) k.head_ta = pos_of[(size_t)k.head_ta];
            if (k.tail_tb >= 0) k.tail_tb = pos_of[(size_t)k.tail_tb];
            k.pad = hparts[(size_t)perm[(size_t)i]];
            k.pad2 = tparts[(size_t)perm[(size_t)i]];
            sorted[(size_t)i] = k;
        }
        ch.swap(sorted);
        for (int32_t& sp : g->plan.h_spans) sp = pos_of[(size_t)sp];
    }
    // entries (a tile reads up to kTileItems + 8 entries past a chunk's start)
    const size_t pad = (size_t)(kTileItems + 16) * sizeof(int32_t);
    if ((rc = g->sw_col.alloc((size_t)nnz * sizeof(int32_t) + pad)) ||
        (g->weighted && (rc = g->sw_w.alloc((size_t)nnz * sizeof(float) + pad))))
        return rc;
    return cuda_ok(cudaGetLastError(), "sweep tables");
}

// The layout's entries: in_col (hub codes already in place) copied behind the
// row offsets, with a placeholder in every empty row.  Stream-ordered; the
// tables must be complete on the device.
int build_sweep_entries(egpr_graph* g, const uint32_t* sorted_dst, cudaStream_t s) {
    const int32_t n = g->n;
    const int32_t nnz = (int32_t)g->sw_nnz;
    const size_t pad = (size_t)(kTileItems + 16) * sizeof(int32_t);
    int rc;
    // every entry is written below; only the padding past the last one is cleared
    if ((rc = cuda_ok(cudaMemsetAsync(g->sw_col.as<int32_t>() + nnz, 0, pad, s), "memset"))) return rc;
    if (g->weighted && (rc = cuda_ok(cudaMemsetAsync(g->sw_w.as<float>() + nnz, 0, pad, s), "memset"))) return rc;
    if (sorted_dst && g->nnz > 0) {
        // entry-parallel: entry i of row r moves by the number of empty rows before r
        k_sweep_cols_by_entry<<<grid_for(g->nnz), kThreads, 0, s>>>(
            sorted_dst, g->in_row.as<int32_t>(), g->in_col.as<int32_t>(), g->weighted ? g->in_w.as<float>() : nullptr,
            g->nnz, g->sw_row.as<int32_t>(), g->sw_col.as<int32_t>(), g->weighted ? g->sw_w.as<float>() : nullptr);
        k_sweep_placeholders<<<grid_for(n), kThreads, 0, s>>>(g->in_row.as<int32_t>(), n, g->sw_row.as<int32_t>(),
                                                             g->sw_col.as<int32_t>(),
                                                             g->weighted ? g->sw_w.as<float>() : nullptr, -(g->nhub + 1));
    } else {
        k_build_sweep_cols<<<grid_for((int64_t)n * 32), kThreads, 0, s>>>(
            g->in_row.as<int32_t>(), g->in_col.as<int32_t>(), g->weighted ? g->in_w.as<float>() : nullptr, n,
            g->sw_row.as<int32_t>(), g->sw_col.as<int32_t>(), g->weighted ? g->sw_w.as<float>() : nullptr,
            -(g->nhub + 1));
    }
    return cuda_ok(cudaGetLastError(), "sweep entries");
}

int build_sweep_layout(egpr_graph* g, int32_t resident_warps, const uint32_t* sorted_dst, cudaStream_t s) {
    int rc;
    if ((rc = build_sweep_tables(g, resident_warps, s)) || (rc = build_sweep_entries(g, sorted_dst, s))) return rc;
    return cuda_ok(cudaStreamSynchronize(s), "sweep layout");
}

// ---- the binned sweep's layout -------------------------------------------------
// Renumbering key of vertex v: the hub block (the first `hubs` vertices of the
// out-degree ranking) first, then everyone else; descending in-degree inside
// each block; the sort is stable, so equal keys keep ascending vertex ids.
__global__ void k_bin_keys(const int32_t* __restrict__ in_row, int32_t n, const uint8_t* __restrict__ hub_flag,
                           uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t deg = (uint32_t)(in_row[v + 1] - in_row[v]);
        key[v] = (hub_flag[v] ? 0u : 0x80000000u) | (0x7fffffffu - deg);
        val[v] = (uint32_t)v;
    }
}

__global__ void k_bin_hub_flags(const uint32_t* __restrict__ ranked, int32_t hubs, uint8_t* __restrict__ flag) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < hubs; i += gridDim.x * blockDim.x) flag[ranked[i]] = 1;
}

// inv: the sorted vertex list; perm[inv[i]] = i; row lengths and FP64
// out-weights in the new order.
__global__ void k_bin_perm(const uint32_t* __restrict__ inv, int32_t n, const int32_t* __restrict__ in_row,
                           const double* __restrict__ outw, int32_t* __restrict__ perm, uint32_t* __restrict__ len,
                           double* __restrict__ outw_new) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)inv[i];
        perm[v] = (int32_t)i;
        len[i] = (uint32_t)(in_row[v + 1] - in_row[v]);
        outw_new[i] = outw[v];
    }
}

// Inbound entry e (destination dst[e], source in_col[e]) to its place in the
// renumbered CSR: same position inside its row, source renumbered.
__global__ void k_bin_entries(const uint32_t* __restrict__ dst, int64_t nnz, const int32_t* __restrict__ in_row,
                              const int32_t* __restrict__ in_col, const float* __restrict__ in_w,
                              const int32_t* __restrict__ perm, const int32_t* __restrict__ row_new,
                              int32_t* __restrict__ col_new, float* __restrict__ w_new) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)dst[e];
        const int64_t pos = (int64_t)row_new[perm[v]] + (e - (int64_t)in_row[v]);
        col_new[pos] = perm[in_col[e]];
        if (w_new) w_new[pos] = in_w[e];
    }
}

// Builds g->bins from the natural inbound CSR (in_row, plain source ids in
// in_col, in_w, outw) and the out-degree ranking of the vertices.  The work
// queue follows in bins_build_items.
int build_bin_layout(egpr_graph* g, const uint32_t* sorted_dst, const uint32_t* ranked, TmpAlloc& tmp,
                     cudaStream_t s) {
    const int32_t n = g->n;
    const int64_t nnz = g->nnz;
    BinLayout* B = new (std::nothrow) BinLayout();
    if (!B) return EGPR_FAILED_TO_ALLOCATE_HOST_MEM;
    g->bins = B;
    B->n = n;
    B->nnz = nnz;
    B->hubs = std::min<int32_t>(n, bin_hub_cap()) & ~3;  // a multiple of 4: the staging copy moves 16-byte units
    if (const char* e = std::getenv("EGPR_BIN_HUBS")) B->hubs = std::min<int32_t>(B->hubs, std::max(0, atoi(e)) & ~3);
    int rc = EGPR_SUCC;
    uint8_t* flag = tmp.get<uint8_t>((size_t)n, &rc);
    uint32_t* key = tmp.get<uint32_t>((size_t)n, &rc);
    uint32_t* val = tmp.get<uint32_t>((size_t)n, &rc);
    uint32_t* key2 = tmp.get<uint32_t>((size_t)n, &rc);
    uint32_t* val2 = tmp.get<uint32_t>((size_t)n, &rc);
    uint32_t* len = tmp.get<uint32_t>((size_t)n + 1, &rc);
    if (rc) return rc;
    // Every array the sweep reads row by row is padded by 16 entries (vector
    // loads near the end); the padding is zero.
    const size_t pad = 16;
    if ((rc = B->perm.alloc((size_t)n * sizeof(int32_t))) || (rc = B->inv.alloc((size_t)n * sizeof(int32_t))) ||
        (rc = B->row.alloc(((size_t)n + 1 + pad) * sizeof(int32_t))) ||
        (rc = B->col.alloc(((size_t)std::max<int64_t>(nnz, 1) + pad) * sizeof(int32_t))) ||
        (rc = B->outw.alloc(((size_t)n + pad) * sizeof(double))) ||
        (g->weighted && (rc = B->w.alloc(((size_t)std::max<int64_t>(nnz, 1) + pad) * sizeof(float)))))
        return rc;
    cudaMemsetAsync(flag, 0, (size_t)n, s);
    cudaMemsetAsync(len, 0, ((size_t)n + 1) * sizeof(uint32_t), s);  // len[n] = 0 closes the scan
    cudaMemsetAsync(B->row.p, 0, B->row.bytes, s);
    cudaMemsetAsync(B->col.p, 0, B->col.bytes, s);
    if (g->weighted) cudaMemsetAsync(B->w.p, 0, B->w.bytes, s);
    if (B->hubs > 0) k_bin_hub_flags<<<grid_for(B->hubs), kThreads, 0, s>>>(ranked, B->hubs, flag);
    k_bin_keys<<<grid_for(n), kThreads, 0, s>>>(g->in_row.as<int32_t>(), n, flag, key, val);
    bool alt = false;
    if ((rc = radix_sort_pairs(key, val, key2, val2, n, 32, s, tmp, &alt, false))) return rc;
    const uint32_t* inv = alt ? val2 : val;
    cudaMemcpyAsync(B->inv.p, inv, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    k_bin_perm<<<grid_for(n), kThreads, 0, s>>>(inv, n, g->in_row.as<int32_t>(), g->outw.as<double>(),
                                                B->perm.as<int32_t>(), len, B->outw.as<double>());
    if ((rc = exclusive_scan_u32(len, reinterpret_cast<uint32_t*>(B->row.as<int32_t>()), (int64_t)n + 1, s)))
        return rc;
    if (nnz > 0)
        k_bin_entries<<<grid_for(nnz), kThreads, 0, s>>>(sorted_dst, nnz, g->in_row.as<int32_t>(),
                                                         g->in_col.as<int32_t>(), g->weighted ? g->in_w.as<float>() : nullptr,
                                                         B->perm.as<int32_t>(), B->row.as<int32_t>(),
                                                         B->col.as<int32_t>(), g->weighted ? B->w.as<float>() : nullptr);
    if ((rc = cuda_ok(cudaGetLastError(), "binned layout"))) return rc;
    if ((rc = bins_build_items(g, s))) return rc;
    return bins_alloc_solve(g, s);
}

// ---- host inputs ------------------------------------------------------------
// A host input array reaches the device in one of three ways:
//  * already page-locked (torch pinned memory, cudaHostAlloc, a registered
//    range): copied by DMA directly;
//  * pageable, with EASYGRAPH_GPU_HOST_REGISTER set to 1/TRUE/ON/YES:
//    page-locked in place for the upload and released after it, as the
//    reference's prepare_h2d_source / release_h2d_source do
//    (gpu_easygraph/common/buffer_cache.h:115-176), for arrays of at least
//    EASYGRAPH_GPU_HOST_REGISTER_MIN_BYTES (default 1 MiB); read-only
//    mappings (memory-mapped bulk CSR files) are registered read-only where
//    the device supports it;
//  * pageable otherwise (the default here; the reference registers by
//    default): copied through a process-wide pool of page-locked staging
//    buffers, host threads filling one buffer while DMA drains the others.
//    Registering pages in place cost about 0.2 s per GB on B200 hosts, several
//    times the copy itself, and it is paid again on every call.
bool host_register_requested() {
    const char* v = std::getenv("EASYGRAPH_GPU_HOST_REGISTER");
    if (!v) return false;
    std::string s(v);
    for (char& c : s) c = (char)std::toupper((unsigned char)c);
    return s == "1" || s == "TRUE" || s == "ON" || s == "YES";
}

size_t host_register_min_bytes() {
    const char* v = std::getenv("EASYGRAPH_GPU_HOST_REGISTER_MIN_BYTES");
    const unsigned long long parsed = v ? std::strtoull(v, nullptr, 10) : 0ull;
    return parsed > 0ull ? (size_t)parsed : (size_t)1 << 20;
}

bool host_page_locked(const void* p) {
    cudaPointerAttributes a = {};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Page-locked staging buffers shared by every upload of the process (one
// upload at a time uses them).
constexpr int kStageSlots = 4;
constexpr size_t kStageBytes = (size_t)32 << 20;
struct StagePool {
    std::mutex mu;
    void* slot[kStageSlots] = {};
};
StagePool& stage_pool() {
    static StagePool* p = new StagePool();  // never destroyed: pinned memory outlives static teardown order
    return *p;
}

void parallel_memcpy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kBlock = (size_t)1 << 20;
    const int64_t blocks = (int64_t)((bytes + kBlock - 1) / kBlock);
    if (blocks <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
#pragma omp parallel for schedule(static) num_threads(std::min<int64_t>(blocks, 16))
    for (int64_t i = 0; i < blocks; ++i) {
        const size_t off = (size_t)i * kBlock;
        std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                    std::min(kBlock, bytes - off));
    }
}

// H2D copy of a pageable host array through the staging pool, enqueued on s.
// Returns once every byte has left the source array (later work on s sees
// the data in stream order).
int staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    StagePool& P = stage_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    for (int k = 0; k < kStageSlots; ++k)
        if (!P.slot[k]) {
            const cudaError_t e = cudaHostAlloc(&P.slot[k], kStageBytes, cudaHostAllocPortable);
            if (e != cudaSuccess) {
                P.slot[k] = nullptr;
                cudaGetLastError();
                // no staging memory: the driver copies from pageable memory
                return cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D (pageable)");
            }
        }
    cudaEvent_t ev[kStageSlots] = {};
    bool used[kStageSlots] = {};
    int rc = EGPR_SUCC;
    for (int k = 0; k < kStageSlots && !rc; ++k)
        rc = cuda_ok(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming), "event");
    size_t off = 0;
    for (int i = 0; off < bytes && !rc; ++i) {
        const int k = i % kStageSlots;
        const size_t len = std::min(kStageBytes, bytes - off);
        if (used[k] && (rc = cuda_ok(cudaEventSynchronize(ev[k]), "staging"))) break;
        parallel_memcpy(P.slot[k], static_cast<const char*>(src) + off, len);
        if ((rc = cuda_ok(cudaMemcpyAsync(static_cast<char*>(dst) + off, P.slot[k], len, cudaMemcpyHostToDevice, s),
                          "H2D (staged)")))
            break;
        if ((rc = cuda_ok(cudaEventRecord(ev[k], s), "event"))) break;
        used[k] = true;
        off += len;
    }
    // the slots are free again once their last copies are done
    for (int k = 0; k < kStageSlots; ++k) {
        if (used[k]) cudaEventSynchronize(ev[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
    }
    return rc;
}

// D2H copy into a pageable host array through the staging pool, after the
// work already enqueued on s: up to kStageSlots chunk copies in flight while
// host threads move finished chunks out.  Returns once every byte is in dst.
int staged_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    // the work that produces the result finishes before the pool is taken, so
    // another thread's upload or download does not wait on this stream's kernels
    int rc0 = cuda_ok(cudaStreamSynchronize(s), "D2H (staged)");
    if (rc0) return rc0;
    StagePool& P = stage_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    for (int k = 0; k < kStageSlots; ++k)
        if (!P.slot[k]) {
            const cudaError_t e = cudaHostAlloc(&P.slot[k], kStageBytes, cudaHostAllocPortable);
            if (e != cudaSuccess) {
                P.slot[k] = nullptr;
                cudaGetLastError();
                int rc = cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "D2H (pageable)");
                return rc ? rc : cuda_ok(cudaStreamSynchronize(s), "D2H (pageable)");
            }
        }
    cudaEvent_t ev[kStageSlots] = {};
    int rc = EGPR_SUCC;
    for (int k = 0; k < kStageSlots && !rc; ++k)
        rc = cuda_ok(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming), "event");
    const size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
    auto issue = [&](size_t i) {
        const int k = (int)(i % kStageSlots);
        const size_t off = i * kStageBytes, len = std::min(kStageBytes, bytes - off);
        int r = cuda_ok(cudaMemcpyAsync(P.slot[k], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, s),
                        "D2H (staged)");
        return r ? r : cuda_ok(cudaEventRecord(ev[k], s), "event");
    };
    for (size_t i = 0; i < std::min<size_t>(chunks, kStageSlots) && !rc; ++i) rc = issue(i);
    for (size_t i = 0; i < chunks && !rc; ++i) {
        const int k = (int)(i % kStageSlots);
        const size_t off = i * kStageBytes, len = std::min(kStageBytes, bytes - off);
        if ((rc = cuda_ok(cudaEventSynchronize(ev[k]), "staging"))) break;
        parallel_memcpy(static_cast<char*>(dst) + off, P.slot[k], len);
        if (i + kStageSlots < chunks) rc = issue(i + kStageSlots);
    }
    if (rc) cudaStreamSynchronize(s);  // no copy may still write into a slot once the pool is unlocked
    for (int k = 0; k < kStageSlots; ++k)
        if (ev[k]) cudaEventDestroy(ev[k]);
    return rc;
}

struct HostInputs {
    cudaStream_t stream;            // the upload's stream: drained before unregistering
    std::vector<void*> registered;  // registered here, unregistered when the upload is done
    int registered_count = 0;
    int already_locked = 0;
    int staged = 0;
    explicit HostInputs(cudaStream_t s) : stream(s) {}
    // Decides how `p` is uploaded; true when it is (now) page-locked.
    bool prepare(const void* p, size_t bytes, int dev) {
        if (!p || bytes == 0) return true;
        if (host_page_locked(p)) {
            ++already_locked;
            return true;
        }
        if (host_register_requested() && bytes >= host_register_min_bytes()) {
            int ro = 0;
            cudaDeviceGetAttribute(&ro, cudaDevAttrHostRegisterReadOnlySupported, dev);
            const unsigned flags = cudaHostRegisterPortable | (ro ? cudaHostRegisterReadOnly : 0u);
            const cudaError_t e = cudaHostRegister(const_cast<void*>(p), bytes, flags);
            if (e == cudaSuccess) {
                registered.push_back(const_cast<void*>(p));
                ++registered_count;
                return true;
            }
            cudaGetLastError();
            if (e == cudaErrorHostMemoryAlreadyRegistered) {  // not ours to unregister
                ++already_locked;
                return true;
            }
        }
        if (bytes >= ((size_t)1 << 20)) ++staged;
        return bytes < ((size_t)1 << 20);  // small arrays: the driver's pageable copy
    }
    ~HostInputs() {
        if (registered.empty()) return;
        cudaStreamSynchronize(stream);  // no copy from these pages may still be in flight
        for (void* p : registered) cudaHostUnregister(p);
        cudaGetLastError();
    }
};

// H2D of [src, src + bytes): direct when `locked`, else through the staging pool.
int upload_h2d(void* dst, const void* src, size_t bytes, bool locked, cudaStream_t s, const char* what) {
    if (bytes == 0) return EGPR_SUCC;
    if (locked) return cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), what);
    return staged_h2d(dst, src, bytes, s);
}

int download_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s, const char* what) {
    if (bytes == 0) return EGPR_SUCC;
    if (bytes < ((size_t)1 << 20) || host_page_locked(dst))
        return cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), what);
    return staged_d2h(dst, src, bytes, s);
}

int prepare_graph(egpr_graph* g, const int32_t* V, const int32_t* E, const double* W) {
    const int32_t n = g->n;
    const int64_t m = g->m_input;
    cudaStream_t s = g->own_stream;
    int rc = EGPR_SUCC;
    const double t0 = wall_seconds();
    // declared before the scratch so that registrations outlive every copy
    // (the stream is synchronised before this function returns)
    HostInputs host(s);
    const bool v_locked = host.prepare(V, ((size_t)n + 1) * sizeof(int32_t), g->device);
    const bool e_locked = host.prepare(E, (size_t)m * sizeof(int32_t), g->device);
    const bool w_locked = host.prepare(W, W ? (size_t)m * sizeof(double) : 0, g->device);
    g->host_inputs_registered = host.registered_count;
    g->host_inputs_locked = host.already_locked;
    g->host_inputs_staged = host.staged;
    cudaEventRecord(g->ev0, s);
    {
        TmpAlloc tmp(s);
        int32_t* dV = tmp.get<int32_t>((size_t)n + 1, &rc);
        int32_t* dE = tmp.get<int32_t>((size_t)m, &rc);
        double* dW = W ? tmp.get<double>((size_t)m, &rc) : nullptr;
        uint32_t* indeg = tmp.get<uint32_t>((size_t)n + 1, &rc);
        uint32_t* keys = tmp.get<uint32_t>((size_t)m, &rc);
        uint32_t* vals = tmp.get<uint32_t>((size_t)m, &rc);
        uint32_t* keys2 = tmp.get<uint32_t>((size_t)m, &rc);
        uint32_t* vals2 = tmp.get<uint32_t>((size_t)m, &rc);
        // weighted: the FP32 weight of every entry moves through the sort with its source
        uint32_t* wbits = W ? tmp.get<uint32_t>((size_t)m, &rc) : nullptr;
        uint32_t* wbits2 = W ? tmp.get<uint32_t>((size_t)m, &rc) : nullptr;
        unsigned long long* counts = tmp.get<unsigned long long>(2, &rc);
        uint32_t* hkey = tmp.get<uint32_t>((size_t)n, &rc);
        uint32_t* hval = tmp.get<uint32_t>((size_t)n, &rc);
        uint32_t* hkey2 = tmp.get<uint32_t>((size_t)n, &rc);
        uint32_t* hval2 = tmp.get<uint32_t>((size_t)n, &rc);
        // weighted: rows whose out-weight is summed sequentially (k_out_weight_exact)
        int32_t* serial_rows = W ? tmp.get<int32_t>((size_t)n, &rc) : nullptr;
        uint32_t* serial_count = W ? tmp.get<uint32_t>(1, &rc) : nullptr;
        int32_t* long_rows = W ? tmp.get<int32_t>((size_t)n, &rc) : nullptr;  // per piece: sources of many entries
        uint32_t* long_count = W ? tmp.get<uint32_t>(1, &rc) : nullptr;
        // per piece: segments of the sources of very many entries, and their accumulators
        OutSegs segs;
        const size_t max_huge = (size_t)(m / kOutWeightHuge) + 1;
        segs.seg = tmp.get<int4>((size_t)(m / kOutWeightSeg) + max_huge, &rc);
        segs.seg_count = tmp.get<uint32_t>(1, &rc);
        segs.acc = tmp.get<HugeAcc>(max_huge, &rc);
        segs.acc_count = tmp.get<uint32_t>(1, &rc);
        if (rc) return rc;
        if (W) cudaMemsetAsync(serial_count, 0, sizeof(uint32_t), s);
        // in_row, hub_slot: bulk copies of a stage's rows may read up to 3 elements past the end.
        if ((rc = g->in_row.alloc(((size_t)n + 8) * sizeof(int32_t))) ||
            (rc = g->outw.alloc((size_t)n * sizeof(double))) ||
            (rc = g->dangling01.alloc((size_t)n * sizeof(int32_t))))
            return rc;
        if ((rc = upload_h2d(dV, V, ((size_t)n + 1) * sizeof(int32_t), v_locked, s, "H2D offsets"))) return rc;
        cudaMemsetAsync(indeg, 0, ((size_t)n + 1) * sizeof(uint32_t), s);
        cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s);
        // the sort carries each entry's source (written from the offsets alone,
        // while E is still arriving) and, when weighted, its FP32 weight
        // (converted as each piece of W arrives), so no gather follows it
        if (m > 0)
            k_expand_src<<<grid_for((int64_t)n * 32), kThreads, 0, s>>>(dV, n, reinterpret_cast<int32_t*>(vals));
        {
            // E (and W) arrive in pieces on a copy stream; the degree passes of
            // each piece run on s while the next one is in flight.  A piece's
            // out-degree pass covers the rows whose entries have all arrived.
            const int pieces = m >= (int64_t)(8 << 20) ? 4 : 1;
            cudaStream_t sc = nullptr;
            std::vector<cudaEvent_t> ev((size_t)pieces, nullptr);
            if (pieces > 1) {
                rc = cuda_ok(cudaStreamCreateWithFlags(&sc, cudaStreamNonBlocking), "stream");
                for (int i = 0; i < pieces && !rc; ++i)
                    rc = cuda_ok(cudaEventCreateWithFlags(&ev[(size_t)i], cudaEventDisableTiming), "event");
                // the copy stream starts after the memsets and the offsets above
                cudaEvent_t start = nullptr;
                if (!rc) rc = cuda_ok(cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "event");
                if (!rc) rc = cuda_ok(cudaEventRecord(start, s), "event");
                if (!rc) rc = cuda_ok(cudaStreamWaitEvent(sc, start, 0), "event");
                if (start) cudaEventDestroy(start);
            }
            int32_t r_done = 0;
            for (int i = 0; i < pieces && !rc; ++i) {
                const int64_t a = m * i / pieces, b = m * (i + 1) / pieces;
                cudaStream_t cs = pieces > 1 ? sc : s;
                if (b > a) {
                    rc = upload_h2d(dE + a, E + a, (size_t)(b - a) * sizeof(int32_t), e_locked, cs, "H2D indices");
                    if (!rc && W)
                        rc = upload_h2d(dW + a, W + a, (size_t)(b - a) * sizeof(double), w_locked, cs, "H2D weights");
                }
                if (!rc && pieces > 1) {
                    rc = cuda_ok(cudaEventRecord(ev[(size_t)i], sc), "event");
                    if (!rc) rc = cuda_ok(cudaStreamWaitEvent(s, ev[(size_t)i], 0), "event");
                }
                if (rc) break;
                // rows [r_done, r_end): V[r_end] <= b, all of them when this is the last piece
                int32_t r_end = n;
                if (i + 1 < pieces) r_end = (int32_t)(std::upper_bound(V, V + n + 1, (int32_t)b) - V) - 1;
                if (r_end > r_done) {
                    cudaMemsetAsync(segs.seg_count, 0, sizeof(uint32_t), s);
                    cudaMemsetAsync(segs.acc_count, 0, sizeof(uint32_t), s);
                    if (dW) {
                        cudaMemsetAsync(long_count, 0, sizeof(uint32_t), s);
                        k_out_weight_exact<<<grid_for((int64_t)(r_end - r_done) * 8), kThreads, 0, s>>>(
                            dV, dE, dW, n, r_done, r_end, g->outw.as<double>(), hkey, hval, serial_rows,
                            serial_count, long_rows, long_count, segs);
                    } else {
                        k_out_degree<<<grid_for((int64_t)(r_end - r_done) * 32), kThreads, 0, s>>>(
                            dV, dE, n, r_done, r_end, g->outw.as<double>(), hkey, hval, segs);
                    }
                    k_out_weight_long<<<148 * 8, kThreads, 0, s>>>(dV, dE, dW, n, long_rows, long_count,
                                                                   g->outw.as<double>(), hkey, hval, serial_rows,
                                                                   serial_count, segs);
                    r_done = r_end;
                }
                if (b > a)
                    k_in_degree_keys<<<grid_for(b - a), kThreads, 0, s>>>(dE, a, b, n, indeg, keys);
                if (b > a && W) k_weight_bits<<<grid_for(b - a), kThreads, 0, s>>>(dW, a, b, wbits);
            }
            if (sc) {
                if (rc) cudaStreamSynchronize(sc);
                cudaStreamDestroy(sc);  // released once its copies are done
            }
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
            if (rc) return rc;
            if (dW && n > 0)
                k_out_weight_serial<<<grid_for(n), kThreads, 0, s>>>(dV, dE, dW, n, serial_rows, serial_count,
                                                                     g->outw.as<double>());
        }
        if ((rc = exclusive_scan_u32(indeg, reinterpret_cast<uint32_t*>(g->in_row.as<int32_t>()), (int64_t)n + 1, s)))
            return rc;
        const uint32_t* sorted_dst = nullptr;  // destination of every inbound entry, in entry order
        int32_t nnz32 = 0;
        if ((rc = cuda_ok(cudaMemcpyAsync(&nnz32, g->in_row.as<int32_t>() + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H nnz")) ||
            (rc = cuda_ok(cudaStreamSynchronize(s), "preparation")))
            return rc;
        g->nnz = nnz32;
        const int64_t nnz = g->nnz;
        // Padding: a stage's bulk copy reads up to 3 entries past the end.
        const size_t pad = 16 * sizeof(int32_t);
        if ((rc = g->in_col.alloc((size_t)std::max<int64_t>(nnz, 1) * sizeof(int32_t) + pad)))
            return rc;
        if (W && (rc = g->in_w.alloc((size_t)std::max<int64_t>(nnz, 1) * sizeof(float) + pad)))
            return rc;
        if (m > 0) {
            // keys are destinations in [0, n), and n for an out-of-range one:
            // the key width covers n only when such an entry exists
            const uint64_t kmax = nnz < m ? (uint64_t)n : (uint64_t)n - 1;
            int bits = 0;
            while (bits < 32 && (kmax >> bits) != 0) ++bits;
            bool alt = false;
            if ((rc = radix_sort_pairs(keys, vals, keys2, vals2, m, bits, s, tmp, &alt, true, wbits, wbits2)))
                return rc;
            const uint32_t* sorted_vals = alt ? vals2 : vals;
            sorted_dst = alt ? keys2 : keys;
            if (nnz > 0 && (rc = cuda_ok(cudaMemcpyAsync(g->in_col.p, sorted_vals, (size_t)nnz * sizeof(int32_t),
                                                         cudaMemcpyDeviceToDevice, s), "inbound sources")))
                return rc;
            if (W && nnz > 0 &&
                (rc = cuda_ok(cudaMemcpyAsync(g->in_w.p, alt ? wbits2 : wbits, (size_t)nnz * sizeof(float),
                                              cudaMemcpyDeviceToDevice, s), "inbound weights")))
                return rc;
        }
        // Hubs: the min(n, kHubCap) sources of largest out-degree (a multiple of 4,
        // the granule of the shared-memory staging copy).
        // EGPR_HUBS=N: hub cache size (0: none); at most kHubCap - 32, which leaves
        // room for the zero slot nhub in a kHubCap-value copy.  By default 24,544
        // hubs, and 16,352 from 2^24 vertices: the shared memory the hubs take is
        // L1 the sweep's other loads lose, and measured on B200 the smaller cache
        // wins once the rank vector no longer fits L2 (R-MAT scale 25 weighted:
        // 2.02 ms per sweep with 16K hubs, 2.06 with 8K, 2.08 with 24K, 2.32 with
        // 32K; scale 22: 0.236, 0.224, 0.222 ms with 8K, 24K, 32K)
        const char* hub_env = std::getenv("EGPR_HUBS");
        const int32_t hub_default = n >= (1 << 24) ? 16384 - 32 : 24576 - 32;
        const int32_t hub_want = hub_env ? std::max(0, std::atoi(hub_env)) : hub_default;
        g->nhub = std::min<int32_t>(std::min<int32_t>(n, hub_want), kHubCap - 32) & ~3;
        if ((rc = g->hub_slot.alloc(((size_t)n + 8) * sizeof(int32_t))) ||
            (rc = g->hub_ids.alloc((size_t)std::max(g->nhub + 1, 4) * sizeof(int32_t))) ||
            (rc = cuda_ok(cudaMemsetAsync(g->hub_slot.p, 0xff, ((size_t)n + 8) * sizeof(int32_t), s), "memset")))
            return rc;
        // the out-degree ranking (descending, ties by id): the hubs of both sweeps
        const bool want_bins = bins_wanted(n, nnz);
        const uint32_t* ranked = nullptr;
        if (g->nhub > 0 || want_bins) {
            bool alt = false;
            if ((rc = radix_sort_pairs(hkey, hval, hkey2, hval2, n, 32, s, tmp, &alt, false))) return rc;
            ranked = alt ? hval2 : hval;
        }
        // the binned layout reads in_col before the hub codes go in
        if (want_bins && (rc = build_bin_layout(g, sorted_dst, ranked, tmp, s))) return rc;
        if (g->nhub > 0) {
            k_hub_slots<<<grid_for(g->nhub), kThreads, 0, s>>>(ranked, g->nhub, g->hub_ids.as<int32_t>(),
                                                               g->hub_slot.as<int32_t>());
            if (nnz > 0)
                k_encode_hubs<<<grid_for(nnz), kThreads, 0, s>>>(g->in_col.as<int32_t>(), nnz, g->hub_slot.as<int32_t>());
        }
        // hub slot nhub is the zero slot of placeholder entries; in the FP64
        // correction sweep it reads z64[n] = 0
        if ((rc = cuda_ok(cudaMemcpyAsync(g->hub_ids.as<int32_t>() + g->nhub, &g->n, sizeof(int32_t),
                                          cudaMemcpyHostToDevice, s), "H2D zero slot")))
            return rc;
        k_dangling<<<grid_for(n), kThreads, 0, s>>>(g->outw.as<double>(), n, g->dangling01.as<int32_t>(), counts);
        // The layout's tables need in_row only (complete since the nnz read
        // above): they are built on a second stream while the inbound sort, the
        // gather and the hub ranking run on s; the entries then follow on s.
        cudaStream_t s2 = nullptr;
        cudaEvent_t e2 = nullptr;
        if ((rc = cuda_ok(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking), "stream")) ||
            (rc = cuda_ok(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming), "event"))) {
            if (s2) cudaStreamDestroy(s2);
            return rc;
        }
        rc = build_sweep_tables(g, sweep_resident_warps(), s2);
        if (!rc) rc = cuda_ok(cudaEventRecord(e2, s2), "event");
        if (!rc) rc = cuda_ok(cudaStreamWaitEvent(s, e2, 0), "event");
        if (!rc) rc = build_sweep_entries(g, sorted_dst, s);
        if (rc) cudaStreamSynchronize(s2);  // nothing of s2 may outlive an early return
        cudaEventDestroy(e2);
        cudaStreamDestroy(s2);  // released once its work is done
        if (rc) return rc;
        unsigned long long hc[2] = {0, 0};
        // a copy into pageable memory returns once it is done, after all of s above
        if ((rc = cuda_ok(cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, s), "D2H counts")))
            return rc;
        g->n_dangling = (int32_t)hc[0];
        g->n_dangling_solve = (int32_t)hc[1];
    }
    cudaEventRecord(g->ev1, s);
    if ((rc = cuda_ok(cudaStreamSynchronize(s), "preparation"))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    g->prep_seconds = ms * 1e-3;
    (void)t0;
    return EGPR_SUCC;
}

// Copies in_col to the host with hub entries decoded back to source ids.
int export_in_col(const egpr_graph* g, int32_t* host, cudaStream_t s) {
    if (g->nnz <= 0) return EGPR_SUCC;
    int32_t* tmp = nullptr;
    int rc = cuda_ok(cudaMallocAsync(&tmp, (size_t)g->nnz * sizeof(int32_t), s), "cudaMallocAsync (export)");
    if (rc) return rc;
    k_decode_hubs<<<grid_for(g->nnz), kThreads, 0, s>>>(g->in_col.as<int32_t>(), g->nnz, g->hub_ids.as<int32_t>(),
                                                        tmp);
    rc = cuda_ok(cudaMemcpyAsync(host, tmp, (size_t)g->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H in_col");
    cudaFreeAsync(tmp, s);
    return rc;
}

}  // namespace egpr
