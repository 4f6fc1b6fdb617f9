// Batched personalised PageRank: k teleport vectors per graph, one CSR x dense
// SpMM per sweep.
//
// Maths per column j (the reference's power iteration, easygraph/functions/
// centrality/pagerank.py:112-139, with the (1-alpha)/n teleport term replaced
// by (1-alpha) * p_j[v]; dangling mass stays uniform):
//     X_new[v][j] = sum_{u -> v} w_uv * alpha * X[u][j] / outw[u]
//                 + (1-alpha) * p_j[v] + alpha * D_j / n
// Column j stops on its own L1 rule err_j < tol*n and keeps its own count.
//
// Layout: columns in panels of 32 (one warp lane per column); X is
// panel-major [panel][vertex][32] FP32, so gathering one source row of a panel
// is one coalesced 128-byte load.  Teleport vectors are sparse per vertex
// (seed sets), so the epilogue reads two offsets per row.
//
// Work split: the single-vector sweep's merge-path sub-tiles, with one warp per
// 256-item slice of a sub-tile instead of one thread per 8 items: every warp
// walks its slice once, its 32 lanes accumulating their 32 columns, with up to
// kBatch gathers in flight.  Rows cut between warps, sub-tiles and chunks are
// combined exactly as in the single-vector sweep (deterministic, no waiting).
// Work units are (panel, chunk) pairs in panel-major order, so all CTAs sweep
// one panel's working set at a time and each inbound entry loaded into shared
// memory feeds 32 columns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "egpr_internal.cuh"

namespace egpr {
namespace {

constexpr int kLanes = 32;
constexpr int kWarpsS = kThreads / 32;
constexpr int kItemsPerWarp = kSubItems / kWarpsS;
constexpr int kBatch = 8;

struct ColState {
    double dmass;
    double dmass_prev;
    double residual;
    double residual64;
    double xsum;
    double dsum;
    int32_t iter;
    int32_t done;
    int32_t converged;
    int32_t active;  // column < k
};

struct SpmmParams {
    const Chunk* chunks;
    int32_t nchunks;
    int32_t npanels;
    int32_t n;
    int32_t max_iter;
    const int32_t* in_row;
    const int32_t* in_col;   // hub entries store -(slot + 1)
    const int32_t* hub_ids;
    const float* in_w;
    const int2* sub_coord;
    const double* outw;
    const float* scale;     // alpha/outw or -1 (dangling)
    const int32_t* tele_ptr;  // n+1
    const int32_t* tele_col;  // entries: column
    const float* tele_val;    // entries: teleport probability
    float* X[2];
    double* out64;
    ColState* cols;
    double alpha;
    double tol_n;
    double* chunk_part;   // [panel][chunk][3][32]
    double* piece;        // [panel][chunk][2][32]
    uint32_t* span_cnt;   // [panel][chunk]
    double* span_part;    // [panel][chunk][3][32]
    uint32_t* panel_arrive;
    Ctl* ctl;
};

template <typename Real>
struct SpmmSmem {
    int32_t col[kSubItems];
    float w[kSubItems];
    float sc[kSubItems];        // FP32 sweep: max(scale, 0) of the source
    double outw[kSubItems];     // FP64 sweep: out-weight of the source
    int32_t rowend[kSubItems + 1];
    Real first_val[kWarpsS][kLanes];
    Real carry_val[kWarpsS][kLanes];
    int32_t first_row[kWarpsS];
    int32_t carry_row[kWarpsS];
    Real sub_carry[kLanes];
    Real head_val[kLanes];
    double red[3][kWarpsS][kLanes];
    int32_t head_pending;
    int32_t unit;
    int32_t is_last;
};

__device__ __forceinline__ size_t pidx(int32_t p, int32_t c, int32_t nchunks) {
    return (size_t)p * (size_t)nchunks + (size_t)c;
}

struct LaneView {
    const float* xin;   // this lane's previous iterate (panel base)
    float* xout;        // FP32 sweep output (panel base)
    double* out64;      // FP64 sweep output (panel base)
    double dmass;
    bool live;          // lane's column takes part
};

template <typename Real>
__device__ __forceinline__ void finish_row_s(const SpmmParams& P, const LaneView& L, int32_t col, int32_t v,
                                             double acc, double& err, double& dsum, double& xsum) {
    if (!L.live) return;
    double t = 0.0;
    const int32_t e0 = P.tele_ptr[v], e1 = P.tele_ptr[v + 1];
    for (int32_t e = e0; e < e1; ++e)
        if (P.tele_col[e] == col) t += (double)P.tele_val[e];
    const double val = (acc + (1.0 - P.alpha) * t) + L.dmass;
    const size_t off = (size_t)v * kLanes + (threadIdx.x & 31);
    const double prev = (double)L.xin[off];
    if constexpr (std::is_same<Real, float>::value) {
        const float xo = (float)val;
        err += fabs((double)xo - prev);
        L.xout[off] = xo;
        if (P.scale[v] < 0.f) dsum += (double)xo;
        xsum += (double)xo;
    } else {
        err += fabs(val - prev);
        L.out64[off] = val;
        xsum += val;
    }
}

// Warp-level span arrival (warp 0 of the CTA); pieces combined lane-wise in chunk order.
template <typename Real>
__device__ void span_arrive_s(const SpmmParams& P, const LaneView& L, int32_t col, int32_t p, int32_t ta,
                              int32_t participants) {
    const int lane = threadIdx.x & 31;
    uint32_t prev = 0;
    if (lane == 0) prev = atomicAdd(&P.span_cnt[pidx(p, ta, P.nchunks)], 1u);
    prev = __shfl_sync(0xffffffffu, prev, 0);
    if (prev != (uint32_t)(participants - 1)) return;
    __threadfence();
    const Chunk cta = P.chunks[ta];
    const int32_t tb = cta.tail_tb;
    double sum = __ldcg(&P.piece[(pidx(p, ta, P.nchunks) * 2 + 1) * kLanes + lane]);
    for (int32_t q = ta + 1; q < tb; ++q) sum += __ldcg(&P.piece[(pidx(p, q, P.nchunks) * 2 + 1) * kLanes + lane]);
    sum += __ldcg(&P.piece[(pidx(p, tb, P.nchunks) * 2) * kLanes + lane]);
    if (lane == 0) P.span_cnt[pidx(p, ta, P.nchunks)] = 0u;
    double e = 0.0, d = 0.0, x = 0.0;
    finish_row_s<Real>(P, L, col, cta.tail_row, sum, e, d, x);
    double* sp = P.span_part + pidx(p, ta, P.nchunks) * 3 * kLanes;
    sp[lane] = e;
    sp[kLanes + lane] = d;
    sp[2 * kLanes + lane] = x;
    __threadfence();
}

template <typename Real>
__device__ void panel_reduce(const SpmmParams& P, SpmmSmem<Real>& S, int32_t p) {
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double e = 0.0, d = 0.0, x = 0.0;
    for (int32_t c = warp; c < P.nchunks; c += kWarpsS) {
        const size_t b = pidx(p, c, P.nchunks) * 3 * kLanes;
        e += __ldcg(&P.chunk_part[b + lane]) + __ldcg(&P.span_part[b + lane]);
        d += __ldcg(&P.chunk_part[b + kLanes + lane]) + __ldcg(&P.span_part[b + kLanes + lane]);
        x += __ldcg(&P.chunk_part[b + 2 * kLanes + lane]) + __ldcg(&P.span_part[b + 2 * kLanes + lane]);
        P.span_part[b + lane] = 0.0;
        P.span_part[b + kLanes + lane] = 0.0;
        P.span_part[b + 2 * kLanes + lane] = 0.0;
    }
    S.red[0][warp][lane] = e;
    S.red[1][warp][lane] = d;
    S.red[2][warp][lane] = x;
    __syncthreads();
    if (warp == 0) {
        e = 0.0; d = 0.0; x = 0.0;
        for (int w = 0; w < kWarpsS; ++w) {
            e += S.red[0][w][lane];
            d += S.red[1][w][lane];
            x += S.red[2][w][lane];
        }
        ColState* cs = P.cols + (size_t)p * kLanes + lane;
        if constexpr (std::is_same<Real, float>::value) {
            if (cs->active && !cs->done) {
                cs->residual = e;
                cs->dsum = d;
                cs->xsum = x;
                cs->dmass_prev = cs->dmass;
                cs->dmass = P.alpha * d / (double)P.n;
                const int32_t it = cs->iter + 1;
                cs->iter = it;
                const bool conv = e < P.tol_n;
                if (conv || it >= P.max_iter) {
                    cs->done = 1;
                    cs->converged = conv ? 1 : 0;
                    atomicSub(&P.ctl->active, 1);
                }
            }
        } else {
            if (cs->active) {
                cs->residual64 = e;
                cs->xsum = x;
            }
        }
        if (lane == 0) P.panel_arrive[p] = 0u;
        __threadfence();
    }
    __syncthreads();
}

template <typename Real>
__device__ void process_unit(const SpmmParams& P, int32_t p, int32_t c, SpmmSmem<Real>& S) {
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int32_t col = p * kLanes + lane;
    const ColState cs = P.cols[col];
    const size_t pbase = (size_t)p * (size_t)P.n * kLanes;
    LaneView L;
    if (!kFinal) {
        L.live = cs.active && !cs.done;
        const unsigned live_mask = __ballot_sync(0xffffffffu, L.live);
        if (live_mask == 0u) return;  // whole panel frozen (same answer in every warp)
        const int src_lane = __ffs(live_mask) - 1;
        const int32_t it = __shfl_sync(0xffffffffu, cs.iter, src_lane);  // active columns share the count
        const int par = it & 1;
        L.xin = P.X[par] + pbase;
        L.xout = P.X[par ^ 1] + pbase;
        L.out64 = nullptr;
        L.dmass = cs.dmass;
    } else {
        L.live = cs.active != 0;
        const int par = (cs.iter - 1) & 1;  // x_{k-1} of this column
        L.xin = P.X[par] + pbase;
        L.xout = nullptr;
        L.out64 = P.out64 + pbase;
        L.dmass = cs.dmass_prev;
    }
    // Gather base: the previous iterate of the active columns (FP32 sweep) or
    // each column's x_{k-1} (FP64 sweep).
    const float* __restrict__ gbase = L.xin;
    const Chunk ck = P.chunks[c];
    double err = 0.0, dsum = 0.0, xsum = 0.0;
    if (tid < kLanes) {
        S.sub_carry[tid] = Real(0);
        S.head_val[tid] = Real(0);
    }
    if (tid == 0) S.head_pending = (ck.flags & kHasHead) ? 1 : 0;
    for (int32_t sidx = ck.sub_begin; sidx < ck.sub_end; ++sidx) {
        const int2 a = P.sub_coord[sidx];
        const int2 b = P.sub_coord[sidx + 1];
        const int32_t ra = a.x, ka = a.y;
        const int32_t nnz_sub = b.y - a.y;
        const int32_t nrows = b.x - a.x;
        for (int32_t i = tid; i < nnz_sub; i += kThreads) {
            const int32_t cu = P.in_col[ka + i];
            const int32_t u = cu >= 0 ? cu : P.hub_ids[-cu - 1];  // hub entries store -(slot + 1)
            S.col[i] = u;
            S.w[i] = P.in_w ? P.in_w[ka + i] : 1.0f;
            if constexpr (kFinal) S.outw[i] = P.outw[u];
            else S.sc[i] = fmaxf(P.scale[u], 0.f);
        }
        for (int32_t i = tid; i < nrows; i += kThreads) S.rowend[i] = P.in_row[ra + i + 1] - ka;
        __syncthreads();
        // This warp's slice of the merge path: [d0, d1).
        const int32_t total = nrows + nnz_sub;
        const int32_t d0 = min(warp * kItemsPerWarp, total);
        const int32_t d1 = min(d0 + kItemsPerWarp, total);
        auto search = [&](int32_t diag) {
            int32_t lo = max(diag - nnz_sub, 0), hi = min(diag, nrows);
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (S.rowend[mid] <= diag - mid - 1) lo = mid + 1;
                else hi = mid;
            }
            return lo;
        };
        const int32_t i0 = search(d0), i1 = search(d1);
        const int32_t j0 = d0 - i0, j1 = d1 - i1;
        int32_t i = i0;
        Real acc = Real(0);
        int32_t first = -1;
        auto complete_row = [&](int32_t r) {
            if (first < 0) {
                first = r;
                S.first_val[warp][lane] = acc;
            } else if (!(r == 0 && S.head_pending)) {
                finish_row_s<Real>(P, L, col, ra + r, (double)acc, err, dsum, xsum);
            }
            acc = Real(0);
        };
        for (int32_t jb = j0; jb < j1; jb += kBatch) {
            Real v[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int32_t jj = jb + q;
                if (jj < j1) {
                    const int32_t u = S.col[jj];
                    if constexpr (kFinal) {
                        const double o = S.outw[jj];
                        const double xv = (double)gbase[(size_t)u * kLanes + lane];
                        v[q] = o <= 1e-15 ? 0.0 : P.alpha * xv / o;
                    } else {
                        v[q] = gbase[(size_t)u * kLanes + lane] * S.sc[jj];
                    }
                } else {
                    v[q] = Real(0);
                }
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int32_t jj = jb + q;
                if (jj < j1) {
                    while (i < i1 && S.rowend[i] <= jj) {
                        complete_row(i);
                        ++i;
                    }
                    acc += (Real)S.w[jj] * v[q];
                }
            }
        }
        while (i < i1) {
            complete_row(i);
            ++i;
        }
        if (lane == 0) {
            S.first_row[warp] = first;
            S.carry_row[warp] = i;
        }
        S.carry_val[warp][lane] = acc;
        __syncthreads();
        // Fix-up of each warp's first completed row with the earlier warps' carries.
        const int32_t fr = S.first_row[warp];
        const Real cin = S.sub_carry[lane];
        if (fr >= 0) {
            Real vsum = S.first_val[warp][lane];
            int32_t t = warp - 1;
            while (t >= 0 && S.carry_row[t] == fr) {
                vsum += S.carry_val[t][lane];
                --t;
            }
            if (t < 0 && fr == 0) vsum += cin;
            if (fr == 0 && S.head_pending) S.head_val[lane] = vsum;
            else finish_row_s<Real>(P, L, col, ra + fr, (double)vsum, err, dsum, xsum);
        }
        Real out_carry = Real(0);
        if (warp == kWarpsS - 1) {
            int32_t t = kWarpsS - 1;
            while (t >= 0 && S.carry_row[t] == nrows) {
                out_carry += S.carry_val[t][lane];
                --t;
            }
            if (t < 0 && nrows == 0) out_carry += cin;
        }
        __syncthreads();
        if (warp == kWarpsS - 1) S.sub_carry[lane] = out_carry;
        if (tid == 0 && nrows > 0) S.head_pending = 0;
    }
    __syncthreads();
    // Per-column partials of this unit (fixed order over warps).
    S.red[0][warp][lane] = err;
    S.red[1][warp][lane] = dsum;
    S.red[2][warp][lane] = xsum;
    __syncthreads();
    if (warp == 0) {
        double e = 0.0, d = 0.0, x = 0.0;
        for (int w = 0; w < kWarpsS; ++w) {
            e += S.red[0][w][lane];
            d += S.red[1][w][lane];
            x += S.red[2][w][lane];
        }
        const size_t u = pidx(p, c, P.nchunks);
        P.chunk_part[u * 3 * kLanes + lane] = e;
        P.chunk_part[u * 3 * kLanes + kLanes + lane] = d;
        P.chunk_part[u * 3 * kLanes + 2 * kLanes + lane] = x;
        const int32_t f = ck.flags;
        if ((f & kHasHead) && !(f & kInterior)) P.piece[(u * 2) * kLanes + lane] = (double)S.head_val[lane];
        if (f & kHasTail) P.piece[(u * 2 + 1) * kLanes + lane] = (double)S.sub_carry[lane];
        __threadfence();
        if (f & kInterior) {
            span_arrive_s<Real>(P, L, col, p, ck.head_ta, ck.tail_tb - ck.head_ta + 1);
        } else {
            if (f & kHasHead) span_arrive_s<Real>(P, L, col, p, ck.head_ta, c - ck.head_ta + 1);
            if (f & kHasTail) span_arrive_s<Real>(P, L, col, p, c, ck.tail_tb - c + 1);
        }
        __threadfence();
        uint32_t prev = 0;
        if (lane == 0) prev = atomicAdd(&P.panel_arrive[p], 1u);
        if (lane == 0) S.is_last = (prev == (uint32_t)(P.nchunks - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (S.is_last) panel_reduce<Real>(P, S, p);
    __syncthreads();
}

template <typename Real>
__global__ void __launch_bounds__(kThreads)
k_spmm(const SpmmParams* __restrict__ Pdev, cudaGraphConditionalHandle cond, int32_t use_cond) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SpmmSmem<Real>& S = *reinterpret_cast<SpmmSmem<Real>*>(smem_raw);
    __shared__ SpmmParams P;
    if (threadIdx.x == 0) P = *Pdev;
    __syncthreads();
    constexpr bool kFinal = std::is_same<Real, double>::value;
    const bool idle = !kFinal && __ldcg(&P.ctl->active) <= 0;
    const int32_t units = P.npanels * P.nchunks;
    if (!idle) {
        for (;;) {
            if (threadIdx.x == 0) S.unit = (int32_t)atomicAdd(&P.ctl->queue, 1u);
            __syncthreads();
            const int32_t u = S.unit;
            __syncthreads();
            if (u >= units) break;
            process_unit<Real>(P, u / P.nchunks, u % P.nchunks, S);
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&P.ctl->exited, 1u);
        if (prev == gridDim.x - 1) {
            P.ctl->queue = 0u;
            P.ctl->exited = 0u;
            if (!kFinal) {
                const int32_t launches = P.ctl->launches + 1;
                P.ctl->launches = launches;
                const int32_t active = __ldcg(&P.ctl->active);
                const bool more = active > 0 && launches < P.ctl->cap;
                if (active > 0 && launches >= P.ctl->cap) P.ctl->error = EGPR_TIMEOUT;
                if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
            }
            __threadfence();
        }
    }
}

// X0 = 1/n on live columns, 0 on padding; column states.
__global__ void k_spmm_init(float* X0, ColState* cols, int32_t n, int32_t npanels, int32_t k, double alpha,
                            int32_t ndang) {
    const float x0 = (float)(1.0 / (double)n);
    const int64_t total = (int64_t)npanels * n * kLanes;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t lane = (int32_t)(i & 31);
        const int32_t p = (int32_t)(i / ((int64_t)n * kLanes));
        X0[i] = (p * kLanes + lane) < k ? x0 : 0.f;
    }
    const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < npanels * kLanes) {
        ColState c;
        c.dsum = (double)ndang * (double)x0;
        c.dmass = alpha * c.dsum / (double)n;
        c.dmass_prev = c.dmass;
        c.residual = 0.0;
        c.residual64 = 0.0;
        c.xsum = 0.0;
        c.iter = 0;
        c.active = j < k ? 1 : 0;
        c.done = j < k ? 0 : 1;
        c.converged = 0;
        cols[j] = c;
    }
}

// out[j*n + v] = final iterate / its sum (panel-major FP64 or FP32 source),
// transposed through shared memory so both sides are coalesced.
__global__ void k_spmm_normalize(const double* __restrict__ out64, const float* X0, const float* X1,
                                 const ColState* __restrict__ cols, int32_t n, int32_t k, int32_t from_fp32,
                                 double* __restrict__ out) {
    __shared__ double tile[32][33];
    const int32_t p = blockIdx.y;
    const int32_t v0 = blockIdx.x * 32;
    const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;  // 8 rows per pass
    const int32_t col = p * kLanes + lane;
    const ColState cs = cols[col];
    const float* xl = (cs.iter & 1) ? X1 : X0;
    const double inv = cs.xsum > 0.0 ? 1.0 / cs.xsum : 0.0;
    const double uni = 1.0 / (double)n;
    for (int r = row; r < 32; r += kThreads / 32) {
        const int32_t v = v0 + r;
        double val = 0.0;
        if (v < n) {
            const size_t off = ((size_t)p * n + v) * kLanes + lane;
            const double raw = from_fp32 ? (double)xl[off] : out64[off];
            val = cs.xsum > 0.0 ? raw * inv : uni;
        }
        tile[r][lane] = val;
    }
    __syncthreads();
    for (int r = row; r < 32; r += kThreads / 32) {
        const int32_t j = p * kLanes + r;
        const int32_t v = v0 + lane;
        if (j < k && v < n) out[(size_t)j * n + v] = tile[lane][r];
    }
}

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? EGPR_SUCC : set_cuda_error(e, what); }

size_t smem_bytes(bool final) {
    return final ? sizeof(SpmmSmem<double>) : sizeof(SpmmSmem<float>);
}

int spmm_grid(bool final) {
    static int cached[2][64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int& c = cached[final ? 1 : 0][dev];
    if (c > 0) return c;
    int sms = 148, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (final) {
        cudaFuncSetAttribute(k_spmm<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(true));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_spmm<double>, kThreads, smem_bytes(true));
    } else {
        cudaFuncSetAttribute(k_spmm<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(false));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_spmm<float>, kThreads, smem_bytes(false));
    }
    c = sms * std::max(per, 1);
    return c;
}

}  // namespace

// Per-handle SpMM workspace (grow-only by panel count).
struct SpmmWork {
    int32_t npanels = 0;
    int32_t nchunks = 0;
    std::vector<Chunk> chunks;
    DevBuf d_chunks, X0, X1, out64, out, cols, chunk_part, piece, span_cnt, span_part, panel_arrive, ctl, tele_ptr,
        tele_col, tele_val, params;
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t cg_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    bool cg_failed = false;
    ~SpmmWork() {
        if (cg_exec) cudaGraphExecDestroy(cg_exec);
        if (cg) cudaGraphDestroy(cg);
    }
};

void spmm_work_release(egpr_graph* g) {
    delete g->spmm;
    g->spmm = nullptr;
}

int ppr_batch_solve(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k,
                    const double* teleport_dense, const int32_t* seed_ptr, const int32_t* seeds, uint32_t flags,
                    double* out, egpr_stats* stats) {
    const double t0 = wall_seconds();
    int rc;
    if ((rc = check_device(g))) return rc;
    if (max_iter < 1) max_iter = 1;
    if (!(tol > 0.0)) tol = 0.0;
    const int32_t n = g->n;
    // Sparse teleport entries grouped by vertex.
    std::vector<int64_t> cnt((size_t)n + 1, 0);
    std::vector<std::vector<std::pair<int32_t, float>>> per_col((size_t)k);
    for (int32_t j = 0; j < k; ++j) {
        auto& ent = per_col[(size_t)j];
        if (teleport_dense) {
            const double* pj = teleport_dense + (size_t)j * n;
            double s = 0.0;
            for (int32_t v = 0; v < n; ++v) {
                if (!(pj[v] >= 0.0) || !std::isfinite(pj[v])) return EGPR_INVALID_ARGUMENT;
                s += pj[v];
            }
            if (!(s > 0.0)) return EGPR_INVALID_ARGUMENT;
            for (int32_t v = 0; v < n; ++v)
                if (pj[v] > 0.0) ent.emplace_back(v, (float)(pj[v] / s));
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
        for (auto& pr : ent) cnt[(size_t)pr.first + 1]++;
    }
    if (g->nnz == 0) {  // pagerank.py:96-98: no edges -> uniform
        for (size_t i = 0; i < (size_t)k * n; ++i) out[i] = 1.0 / n;
        if (stats)
            for (int32_t j = 0; j < k; ++j) {
                std::memset(&stats[j], 0, sizeof(egpr_stats));
                stats[j].total_seconds = wall_seconds() - t0;
            }
        return EGPR_SUCC;
    }
    for (int32_t v = 0; v < n; ++v) cnt[(size_t)v + 1] += cnt[(size_t)v];
    const int64_t nent = cnt[(size_t)n];
    std::vector<int32_t> tptr((size_t)n + 1), tcol((size_t)std::max<int64_t>(nent, 1));
    std::vector<float> tval((size_t)std::max<int64_t>(nent, 1));
    {
        std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
        for (int32_t j = 0; j < k; ++j)
            for (auto& pr : per_col[(size_t)j]) {
                const int64_t pos = cur[(size_t)pr.first]++;
                tcol[(size_t)pos] = j;
                tval[(size_t)pos] = pr.second;
            }
        for (int32_t v = 0; v <= n; ++v) tptr[(size_t)v] = (int32_t)cnt[(size_t)v];
    }
    cudaStream_t s = g->stream;
    const int32_t npanels = (k + kLanes - 1) / kLanes;
    if (!g->spmm) g->spmm = new SpmmWork();
    SpmmWork& w = *g->spmm;
    if (w.npanels < npanels || w.chunks.empty()) {
        // Coarser chunks than the single-vector sweep: units = panels x chunks.
        const int grid = spmm_grid(false);
        const int32_t target = std::max(1, (2 * grid + npanels - 1) / npanels);
        const int32_t chunk_subs = std::max<int32_t>(1, (g->nsub + target - 1) / target);
        if ((rc = build_chunk_table(g, chunk_subs, w.chunks, s))) return rc;
        w.nchunks = (int32_t)w.chunks.size();
        const size_t units = (size_t)npanels * w.nchunks;
        const size_t xs = (size_t)npanels * n * kLanes;
        if ((rc = w.d_chunks.alloc(w.chunks.size() * sizeof(Chunk))) || (rc = w.X0.alloc(xs * sizeof(float))) ||
            (rc = w.X1.alloc(xs * sizeof(float))) || (rc = w.out64.alloc(xs * sizeof(double))) ||
            (rc = w.cols.alloc((size_t)npanels * kLanes * sizeof(ColState))) ||
            (rc = w.chunk_part.alloc(units * 3 * kLanes * sizeof(double))) ||
            (rc = w.piece.alloc(units * 2 * kLanes * sizeof(double))) ||
            (rc = w.span_cnt.alloc(units * sizeof(uint32_t))) ||
            (rc = w.span_part.alloc(units * 3 * kLanes * sizeof(double))) ||
            (rc = w.panel_arrive.alloc((size_t)npanels * sizeof(uint32_t))) || (rc = w.ctl.alloc(sizeof(Ctl))) ||
            (rc = w.params.alloc(sizeof(SpmmParams))))
            return rc;
        if ((rc = cuda_ok(cudaMemcpyAsync(w.d_chunks.p, w.chunks.data(), w.chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice, s), "H2D chunks")) ||
            (rc = cuda_ok(cudaMemsetAsync(w.span_cnt.p, 0, units * sizeof(uint32_t), s), "memset")) ||
            (rc = cuda_ok(cudaMemsetAsync(w.span_part.p, 0, units * 3 * kLanes * sizeof(double), s), "memset")) ||
            (rc = cuda_ok(cudaMemsetAsync(w.panel_arrive.p, 0, (size_t)npanels * sizeof(uint32_t), s), "memset")))
            return rc;
        if (w.cg_exec) cudaGraphExecDestroy(w.cg_exec);
        if (w.cg) cudaGraphDestroy(w.cg);
        w.cg_exec = nullptr;
        w.cg = nullptr;
        w.cg_failed = false;
        w.npanels = npanels;
    }
    if ((size_t)k * n * sizeof(double) > w.out.bytes && (rc = w.out.alloc((size_t)k * n * sizeof(double)))) return rc;
    if ((rc = w.tele_ptr.alloc(tptr.size() * sizeof(int32_t))) || (rc = w.tele_col.alloc(tcol.size() * sizeof(int32_t))) ||
        (rc = w.tele_val.alloc(tval.size() * sizeof(float))))
        return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(w.tele_ptr.p, tptr.data(), tptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D teleport")) ||
        (rc = cuda_ok(cudaMemcpyAsync(w.tele_col.p, tcol.data(), tcol.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D teleport")) ||
        (rc = cuda_ok(cudaMemcpyAsync(w.tele_val.p, tval.data(), tval.size() * sizeof(float), cudaMemcpyHostToDevice, s), "H2D teleport")))
        return rc;
    // Per-vertex scale for this alpha (the single-vector set-up kernel writes it).
    if ((rc = launch_init(g->plan, alpha, max_iter, tol, false, s))) return rc;

    SpmmParams P;
    P.chunks = w.d_chunks.as<Chunk>();
    P.nchunks = w.nchunks;
    P.npanels = npanels;
    P.n = n;
    P.max_iter = max_iter;
    P.in_row = g->in_row.as<int32_t>();
    P.in_col = g->in_col.as<int32_t>();
    P.hub_ids = g->hub_ids.as<int32_t>();
    P.in_w = g->weighted ? g->in_w.as<float>() : nullptr;
    P.sub_coord = g->sub_coord.as<int2>();
    P.outw = g->outw.as<double>();
    P.scale = g->scale.as<float>();
    P.tele_ptr = w.tele_ptr.as<int32_t>();
    P.tele_col = w.tele_col.as<int32_t>();
    P.tele_val = w.tele_val.as<float>();
    P.X[0] = w.X0.as<float>();
    P.X[1] = w.X1.as<float>();
    P.out64 = w.out64.as<double>();
    P.cols = w.cols.as<ColState>();
    P.alpha = alpha;
    P.tol_n = tol * (double)n;
    P.chunk_part = w.chunk_part.as<double>();
    P.piece = w.piece.as<double>();
    P.span_cnt = w.span_cnt.as<uint32_t>();
    P.span_part = w.span_part.as<double>();
    P.panel_arrive = w.panel_arrive.as<uint32_t>();
    P.ctl = w.ctl.as<Ctl>();
    if ((rc = cuda_ok(cudaMemcpyAsync(w.params.p, &P, sizeof(P), cudaMemcpyHostToDevice, s), "H2D params"))) return rc;
    const SpmmParams* Pd = w.params.as<SpmmParams>();
    const int units = npanels * w.nchunks;
    const int grid = std::max(1, std::min(units, spmm_grid(false)));
    const int grid_final = std::max(1, std::min(units, spmm_grid(true)));
    if ((rc = cuda_ok(cudaEventRecord(g->ev0, s), "event"))) return rc;
    {
        const int64_t total = (int64_t)npanels * n * kLanes;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((total + kThreads - 1) / kThreads, 148 * 16));
        const int need = (npanels * kLanes + kThreads - 1) / kThreads;
        k_spmm_init<<<std::max(blocks, need), kThreads, 0, s>>>(w.X0.as<float>(), w.cols.as<ColState>(), n, npanels, k,
                                                                 alpha, g->n_dangling_solve);
    }
    // Control block: active columns = k, cap = max_iter + 1 sweeps.
    {
        Ctl c{};
        c.active = k;
        c.cap = max_iter + 1;
        if ((rc = cuda_ok(cudaMemcpyAsync(w.ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, s), "H2D ctl"))) return rc;
    }
    // The sweep loop: a CUDA-graph while node whose body is one k_spmm launch,
    // built once per workspace (its only argument is the parameter block).
    if (!w.cg_exec && !w.cg_failed) {
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
            kp.func = (void*)k_spmm<float>;
            kp.gridDim = dim3((unsigned)grid);
            kp.blockDim = dim3(kThreads);
            kp.sharedMemBytes = (unsigned)smem_bytes(false);
            kp.kernelParams = args;
            ok = cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp) == cudaSuccess &&
                 cudaGraphInstantiate(&ex, cg, 0) == cudaSuccess;
        }
        if (ok) {
            w.cg = cg;
            w.cg_exec = ex;
            w.cond = h;
        } else {
            cudaGetLastError();
            if (cg) cudaGraphDestroy(cg);
            w.cg_failed = true;
        }
    }
    int32_t launches = 2;  // set-up kernels
    if (w.cg_exec) {
        if ((rc = cuda_ok(cudaGraphLaunch(w.cg_exec, s), "graph launch"))) return rc;
    } else {
        for (int32_t it = 0; it < max_iter; ++it)
            k_spmm<float><<<grid, kThreads, smem_bytes(false), s>>>(Pd, 0, 0);
        if ((rc = cuda_ok(cudaGetLastError(), "spmm launch"))) return rc;
    }
    const bool correction = (flags & EGPR_FLAG_NO_CORRECTION) == 0;
    if (correction) {
        k_spmm<double><<<grid_final, kThreads, smem_bytes(true), s>>>(Pd, 0, 0);
        launches += 1;
    }
    {
        dim3 gr((unsigned)((n + 31) / 32), (unsigned)npanels);
        k_spmm_normalize<<<gr, kThreads, 0, s>>>(w.out64.as<double>(), w.X0.as<float>(), w.X1.as<float>(),
                                                 w.cols.as<ColState>(), n, k, correction ? 0 : 1, w.out.as<double>());
        launches += 1;
    }
    if ((rc = cuda_ok(cudaGetLastError(), "spmm finish"))) return rc;
    if ((rc = cuda_ok(cudaEventRecord(g->ev1, s), "event"))) return rc;
    if ((rc = cuda_ok(cudaMemcpyAsync(out, w.out.p, (size_t)k * n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H ranks")))
        return rc;
    std::vector<ColState> hc((size_t)npanels * kLanes);
    Ctl ctl;
    if ((rc = cuda_ok(cudaMemcpyAsync(hc.data(), w.cols.p, hc.size() * sizeof(ColState), cudaMemcpyDeviceToHost, s), "D2H cols")) ||
        (rc = cuda_ok(cudaMemcpyAsync(&ctl, w.ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s), "D2H ctl")) ||
        (rc = cuda_ok(cudaStreamSynchronize(s), "batch solve")))
        return rc;
    if (ctl.error) return ctl.error;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    if (stats) {
        const int64_t bytes = 4 * ((int64_t)n + 1) + 4 * g->nnz * (g->weighted ? 2 : 1) + 4 * (int64_t)n +
                              12 * (int64_t)n * k;
        for (int32_t j = 0; j < k; ++j) {
            egpr_stats& st = stats[j];
            st.iterations = hc[(size_t)j].iter;
            st.converged = hc[(size_t)j].converged;
            st.residual = hc[(size_t)j].residual;
            st.kernel_seconds = ms * 1e-3;
            st.total_seconds = wall_seconds() - t0;
            st.bytes_per_iter = bytes;
            st.launches = launches + ctl.launches;
            st.reserved = 0;
        }
    }
    return EGPR_SUCC;
}

}  // namespace egpr
