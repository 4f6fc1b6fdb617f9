// Seeded synthetic graph generators for the PageRank workloads (host C++,
// OpenMP).  They write an out-edge CSR in the layout the reference's C++
// graph produces from gen_CSR (cpp_easygraph/classes/graph.cpp:719-886):
// int32 offsets V[n+1], int32 destinations E[m] sorted ascending inside each
// row, no duplicate pairs, and (when asked) one weight per entry as FP64.
//
// Randomness is counter based (SplitMix64 over (seed, sample index)), so a
// graph depends only on its parameters and never on the thread count.
//
//   egpr_synth_rmat  R-MAT: edgefactor * 2^scale sampled (src, dst) pairs,
//                    each of the `scale` bit levels picks a quadrant with
//                    probabilities a/b/c/d (d = 1-a-b-c), most significant
//                    bit first, no noise, no permutation.  Self-loops are
//                    dropped and directed duplicates removed.  keep_n > 0
//                    keeps vertices [0, keep_n) and drops every sampled pair
//                    with an endpoint >= keep_n (non-power-of-two sizes).
//   egpr_synth_er    Erdos-Renyi G(n, M): M uniform (src, dst) pairs, then the
//                    same self-loop / duplicate rules.
//   weights          w = 1 - U with U uniform in [0, 1) rounded to FP32, so
//                    w lies in (0, 1]; drawn per final CSR entry index.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

inline double unit_double(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Turns sampled (src, dst) pairs into a deduplicated CSR with sorted rows.
// src/dst entries < 0 mark dropped samples.  Returns m.
int64_t pairs_to_csr(int32_t n, int64_t samples, const int32_t* src, const int32_t* dst,
                     int32_t* V, int32_t* E) {
    std::vector<int64_t> count((size_t)n + 1, 0);
    for (int64_t i = 0; i < samples; ++i)
        if (src[i] >= 0) count[(size_t)src[i] + 1]++;
    for (int32_t i = 0; i < n; ++i) count[(size_t)i + 1] += count[(size_t)i];
    std::vector<int64_t> cur(count.begin(), count.end() - 1);
    std::vector<int32_t> tmp((size_t)count[(size_t)n]);
    for (int64_t i = 0; i < samples; ++i)
        if (src[i] >= 0) tmp[(size_t)cur[(size_t)src[i]]++] = dst[i];
    std::vector<int64_t> kept((size_t)n, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t u = 0; u < n; ++u) {
        int32_t* b = tmp.data() + count[(size_t)u];
        int32_t* e = tmp.data() + count[(size_t)u + 1];
        std::sort(b, e);
        kept[(size_t)u] = std::unique(b, e) - b;
    }
    V[0] = 0;
    int64_t m = 0;
    for (int32_t u = 0; u < n; ++u) {
        m += kept[(size_t)u];
        V[u + 1] = (int32_t)m;
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t u = 0; u < n; ++u)
        std::memcpy(E + V[u], tmp.data() + count[(size_t)u], sizeof(int32_t) * (size_t)kept[(size_t)u]);
    return m;
}

void fill_weights(uint64_t seed, int64_t m, double* W) {
    const uint64_t wseed = splitmix64(seed ^ 0x5DEECE66Dull);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < m; ++p) {
        float u = (float)unit_double(splitmix64(wseed + (uint64_t)p * 0x9E3779B97F4A7C15ull));
        float w = 1.0f - u;  // (0, 1]
        if (w <= 0.0f) w = 1.0f;
        W[p] = (double)w;
    }
}

}  // namespace

extern "C" {

// Upper bound for E's capacity: edgefactor << scale samples.
int64_t egpr_synth_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c,
                        uint64_t seed, int32_t keep_n, int32_t* V, int32_t* E, double* W) {
    if (scale < 1 || scale > 30 || edgefactor < 1) return -1;
    const int32_t n_full = (int32_t)1 << scale;
    const int32_t n = keep_n > 0 ? std::min(keep_n, n_full) : n_full;
    const int64_t samples = (int64_t)edgefactor << scale;
    std::vector<int32_t> src((size_t)samples), dst((size_t)samples);
    const double ab = a + b, abc = a + b + c;
    const uint64_t base = splitmix64(seed);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < samples; ++i) {
        uint64_t s = base + (uint64_t)i * 0xD1B54A32D192ED03ull;
        int32_t r = 0, q = 0;
        for (int32_t lvl = 0; lvl < scale; ++lvl) {
            s = splitmix64(s);
            const double u = unit_double(s);
            const int32_t bit = 1 << (scale - 1 - lvl);
            if (u < a) {
            } else if (u < ab) {
                q |= bit;
            } else if (u < abc) {
                r |= bit;
            } else {
                r |= bit;
                q |= bit;
            }
        }
        if (r == q || r >= n || q >= n) {
            src[(size_t)i] = -1;
            dst[(size_t)i] = -1;
        } else {
            src[(size_t)i] = r;
            dst[(size_t)i] = q;
        }
    }
    const int64_t m = pairs_to_csr(n, samples, src.data(), dst.data(), V, E);
    if (W) fill_weights(seed, m, W);
    return m;
}

// Upper bound for E's capacity: m_samples.
int64_t egpr_synth_er(int32_t n, int64_t m_samples, uint64_t seed, int32_t* V, int32_t* E,
                      double* W) {
    if (n < 1 || m_samples < 0) return -1;
    std::vector<int32_t> src((size_t)m_samples), dst((size_t)m_samples);
    const uint64_t base = splitmix64(seed ^ 0xA0761D6478BD642Full);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m_samples; ++i) {
        uint64_t r1 = splitmix64(base + (uint64_t)(2 * i) * 0x9E3779B97F4A7C15ull);
        uint64_t r2 = splitmix64(base + (uint64_t)(2 * i + 1) * 0x9E3779B97F4A7C15ull);
        int32_t u = (int32_t)((r1 >> 32) * (uint64_t)n >> 32);
        int32_t v = (int32_t)((r2 >> 32) * (uint64_t)n >> 32);
        if (u == v) {
            u = -1;
            v = -1;
        }
        src[(size_t)i] = u;
        dst[(size_t)i] = v;
    }
    const int64_t m = pairs_to_csr(n, m_samples, src.data(), dst.data(), V, E);
    if (W) fill_weights(seed, m, W);
    return m;
}

}  // extern "C"
