// Test-infrastructure shim (oracle only, never shipped): compiles the
// reference's own PageRank translation unit and exposes two of its functions
// with C linkage so the oracle tests can call them directly.
//
//  * ref_build_inbound  -> build_inbound_from_csr
//                          (gpu_easygraph/functions/centrality/pagerank.cu:286-347),
//                          the reference's host-side CSR -> inbound-CSR preparation.
//  * ref_cuda_pagerank  -> cuda_pagerank
//                          (gpu_easygraph/functions/centrality/pagerank.cu:352-713),
//                          the reference's cuSPARSE/cuBLAS GPU solve.
//
// The reference sources are #included from their location in the reference
// tree (include path given by oracle/Makefile.ref); nothing is copied.
#include "functions/centrality/pagerank.cu"

#include <cstdint>
#include <cstring>

extern "C" int ref_build_inbound(const int* V, const int* E, const double* W,
                                 int n, int m, double alpha,
                                 int* in_row /* n+1 */, int* in_col /* m */,
                                 float* in_val /* m */, int* dangling01 /* n */,
                                 int* out_nnz) {
    std::vector<int> row, col, dang;
    std::vector<float> val;
    gpu_easygraph::build_inbound_from_csr(V, E, W, n, m, alpha, row, col, val, dang);
    std::memcpy(in_row, row.data(), sizeof(int) * (size_t)(n + 1));
    if (!col.empty()) {
        std::memcpy(in_col, col.data(), sizeof(int) * col.size());
        std::memcpy(in_val, val.data(), sizeof(float) * val.size());
    }
    if (n > 0) std::memcpy(dangling01, dang.data(), sizeof(int) * (size_t)n);
    *out_nnz = (int)col.size();
    return 0;
}

extern "C" int ref_cuda_pagerank(const int* V, const int* E, const double* W,
                                 int n, int m, double alpha, int max_iter,
                                 double threshold, double* out /* n */,
                                 double* kernel_seconds) {
    std::vector<double> pr;
    int rc = gpu_easygraph::cuda_pagerank(V, E, W, n, m, alpha, max_iter, threshold, pr,
                                          kernel_seconds);
    if (rc == 0 && (int)pr.size() == n && n > 0) std::memcpy(out, pr.data(), sizeof(double) * (size_t)n);
    return rc;
}
