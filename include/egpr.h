/*
 * egpr.h — C ABI of the B200 PageRank engine (libegpr.so).
 *
 * This is the native boundary that replaces the reference's PageRank
 * binding and library entry:
 *
 *   cpp_easygraph.cpp_gpu_pagerank_dense(G, alpha, max_iterator, threshold, weight)
 *       cpp_easygraph/cpp_easygraph.cpp:120,
 *       impl cpp_easygraph/functions/pagerank/pagerank.cpp:176-223
 *   int gpu_easygraph::pagerank(V, E, W, alpha, max_iter_num, threshold, PR, kernel_seconds)
 *       gpu_easygraph/gpu_easygraph.h:95-104,
 *       impl gpu_easygraph/functions/centrality/centrality.cpp:150-179 and
 *            gpu_easygraph/functions/centrality/pagerank.cu:352-713
 *
 * Conventions: plain pointers and sizes only; every pointer argument is a
 * HOST pointer; no device pointer ever crosses this ABI; no exception or
 * longjmp crosses it.  Every call returns an int status (EGPR_*), whose
 * values 0..6 keep the numbering of the reference's EG_GPU_STATUS_CODE
 * (gpu_easygraph/common/err.h:7-15).  A graph handle is bound to the CUDA
 * device that was current when it was created; calling it while another
 * device is current returns EGPR_DEVICE_ERR (the reference's fixed-device
 * rule, pagerank.cu:369-378).  Calls on one handle are serialised by the
 * library; distinct handles may be used from distinct host threads at once.
 *
 * Arithmetic: the maths of the reference's EasyGraph power iteration
 * (easygraph/functions/centrality/pagerank.py:75-139): uniform start 1/n,
 * out-weight normalisation, uniform redistribution of dangling mass, the
 * (1-alpha)/n teleport term, the L1 stop rule err < tol*n checked after each
 * sweep, at most max(1, max_iter) sweeps, one final normalisation.  Ranks and
 * the sparse products are FP32; dangling mass, residual and sums are FP64; a
 * final FP64 sweep recomputes the last iterate unless disabled.
 */
#ifndef EGPR_H
#define EGPR_H

#include <stdint.h>

#if defined(__GNUC__)
#define EGPR_API __attribute__((visibility("default")))
#else
#define EGPR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  0..6 = gpu_easygraph EG_GPU_STATUS_CODE (err.h:7-15). */
#define EGPR_SUCC 0
#define EGPR_FAILED_TO_ALLOCATE_HOST_MEM 1
#define EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM 2
#define EGPR_DEVICE_ERR 3
#define EGPR_UNKNOWN_ERROR 4
#define EGPR_UNSUPPORTED_GRAPH 5
#define EGPR_NEGATIVE_CYCLE 6
/* Added by this engine. */
#define EGPR_TIMEOUT 7          /* a bounded device wait gave up */
#define EGPR_INVALID_ARGUMENT 8 /* malformed CSR, bad sizes, NULL output ... */

/* Solve flags (egpr_solve_opts.flags). */
#define EGPR_FLAG_NO_CORRECTION 1u /* skip the final FP64 sweep */

typedef struct egpr_graph egpr_graph; /* opaque prepared graph (device resident) */

typedef struct egpr_stats {
    int32_t iterations;    /* sweeps run, counted like pagerank.py's loop */
    int32_t converged;     /* 1 when the L1 rule stopped the loop, else 0 */
    double residual;       /* FP64 L1 difference of the last sweep */
    double kernel_seconds; /* device time of the solve (CUDA events) */
    double total_seconds;  /* host wall time of the call */
    int64_t bytes_per_iter;/* algorithmic HBM bytes of one sweep */
    int32_t launches;      /* kernels this library launched for the solve */
    int32_t reserved;
} egpr_stats;

typedef struct egpr_graph_info {
    int32_t n;             /* vertices */
    int32_t device;        /* CUDA device the handle lives on */
    int64_t m_input;       /* entries of the out-edge CSR given at create */
    int64_t nnz;           /* inbound entries kept (valid endpoints) */
    int32_t weighted;      /* 1 if a weight array was given */
    int32_t n_dangling;    /* vertices with out-weight sum <= 0 */
    int64_t device_bytes;  /* device memory held by the handle */
    double prep_seconds;   /* device time of the preparation */
} egpr_graph_info;

typedef struct egpr_cache_stats {
    int64_t graphs;        /* live prepared graphs (all handles) */
    int64_t device_bytes;  /* device bytes they hold */
    int64_t hits;          /* egpr_pagerank_csr reuses of a prepared graph */
    int64_t misses;        /* egpr_pagerank_csr preparations */
    int64_t evictions;     /* prepared graphs dropped by the csr cache */
    int64_t budget_bytes;  /* byte budget of the csr cache */
} egpr_cache_stats;

/* ---- status -------------------------------------------------------- */

/* Replaces gpu_easygraph::err_code_detail (gpu_easygraph/common/err.cpp:9-31). */
EGPR_API const char* egpr_status_string(int status);

/* Text of the last CUDA error seen on this host thread ("" if none). */
EGPR_API const char* egpr_last_error(void);

/* ---- prepared graphs ------------------------------------------------ */

/*
 * Uploads an out-edge CSR and prepares it on the current device: FP64
 * out-weight sums, inbound CSR with entries in ascending source order,
 * dangling mask, and the sweep's layout (rows padded to end on an entry of
 * their own, 256-entry warp tiles, cost-balanced chunks).  Replaces the host-side
 * build_inbound_from_csr + H2D of pagerank.cu:286-347,472-518, done on the
 * GPU.  V[n+1] must be non-decreasing with V[0]==0 and V[n]==m (the CSR the
 * reference's gen_CSR / load_csr_files produce); destinations outside [0,n)
 * are skipped like pagerank.cu:310; non-finite or negative weights count as
 * 0 (pagerank.cu:311).  W may be NULL (unit weights, centrality.cpp:170).
 */
EGPR_API int egpr_graph_create(const int32_t* V, const int32_t* E, const double* W, int32_t n, int64_t m,
                      egpr_graph** out);
EGPR_API int egpr_graph_destroy(egpr_graph* g);
EGPR_API int egpr_graph_info_get(const egpr_graph* g, egpr_graph_info* info);

/*
 * Copies the prepared inbound CSR back to the host, for parity checks
 * against build_inbound_from_csr (pagerank.cu:286-347).  in_w may be NULL;
 * every other pointer must hold the sizes given by egpr_graph_info_get.
 */
EGPR_API int egpr_graph_export_inbound(const egpr_graph* g, int32_t* in_row /* n+1 */,
                              int32_t* in_col /* nnz */, float* in_w /* nnz, nullable */,
                              int32_t* dangling01 /* n */, double* out_weight_sum /* n */);

/*
 * Runs launches on the given cudaStream_t (passed as void*) instead of the
 * handle's own stream; NULL restores the handle's stream.
 */
EGPR_API int egpr_graph_set_stream(egpr_graph* g, void* stream);

/* ---- layout tuning (no counterpart in the reference) ------------------- */

/*
 * The work-layout parameters of a prepared graph.  The reference has no such
 * layer: its PageRank kernel takes one thread per row with fixed launch
 * shapes (pagerank.cu), so nothing there is tuned per graph.
 */
typedef struct egpr_tuning {
    int32_t chunks_per_warp; /* single-vector sweep: work-queue chunks per resident warp */
    int32_t row_cost;        /* single-vector sweep: cost of finishing a row, in entries, when cutting chunks */
    int32_t spmm_chunk;      /* batched solve: inbound entries per work unit (the tile along the entries) */
    int32_t configs_tried;   /* egpr_graph_autotune: layouts measured */
    double sweep_ms;         /* egpr_graph_autotune: per-sweep device time of the chosen sweep layout */
    double spmm_sweep_ms;    /* egpr_graph_autotune: per-sweep device time of the chosen batched layout
                                (one 32-column panel) */
} egpr_tuning;

#define EGPR_TUNE_SWEEP 1u /* tune the single-vector sweep layout */
#define EGPR_TUNE_SPMM 2u  /* tune the batched solve's tile */

/*
 * Measures candidate layouts on this graph (a few fixed-count sweeps each,
 * timed on the device) and keeps the fastest: chunks_per_warp in {4, 8, 16}
 * x row_cost in {2, 4, 8} for the sweep, spmm_chunk in {512, 1024, 2048} for
 * the batched solve.  Results do not depend on the layout beyond FP32
 * rounding.  out (nullable) receives the chosen parameters and timings.
 * The choice is recorded per GPU model and graph-shape bucket (log2 of n,
 * log2 of the mean degree, weighted or not) in the file EGPR_TUNE_CACHE
 * names (default $XDG_CACHE_HOME/eggpu_b200/tuning.txt or
 * ~/.cache/eggpu_b200/tuning.txt; EGPR_TUNE_CACHE=0 turns recording off), and
 * every graph prepared later whose shape falls in a recorded bucket, through
 * egpr_graph_create or egpr_pagerank_csr, starts with that layout (unless
 * EGPR_CHUNKS_PER_WARP, EGPR_ROW_COST or EGPR_SPMM_CHUNK fix it).
 */
EGPR_API int egpr_graph_autotune(egpr_graph* g, uint32_t what, egpr_tuning* out);
/* Reads / applies layout parameters (values outside their ranges are refused). */
EGPR_API int egpr_graph_get_tuning(const egpr_graph* g, egpr_tuning* out);
EGPR_API int egpr_graph_set_tuning(egpr_graph* g, const egpr_tuning* in);

/* ---- solves ---------------------------------------------------------- */

/*
 * PageRank / personalised PageRank on a prepared graph.  personalization
 * (nullable, n values >= 0, not all zero) replaces the uniform teleport
 * vector after normalisation to sum 1; dangling mass stays uniform.
 * out_ranks[n] receives the normalised FP64 ranks.  stats may be NULL.
 */
EGPR_API int egpr_pagerank(egpr_graph* g, double alpha, int32_t max_iter, double tol,
                  const double* personalization, uint32_t flags, double* out_ranks,
                  egpr_stats* stats);

/*
 * Asynchronous form of egpr_pagerank without personalisation: enqueues the
 * whole solve on the handle's stream and returns; egpr_pagerank_collect
 * waits for it and copies the ranks (out_ranks may be NULL to skip the copy).
 * Enqueueing again before collecting is allowed: the solves run back to back
 * in stream order on the same workspace and collect reports the last one.
 */
EGPR_API int egpr_pagerank_enqueue(egpr_graph* g, double alpha, int32_t max_iter, double tol,
                          uint32_t flags);
EGPR_API int egpr_pagerank_collect(egpr_graph* g, double* out_ranks, egpr_stats* stats);

/*
 * Batched personalised PageRank: k teleport vectors solved together as one
 * CSR x dense SpMM per sweep (each inbound entry is loaded once per sweep
 * for a tile of columns).  teleport is k*n row-major (vector j at j*n);
 * every vector is normalised to sum 1.  Each column stops on its own L1
 * rule and keeps its own iteration count.  out is k*n.  stats (nullable)
 * holds k entries.
 */
EGPR_API int egpr_pagerank_batch(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k,
                        const double* teleport, uint32_t flags, double* out, egpr_stats* stats);

/*
 * Batched personalised PageRank with sparse seed sets: column j teleports
 * uniformly to seeds[seed_ptr[j] .. seed_ptr[j+1]) (vertex ids, duplicates
 * count once).  Same maths and outputs as egpr_pagerank_batch.
 */
EGPR_API int egpr_pagerank_seeds(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k,
                        const int32_t* seed_ptr, const int32_t* seeds, uint32_t flags, double* out,
                        egpr_stats* stats);

/* ---- continuous batching of personalised PageRank ---------------------- */

/*
 * No counterpart in the reference.  A session keeps one batched solve of a
 * prepared graph running so that requests can join it while it runs: slots
 * (columns of the CSR x dense SpMM, 1..512, rounded up to a multiple of 32)
 * are filled by egpr_session_admit between steps, egpr_session_step runs a
 * few sweeps of every running column, and a finished column is collected
 * (FP64 correction sweep unless EGPR_FLAG_NO_CORRECTION, normalisation, copy
 * to the host) and its slot freed while the other columns keep sweeping.
 * Every column has the maths, stop rule (err < tol * n) and sweep limit of a
 * seed-set solve of egpr_pagerank_seeds on its own; alpha and tol are the
 * session's.  Calls on a session lock its graph.  A graph with live sessions
 * refuses egpr_graph_destroy and layout changes of the batched solve.
 */
typedef struct egpr_session egpr_session;

EGPR_API int egpr_session_create(egpr_graph* g, double alpha, double tol, int32_t slots, egpr_session** out);
/* count requests with seed sets seeds[seed_ptr[i] .. seed_ptr[i+1]) each, up
 * to max_iter sweeps of their own; slots_out[count] receives their slots.
 * Fails (EGPR_INVALID_ARGUMENT) without admitting any when fewer slots are free. */
EGPR_API int egpr_session_admit(egpr_session* s, int32_t count, const int32_t* seed_ptr, const int32_t* seeds,
                                int32_t max_iter, int32_t* slots_out);
/* Runs up to `sweeps` sweeps of the running columns; done_slots (capacity:
 * the session's slots) receives every finished, not yet collected slot. */
EGPR_API int egpr_session_step(egpr_session* s, int32_t sweeps, int32_t* done_slots, int32_t* ndone);
/* Results of finished slots: out is count x n (row i = slots[i]); stats
 * (nullable) count entries, iterations counted from each column's start. */
EGPR_API int egpr_session_collect(egpr_session* s, int32_t count, const int32_t* slots, uint32_t flags, double* out,
                                  egpr_stats* stats);
EGPR_API int egpr_session_info(const egpr_session* s, int32_t* slots, int32_t* running, int32_t* done);
EGPR_API int egpr_session_destroy(egpr_session* s);

/*
 * Many independent graphs in one persistent launch per sweep: the work
 * tiles of all graphs form one queue; every graph keeps its own residual,
 * stop rule and iteration count.  outs[i] receives graph i's n_i ranks.
 * stats (nullable) holds count entries.
 */
EGPR_API int egpr_pagerank_multi(int32_t count, egpr_graph* const* graphs, double alpha, int32_t max_iter,
                        double tol, uint32_t flags, double* const* outs, egpr_stats* stats);

/* ---- drop-in for gpu_easygraph::pagerank ----------------------------- */

/*
 * Same contract as int gpu_easygraph::pagerank(V, E, W, alpha,
 * max_iter_num, threshold, PR, kernel_seconds) (gpu_easygraph.h:95-104):
 * len_V = n+1, W NULL when the reference passes an empty vector, PR[n]
 * receives FP64 ranks, *kernel_seconds the device time (nullable).  n <= 0
 * returns EGPR_SUCC with nothing written (centrality.cpp:160-165).
 * graph_id names one immutable host CSR, as CSRGraph::cache_id does
 * (cpp_easygraph/classes/csr_graph.h:33-47): calls with the same id and the
 * same CSR signature reuse the prepared device graph (alpha is not part of
 * the key: nothing prepared depends on it).
 */
EGPR_API int egpr_pagerank_csr(const int32_t* V, int32_t len_V, const int32_t* E, int64_t len_E,
                      const double* W, uint64_t graph_id, double alpha, int32_t max_iter_num,
                      double threshold, double* PR, double* kernel_seconds);

/* ---- solve without allocating --------------------------------------- */

/*
 * No counterpart in the reference.  PageRank for callers that may not call
 * cudaMalloc: code inside a framework that owns all device memory through
 * its own pool, a serving thread with a fixed memory budget, a plug-in whose
 * host forbids allocations while a request runs.  The caller passes device
 * pointers: the inbound CSR in_row[n+1] / in_col[nnz] (entries are source
 * ids, as egpr_graph_export_inbound returns them), optional FP32 weights
 * in_w[nnz] (NULL = unit weights), the FP64 out-weight sum of every source
 * out_weight[n], and ranks[n] for the normalised FP64 result.  Same maths,
 * stop rule and flags as egpr_pagerank (uniform teleport only).
 *
 * Nothing is allocated: the solve's buffers live in one fixed device array
 * compiled into the library (4 MiB + 256 bytes, held on every GPU that loads
 * the library until the process exits).  Hence the limit n <= 262144; a
 * larger n returns EGPR_INVALID_ARGUMENT.  The first call on a device looks
 * up that array's device address (make it before any stream capture).  Every
 * call reuses the array, so calls that overlap on the GPU (other threads or
 * other streams) race and give wrong results: serialise them.  Work is
 * enqueued on `stream` (a cudaStream_t, NULL = default stream); with stats
 * non-NULL the call waits for it and fills stats (kernel_seconds: device time
 * from the first to the last kernel of the solve, read from the GPU's global
 * timer; n <= 0 zeroes stats).  Every one of the max_iter sweeps is launched:
 * sweeps after convergence return at once but each still costs a kernel
 * launch (a few microseconds), so pick max_iter near the sweeps needed.  The
 * array's device address is cached per device for the life of the process;
 * after cudaDeviceReset on that device the cached address is stale, so do not
 * reset a device between calls.
 */
EGPR_API int egpr_pagerank_device_noalloc(int32_t n, int64_t nnz, const int32_t* in_row, const int32_t* in_col,
                                          const float* in_w, const double* out_weight, double alpha,
                                          int32_t max_iter, double tol, uint32_t flags, double* ranks,
                                          void* stream, egpr_stats* stats);

/* Counters of the prepared-graph cache behind egpr_pagerank_csr. */
EGPR_API int egpr_cache_stats_get(egpr_cache_stats* out);
/* Drops every graph held by the egpr_pagerank_csr cache. */
EGPR_API int egpr_cache_reset(void);
/* Byte budget of that cache (0 = max(free/4, 256 MiB) at first use). */
EGPR_API int egpr_cache_set_budget(int64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* EGPR_H */
