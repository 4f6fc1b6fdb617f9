// Internal declarations shared by the CUDA translation units of libegpr.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/egpr.h"

namespace egpr {

// ---------------------------------------------------------------------------
// Work decomposition of the single-vector sweep.
//
// The sweep reads the inbound CSR with one placeholder entry in every empty
// row, in warp tiles of kTileItems entries.  Runs of tiles form chunks, cut at
// equal cost (entries plus a weight per row), the unit of the persistent work
// queue.  A row cut by a chunk boundary is a "span": each chunk it touches
// adds its piece, and the last of them to arrive finishes the row (no
// waiting; the pieces are exact fixed point, so the order does not matter).
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;  // threads of the preparation and helper kernels

// Chunk flags.
constexpr int32_t kHasHead = 1;    // the chunk's first row began in an earlier chunk
constexpr int32_t kHasTail = 2;    // the chunk's last row continues into a later chunk
constexpr int32_t kInterior = 4;   // the chunk lies inside one row (head and tail are that row)

struct Chunk {
    int32_t tile_begin;  // first warp tile of the chunk
    int32_t tile_end;    // one past its last warp tile
    int32_t graph;       // slot in the plan's graph table
    int32_t flags;
    int32_t head_ta;     // global chunk id where the head row's span starts
    int32_t tail_tb;     // global chunk id where the tail row's span ends
    int32_t tail_row;    // vertex id of the tail row (span rows are finalised by row id)
    int32_t pad2;        // sweep chunk: chunks of its tail row's span
    int32_t nnz_begin;   // entries [nnz_begin, nnz_end) belong to the chunk
    int32_t nnz_end;
    int32_t row_end;     // sweep chunk: rows before row_end are finished by the chunk
    int32_t pad;         // sweep chunk: chunks of its head row's span (estimated cost while preparing)
};

// The sweep's warp tiles: kTileItems entries, lane l owning entries 8l..8l+7.
constexpr int kLaneItems = 8;
constexpr int kTileItems = 32 * kLaneItems;
// Per-tile words of the tile table: 8 words of row-end marks (one byte per
// lane), then 8 words with, per lane, the marks of the lanes below it.
constexpr int kTileWords = 16;
// Hub cache: the carried values of the (up to kHubCap - 32) sources with the
// largest out-degree are kept in shared memory by the sweep; inbound entries
// from a hub store -(slot + 1) instead of the source id.  Slot nhub holds 0 and
// is read by the placeholder entry of every row without entries.
constexpr int kHubCap = 49152;      // largest hub cache (values) a sweep CTA stages

// Per-graph device view used by the sweep kernels.
struct GraphDev {
    const int32_t* cols;        // sweep entries: hub-encoded sources, a placeholder in every empty row
    const float* w;             // their weights, NULL = unit weights
    const uint32_t* tile_bits;  // per warp tile: kTileWords words (row-end marks, per-lane mark offsets)
    const int32_t* tile_row;    // per warp tile: the row its first mark ends
    const double* outw;      // n, FP64 out-weight sums
    const float* scale;      // n, alpha/outw (FP32) or -1 for dangling vertices
    const float* tele;       // n, personalisation (NULL = uniform)
    float* x[2];             // ranks, double-buffered
    float* z[2];             // x * scale: the value each out-edge carries
    double* out;             // n, FP64 result
    double* z64;             // n, FP64 carried values for the correction sweep
    const int32_t* hub_ids;  // nhub source ids of the hub slots
    const int32_t* hub_slot; // n, slot of each vertex or -1
    float* hubz[2];          // nhub carried values of the hubs, double-buffered with z
    double* hubz64;          // nhub + 1: the hubs' FP64 carried values for the correction sweep (slot nhub = 0)
    int32_t nhub;
    int32_t n;
    int32_t chunk_begin;     // this graph's global chunk id range
    int32_t chunk_end;
    int32_t span_begin;      // this graph's entries of the span list (span start stages)
    int32_t span_end;
};

struct GraphState {
    double alpha;
    double c1;         // (1 - alpha) / n
    double tol_n;      // tol * n
    double dmass;      // alpha * (dangling mass) / n for the next sweep
    double dmass_prev; // the value used by the last completed sweep
    double residual;   // L1 of the last sweep
    double residual64; // L1 of the FP64 correction sweep against x_{k-1}
    double xsum;       // sum of the last sweep's ranks (FP64 sweep: of the result)
    double dsum;       // dangling mass of the last sweep's ranks
    int32_t iter;
    int32_t max_iter;
    int32_t done;
    int32_t converged;
    uint32_t arrive;   // chunk arrivals in the running launch
    int32_t personalised;  // teleport from GraphDev::tele instead of 1/n
};

struct Ctl {
    uint32_t queue;    // work-queue head
    uint32_t exited;   // CTAs that left the queue loop
    int32_t active;    // graphs still iterating
    int32_t launches;  // sweep launches so far
    int32_t cap;       // hard cap on sweep launches
    int32_t error;
};

constexpr int kAccWords = 8;  // words per accumulator slot (6 used; 64-byte slots)

struct SweepParams {
    const Chunk* chunks;     // in queue order (costliest chunks of a graph first)
    int32_t nchunks;
    int32_t mode;            // 0 = FP32 sweep, 1 = FP64 correction sweep
    const GraphDev* graphs;
    GraphState* states;
    // FP64 sums are accumulated as two's-complement fixed point (2 words: units
    // of 2^-32 and of 2^-64) with integer atomics, so their order does not
    // change the result.
    unsigned long long* acc;       // kAccWords per slot: err, dangling, rank sums
    unsigned long long* span_acc;  // 2 per chunk (span start chunk): the cut row's sum
    uint32_t* span_cnt;            // per chunk (span start chunk): pieces added so far
    const int32_t* span_list;  // span start stages
    int32_t nspans;
    int32_t acc_sub;           // accumulator slots per graph
    Ctl* ctl;
    cudaGraphConditionalHandle cond;
    int32_t use_cond;
    int32_t ngraphs;
    int32_t hub_count;       // hub slots staged in shared memory (0: hubs read from global memory)
};

// ---- device buffers --------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int dev = -1;         // device of the allocation
    bool pooled = false;  // from device_pool() (else cudaMalloc)
    int alloc(size_t b);
    void release();
    // Stream-ordered forms for buffers used by one stream only: grow_on keeps
    // a large enough buffer and otherwise frees and allocates in the order of
    // stream s; neither waits for the device.
    int grow_on(size_t b, cudaStream_t s);
    void release_on(cudaStream_t s);
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// ---- the work plan over one or more prepared graphs -------------------------
struct Plan {
    int32_t ngraphs = 0;
    int32_t nchunks = 0;
    int32_t grid = 0;        // CTAs of a sweep
    int32_t any_weighted = 0;
    int32_t hub_count = 0;   // hubs of the plan's graph (one-graph plans)
    int32_t max_n = 0;
    DevBuf d_chunks, d_graphs, d_states, d_ndang, d_ctl, d_span_list, d_acc, d_span_acc, d_span_cnt;
    std::vector<Chunk> h_chunks;      // a graph's own chunk table (local ids)
    std::vector<int32_t> h_spans;     // a graph's span start chunks (local ids)
    std::vector<Chunk> h_chunks_all;  // the plan's table (global ids)
    int32_t nspans = 0;
    int32_t nacc = 0;                 // accumulator slots
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t cg_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    bool cg_failed = false;
    void* l2_base = nullptr;  // persisting L2 window over the gathered vectors
    size_t l2_bytes = 0;
    float l2_hit_ratio = 0.f;
    ~Plan();
    void release();
    void release_on(cudaStream_t s);  // buffers used by stream s only: freed in its order
};

struct SpmmWork;  // batched personalised PageRank workspace (spmm.cu)

// ---------------------------------------------------------------------------
// The binned single-graph sweep (bins.cu; layout built in prep.cu).
//
// Vertices are renumbered: first the H sources of largest out-degree (the hub
// block, whose carried values the sweep stages in shared memory, so a source
// id below H is a shared-memory read), then every other vertex; inside each
// block vertices go by descending in-degree.  The inbound CSR in that order
// keeps, per row, the entries in ascending original-source order.  Rows of
// one length class are then contiguous, and the work queue holds:
//   kBinPiece  a piece of a long row (>= bin_piece entries), one warp; a row cut
//              into several pieces is finished by the last piece to arrive
//              (pieces add exact fixed-point sums)
//   kBinGroup  rows [r0, r1) of one length class, G lanes per row with G a
//              power of two sized so that each lane gathers 4..8 entries
//   kBinEmpty  rows [r0, r1) without inbound entries (teleport and dangling
//              terms only)
// ---------------------------------------------------------------------------
constexpr int32_t kBinPiece = 0;
constexpr int32_t kBinGroup = 1;
constexpr int32_t kBinEmpty = 2;

struct BinItem {
    int32_t kind;
    int32_t r0, r1;  // rows [r0, r1); kBinPiece: r0 is the row
    int32_t e0, e1;  // kBinPiece: entries [e0, e1)
    int32_t span;    // kBinPiece: span slot of a row cut into several pieces, -1 for one piece
    int32_t parts;   // kBinPiece: pieces of the row; kBinGroup: lanes per row (G)
    int32_t pad;
};

struct BinLayout {
    int32_t n = 0;
    int32_t hubs = 0;            // hub block [0, hubs)
    int64_t nnz = 0;
    DevBuf perm;                 // n: new id of each vertex
    DevBuf inv;                  // n: vertex of each new id
    DevBuf row;                  // n + 1 (+ pad): offsets of the renumbered inbound CSR
    DevBuf col;                  // nnz (+ pad): renumbered sources
    DevBuf w;                    // nnz (+ pad): FP32 weights (weighted graphs)
    DevBuf outw;                 // n: FP64 out-weight sums, renumbered
    std::vector<int32_t> h_row_bounds;  // row offsets at the class boundaries (host copy, item building)
    // work queue
    DevBuf items;
    int32_t nitems = 0;
    int32_t nspans = 0;
    int32_t piece = 2048;        // entries per piece of a long row (tuning)
    int32_t group_entries = 4096;  // target entries of a kBinGroup item (tuning)
    // per-solve state (renumbered)
    DevBuf scale, tele, x, z, z64, out64, states, ctl, acc, span_acc, span_cnt;
    int32_t acc_slots = 0;
    int32_t grid = 0;
    cudaGraph_t cg = nullptr;
    cudaGraphExec_t cg_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    bool cg_failed = false;
    int64_t device_bytes() const {
        int64_t b = 0;
        for (const DevBuf* d : {&perm, &inv, &row, &col, &w, &outw, &items, &scale, &tele, &x, &z, &z64, &out64, &states,
                                &ctl, &acc, &span_acc, &span_cnt})
            b += (int64_t)d->bytes;
        return b;
    }
    ~BinLayout();
};

// ---- prepared graph handle ---------------------------------------------------
}  // namespace egpr

struct egpr_graph {
    std::mutex mu;
    int device = -1;
    int32_t n = 0;
    int64_t m_input = 0;
    int64_t nnz = 0;
    int32_t weighted = 0;
    int32_t n_dangling = 0;        // out-weight <= 0 (reference mask)
    int32_t n_dangling_solve = 0;  // out-weight <= 1e-15 (EasyGraph CPU rule)
    double prep_seconds = 0.0;
    int32_t host_inputs_registered = 0;  // host input arrays page-locked for the upload
    int32_t host_inputs_locked = 0;      // host input arrays that were page-locked already
    int32_t host_inputs_staged = 0;      // host input arrays copied through the staging pool
    // prepared graph
    egpr::DevBuf in_row, in_col, in_w, outw, dangling01, hub_ids, hub_slot, hubz, hubz64;
    // the sweep's layout (see build_sweep_layout)
    egpr::DevBuf sw_row, sw_col, sw_w, tile_bits, tile_row;
    int64_t sw_nnz = 0;
    int32_t ntiles = 0;
    int32_t nhub = 0;
    // layout parameters (egpr_tuning); defaults from the environment
    int32_t tune_cpw = 8;           // sweep: work-queue chunks per resident warp
    int32_t tune_rc = 4;            // sweep: cost of finishing a row, in entries
    int32_t tune_spmm_chunk = 1024; // batched solve: entries per work unit
    int32_t tuning_recorded = 0;    // the layout came from the persisted tuner choices
    // solve workspace
    egpr::DevBuf scale, tele, x0, x1, z0, z1, out, z64;
    egpr::DevBuf seed_ids;         // seed set of a single-vector PPR solve
    egpr::Plan plan;               // single-graph plan
    egpr::SpmmWork* spmm = nullptr; // batched personalised PageRank workspace
    egpr::BinLayout* bins = nullptr; // binned single-graph sweep (null: the tile sweep serves single solves)
    int32_t sessions = 0;            // live batched-solve sessions (egpr_session_*) on this graph
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr; // active stream (own or user-given)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // state of an enqueued solve
    bool pending = false;
    int32_t pending_launches = 0;
    double pending_t0 = 0.0;
    int64_t device_bytes() const;
};

namespace egpr {

// The library's memory pool of the current device: device buffers and
// preparation scratch come from it, and it keeps up to EGPR_POOL_KEEP_MB
// (default: a quarter of the device) MiB of freed memory for reuse (null if
// pools are unavailable).
cudaMemPool_t device_pool();

// Status helpers.
int set_cuda_error(cudaError_t e, const char* what);
int arg_error(const char* why);  // EGPR_INVALID_ARGUMENT with a message
bool graph_loop_enabled();       // sweeps loop in a CUDA-graph while node (EGPR_GRAPH_LOOP != 0)
int check_device(const egpr_graph* g);
double wall_seconds();

// Preparation (prep.cu).
int prepare_graph(egpr_graph* g, const int32_t* V, const int32_t* E, const double* W);
int build_sweep_layout(egpr_graph* g, int32_t resident_warps, const uint32_t* sorted_dst, cudaStream_t s);
int default_chunks_per_warp();  // EGPR_CHUNKS_PER_WARP, else 8
int default_row_cost();         // EGPR_ROW_COST, else 4
int32_t default_spmm_chunk();   // EGPR_SPMM_CHUNK, else 1024
int export_in_col(const egpr_graph* g, int32_t* host, cudaStream_t s);
// D2H of a result after the work enqueued on s: a plain async copy into
// page-locked memory (or under 1 MiB); into pageable memory through the
// page-locked staging pool, returning once the bytes are in dst.
int download_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s, const char* what);

// Binned single-graph sweep (bins.cu).
bool bins_wanted(int32_t n, int64_t nnz);  // build the binned layout for this graph (EGPR_BINS, size)
int32_t bin_hub_cap();                      // hub block size limit (shared memory of one CTA)
int bins_build_items(egpr_graph* g, cudaStream_t s);
int bins_alloc_solve(egpr_graph* g, cudaStream_t s);
int bins_upload_tele(egpr_graph* g, cudaStream_t s);  // renumbers g->tele into the layout's order
int bins_enqueue(egpr_graph* g, double alpha, int32_t max_iter, double tol, bool personalised, uint32_t flags,
                 cudaStream_t s, int32_t* host_launches);
int bins_read_state(egpr_graph* g, cudaStream_t s, int32_t* iterations, int32_t* converged, double* residual,
                    int32_t* launches, int32_t* error);

// Plans and sweeps (sweep.cu).
int sweep_grid();
int sweep_resident_warps();
int work_grid(int64_t entries, int full);  // CTAs of a launch over that many entries
int32_t hub_stride(int32_t nhub);  // floats per parity of the hub copy (zero slot included)
int plan_build(Plan& plan, egpr_graph* const* graphs, int32_t count, cudaStream_t stream);
int plan_capture_loop(Plan& plan, cudaStream_t stream);
void plan_set_l2_window(Plan& plan, void* base, size_t bytes);
GraphDev graph_dev_view(const egpr_graph* g);
int launch_init(Plan& plan, double alpha, int32_t max_iter, double tol, bool personalised,
                cudaStream_t stream);
int launch_loop(Plan& plan, int32_t max_iter, cudaStream_t stream, int32_t* launches);
int launch_finish(Plan& plan, bool correction, cudaStream_t stream, int32_t* launches);

// SpMM personalised PageRank (spmm.cu).  A batched sweep gathers a whole
// 32-column panel per entry, about seven single-vector sweeps' worth, so
// batches of fewer columns run as single-vector solves.
constexpr int32_t kSpmmMinColumns = 6;
void spmm_work_release(egpr_graph* g);
int ppr_batch_solve(egpr_graph* g, double alpha, int32_t max_iter, double tol, int32_t k,
                    const double* teleport_dense, const int32_t* seed_ptr, const int32_t* seeds,
                    uint32_t flags, double* out, egpr_stats* stats);

// Scan / sort helpers (prep.cu), exposed for the SpMM set-up.
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t len, cudaStream_t s);

}  // namespace egpr
