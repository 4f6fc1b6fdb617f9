// Batched personalised PageRank (placeholder until the SpMM kernel lands).
#include "egpr_internal.cuh"

namespace egpr {

int ppr_batch_solve(egpr_graph*, double, int32_t, double, int32_t, const double*, const int32_t*, const int32_t*,
                    uint32_t, double*, egpr_stats*) {
    return EGPR_UNSUPPORTED_GRAPH;
}

}  // namespace egpr
