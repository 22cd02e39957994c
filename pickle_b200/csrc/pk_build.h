// Batched insertion kernels (pk_build.cu): argument blocks and launchers.
#pragma once

#include "pk_internal.h"

namespace pk {

struct BuildEnt {
    float d;
    int32_t id;
};

// Kernel 1: per-node descent, layer searches and SelectHeuristic.
struct InsertSearchArgs {
    int32_t nb;               // nodes in the batch
    int32_t pos0;             // layer-0 id (= vec0 row) of the batch's first node
    const uint8_t *levels;    // [nb]
    int32_t enter_level;      // of the graph before the batch
    int32_t graph_nonempty;
    int32_t efc;
    int32_t top_k0;           // 2M (layer 0); upper layers keep M
    int32_t max_levels;       // stride of out / counts / node_id per node
    const int32_t *node_id;   // [nb * max_levels] each node's new id per layer
    void *out;                // BuildEnt[nb * max_levels * top_k0]: R then Pruned
    int32_t *counts;          // [nb * max_levels]: nR | nP << 16
    int32_t *work;            // [0] node counter, [1] scratch overflows
    WarpGlobalScratch gs;
    int32_t wcap;
    // layer 0 from a walk's candidate lists instead of the exact search:
    // node i's efc best traversal candidates at l0_cand[i * l0_stride]
    // (layer-0 ids, -1 = none); null = the exact search
    const int32_t *l0_cand;
    int32_t l0_stride;
};

// Kernel 2: AddNode for each (node, layer <= its level).  With meta_only it
// writes only the node's bookkeeping (run before kernel 1).
struct AddNodeArgs {
    int32_t meta_only;
    int64_t nitems;
    const int32_t *item_node;   // batch index
    const int32_t *item_level;
    const int32_t *item_id;     // its new internal id on that layer
    const int32_t *item_down;   // its internal id one layer down
    const int32_t *ext_ids;     // [nb]
    const int32_t *top_inserted;  // [nb]
    int32_t pos0;
    int32_t max_levels;
    int32_t top_k0;
    const void *out;
    const int32_t *counts;
};

struct EdgeKeyArgs {
    int64_t nslots;             // nb * max_levels * top_k0
    int32_t max_levels, top_k0;
    const uint8_t *levels;
    const int32_t *top_inserted;
    const int32_t *counts;
    const void *out;
    const int32_t *node_id;     // [nb * max_levels] new internal id per layer
    uint64_t *keys;             // [nslots]
    void *edges;                // BuildEnt[nslots]: (distance, new node id)
};

struct AddEdgeArgs {
    const uint64_t *keys;       // sorted
    const void *edges;
    const int64_t *seg_start;   // [nseg + 1]
    const int32_t *nseg;
    int32_t capmax;
};

struct EdgeWork {
    void *temp;
    size_t temp_bytes;
    uint64_t *keys_sorted;
    int32_t *flags, *scan;
    int64_t *seg_start;
    int32_t *nseg;
};

__host__ __device__ inline int insert_smem_per_warp(int wcap, int top_k0, int64_t row_bytes) {
    return search_smem_per_warp(wcap, row_bytes) + align16((int64_t)top_k0 * 8);
}
__host__ __device__ inline int add_edge_smem_per_warp(int capmax) {
    return (((capmax + 2) * 8) * 2 + (capmax + 2) * 4 * 2 + 15) & ~15;
}

int insert_search_blocks_per_sm(int dtype, const LaneCfg &lc, int wpb, size_t smem);
cudaError_t launch_insert_search(const DevGraph *g, int dtype, const LaneCfg &lc, const InsertSearchArgs &a, int grid,
                                 int wpb, size_t smem, cudaStream_t s);
cudaError_t launch_add_node(DevGraph *g, const AddNodeArgs &a, cudaStream_t s);
cudaError_t launch_add_edges(DevGraph *g, int dtype, const LaneCfg &lc, EdgeWork &w, const EdgeKeyArgs &ka,
                             int capmax, cudaStream_t s);
size_t edge_sort_temp_bytes(int64_t n);

}  // namespace pk
