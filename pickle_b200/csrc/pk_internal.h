// Internal definitions shared by the host code and the CUDA kernels of
// libpickle_b200.so.  Not part of the public interface (include/pickle_b200.h).
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "pickle_b200.h"

namespace pk {

constexpr int kMaxLayers = 32;   // levels drawn for M >= 2 stay far below this
constexpr int kWarpSize = 32;

// One HNSW layer as the kernels see it (device pointers).
//
// The reference keeps, per layer, a fixed-stride adjacency array of cap slots
// per node plus a degree per node (include/hnsw_layer.hpp:76-78, :192-195), and
// reads a node's list as adj[v*cap, v*cap + degree[v]).  Its reverse-edge
// insertion can grow degree past cap, so a list may run on into the following
// rows; reading the flat array the same way reproduces that.  `alloc_rows`
// rows are allocated (>= lcap plus a tail of spare rows).
struct DevLayer {
    int32_t *adj;    // [alloc_rows * cap], -1 where unset
    float *dist;     // [alloc_rows * cap], FLT_MAX where unset
    int32_t *deg;    // [alloc_rows]
    int32_t *heu;    // [alloc_rows] size of the heuristic prefix
    int32_t *ext;    // [alloc_rows] internal -> external id
    int32_t *vrow;   // [alloc_rows] layer-0 row of this node's vector in this
                     // layer, or -1 for the zero row (upper layers only)
    int32_t *down;   // [alloc_rows] internal id of the same node one layer
                     // down (upper layers only)
    int64_t n;       // nodes present
    int64_t lcap;    // capacity in nodes (ids in [0, lcap) are addressable)
    int64_t cap;     // slots per node
    int32_t ent;     // entry id (GetEntInID, include/hnsw_layer.hpp:186-190)
    int32_t pad_;
};

// The whole index as the kernels see it; passed by value.
struct DevGraph {
    const uint8_t *vec0;    // layer-0 rows, row_bytes apart, zero padded
    const uint8_t *zero_row;
    int64_t row_bytes;
    int32_t dim;
    int32_t dtype;          // PK_DTYPE_*
    int32_t metric;         // PK_METRIC_*
    int32_t enter_level;
    int32_t num_layers;
    int32_t pad_;
    DevLayer L[kMaxLayers];
};

// Lane layout of the distance kernels: a row of C 16-byte chunks is handled by
// a group of G lanes (G a power of two), lane g of the group taking chunks
// g, g + G, g + 2G, ... (K of them).  32 / G rows are processed per step.
struct LaneCfg {
    int G;
    int K;
    int C;
    int KMAX;
};

inline LaneCfg lane_config(int64_t row_bytes) {
    LaneCfg c;
    c.C = (int)(row_bytes / 16);
    int want = (c.C + 3) / 4;
    int G = 2;
    while (G < want && G < 32) G *= 2;
    c.G = G;
    c.K = (c.C + G - 1) / G;
    int km = 1;
    while (km < c.K) km *= 2;
    c.KMAX = km;
    return c;
}

inline int64_t elem_size(int dtype) {
    switch (dtype) {
        case PK_DTYPE_U8:
        case PK_DTYPE_I8: return 1;
        case PK_DTYPE_F32: return 4;
        case PK_DTYPE_F16: return 2;
        default: return 0;
    }
}

// Global scratch of the search warps: per warp a visited bitmap, the list of
// ids marked in the current layer search, and the spill of the candidate heap.
struct WarpGlobalScratch {
    uint32_t *bitmap;           // warps * bm_words
    int64_t bm_words;           // >= layer-0 capacity / 32
    int32_t *vlist;             // warps * vl_cap
    int32_t vl_cap;
    void *cand_tail;            // warps * cand_tail_cap entries of 8 bytes
    int32_t cand_tail_cap;
};

// Search launch parameters (see pk_search.cu).
struct SearchArgs {
    const uint8_t *queries;     // nq rows of row_bytes (padded staging copy)
    int64_t nq;
    const int32_t *qlist;       // optional: indices of the queries to run
    int32_t k, ef;              // uniform values (used when the arrays are null)
    const int32_t *k_arr, *ef_arr;
    int32_t out_stride;
    int32_t *out_ids;
    float *out_dists;
    const int32_t *ext0;        // layer-0 internal -> external id
    int32_t *counters;          // nq * 6 or null
    uint8_t *status;            // nq: 0 done, 1 scratch overflow (retry)
    int32_t *work;              // [0] work counter, [1] overflow count
    WarpGlobalScratch gs;
    int32_t wcap;               // result-heap capacity in shared memory
};

// Kernel launchers (pk_search.cu).
// g is a device pointer to the index's DevGraph.
int search_blocks_per_sm(int dtype, const LaneCfg &lc, int warps_per_block, size_t smem);
cudaError_t launch_search_exact(const DevGraph *g, int dtype, const LaneCfg &lc, const SearchArgs &a, int grid,
                                int warps_per_block, size_t smem, cudaStream_t s);
constexpr int kCandTop = 256;   // candidate-heap entries kept in shared memory
constexpr int kStageBytes = 32 * 4 * 3;  // per-warp staging of one adjacency chunk
constexpr int kStageRows = 16;           // vector rows staged in shared memory at once
// Shared memory of one search warp: result heap (wcap entries of 8 bytes),
// top of the candidate heap, staging of one adjacency chunk (ids, rows,
// distances), then kStageRows vector rows.  Every region starts on a 16-byte
// boundary: the row buffer is read and written with 16-byte accesses.
__host__ __device__ inline int align16(int64_t x) { return (int)((x + 15) & ~(int64_t)15); }
__host__ __device__ inline int search_stage_off(int wcap) { return align16((int64_t)(wcap + kCandTop) * 8); }
__host__ __device__ inline int search_rowbuf_off(int wcap) { return search_stage_off(wcap) + kStageBytes; }
__host__ __device__ inline int search_smem_per_warp(int wcap, int64_t row_bytes) {
    return align16(search_rowbuf_off(wcap) + kStageRows * row_bytes);
}

// A read-only view of an index handle (pk_index.cu), for entry points
// defined outside that file.
struct IndexView {
    int device;
    int num_sms;
    int dtype;
    int64_t dim, esz, row_bytes;
    LaneCfg lc;
    const DevGraph *dg;
    const int32_t *ext0;
    int64_t n0;
    int64_t lcap0;  // layer-0 capacity: ids stay below it
};
IndexView index_view(const pk_index *h);
void set_error(const char *msg);

}  // namespace pk
