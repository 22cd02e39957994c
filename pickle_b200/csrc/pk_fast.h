// Batched low-precision search (pk_fast.cu): arguments and launchers.
#pragma once

#include "pk_internal.h"

namespace pk {

constexpr int kTravF16 = 1;   // traversal copy in FP16
constexpr int kTravE4M3 = 2;  // traversal copy in FP8 E4M3 with per-dimension scales

struct TravCfgHost {
    int GT, KT, CT, KTMAX;
};
TravCfgHost trav_config(int64_t trav_row_bytes, int trav);

struct FastArgs {
    int64_t nq;
    int32_t k, ef;                 // uniform values (ef also bounds ef_arr)
    const int32_t *k_arr, *ef_arr;
    int32_t out_stride;
    int32_t *out_ids;
    float *out_dists;
    const int32_t *ext0;
    int32_t *counters;             // nq * 6 or null
    int32_t *work;                 // [0] query counter
    WarpGlobalScratch gs;          // visited bitmaps and id lists
    int32_t list_cap;              // a power of two >= every ef
    int32_t rowbuf_bytes;          // kStageRows * max(row_bytes, trav_row_bytes)
    int32_t expand;                // entries expanded per iteration (1..4)
    const uint8_t *queries;        // exact queries, padded rows of row_bytes
    const uint8_t *tq_rows;        // traversal queries
    int64_t tq_row_bytes;
    const float *qnorm;            // E4M3: sum of squares of each query
    const uint8_t *trav;           // traversal copy of the vectors
    const uint8_t *trav_zero;      // a zero row of the traversal copy
    int64_t trav_row_bytes;
    const float *rownorm;          // E4M3: per-row norm of the stored copy
};

// Shared memory of one warp: two lists of list_cap (distance, id) entries, 32
// staged new entries, a Stage block, and the row buffer.
__host__ __device__ inline int fast_smem_per_warp(int list_cap, int rowbuf_bytes) {
    return align16((int64_t)16 * list_cap + 256 + kStageBytes) + align16(rowbuf_bytes);
}

int fast_blocks_per_sm(int dtype, const LaneCfg &lc, int trav, const TravCfgHost &tc, int wpb, size_t smem);
cudaError_t launch_search_fast(const DevGraph *g, int dtype, const LaneCfg &lc, int trav, const TravCfgHost &tc,
                               const FastArgs &a, int grid, int wpb, size_t smem, cudaStream_t s);
cudaError_t launch_absmax(int dtype, const uint8_t *vec0, int64_t row_bytes, int64_t n, int dim, uint32_t *out,
                          cudaStream_t s);
cudaError_t launch_convert_rows(int dtype, int trav, const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1,
                                int dim, const float *scale, uint8_t *trav_rows, int64_t trav_row_bytes,
                                float *rownorm, cudaStream_t s);
cudaError_t launch_prep_queries(int dtype, int trav, const uint8_t *q, int64_t row_bytes, int64_t nq, int dim,
                                const float *scale, uint8_t *out, int64_t out_row_bytes, float *qnorm,
                                cudaStream_t s);

}  // namespace pk
