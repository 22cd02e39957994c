// Batched low-precision search (pk_fast.cu): arguments and launchers.
#pragma once

#include "pk_internal.h"

namespace pk {

constexpr int kTravF16 = 1;   // traversal copy in FP16
constexpr int kTravE4M3 = 2;  // traversal copy in FP8 E4M3 with per-dimension scales

constexpr int kFastMaxEf = 1024;  // the walk's register list holds up to 32 * 32 entries

// Bytes of a traversal query row: FP16 = the values; E4M3 = the query's two
// E4M3 parts and a 16-byte chunk holding its power-of-two factor.
__host__ __device__ inline int64_t trav_query_bytes(int trav, int64_t trav_data_bytes) {
    return trav == kTravF16 ? trav_data_bytes : 2 * trav_data_bytes + 16;
}

// Walk launch parameters.
struct WalkArgs {
    int64_t nq;
    int32_t ef;                 // uniform ef, or the bound of ef_arr
    int32_t expand;             // list entries expanded per iteration (1..4)
    const int32_t *ef_arr;
    int32_t *counters;          // nq * 6 or null
    int32_t *work;              // this launch's query counter
    int32_t *status;            // set to 1 when a row fetch timed out
    const int32_t *qlist;       // the queries this launch takes (null: 0 .. nq-1)
    const int32_t *qcount;      // their number, on the device (null: nq)
    int32_t *cand;              // nq * cand_stride: each query's final list (ids, -1 = empty)
    int32_t cand_stride;        // 32 * list slots per lane
    int32_t rb;                 // rows per fetch batch
    int32_t hlog2;              // log2 of the recently-seen table's id slots
    int32_t tag16;              // 1: 16-bit tags in 4-way sets, 0: 32-bit ids in 2-way sets
    int32_t idbits;             // bits of the largest node id (tag16)
    const uint8_t *tq_rows;     // traversal queries
    int64_t tq_row_bytes;
    const float *qnorm;         // sum of squares of each traversal query (L2)
    const uint8_t *trav;        // traversal copy of the vectors
    const uint8_t *trav_zero;   // a zero row of the traversal copy
    int64_t trav_row_bytes;
    int64_t trav_rows;          // rows in the traversal copy; node ids stay below it
    int64_t trav_data_bytes;    // the values of a row; E4M3 L2 rows have their norm after them (float)
    // second level of the visited filter: per warp (blockIdx.x * warps per
    // block + warp) 2^vt_log2sets sets of eight 16-bit tags in global memory,
    // small enough to stay in L2; null = the shared-memory table alone
    void *vt;
    int32_t vt_log2sets;
    int32_t vt_tbits;           // tag bits: the id's bits beyond the set index (<= 15)
    uint32_t vt_bmask;          // 2^(vt_log2sets + vt_tbits) - 1
    // a batch's winners (candidates below the list's last entry) are merged
    // into the list at once when at least merge_min of a 32-candidate chunk
    // win (lists of kMergeMinSlots or more slots), else inserted one by one
    int32_t merge_min;
};

// Sets (of eight 16-bit tags, 16 bytes) of a walk warp's visited table in
// global memory for lists of `slots` per lane over `ids` node ids.  A walk at
// ef meets about 1.5k + 16 ef distinct nodes on 128-dimensional data with
// 64 neighbours per node; the table holds about 1.25x that for the widest
// ef of the width (8-way sets: few overflow), at most twice the ids, and at
// least enough sets that the tag (the id's remaining bits) fits in 15 bits.
__host__ __device__ inline int visited_log2sets(int slots, int64_t ids) {
    const int64_t cap = 32 * (int64_t)slots;
    int64_t want = (1536 + 16 * cap) * 5 / 4;
    if (want > 2 * ids) want = 2 * ids;
    int l = 0;
    while (((int64_t)8 << l) < want) l++;
    int b = 1;
    while (b < 32 && ((int64_t)1 << b) < ids) b++;
    if (b - l > 15) l = b - 15;
    return l;
}

// Shared-memory stride of a staged traversal row: the row padded to an odd
// number of 16-byte chunks, so that 8 consecutive rows start in 8 different
// groups of banks (conflict-free ldmatrix and 16-byte loads).
__host__ __device__ inline int64_t stage_stride(int64_t trav_row_bytes) {
    return ((trav_row_bytes / 16) & 1) ? trav_row_bytes : trav_row_bytes + 16;
}

// Exact 16-bit tags fit when an id's bits beyond the set index (4-way sets:
// hlog2 - 2 index bits) are at most 15.  idbits_for(n) = bits of ids below n.
__host__ __device__ inline int idbits_for(int64_t n) {
    int b = 1;
    while (b < 32 && ((int64_t)1 << b) < n) b++;
    return b;
}
__host__ __device__ inline bool seen_tag16(int64_t n, int hlog2) {
    const int b = idbits_for(n) > hlog2 - 2 ? idbits_for(n) : hlog2 - 2;
    return b - (hlog2 - 2) <= 15;
}

// Lists of at least this many slots per lane merge a batch's winning
// candidates into the list at once when there are enough of them (one merge
// costs about as much as two or three one-at-a-time insertions at 16 slots).
constexpr int kMergeMinSlots = 6;

// Default winners of a chunk from which a list of `slots` per lane merges
// them at once (below it, one-by-one insertions are cheaper).
__host__ __device__ inline int merge_min_for(int slots) { return slots >= 12 ? 3 : slots >= 8 ? 4 : 5; }

// Shared memory the merge works in: the list (32 * slots packed entries), the
// winners (32 packed), the destination masks and the expanded marks (32 words
// each).  It reuses the staged rows' space, which is free between a batch's
// distances and the next fetch.
__host__ __device__ inline int64_t walk_merge_bytes(int slots) {
    return slots >= kMergeMinSlots ? 8 * 32 * (int64_t)slots + 8 * 32 + 4 * 32 + 4 * 32 : 0;
}

// Shared memory of one walk warp: the staged rows (rb rows, stride apart; at
// least the merge's working space for the list width), the query in the
// traversal format, the recently-seen table, the pending batch (rows, ids,
// distances), the mbarrier.  Every region starts on a 16-byte boundary (bulk
// copies land on 16-byte boundaries).
struct WalkLayout {
    int rowbuf, qbuf, tab, crow, cid, cd, bar, total;
    int64_t stride;
};
__host__ __device__ inline WalkLayout walk_layout(int rb, int64_t trav_row_bytes, int64_t query_bytes, int hlog2,
                                                  bool tag16, int slots) {
    WalkLayout w;
    w.stride = stage_stride(trav_row_bytes);
    w.rowbuf = 0;
    const int64_t rows = (int64_t)rb * w.stride, mb = walk_merge_bytes(slots);
    w.qbuf = align16(rows > mb ? rows : mb);
    w.tab = w.qbuf + align16(query_bytes);
    w.crow = w.tab + ((tag16 ? 2 : 4) << hlog2);
    w.cid = w.crow + align16(4 * (int64_t)rb);
    w.cd = w.cid + align16(4 * (int64_t)rb);
    w.bar = w.cd + align16(4 * (int64_t)rb);
    w.total = w.bar + 16;
    return w;
}

// Re-rank launch parameters.
struct RerankArgs {
    int64_t nq;
    int32_t k, ef;              // uniform values (ef also bounds ef_arr)
    const int32_t *k_arr, *ef_arr;
    int32_t out_stride;
    int32_t cand_stride;        // ints between two queries' lists in cand
    int32_t cand_cap;           // entries a list may hold (<= cand_stride; 0 = cand_stride): bounds ef, sizes the sort
    int32_t *out_ids;
    float *out_dists;
    const int32_t *ext0;
    const int32_t *cand;
    const int32_t *status;      // the walk's status: nonzero = its lists are incomplete
    const uint8_t *queries;     // exact queries, padded rows of row_bytes
    int64_t row_bytes;
    const int32_t *qlist;       // the queries to re-rank (null: 0 .. nq-1)
    const int32_t *qcount;      // device count of qlist's entries (null: nq)
};

__host__ __device__ inline int pow2_at_least(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Shared memory of one re-rank warp: a Stage block, the sort buffers (the
// bitonic sort pads a list to a power of two, so pow2_at_least(cand_stride)
// distances and ids), kStageRows exact rows.
struct RerankLayout {
    int sd, sid, rowbuf, total;
};
__host__ __device__ inline RerankLayout rerank_layout(int cand_stride, int64_t row_bytes) {
    RerankLayout r;
    const int64_t sort_cap = pow2_at_least(cand_stride);
    r.sd = kStageBytes;
    r.sid = r.sd + align16(4 * sort_cap);
    r.rowbuf = r.sid + align16(4 * sort_cap);
    r.total = align16(r.rowbuf + kStageRows * row_bytes);
    return r;
}

// List widths: slots per lane of the register list, which holds 32 entries
// per slot.  A query takes the narrowest width that holds its ef, so its list
// is at most twice ef (ef <= 64) or half again as wide (ef > 64).
constexpr int kSlotClasses = 10;
__host__ __device__ inline int slot_class_width(int c) {  // 1 2 3 4 6 8 12 16 24 32
    return c < 3 ? c + 1 : c == 3 ? 4 : c == 4 ? 6 : c == 5 ? 8 : c == 6 ? 12 : c == 7 ? 16 : c == 8 ? 24 : 32;
}
__host__ __device__ inline int slot_class(int ef) {
    int c = 0;
    while (c < kSlotClasses - 1 && 32 * slot_class_width(c) < ef) c++;
    return c;
}
__host__ __device__ inline int list_slots(int ef) { return slot_class_width(slot_class(ef)); }

int walk_blocks_per_sm(int trav, int slots, int expand, int wpb, size_t smem);
// Sorts the queries by list width class: lists[c * nq + i] = the i-th query
// of class c, counts[c] = how many (counts zeroed by the caller).
cudaError_t launch_bin_by_slots(const int32_t *ef_arr, int32_t ef_bound, int64_t nq, int32_t *counts,
                                int32_t *lists, cudaStream_t s);
cudaError_t launch_walk(const DevGraph *g, int trav, int slots, const WalkArgs &a, int grid, int wpb, size_t smem,
                        cudaStream_t s);
int rerank_blocks_per_sm(int dtype, const LaneCfg &lc, int wpb, size_t smem);
cudaError_t launch_rerank(const DevGraph *g, int dtype, const LaneCfg &lc, const RerankArgs &a, int grid, int wpb,
                          size_t smem, cudaStream_t s);
cudaError_t launch_absmax(int dtype, const uint8_t *vec0, int64_t row_bytes, int64_t n, int dim, uint32_t *out,
                          cudaStream_t s);
// Rows [r0, r1) into the traversal copy; each row's sum of squares of the
// stored values goes to rownorm[r] and, when norm_off >= 0, into the row at
// byte norm_off.
cudaError_t launch_convert_rows(int dtype, int trav, const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1,
                                int dim, const float *scale, uint8_t *trav_rows, int64_t trav_row_bytes,
                                int64_t norm_off, float *rownorm, cudaStream_t s);
cudaError_t launch_prep_queries(int dtype, int trav, const uint8_t *q, int64_t row_bytes, int64_t nq, int dim,
                                const float *scale, uint8_t *out, int64_t out_row_bytes, int64_t data_bytes,
                                float *qnorm, cudaStream_t s);

}  // namespace pk
