/*
 * CPU restatement of pickle's v2 HNSW query and insert path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product (libpickle_b200.so) neither links nor calls it.
 *
 * Parity pins: this restatement is itself checked against the reference's own
 * code, compiled from its headers into oracle/_ref/pk_ref by oracle/Makefile
 * (tests/test_oracle_pins.py) and against the committed fixtures in
 * tests/golden/ that pk_ref produced.
 */
#ifndef PK_ORACLE_H
#define PK_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Adjacency growth on reverse-edge insertion.
 * ORA_GROWTH_REFERENCE: the reference's behaviour.  Its heuristic re-prune in
 *   AddEdge appends every kept neighbour without checking the slot count
 *   (include/hnsw_layer.hpp:441-447), so a node's list can outgrow its cap and
 *   run on into the following nodes' rows of the fixed-stride array.
 * ORA_GROWTH_CAPPED: the same algorithm with the heuristic prefix bounded by
 *   the cap (no spill).  This is what the device build implements. */
enum { ORA_GROWTH_REFERENCE = 0, ORA_GROWTH_CAPPED = 1 };

typedef struct ora_graph ora_graph;

/* Load a v2 graph file; *rc receives pkf_read's status. */
ora_graph *ora_load(const char *path, int *rc);
/* An empty index for sequential insertion with fixed per-node levels. */
ora_graph *ora_new(int metric, int dtype, int64_t dim, int64_t M, int64_t efc, int64_t capacity,
                   const uint8_t *levels, int growth);
void ora_free(ora_graph *g);
int ora_save(const ora_graph *g, const char *path);
/* out[0..7] = n0, num_layers, enter_level, capacity, dim, M, metric, dtype */
int ora_info(const ora_graph *g, int64_t *out);

/* HNSWGraph::Insert for one external id; data is the whole external-id
 * indexed matrix (row ext_id is inserted). */
int ora_insert(ora_graph *g, int32_t ext_id, const void *data);
/* Insert order[0..n) one after another (a one-thread HNSWGraph::Build). */
int ora_build(ora_graph *g, const void *data, const int32_t *order, int64_t n);

/* Batch AnnSearch.  ids/dists are nq*k, padded with -1 / FLT_MAX when fewer
 * than k results exist.  counters (nullable) is nq*6:
 * {hops upper, dists upper, neighbours upper, hops l0, dists l0, neighbours l0},
 * the per-level Profiler quantities of include/profiler.hpp:60-68. */
int ora_search(const ora_graph *g, const void *queries, int64_t nq, int k, int ef, int nthreads, int32_t *ids,
               float *dists, int64_t *counters);

/* pickle::Distance for one pair (L2 squared or negative inner product). */
float ora_distance(int dtype, int metric, const void *a, const void *b, int64_t dim);

/* Summation order of float32 / float16 distances (integer types are exact in
 * any order).  ORA_ORDER_SOURCE: the reference's source order (16 lanes, then
 * a left-to-right lane sum; the default).  ORA_ORDER_DEVICE: the order of the
 * device library's kernels, so that a search or build of the restatement can
 * be replayed with the device's own distances.  Process-wide; set it before a
 * call, not during one. */
enum { ORA_ORDER_SOURCE = 0, ORA_ORDER_DEVICE = 1, ORA_ORDER_TABLE = 2 };
void ora_set_float_order(int order);

/* Fork detector for float parity.  Replays AnnSearch for each query with two
 * sets of distances at once: order_a (ORA_ORDER_SOURCE or ORA_ORDER_DEVICE)
 * drives every decision, and each comparison of two distances (SlideLayer's
 * '<', the early exit, the admission test and every heap comparison) is also
 * evaluated with order_b's distances (ORA_ORDER_SOURCE, ORA_ORDER_DEVICE, or
 * ORA_ORDER_TABLE = values looked up per query in a table of (row key,
 * distance) pairs, key = the row's external id or -1 for the zero row, keys
 * sorted within each query's range tb_off[q]..tb_off[q+1]).  The first
 * comparison whose outcome differs is the point where the two searches fork;
 * fork[q*6 + 0..5] = {1 if forked else 0, where (1 slide, 2 early exit,
 * 3 admission, 4 heap order; 5 a table lookup missed), the two operands in
 * order a, the same two in order b}.  ids / dists (nq*k) are order_a's
 * results (those of ora_search in that order).  touched (nullable,
 * nq*touched_cap) receives the keys of the rows whose distances the order_a
 * search evaluated, touched_n[q] their count (may exceed touched_cap: then
 * the list is truncated). */
int ora_search_fork(const ora_graph *g, const void *queries, int64_t nq, int k, int ef, int order_a, int order_b,
                    const int64_t *tb_off, const int32_t *tb_key, const float *tb_val, int nthreads, int32_t *ids,
                    float *dists, double *fork, int32_t *touched, int64_t touched_cap, int64_t *touched_n);

/* The reference's level distribution: get_cumulative_probability(M)
 * (include/util.hpp:13-25).  Writes up to maxn values, returns the count. */
int ora_cumulative_probability(int64_t M, double *out, int maxn);

/* Read access to one layer, for structural comparisons in tests.
 * Pointers stay valid until ora_free. */
int ora_layer(const ora_graph *g, int level, int64_t *n, int64_t *cap, const int32_t **ext, const int16_t **degree,
              const int16_t **heuristic, const int32_t **adj, const float **dist);

#ifdef __cplusplus
}
#endif
#endif
