/*
 * pickle_b200 — C ABI of the B200 HNSW index (query and insert path).
 *
 * The reference (juelinl/pickle) exposes its HNSW index only as a header-only
 * C++ template class, pickle::v2::HNSWGraph (include/hnsw.hpp:23-220).  This
 * library implements the same index on the GPU and exposes it through plain C
 * entry points, so that any host language can bind it (ctypes, cgo, JNI, a C++
 * header such as include/pickle_b200/hnsw.hpp).  Each entry point below names
 * the reference interface it replaces.
 *
 * Conventions
 *  - Every call returns an int status: PK_OK (0) or a negative PK_ERR_* code.
 *    pk_last_error() gives a message for the calling thread's last failure.
 *    The reference has no error codes (it asserts or calls exit(-1),
 *    include/marco.hpp:20-68); here nothing aborts the process.
 *  - Enumerations keep the reference's numeric values: metric is DistFunc
 *    (1 = L2, 2 = IP; include/common.hpp:28-33), dtype is DataType
 *    (0 = uint8, 1 = int8, 2 = float32, 3 = float16; include/common.hpp:21-26).
 *  - Distances are returned as the reference returns them: squared L2, or the
 *    negated inner product (include/distance/avx512.hpp:233-243), ascending.
 *  - Vectors are row-major, dim elements per row, element type = dtype.
 *  - The index owns its device memory; caller buffers are only borrowed for
 *    the duration of a call (host variants) or until the given stream reaches
 *    the end of the call's work (device variants).
 *  - A handle may be used by one thread at a time.
 */
#ifndef PICKLE_B200_H
#define PICKLE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PK_OK 0
#define PK_ERR_ARG (-1)         /* bad argument */
#define PK_ERR_OOM (-2)         /* host or device allocation failed */
#define PK_ERR_IO (-3)          /* file could not be opened / read / written */
#define PK_ERR_FORMAT (-4)      /* not a v2 graph file, bad header, bad checksum */
#define PK_ERR_CUDA (-5)        /* a CUDA call failed */
#define PK_ERR_STATE (-6)       /* call not valid in the index's state */
#define PK_ERR_TIMEOUT (-7)     /* a device-side wait ran out of its budget */
#define PK_ERR_OVERFLOW (-8)    /* a search outgrew its scratch even after retry */
#define PK_ERR_NO_DEVICE (-9)   /* no CUDA device */
#define PK_ERR_CAPACITY (-10)   /* external id beyond the reserved capacity */

#define PK_METRIC_L2 1
#define PK_METRIC_IP 2

#define PK_DTYPE_U8 0
#define PK_DTYPE_I8 1
#define PK_DTYPE_F32 2
#define PK_DTYPE_F16 3

typedef struct pk_index pk_index;

/* Message for the calling thread's most recent failed call ("" if none). */
const char *pk_last_error(void);

/* Library version: major * 10000 + minor * 100 + patch. */
int pk_version(void);

/* Replaces HNSWGraph(max_degree, build_ef, DistFunc) / HNSWGraph::Init
 * (include/hnsw.hpp:27-36).  M is the upper-layer degree cap; layer 0 holds
 * 2*M slots per node (include/hnsw.hpp:235).  The index is bound to the
 * current CUDA device. */
int pk_index_create(pk_index **out, int metric, int dtype, int64_t dim, int64_t M, int64_t ef_construction);

/* Frees the handle and all its device memory.  NULL is accepted. */
int pk_index_destroy(pk_index *h);

/* Sets the seed of the per-node level draw (default 0).  The reference draws
 * levels from std::random_device (include/util.hpp:38-64); here level(ext_id)
 * is a pure function of (seed, ext_id) with the same distribution, so builds
 * are reproducible.  Must be called before the first insertion. */
int pk_index_set_seed(pk_index *h, uint64_t seed);

/* Sets per-node levels explicitly for external ids [0, n) (one byte each).
 * Replaces the level draw of InitBuffer (include/hnsw.hpp:222-245); used to
 * reproduce a given build.  Must be called before the first insertion. */
int pk_index_set_levels(pk_index *h, const uint8_t *levels, int64_t n);

/* Replaces HNSWGraph::Build (include/hnsw.hpp:497-507): inserts the rows of
 * data (n rows, host memory, indexed by external id) in the order given by
 * ext_ids (NULL = 0, 1, ..., n-1).  External ids must lie in [0, n).
 * Insertion runs on the GPU in batches of at most max_batch nodes
 * (0 = automatic); max_batch = 1 reproduces a one-thread build of the
 * reference algorithm exactly (with adjacency lists bounded by their caps). */
int pk_index_build(pk_index *h, const void *data, int64_t n, const int32_t *ext_ids, int32_t max_batch);

/* Replaces HNSWGraph::Insert (include/hnsw.hpp:247-302) for a batch: inserts
 * n new rows (host memory, row i has external id ext_ids[i]) into an existing
 * index.  External ids must be unused; the index grows as needed. */
int pk_index_add(pk_index *h, const void *rows, int64_t n, const int32_t *ext_ids, int32_t max_batch);

/* Replaces HNSWGraph::AnnSearch(top_k, search_ef, NDArray) (include/hnsw.hpp:528-541).
 * Host buffers: queries nq*dim, out_ids / out_dists nq*k.  Rows with fewer than
 * k results are padded with id -1 and distance FLT_MAX.  Synchronous. */
int pk_index_search(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                    float *out_dists);

/* pk_index_search with a k and an ef per query: the reference's batch loop
 * (include/hnsw.hpp:528-541) over its single-query AnnSearch (:509-525) with
 * each query's own values.  Host buffers: queries nq*dim, out_ids / out_dists
 * nq*out_stride (out_stride >= the largest k; row i holds k_per_query[i]
 * results, then -1 / FLT_MAX).  Synchronous. */
int pk_index_search_var(pk_index *h, const void *queries, int64_t nq, const int32_t *k_per_query,
                        const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids, float *out_dists);

/* Device-resident batch search, asynchronous on `stream` (a cudaStream_t,
 * NULL = legacy default stream).  All pointers are device pointers.
 *  k_per_query / ef_per_query: nq values each, or NULL to use k / ef for all.
 *  Results for query i go to out_ids/out_dists + i*out_stride (out_stride >=
 *  the largest k).  counters (nullable) receives nq*6 int32 values per query:
 *  hops, distance evaluations and neighbours scanned on the upper layers,
 *  then the same three on layer 0 (the Profiler quantities of
 *  include/profiler.hpp:13-69).
 *  Results are identical to pk_index_search's.  The call may synchronise
 *  `stream` once to retry the rare queries that outgrow their scratch. */
int pk_index_search_device(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                           const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride,
                           int32_t *out_ids, float *out_dists, int32_t *counters, void *stream);

/* Traversal precisions of the batched low-precision search. */
#define PK_TRAVERSAL_F16 1   /* FP16 copy of the vectors */
#define PK_TRAVERSAL_FP8 2   /* FP8 E4M3 copy, scaled per dimension */

/* Builds the low-precision copy of the vectors that pk_index_search_fast
 * walks the graph with (FP16, or FP8 E4M3 with one scale per dimension taken
 * from the rows present now; rows inserted later reuse those scales).
 * Synchronous.  Extends the reference, which walks with the original vectors
 * only (include/hnsw.hpp:373-444). */
int pk_index_prepare_fast(pk_index *h, int traversal);

/* Batched search that walks the graph with the low-precision copy and
 * re-ranks the ef listed candidates with exact distances from the original
 * vectors (the returned distances are exact; the ids may differ from the
 * exact search's where low-precision distances reorder the walk).  Arguments
 * as pk_index_search_device; `ef` bounds ef_per_query; expand = list entries
 * expanded per step (1..4, 0 = 1); ef <= 1024.  Fully asynchronous on `stream` (no host
 * synchronisation), so it can be captured in a CUDA graph once buffers have
 * grown to the batch size by an earlier call.  Successive calls on one
 * handle share its scratch: order them on one stream. */
int pk_index_search_fast(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                         const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride,
                         int32_t *out_ids, float *out_dists, int32_t *counters, int32_t expand, void *stream);

/* pk_index_search_fast with host buffers (queries nq*dim in, out_ids /
 * out_dists nq*k out); synchronous.  PK_ERR_TIMEOUT if a row fetch of the
 * walk did not complete within its bound (the results are then -1). */
int pk_index_search_fast_host(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                              float *out_dists, int32_t expand);

/* pk_index_search_fast with host buffers and a k and an ef per query (the
 * reference's batch AnnSearch takes one k and one ef for the whole batch,
 * include/hnsw.hpp:528-541; its single-query AnnSearch, :509-525, takes them
 * per call): queries nq*dim in, out_ids / out_dists nq*out_stride out
 * (out_stride >= the largest k; row i holds k_per_query[i] results, then
 * -1 / FLT_MAX).  Synchronous; PK_ERR_TIMEOUT as pk_index_search_fast_host. */
int pk_index_search_fast_host_var(pk_index *h, const void *queries, int64_t nq, const int32_t *k_per_query,
                                  const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids,
                                  float *out_dists, int32_t expand);

/* Launch shape of pk_index_search_fast's walk (0 keeps the default):
 * rows_per_batch = vector rows fetched per round trip (1..256; default
 * min(32, 12 KiB / row)); filter_log2 = log2 of the slots of the per-query
 * table of recently seen ids (5..15; default 10); warps_per_block (1..8;
 * default 4).  The results do not depend on the shape (the table only saves
 * recomputed distances); the speed does.  Clears the per-class shapes of
 * pk_index_tune_fast_classes.  No counterpart in the reference. */
int pk_index_set_fast_params(pk_index *h, int32_t rows_per_batch, int32_t filter_log2, int32_t warps_per_block);

/* Second level of the walk's visited filter: besides its table of recently
 * seen ids in shared memory, each walk warp keeps a larger table of the ids it
 * met in global memory (8-way sets of exact 16-bit tags, cleared per query,
 * a few to a few tens of KB per warp so that the resident warps' tables stay
 * in L2), which spares the walk most of the rows it would otherwise fetch and
 * score again after the shared-memory table forgot them.  log2_sets = 0 sizes
 * each width's tables by its list width (the default), -1 turns them off,
 * 1..20 gives every width 2^log2_sets sets of 16 bytes.  The tables are
 * allocated with the search's other buffers (their size grows with the warps
 * of a launch, not with the batch); when that allocation fails the walk runs
 * without them.  The autotuners (pk_index_tune_fast[_classes]) also time each
 * width without the tables and turn them off for a width where that is
 * faster; this call clears those choices.  The results do not depend on this
 * setting.  No counterpart in the reference. */
int pk_index_set_fast_visited(pk_index *h, int32_t log2_sets);

/* Layer-0 searches of batched insertion (pk_index_build / pk_index_add with
 * max_batch != 1), opt-in: with min_batch > 0 the nodes of every batch of at
 * least min_batch nodes take their ef_construction candidates at layer 0 from
 * the FP16 walk of pk_index_search_fast (run with the batch's own rows as
 * queries against the graph as it stood before the batch), whose exact
 * distances then feed SelectHeuristic as the exact search's result set
 * would; smaller batches, and every batch when max_batch == 1, use the exact
 * search that replays the reference's heaps.  The build makes the FP16
 * traversal copy it needs (as pk_index_prepare_fast(h, PK_TRAVERSAL_F16)
 * would) unless an FP8 copy is prepared, in which case it keeps the exact
 * search.  0 = off (the default).  On 10M x 128 FP16 rows (M=32, efC=200)
 * with min_batch = 256 the build took 53.0 s instead of 62.7 s, and the
 * graph's recall@10 at ef 64-96 was 0.005 lower.  No counterpart in the
 * reference. */
int pk_index_set_build_walk(pk_index *h, int64_t min_batch);

/* Insertion into the walk's result list: a list of 6 or more slots of 32
 * entries per lane (ef > 160) takes the winners of a 32-candidate chunk (the
 * candidates that beat its last entry) one at a time, or, when at least
 * min_winners of them win, all at once by a merge (sorted across the warp,
 * ranked in the list by binary search, moved through shared memory).  Either
 * way the list afterwards is the same.  0 = a threshold by list width (the
 * default), -1 = never merge, 1..32 = merge from that many winners.  No
 * counterpart in the reference. */
int pk_index_set_fast_merge(pk_index *h, int32_t min_winners);

/* Measurement: with timing enabled, each pk_index_search_fast /
 * pk_index_search_fast_host call on the handle records CUDA events on its
 * stream around the walk kernel and the re-rank kernel;
 * pk_index_fast_timing waits for the last call's events and returns the two
 * device durations in milliseconds.  With per-query ef each list width's
 * re-rank follows its walk on that width's stream: the walk time is then the
 * span until the last width's walk ends (the earlier widths' re-ranks run
 * inside it), the re-rank time what follows it.  Off by default (serving
 * slots never record).  No counterpart in the reference. */
int pk_index_set_fast_timing(pk_index *h, int enable);
int pk_index_fast_timing(pk_index *h, float *walk_ms, float *rerank_ms);

/* Autotuner: runs pk_index_search_fast on this batch (queries in device
 * memory, uniform k and ef, `expand` as given) for a grid of launch shapes,
 * times each with CUDA events on `stream`, and keeps the fastest as the
 * handle's shape (as pk_index_set_fast_params would).  out_shape (3 ints,
 * may be null) receives rows_per_batch, filter_log2, warps_per_block; out_ms
 * (may be null) the batch time.  Synchronous; results of later searches are
 * the same as with any other shape.  No counterpart in the reference. */
int pk_index_tune_fast(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t expand,
                       int32_t *out_shape, float *out_ms, void *stream);

/* Autotuner for batches whose queries carry their own ef: the walk runs one
 * launch per list width (1, 2, 3, 4, 6, 8, 12, 16, 24, 32 slots of 32 entries per
 * lane), and this tunes each width class up to max_ef separately on the given
 * queries (each class at its widest ef, k = min(k, that ef)), keeping one
 * launch shape per class.  out_shapes (10 x 3 ints, may be null) receives
 * rows_per_batch, filter_log2, warps_per_block per class (zeros for classes
 * above max_ef), out_ms (10 floats, may be null) each class's batch time.
 * pk_index_set_fast_params and pk_index_tune_fast clear the per-class shapes.
 * No counterpart in the reference. */
int pk_index_tune_fast_classes(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t max_ef,
                               int32_t expand, int32_t *out_shapes, float *out_ms, void *stream);

/* Sets the launch shape of one list-width class (0..9, see above) as
 * pk_index_tune_fast_classes would; all three values 0 = the handle's shape.
 * No counterpart in the reference. */
int pk_index_set_fast_class_params(pk_index *h, int32_t width_class, int32_t rows_per_batch, int32_t filter_log2,
                                   int32_t warps_per_block);

/* Serving: continuous batching over pk_index_search_fast.  No counterpart
 * in the reference (its batch AnnSearch is a blocking OpenMP loop,
 * include/hnsw.hpp:528-541).  A worker thread owns `slots` streams and one
 * arena of device memory.  Submitted requests (nq queries sharing one
 * k <= max_k and one ef <= max_ef <= 1024) wait in FIFO order; whenever a
 * stream is free, queued requests are packed into a batch of up to max_batch
 * queries for as long as the batch's device buffers - sized from the batch's
 * own query count, largest k and largest ef (pk_server_request_bytes gives a
 * request's share) - fit the arena's free space; batches in flight overlap on
 * the GPU and give their memory back when they finish.  Admission is thus by
 * device memory: a request that does not fit waits (deferred for memory, see
 * pk_server_memory) even while streams are free, and one larger than the
 * whole arena is refused at submission with PK_ERR_CAPACITY.  The arena is
 * device_bytes (pk_server_create_with_memory) or, for pk_server_create, enough
 * for every stream's full batch at max_k and max_ef but at most half of the
 * device memory free at creation; pk_server_create also gives each stream the
 * walk's visited tables in L2 (pk_index_set_fast_visited) for a full batch at
 * max_ef, outside the arena, where they can be allocated (without them a
 * stream's batches return the same results, more slowly), while
 * pk_server_create_with_memory with device_bytes > 0 takes device_bytes and
 * nothing more (device_bytes = 0: as pk_server_create).  Each
 * result equals what
 * pk_index_search_fast returns for that request alone.  A batch that does not
 * finish within the watchdog period (30 s) fails its requests with
 * PK_ERR_TIMEOUT.  The index must not be modified while a server uses it.
 * submit copies the queries and returns a ticket at once; wait blocks until
 * the ticket's results are ready (timeout_ms < 0: no limit), copies nq*k ids
 * and distances out, and reports the latency from submit to completion.
 * stats: out[0..4] = batches launched, queries served, most batches in flight
 * at once, requests queued, error status. */
typedef struct pk_server pk_server;
int pk_server_create(pk_server **out, pk_index *h, int traversal, int slots, int32_t max_batch, int32_t max_k,
                     int32_t max_ef, int32_t expand);
int pk_server_submit(pk_server *s, const void *queries, int32_t nq, int32_t k, int32_t ef, int64_t *ticket);
int pk_server_wait(pk_server *s, int64_t ticket, int32_t *out_ids, float *out_dists, double *latency_ms,
                   int32_t timeout_ms);
int pk_server_stats(pk_server *s, int64_t *out);
int pk_server_create_with_memory(pk_server **out, pk_index *h, int traversal, int slots, int32_t max_batch,
                                 int32_t max_k, int32_t max_ef, int32_t expand, int64_t device_bytes);
/* out[0..3] = arena bytes, bytes in use now, most bytes in use at once,
 * requests that had to wait for device memory. */
int pk_server_memory(pk_server *s, int64_t *out);
/* Device bytes a request of nq queries at k and ef takes while it runs (the
 * share admission checks against the arena). */
int pk_server_request_bytes(pk_server *s, int32_t nq, int32_t k, int32_t ef, int64_t *bytes);
/* Replays a timed request trace through the server: request i (nq[i]
 * consecutive rows of `queries`, k[i], ef[i]) is submitted arrival_us[i]
 * microseconds after the call starts, by a producer thread that waits for each
 * arrival time; results land in out_ids / out_dists (rows of out_stride, may
 * be NULL) and each request's submit-to-completion latency in latency_ms[i].
 * For measuring latency under a given arrival process (e.g. Poisson). */
int pk_server_replay(pk_server *s, const void *queries, int64_t n, const int32_t *nq, const double *arrival_us,
                     const int32_t *k, const int32_t *ef, int32_t *out_ids, float *out_dists, int32_t out_stride,
                     double *latency_ms);
/* Watchdog period in seconds (default 30): how long a slot may stay in flight
 * before its requests fail with PK_ERR_TIMEOUT. */
int pk_server_set_watchdog(pk_server *s, double seconds);
int pk_server_destroy(pk_server *s);

/* No counterpart in the reference.  The exact device search of
 * pk_index_search_device (uniform k and ef, device pointers, asynchronous work
 * on `stream` but the call waits for it) without any device allocation: for
 * callers that cannot let a library call cudaMalloc / cudaFree, such as a
 * serving loop that must not take the allocator's implicit device-wide
 * synchronisation, or a process whose device memory is already reserved by
 * another allocator.  All scratch comes from one fixed 64 MiB array in the
 * library image, held by every GPU that loads the library until exit.
 * Limits: nq <= 65536 and ef <= 1024 (PK_ERR_ARG beyond them); a query that
 * outgrows the fixed scratch is not retried (PK_ERR_OVERFLOW; fall back to
 * pk_index_search_device).  The index's device must be current.  The first
 * call on a device looks up the array's address there, and every call waits
 * for its work on the stream before it returns.  All calls on a device share the array and keep its
 * contents between calls (the call clears what must start at zero); calls
 * that overlap on the GPU race on it, so serialise them.  Results equal
 * pk_index_search_device's. */
int pk_index_search_noalloc(const pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                            int32_t *out_ids, float *out_dists, void *stream);

/* Replaces the Serializer::to_disk / from_disk pair that the reference names
 * for persistence (include/serializer.hpp:21-25) but only implements for its
 * retired v0 layer.  Writes / reads the v2 graph file: a versioned header,
 * per layer the reference's record layout (include/serializer.hpp:27-55)
 * extended with the v2 layer's fields, the layer-0 vectors and a checksum (the
 * byte layout is written out in pickle_b200/csrc/pk_format.cpp). */
int pk_index_save(const pk_index *h, const char *path);
int pk_index_load(pk_index **out, const char *path);

/* out[0..11] = n (nodes), num_layers, enter_level, capacity, dim, M,
 * ef_construction, metric, dtype, device bytes held, layer-0 cap, entry id. */
int pk_index_info(const pk_index *h, int64_t *out);

/* Copies one layer's structure to host buffers (each may be NULL):
 * ext[n], degree[n], heuristic[n], has_vector[n], adj[layer_capacity*cap],
 * dist[layer_capacity*cap].  *n, *layer_capacity and *cap are always written. */
int pk_index_layer(const pk_index *h, int level, int64_t *n, int64_t *layer_capacity, int64_t *cap, int32_t *ext,
                   int16_t *degree, int16_t *heuristic, uint8_t *has_vector, int32_t *adj, float *dist);

#ifdef __cplusplus
}
#endif
#endif
