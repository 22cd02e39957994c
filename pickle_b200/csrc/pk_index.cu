// Host side of libpickle_b200.so: the index handle, its device memory, the
// batched build, search dispatch and the C ABI of include/pickle_b200.h.
//
// Device layout (one index):
//   vec0      layer-0 vectors, one row per layer-0 internal id (= insertion
//             order), rows padded with zeros to a multiple of 16 bytes;
//   per layer adj / dist (fixed stride cap, as the reference's
//             include/hnsw_layer.hpp:76-78), deg, heu, ext, and for upper
//             layers vrow (the vec0 row holding that layer's copy of the
//             vector, -1 = the zero row) and down (the node's id one layer
//             down, replacing the reference's ext2in lookups);
//   a DevGraph block holding all of the above, read by the kernels.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <new>
#include <stdexcept>
#include <vector>

#include "pk_build.h"
#include "pk_fast.h"
#include "pk_format.h"
#include "pk_internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define PK_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? PK_ERR_OOM : PK_ERR_CUDA,                \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
        }                                                                                          \
    } while (0)

#define PK_TRY(call)               \
    do {                           \
        int rc_ = (call);          \
        if (rc_ != PK_OK) return rc_; \
    } while (0)

__global__ void fill_i32_kernel(int32_t *p, int64_t n, int32_t v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void fill_f32_kernel(float *p, int64_t n, float v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

cudaError_t fill_i32(int32_t *p, int64_t n, int32_t v, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
    fill_i32_kernel<<<grid, 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}
cudaError_t fill_f32(float *p, int64_t n, float v, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
    fill_f32_kernel<<<grid, 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}

// splitmix64: the per-node random stream of the level draw.
inline uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Scratch of one kind of search launch (queries, or insertion searches):
// per warp a visited bitmap, a list of marked ids, and a candidate-heap spill.
struct SearchScratch {
    int64_t warps = 0;
    int64_t bm_words = 0;
    int64_t vl_cap = 0;
    int64_t tail_cap = 0;
    uint32_t *bitmap = nullptr;
    int32_t *vlist = nullptr;
    void *cand_tail = nullptr;
    int32_t *work = nullptr;
    pk::WarpGlobalScratch view() const {
        return pk::WarpGlobalScratch{bitmap, bm_words, vlist, (int32_t)vl_cap, cand_tail, (int32_t)tail_cap};
    }
};

// Per-launch working set of the fast search: scratch and query staging.  The
// handle owns one; each serving slot owns its own, so slots can overlap.
// Layout of FastCtx::d_work: the walk's status, the query count of each list
// width class, the work counter of each class's launch.
constexpr int kWorkStatus = 0;
constexpr int kWorkCounts = 2;
constexpr int kWorkCounters = kWorkCounts + pk::kSlotClasses;
constexpr int kWorkInts = kWorkCounters + pk::kSlotClasses;

struct FastCtx {
    int32_t *d_work = nullptr;     // kWorkInts ints (above)
    int64_t work_n = 0;
    int32_t *d_lists = nullptr;    // per-query ef: the queries of each list width class
    int64_t lists_n = 0;
    int32_t *d_cand = nullptr;     // the walk's final lists, nq * 32 * slots ids
    int64_t cand_n = 0;
    uint8_t *d_fq = nullptr, *d_tq = nullptr;
    int64_t fq_n = 0, tq_n = 0;
    float *d_qn = nullptr;
    int64_t qn_n = 0;
    // the walk's visited tables in L2 (per warp of each width's launch);
    // a context with vt_fixed never allocates them (it uses what d_vt holds,
    // or runs with the shared-memory table alone)
    uint8_t *d_vt = nullptr;
    int64_t vt_n = 0;
    bool vt_fixed = false;
    // optional timing of the last launch: before the walk, after it, after
    // the re-rank (created on first use)
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    // per-query ef: one stream per list width, so that the widths' launches
    // run side by side and one width's tail does not hold the next back
    // (forked from and joined to the caller's stream with events; created on
    // first use)
    cudaStream_t aux[pk::kSlotClasses] = {};
    cudaEvent_t fork = nullptr, join[pk::kSlotClasses] = {};
    // timed per-width launches: the end of each width's walk (its re-rank
    // follows on the same stream), for the widths in wend_mask
    cudaEvent_t wend[pk::kSlotClasses] = {};
    uint32_t wend_mask = 0;
};

// Releases a context's streams and events (not its buffers).
void release_ctx_sync(FastCtx &c) {
    for (cudaEvent_t &e : c.ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t &e : c.join)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t &e : c.wend)
        if (e) cudaEventDestroy(e);
    if (c.fork) cudaEventDestroy(c.fork);
    for (cudaStream_t &t : c.aux)
        if (t) cudaStreamDestroy(t);
}

}  // namespace

struct pk_index {
    int device = 0;
    int num_sms = 0;
    int metric = 0, dtype = 0;
    int64_t dim = 0, M = 0, efc = 0, esz = 0, row_bytes = 0;
    pk::LaneCfg lc{};
    uint64_t seed = 0;
    std::vector<uint8_t> level_override;
    bool touched = false;   // an insertion happened (seed / levels are frozen)
    cudaStream_t stream = nullptr;

    // graph
    pk::DevGraph hg{};             // host copy holding device pointers
    pk::DevGraph *dg = nullptr;    // device copy
    int64_t alloc_rows[pk::kMaxLayers] = {};
    int num_layers = 0;
    int64_t vec_rows = 0;          // rows allocated in vec0
    int64_t capacity = 0;          // external ids in [0, capacity)
    std::vector<int32_t> ext_in0;  // external id -> layer-0 id (-1 absent)
    std::vector<uint8_t> ext_level;
    uint8_t *zero_row = nullptr;

    // scratch
    SearchScratch qs, bs;
    uint8_t *d_qstage = nullptr;
    int64_t qstage_rows = 0;
    int32_t *d_ids = nullptr;
    float *d_dists = nullptr;
    int64_t ids_n = 0, dists_n = 0;
    uint8_t *d_status = nullptr;
    int64_t status_n = 0;
    int32_t *d_qlist = nullptr;
    int64_t qlist_n = 0;

    // low-precision traversal copy and the fast path's scratch
    int trav = 0;                  // 0 none, pk::kTravF16, pk::kTravE4M3
    int64_t trav_row_bytes = 0, trav_rows = 0, trav_cap = 0;
    int64_t trav_data_bytes = 0;   // the traversal values; E4M3 L2 rows add a 32-byte chunk with the row's norm
    uint8_t *d_trav = nullptr, *d_trav_zero = nullptr;
    float *d_scale = nullptr, *d_rownorm = nullptr;
    float trav_f16_scale = 1.0f;   // FP16 copy = vectors / this power of two
    FastCtx fctx;
    int32_t *d_fids = nullptr;
    float *d_fdists = nullptr;
    int64_t fids_n = 0, fdists_n = 0;
    int32_t *d_karr = nullptr, *d_efarr = nullptr;  // per-query k / ef of host calls
    int64_t karr_n = 0, efarr_n = 0;
    // walk launch shape (0 = the default): rows per fetch batch, log2 of the
    // visited-filter slots, warps per block
    int fast_rb = 0, fast_hlog2 = 0, fast_wpb = 0;
    // per list-width class (pk::slot_class): a shape that overrides the one
    // above for that class's launch (0 = none)
    int cls_rb[pk::kSlotClasses] = {}, cls_hlog2[pk::kSlotClasses] = {}, cls_wpb[pk::kSlotClasses] = {};
    bool fast_timing = false;      // record events around the walk and the re-rank
    // the walk's visited tables in L2: 0 = sized by list width, -1 = off,
    // > 0 = log2 of the sets for every width
    int fast_vt = 0;
    // per list-width class: -1 = the tuner found the width faster without
    // the L2 tables (0 = as fast_vt)
    int cls_vt[pk::kSlotClasses] = {};
    // winners of a 32-candidate chunk from which the walk merges them into a
    // wide list at once: 0 = by list width, -1 = never (one by one)
    int fast_merge = 0;
    // insertion batches of at least this many nodes take their layer-0
    // candidates from the FP16 walk (0 = none: the exact search throughout)
    int64_t build_walk = 0;

    size_t dev_bytes = 0;

    int64_t n0() const { return hg.L[0].n; }
};

namespace {

int dalloc(pk_index *h, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PK_ERR_OOM, "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    h->dev_bytes += bytes;
    return PK_OK;
}

void dfree(pk_index *h, void *p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    h->dev_bytes -= std::min(h->dev_bytes, bytes == 0 ? (size_t)16 : bytes);
}

int push_graph(pk_index *h) {
    PK_CUDA(cudaMemcpy(h->dg, &h->hg, sizeof(pk::DevGraph), cudaMemcpyHostToDevice));
    return PK_OK;
}

// Make layer l hold at least rows node slots (plus a spare tail row).
int ensure_layer(pk_index *h, int l, int64_t rows, int64_t cap) {
    pk::DevLayer &L = h->hg.L[l];
    if (l >= h->num_layers) {
        L = pk::DevLayer{};
        L.cap = cap;
        h->alloc_rows[l] = 0;
        h->num_layers = l + 1;
        h->hg.num_layers = h->num_layers;
    }
    const int64_t want = rows + 1;
    if (h->alloc_rows[l] >= want) {
        L.lcap = std::max(L.lcap, rows);
        return PK_OK;
    }
    int64_t nr = std::max<int64_t>(want, h->alloc_rows[l] + h->alloc_rows[l] / 2);
    nr = std::max<int64_t>(nr, 16);
    const int64_t old = h->alloc_rows[l];
    const int64_t c = L.cap;
    pk::DevLayer N = L;
    PK_TRY(dalloc(h, (void **)&N.adj, sizeof(int32_t) * nr * c));
    PK_TRY(dalloc(h, (void **)&N.dist, sizeof(float) * nr * c));
    PK_TRY(dalloc(h, (void **)&N.deg, sizeof(int32_t) * nr));
    PK_TRY(dalloc(h, (void **)&N.heu, sizeof(int32_t) * nr));
    PK_TRY(dalloc(h, (void **)&N.ext, sizeof(int32_t) * nr));
    PK_TRY(dalloc(h, (void **)&N.vrow, sizeof(int32_t) * nr));
    PK_TRY(dalloc(h, (void **)&N.down, sizeof(int32_t) * nr));
    cudaStream_t s = h->stream;
    PK_CUDA(fill_i32(N.adj, nr * c, -1, s));
    PK_CUDA(fill_f32(N.dist, nr * c, FLT_MAX, s));
    PK_CUDA(cudaMemsetAsync(N.deg, 0, sizeof(int32_t) * nr, s));
    PK_CUDA(cudaMemsetAsync(N.heu, 0, sizeof(int32_t) * nr, s));
    PK_CUDA(fill_i32(N.ext, nr, -1, s));
    PK_CUDA(fill_i32(N.vrow, nr, -1, s));
    PK_CUDA(fill_i32(N.down, nr, -1, s));
    if (old > 0) {
        PK_CUDA(cudaMemcpyAsync(N.adj, L.adj, sizeof(int32_t) * old * c, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.dist, L.dist, sizeof(float) * old * c, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.deg, L.deg, sizeof(int32_t) * old, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.heu, L.heu, sizeof(int32_t) * old, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.ext, L.ext, sizeof(int32_t) * old, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.vrow, L.vrow, sizeof(int32_t) * old, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaMemcpyAsync(N.down, L.down, sizeof(int32_t) * old, cudaMemcpyDeviceToDevice, s));
        PK_CUDA(cudaStreamSynchronize(s));
        dfree(h, L.adj, sizeof(int32_t) * old * c);
        dfree(h, L.dist, sizeof(float) * old * c);
        dfree(h, L.deg, sizeof(int32_t) * old);
        dfree(h, L.heu, sizeof(int32_t) * old);
        dfree(h, L.ext, sizeof(int32_t) * old);
        dfree(h, L.vrow, sizeof(int32_t) * old);
        dfree(h, L.down, sizeof(int32_t) * old);
    }
    N.lcap = std::max(L.lcap, rows);
    L = N;
    h->alloc_rows[l] = nr;
    return PK_OK;
}

int ensure_vec(pk_index *h, int64_t rows) {
    if (h->vec_rows >= rows) return PK_OK;
    int64_t nr = std::max<int64_t>(rows, h->vec_rows + h->vec_rows / 2);
    nr = std::max<int64_t>(nr, 16);
    uint8_t *nv = nullptr;
    PK_TRY(dalloc(h, (void **)&nv, (size_t)(nr * h->row_bytes)));
    PK_CUDA(cudaMemsetAsync(nv, 0, (size_t)(nr * h->row_bytes), h->stream));
    if (h->vec_rows > 0) {
        PK_CUDA(cudaMemcpyAsync(nv, h->hg.vec0, (size_t)(h->vec_rows * h->row_bytes), cudaMemcpyDeviceToDevice,
                                h->stream));
        PK_CUDA(cudaStreamSynchronize(h->stream));
        dfree(h, (void *)h->hg.vec0, (size_t)(h->vec_rows * h->row_bytes));
    }
    h->hg.vec0 = nv;
    h->vec_rows = nr;
    return PK_OK;
}

void free_scratch(pk_index *h, SearchScratch &s) {
    dfree(h, s.bitmap, 4 * (size_t)s.warps * (size_t)s.bm_words);
    dfree(h, s.vlist, 4 * (size_t)s.warps * (size_t)s.vl_cap);
    dfree(h, s.cand_tail, 8 * (size_t)s.warps * (size_t)s.tail_cap);
    dfree(h, s.work, sizeof(int32_t) * 4);
    s = SearchScratch{};
}

// At least `warps` warps of scratch with bitmaps of bm_words words, lists of
// vl_cap ids and candidate spills of tail_cap entries.  Bitmaps start zeroed
// and every layer search leaves them zeroed.
int ensure_scratch(pk_index *h, SearchScratch &s, int64_t warps, int64_t bm_words, int64_t vl_cap, int64_t tail_cap) {
    if (s.bitmap && s.warps >= warps && s.bm_words >= bm_words && s.vl_cap >= vl_cap && s.tail_cap >= tail_cap)
        return PK_OK;
    const int64_t w = std::max(warps, s.warps), bw = std::max(bm_words, s.bm_words);
    const int64_t vc = std::max(vl_cap, s.vl_cap), tc = std::max(tail_cap, s.tail_cap);
    if (s.bitmap) {
        PK_CUDA(cudaStreamSynchronize(h->stream));
        PK_CUDA(cudaDeviceSynchronize());
        free_scratch(h, s);
    }
    PK_TRY(dalloc(h, (void **)&s.bitmap, 4 * (size_t)w * (size_t)bw));
    PK_TRY(dalloc(h, (void **)&s.vlist, 4 * (size_t)w * (size_t)vc));
    PK_TRY(dalloc(h, &s.cand_tail, 8 * (size_t)w * (size_t)tc));
    PK_TRY(dalloc(h, (void **)&s.work, sizeof(int32_t) * 4));
    PK_CUDA(cudaMemsetAsync(s.bitmap, 0, 4 * (size_t)w * (size_t)bw, h->stream));
    PK_CUDA(cudaStreamSynchronize(h->stream));
    s.warps = w;
    s.bm_words = bw;
    s.vl_cap = vc;
    s.tail_cap = tc;
    return PK_OK;
}

template <class T>
int ensure_buf(pk_index *h, T **p, int64_t &have, int64_t need) {
    if (have >= need && *p) return PK_OK;
    if (*p) {
        PK_CUDA(cudaStreamSynchronize(h->stream));
        dfree(h, *p, sizeof(T) * have);
        *p = nullptr;
    }
    int64_t n = std::max<int64_t>(need, have + have / 2);
    PK_TRY(dalloc(h, (void **)p, sizeof(T) * n));
    have = n;
    return PK_OK;
}

// ---------------------------------------------------------------- levels ----

// get_cumulative_probability (include/util.hpp:13-25).
std::vector<double> cumulative_probability(int64_t M) {
    std::vector<double> ret;
    const double r = 1.0 / std::log((double)M);
    double c = 0.0;
    for (;;) {
        const double delta = std::exp(-1.0 * (double)ret.size() / r) * (1 - std::exp(-1.0 / r));
        if (delta < 1e-9) break;
        c += delta;
        ret.push_back(c);
    }
    return ret;
}

// The level of one node: a fresh uniform draw per level, compared with the
// cumulative probability (the scheme of get_random_levels,
// include/util.hpp:38-64), from a stream keyed by (seed, external id).
int draw_level(const std::vector<double> &cp, uint64_t seed, int32_t ext) {
    uint64_t s = seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)(uint32_t)ext + 0x8CB92BA72F3D8DD7ULL);
    for (size_t l = 0; l < cp.size(); l++) {
        const double u = (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
        if (u < cp[l]) return (int)l;
    }
    return (int)cp.size() - 1;
}

// ---------------------------------------------------------------- search ----

int run_search(pk_index *h, const uint8_t *d_q, int64_t nq, int32_t k, int32_t ef, const int32_t *k_arr,
               const int32_t *ef_arr, int32_t stride, int32_t *ids, float *dists, int32_t *counters, cudaStream_t s) {
    if (nq == 0) return PK_OK;
    const int ef_max = std::max(ef, 1);
    const int wcap = ef_max + 2;
    int wpb = 4;
    size_t smem = (size_t)wpb * pk::search_smem_per_warp(wcap, h->row_bytes);
    while (wpb > 1 && smem > 200 * 1024) {
        wpb /= 2;
        smem = (size_t)wpb * pk::search_smem_per_warp(wcap, h->row_bytes);
    }
    if (smem > 220 * 1024) return fail(PK_ERR_ARG, "ef too large for shared memory: " + std::to_string(ef));
    const int nb = pk::search_blocks_per_sm(h->dtype, h->lc, wpb, smem);
    if (nb <= 0) return fail(PK_ERR_CUDA, "search kernel cannot be resident");
    const int64_t grid = std::min<int64_t>((int64_t)nb * h->num_sms, (nq + wpb - 1) / wpb);
    PK_TRY(ensure_buf(h, &h->d_status, h->status_n, nq));

    const int64_t bm_words = (h->hg.L[0].lcap + 31) / 32 + 1;
    const int64_t vl_cap = std::max<int64_t>(8192, 64LL * ef_max);
    int64_t tail = std::max<int64_t>(4096, 32LL * ef_max);
    const int32_t *qlist = nullptr;
    int64_t todo = nq;
    for (int attempt = 0; attempt < 4; attempt++) {
        PK_TRY(ensure_scratch(h, h->qs, grid * wpb, bm_words, vl_cap, tail));
        PK_CUDA(cudaMemsetAsync(h->qs.work, 0, sizeof(int32_t) * 2, s));
        pk::SearchArgs a{};
        a.queries = d_q;
        a.nq = todo;
        a.qlist = qlist;
        a.k = k;
        a.ef = ef_max;
        a.k_arr = k_arr;
        a.ef_arr = ef_arr;
        a.out_stride = stride;
        a.out_ids = ids;
        a.out_dists = dists;
        a.ext0 = h->hg.L[0].ext;
        a.counters = counters;
        a.status = h->d_status;
        a.work = h->qs.work;
        a.gs = h->qs.view();
        a.wcap = wcap;
        const int64_t g = std::min<int64_t>(grid, (todo + wpb - 1) / wpb);
        PK_CUDA(pk::launch_search_exact(h->dg, h->dtype, h->lc, a, (int)g, wpb, smem, s));
        int32_t over = 0;
        PK_CUDA(cudaMemcpyAsync(&over, h->qs.work + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        PK_CUDA(cudaStreamSynchronize(s));
        if (over == 0) return PK_OK;
        // rerun the queries whose candidate heap outgrew its spill, with 4x the room
        std::vector<uint8_t> st(nq);
        PK_CUDA(cudaMemcpy(st.data(), h->d_status, nq, cudaMemcpyDeviceToHost));
        std::vector<int32_t> list;
        for (int64_t i = 0; i < nq; i++)
            if (st[i]) list.push_back((int32_t)i);
        PK_TRY(ensure_buf(h, &h->d_qlist, h->qlist_n, (int64_t)list.size()));
        PK_CUDA(cudaMemcpy(h->d_qlist, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice));
        PK_CUDA(cudaMemsetAsync(h->d_status, 0, nq, s));
        qlist = h->d_qlist;
        todo = (int64_t)list.size();
        tail *= 4;
        if (tail > (1LL << 24)) break;
    }
    return fail(PK_ERR_OVERFLOW, "search outgrew its scratch after retries");
}

// Copies nq rows of dim*esz bytes into the padded staging buffer.
int stage_queries(pk_index *h, const void *q, int64_t nq, cudaMemcpyKind kind, cudaStream_t s) {
    PK_TRY(ensure_buf(h, &h->d_qstage, h->qstage_rows, nq * h->row_bytes));
    const size_t w = (size_t)(h->dim * h->esz);
    if (w != (size_t)h->row_bytes) PK_CUDA(cudaMemsetAsync(h->d_qstage, 0, (size_t)(nq * h->row_bytes), s));
    PK_CUDA(cudaMemcpy2DAsync(h->d_qstage, (size_t)h->row_bytes, q, w, w, (size_t)nq, kind, s));
    return PK_OK;
}

// ---------------------------------------------------------------- insert ----

struct BatchBufs {
    uint8_t *levels = nullptr;
    int32_t *ext = nullptr, *top_ins = nullptr, *node_id = nullptr;
    int32_t *item_node = nullptr, *item_level = nullptr, *item_id = nullptr, *item_down = nullptr;
    void *out = nullptr;
    int32_t *counts = nullptr;
    uint64_t *keys = nullptr;
    void *edges = nullptr;
    pk::EdgeWork ew{};
    int64_t nb_cap = 0, max_levels = 0, top_k0 = 0;
};

int alloc_batch(pk_index *h, BatchBufs &b, int64_t nb, int64_t max_levels, int64_t top_k0) {
    b.nb_cap = nb;
    b.max_levels = max_levels;
    b.top_k0 = top_k0;
    const int64_t nl = nb * max_levels, ns = nl * top_k0;
    PK_TRY(dalloc(h, (void **)&b.levels, nb));
    PK_TRY(dalloc(h, (void **)&b.ext, 4 * nb));
    PK_TRY(dalloc(h, (void **)&b.top_ins, 4 * nb));
    PK_TRY(dalloc(h, (void **)&b.node_id, 4 * nl));
    PK_TRY(dalloc(h, (void **)&b.item_node, 4 * nl));
    PK_TRY(dalloc(h, (void **)&b.item_level, 4 * nl));
    PK_TRY(dalloc(h, (void **)&b.item_id, 4 * nl));
    PK_TRY(dalloc(h, (void **)&b.item_down, 4 * nl));
    PK_TRY(dalloc(h, &b.out, 8 * ns));
    PK_TRY(dalloc(h, (void **)&b.counts, 4 * nl));
    PK_TRY(dalloc(h, (void **)&b.keys, 8 * ns));
    PK_TRY(dalloc(h, &b.edges, 8 * ns));
    b.ew.temp_bytes = pk::edge_sort_temp_bytes(ns);
    PK_TRY(dalloc(h, &b.ew.temp, b.ew.temp_bytes));
    PK_TRY(dalloc(h, (void **)&b.ew.keys_sorted, 8 * ns));
    PK_TRY(dalloc(h, (void **)&b.ew.flags, 4 * ns));
    PK_TRY(dalloc(h, (void **)&b.ew.scan, 4 * ns));
    PK_TRY(dalloc(h, (void **)&b.ew.seg_start, 8 * (ns + 1)));
    PK_TRY(dalloc(h, (void **)&b.ew.nseg, 4));
    return PK_OK;
}

void free_batch(pk_index *h, BatchBufs &b) {
    const int64_t nb = b.nb_cap, nl = nb * b.max_levels, ns = nl * b.top_k0;
    dfree(h, b.levels, nb);
    dfree(h, b.ext, 4 * nb);
    dfree(h, b.top_ins, 4 * nb);
    dfree(h, b.node_id, 4 * nl);
    dfree(h, b.item_node, 4 * nl);
    dfree(h, b.item_level, 4 * nl);
    dfree(h, b.item_id, 4 * nl);
    dfree(h, b.item_down, 4 * nl);
    dfree(h, b.out, 8 * ns);
    dfree(h, b.counts, 4 * nl);
    dfree(h, b.keys, 8 * ns);
    dfree(h, b.edges, 8 * ns);
    dfree(h, b.ew.temp, b.ew.temp_bytes);
    dfree(h, b.ew.keys_sorted, 8 * ns);
    dfree(h, b.ew.flags, 4 * ns);
    dfree(h, b.ew.scan, 4 * ns);
    dfree(h, b.ew.seg_start, 8 * (ns + 1));
    dfree(h, b.ew.nseg, 4);
    b = BatchBufs{};
}

int build_traversal(pk_index *h, int trav);
int refresh_traversal(pk_index *h);
int run_search_fast(pk_index *h, FastCtx &c, const void *queries, bool host_queries, int64_t nq, int32_t k,
                    int32_t ef, const int32_t *k_arr, const int32_t *ef_arr, int32_t stride, int32_t *ids,
                    float *dists, int32_t *counters, int32_t expand, cudaStream_t s, bool walk_only = false);
int fast_status(pk_index *h, FastCtx &c, cudaStream_t s);

// Inserts count rows, row i taken from rows + i*dim*esz with external id
// ext[i], in that order.
int insert_rows(pk_index *h, const uint8_t *rows, const int32_t *ext, int64_t count, int32_t max_batch) {
    if (count == 0) return PK_OK;
    cudaStream_t s = h->stream;
    const std::vector<double> cp = cumulative_probability(h->M);
    // levels and bookkeeping
    int64_t max_ext = -1;
    for (int64_t i = 0; i < count; i++) {
        if (ext[i] < 0) return fail(PK_ERR_ARG, "negative external id");
        max_ext = std::max<int64_t>(max_ext, ext[i]);
    }
    if (max_ext >= h->capacity) {
        h->capacity = max_ext + 1;
        h->ext_in0.resize(h->capacity, -1);
        h->ext_level.resize(h->capacity, 0);
    }
    std::vector<uint8_t> lv(count);
    int top = 0;
    for (int64_t i = 0; i < count; i++) {
        if (h->ext_in0[ext[i]] >= 0) return fail(PK_ERR_ARG, "external id inserted twice: " + std::to_string(ext[i]));
        int l;
        if (!h->level_override.empty()) {
            if (ext[i] >= (int64_t)h->level_override.size())
                return fail(PK_ERR_ARG, "no level given for external id " + std::to_string(ext[i]));
            l = h->level_override[ext[i]];
        } else {
            l = draw_level(cp, h->seed, ext[i]);
        }
        if (l >= pk::kMaxLayers) return fail(PK_ERR_ARG, "level too high");
        lv[i] = (uint8_t)l;
        top = std::max(top, l);
    }
    {
        std::vector<int32_t> sorted(ext, ext + count);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            return fail(PK_ERR_ARG, "duplicate external id in one call");
    }
    h->touched = true;
    // capacity per layer
    std::vector<int64_t> add_per(top + 1, 0);
    for (int64_t i = 0; i < count; i++)
        for (int l = 0; l <= lv[i]; l++) add_per[l]++;
    const int64_t n0_before = h->n0();
    for (int l = 0; l <= top; l++) {
        const int64_t have = l < h->num_layers ? h->hg.L[l].n : 0;
        PK_TRY(ensure_layer(h, l, have + add_per[l], l == 0 ? 2 * h->M : h->M));
    }
    // vectors, in insertion order
    PK_TRY(ensure_vec(h, n0_before + count));
    {
        const int64_t chunk = std::max<int64_t>(1, (256LL << 20) / h->row_bytes);
        std::vector<uint8_t> tmp;
        const size_t w = (size_t)(h->dim * h->esz);
        for (int64_t i0 = 0; i0 < count; i0 += chunk) {
            const int64_t c = std::min(chunk, count - i0);
            PK_CUDA(cudaMemcpy2D((uint8_t *)h->hg.vec0 + (n0_before + i0) * h->row_bytes, (size_t)h->row_bytes,
                                 rows + (size_t)i0 * w, w, w, (size_t)c, cudaMemcpyHostToDevice));
        }
    }
    PK_TRY(push_graph(h));

    // batch buffers
    const int64_t top_k0 = 2 * h->M;
    const int64_t max_levels = std::max(top, h->num_layers - 1) + 1;
    const int wcap = (int)h->efc + 2;
    int wpb = 4;
    size_t smem = (size_t)wpb * pk::insert_smem_per_warp(wcap, (int)top_k0, h->row_bytes);
    while (wpb > 1 && smem > 200 * 1024) {
        wpb /= 2;
        smem = (size_t)wpb * pk::insert_smem_per_warp(wcap, (int)top_k0, h->row_bytes);
    }
    const int bpsm = pk::insert_search_blocks_per_sm(h->dtype, h->lc, wpb, smem);
    if (bpsm <= 0) return fail(PK_ERR_CUDA, "insert kernel cannot be resident");
    const int64_t resident = (int64_t)bpsm * h->num_sms * wpb;
    // batches are capped: every node also compares itself with all earlier
    // nodes of its batch, which grows with the square of the batch
    int64_t bmax = max_batch > 0 ? max_batch : std::min<int64_t>(resident, 4096);
    bmax = std::max<int64_t>(1, std::min<int64_t>(bmax, count));
    BatchBufs bb;
    PK_TRY(alloc_batch(h, bb, bmax, max_levels, top_k0));
    struct Guard {
        pk_index *h;
        BatchBufs *b;
        ~Guard() {
            cudaStreamSynchronize(h->stream);
            free_batch(h, *b);
        }
    } guard{h, &bb};
    // every launched warp owns a scratch slot, including the ones that find
    // no work: size the scratch by the largest grid this call launches
    const int64_t max_grid = std::min<int64_t>((bmax + wpb - 1) / wpb, (int64_t)bpsm * h->num_sms);
    const int64_t bm_words = (h->hg.L[0].lcap + 31) / 32 + 1;
    const int64_t vl_cap = std::max<int64_t>(8192, 64LL * h->efc);
    int64_t tail = std::max<int64_t>(4096, 32LL * h->efc);
    PK_TRY(ensure_scratch(h, h->bs, max_grid * wpb, bm_words, vl_cap, tail));

    const int capmax = (int)top_k0;
    // layer-0 candidates from the FP16 walk for large batches (an FP8 copy,
    // or one-node batches, keep the exact search)
    const int64_t walk_min = h->build_walk > 0 ? h->build_walk : INT64_MAX;
    const bool walk_ok = max_batch != 1 && h->efc <= pk::kFastMaxEf && (h->trav == 0 || h->trav == pk::kTravF16);
    std::vector<int32_t> node_id, item_node, item_level, item_id, item_down, top_ins, bext;
    int64_t done = 0, bsize = 1;
    while (done < count) {
        const int64_t nb = std::min(std::min(bsize, bmax), count - done);
        const bool nonempty = h->n0() > 0;
        const int L = h->hg.enter_level;
        node_id.assign(nb * max_levels, -1);
        item_node.clear();
        item_level.clear();
        item_id.clear();
        item_down.clear();
        top_ins.assign(nb, 0);
        bext.assign(ext + done, ext + done + nb);
        std::vector<int64_t> next(max_levels, 0);
        for (int l = 0; l < max_levels; l++) next[l] = l < h->num_layers ? h->hg.L[l].n : 0;
        for (int64_t b = 0; b < nb; b++) {
            const int l = lv[done + b];
            top_ins[b] = nonempty ? std::min(l, L) : 0;
            for (int x = 0; x <= l; x++) {
                const int32_t id = (int32_t)next[x]++;  // NewInID in batch order
                node_id[b * max_levels + x] = id;
                item_node.push_back((int32_t)b);
                item_level.push_back(x);
                item_id.push_back(id);
                item_down.push_back(x > 0 ? node_id[b * max_levels + x - 1] : -1);
            }
        }
        PK_CUDA(cudaMemcpyAsync(bb.levels, lv.data() + done, nb, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.ext, bext.data(), 4 * nb, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.top_ins, top_ins.data(), 4 * nb, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.node_id, node_id.data(), 4 * nb * max_levels, cudaMemcpyHostToDevice, s));
        const int64_t ni = (int64_t)item_node.size();
        PK_CUDA(cudaMemcpyAsync(bb.item_node, item_node.data(), 4 * ni, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.item_level, item_level.data(), 4 * ni, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.item_id, item_id.data(), 4 * ni, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(bb.item_down, item_down.data(), 4 * ni, cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemsetAsync(bb.counts, 0, 4 * nb * max_levels, s));

        pk::AddNodeArgs na{};
        na.nitems = ni;
        na.item_node = bb.item_node;
        na.item_level = bb.item_level;
        na.item_id = bb.item_id;
        na.item_down = bb.item_down;
        na.ext_ids = bb.ext;
        na.top_inserted = bb.top_ins;
        na.pos0 = (int32_t)(n0_before + done);
        na.max_levels = (int32_t)max_levels;
        na.top_k0 = (int32_t)top_k0;
        na.out = bb.out;
        na.counts = bb.counts;
        na.meta_only = 1;
        PK_CUDA(pk::launch_add_node(h->dg, na, s));
        // 0. for a large batch on a graph of some size, the walk's layer-0
        // candidate lists for the batch's nodes (their rows are the queries)
        const bool use_walk = walk_ok && nonempty && nb >= walk_min && h->n0() >= 4 * h->efc;
        if (use_walk) {
            if (h->trav == 0) PK_TRY(build_traversal(h, pk::kTravF16));
            PK_TRY(run_search_fast(h, h->fctx, h->hg.vec0 + (n0_before + done) * h->row_bytes, false, nb, 1,
                                   (int32_t)h->efc, nullptr, nullptr, 1, nullptr, nullptr, nullptr, 1, s, true));
        }
        // 1. searches + SelectHeuristic (retried with more scratch on overflow)
        for (int attempt = 0;; attempt++) {
            PK_CUDA(cudaMemsetAsync(h->bs.work, 0, sizeof(int32_t) * 2, s));
            pk::InsertSearchArgs a{};
            a.nb = (int32_t)nb;
            a.pos0 = (int32_t)(n0_before + done);
            a.levels = bb.levels;
            a.enter_level = L;
            a.graph_nonempty = nonempty;
            a.efc = (int32_t)h->efc;
            a.top_k0 = (int32_t)top_k0;
            a.max_levels = (int32_t)max_levels;
            a.node_id = bb.node_id;
            a.out = bb.out;
            a.counts = bb.counts;
            a.work = h->bs.work;
            a.gs = h->bs.view();
            a.wcap = wcap;
            a.l0_cand = use_walk ? h->fctx.d_cand : nullptr;
            a.l0_stride = 32 * pk::list_slots((int)std::min<int64_t>(h->efc, pk::kFastMaxEf));
            const int64_t grid = std::min<int64_t>((nb + wpb - 1) / wpb, max_grid);
            PK_CUDA(pk::launch_insert_search(h->dg, h->dtype, h->lc, a, (int)grid, wpb, smem, s));
            int32_t over = 0;
            PK_CUDA(cudaMemcpyAsync(&over, h->bs.work + 1, 4, cudaMemcpyDeviceToHost, s));
            PK_CUDA(cudaStreamSynchronize(s));
            if (over == 0) break;
            if (attempt >= 3 || tail >= (1LL << 24)) return fail(PK_ERR_OVERFLOW, "insertion search outgrew scratch");
            // (the walk's candidates stay valid for the retry)
            tail *= 4;
            PK_TRY(ensure_scratch(h, h->bs, max_grid * wpb, bm_words, vl_cap, tail));
            PK_CUDA(cudaMemsetAsync(bb.counts, 0, 4 * nb * max_levels, s));
        }
        // a walk whose row fetch timed out left incomplete lists
        if (use_walk) PK_TRY(fast_status(h, h->fctx, s));
        // 2. AddNode for every (node, layer)
        na.meta_only = 0;
        PK_CUDA(pk::launch_add_node(h->dg, na, s));
        // 3. reverse edges, grouped by target
        pk::EdgeKeyArgs ka{};
        ka.nslots = nb * max_levels * top_k0;
        ka.max_levels = (int32_t)max_levels;
        ka.top_k0 = (int32_t)top_k0;
        ka.levels = bb.levels;
        ka.top_inserted = bb.top_ins;
        ka.counts = bb.counts;
        ka.out = bb.out;
        ka.node_id = bb.node_id;
        ka.keys = bb.keys;
        ka.edges = bb.edges;
        if (nonempty) PK_CUDA(pk::launch_add_edges(h->dg, h->dtype, h->lc, bb.ew, ka, capmax, s));
        // bookkeeping
        for (int l = 0; l < max_levels; l++)
            if (l < h->num_layers) h->hg.L[l].n = next[l];
        for (int64_t b = 0; b < nb; b++) {
            h->ext_in0[bext[b]] = (int32_t)node_id[b * max_levels];
            h->ext_level[bext[b]] = lv[done + b];
            if (lv[done + b] > h->hg.enter_level) h->hg.enter_level = lv[done + b];
        }
        PK_TRY(push_graph(h));
        done += nb;
        bsize = std::min<int64_t>(bsize * 2, bmax);
    }
    PK_CUDA(cudaStreamSynchronize(s));
    return PK_OK;
}

// ------------------------------------------------------------ fast path -----

// Per-dimension largest magnitude of rows [r0, r1) of the vectors.
int rows_absmax(pk_index *h, int64_t r0, int64_t r1, std::vector<float> &m) {
    cudaStream_t s = h->stream;
    m.assign(h->dim, 0.f);
    if (r1 <= r0) return PK_OK;
    uint32_t *amax = nullptr;
    PK_TRY(dalloc(h, (void **)&amax, 4 * (size_t)h->dim));
    PK_CUDA(cudaMemsetAsync(amax, 0, 4 * (size_t)h->dim, s));
    PK_CUDA(pk::launch_absmax(h->dtype, h->hg.vec0 + r0 * h->row_bytes, h->row_bytes, r1 - r0, (int)h->dim, amax,
                              s));
    PK_CUDA(cudaMemcpyAsync(m.data(), amax, 4 * (size_t)h->dim, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    dfree(h, amax, 4 * (size_t)h->dim);
    return PK_OK;
}

// FP16 traversal scale: the power of two sc with max|x| / sc in [4, 8), so
// that half-precision products and squares stay far inside FP16's range (1
// for an all-zero or non-finite maximum).
float f16_scale(const std::vector<float> &m) {
    float mx = 0.f;
    for (float v : m) mx = std::max(mx, v);
    if (!(mx > 0.f) || !std::isfinite(mx)) return 1.0f;
    int e = 0;
    std::frexp(mx / 8.0f, &e);  // mx / 8 = f * 2^e with f in [0.5, 1)
    return std::ldexp(1.0f, e);
}

// (Re)builds the traversal copy of rows [0, n0): scales from the rows present
// now (per dimension for FP8, one power of two for FP16), then every row
// converted, with its stored norm.
int build_traversal(pk_index *h, int trav) {
    cudaStream_t s = h->stream;
    // values padded with zeros to whole 32-byte steps of the tensor-core dot
    // products (16 FP16 or 32 E4M3 elements); for L2 in E4M3 a 32-byte chunk
    // after them holds the row's sum of squares (in original units, which the
    // per-dimension scales keep from being a function of the codes), so a
    // row's bulk copy brings its norm along and rows stay on whole 32-byte
    // sectors.  FP16 rows need no norm: the walk takes it from the Gram
    // diagonal of the staged rows.
    const int64_t tdb = trav == pk::kTravF16 ? (h->dim * 2 + 31) / 32 * 32 : (h->dim + 31) / 32 * 32;
    const int64_t trb = tdb + (h->metric == PK_METRIC_L2 && trav == pk::kTravE4M3 ? 32 : 0);
    const int64_t rows = std::max<int64_t>(h->vec_rows, 1);
    PK_CUDA(cudaStreamSynchronize(s));
    dfree(h, h->d_trav, (size_t)(h->trav_cap * h->trav_row_bytes));
    dfree(h, h->d_rownorm, 4 * (size_t)h->trav_cap);
    dfree(h, h->d_trav_zero, (size_t)h->trav_row_bytes);
    dfree(h, h->d_scale, 4 * (size_t)h->dim);
    h->d_trav = nullptr;
    h->trav = 0;
    PK_TRY(dalloc(h, (void **)&h->d_trav, (size_t)(rows * trb)));
    PK_TRY(dalloc(h, (void **)&h->d_rownorm, 4 * (size_t)rows));
    PK_TRY(dalloc(h, (void **)&h->d_trav_zero, (size_t)trb));
    PK_TRY(dalloc(h, (void **)&h->d_scale, 4 * (size_t)h->dim));
    PK_CUDA(cudaMemsetAsync(h->d_trav, 0, (size_t)(rows * trb), s));
    PK_CUDA(cudaMemsetAsync(h->d_trav_zero, 0, (size_t)trb, s));
    PK_CUDA(cudaMemsetAsync(h->d_rownorm, 0, 4 * (size_t)rows, s));
    std::vector<float> m, scale(h->dim, 1.0f);
    PK_TRY(rows_absmax(h, 0, h->n0(), m));
    if (trav == pk::kTravE4M3) {
        // E4M3's largest finite value is 448: map each dimension's largest
        // magnitude onto it
        for (int64_t d = 0; d < h->dim; d++) scale[d] = m[d] > 0.f ? m[d] / 448.0f : 1.0f;
    } else {
        const float sc = f16_scale(m);
        for (int64_t d = 0; d < h->dim; d++) scale[d] = sc;
        h->trav_f16_scale = sc;
    }
    PK_CUDA(cudaMemcpyAsync(h->d_scale, scale.data(), 4 * (size_t)h->dim, cudaMemcpyHostToDevice, s));
    PK_CUDA(pk::launch_convert_rows(h->dtype, trav, h->hg.vec0, h->row_bytes, 0, h->n0(), (int)h->dim, h->d_scale,
                                    h->d_trav, trb, trb > tdb ? tdb : -1, h->d_rownorm, s));
    PK_CUDA(cudaStreamSynchronize(s));
    h->trav = trav;
    h->trav_row_bytes = trb;
    h->trav_data_bytes = tdb;
    h->trav_rows = h->n0();
    h->trav_cap = rows;
    return PK_OK;
}

// Rows inserted since the copy was built are converted with the same scales,
// unless (FP16) they reach past 32 in scaled units, where half-precision
// squares could overflow: then the copy is rebuilt with a new scale.
int refresh_traversal(pk_index *h) {
    if (h->trav_rows == h->n0()) return PK_OK;
    if (h->vec_rows > h->trav_cap) return build_traversal(h, h->trav);
    if (h->trav == pk::kTravF16) {
        std::vector<float> m;
        PK_TRY(rows_absmax(h, h->trav_rows, h->n0(), m));
        float mx = 0.f;
        for (float v : m) mx = std::max(mx, v);
        if (!(mx <= 32.0f * h->trav_f16_scale)) return build_traversal(h, h->trav);
    }
    PK_CUDA(pk::launch_convert_rows(h->dtype, h->trav, h->hg.vec0, h->row_bytes, h->trav_rows, h->n0(), (int)h->dim,
                                    h->d_scale, h->d_trav, h->trav_row_bytes,
                                    h->trav_row_bytes > h->trav_data_bytes ? h->trav_data_bytes : -1, h->d_rownorm,
                                    h->stream));
    PK_CUDA(cudaStreamSynchronize(h->stream));
    h->trav_rows = h->n0();
    return PK_OK;
}

// Shape of the walk launch for this index: rows per fetch batch, visited
// filter size, warps per block, and the shared memory that takes.
struct WalkShape {
    int rb, hlog2, wpb;
    bool tag16;
    int idbits;
    size_t smem;
};
int walk_shape(const pk_index *h, WalkShape &w, int cls = -1) {
    const int64_t trb = h->trav_row_bytes;
    const bool own = cls >= 0 && cls < pk::kSlotClasses && h->cls_rb[cls] > 0;
    const int rb = own ? h->cls_rb[cls] : h->fast_rb;
    const int hl = own ? h->cls_hlog2[cls] : h->fast_hlog2;
    const int wp = own ? h->cls_wpb[cls] : h->fast_wpb;
    w.rb = rb > 0 ? rb : (int)std::max<int64_t>(8, std::min<int64_t>(32, 12288 / trb));
    w.hlog2 = hl > 0 ? hl : 10;
    w.wpb = wp > 0 ? wp : 4;
    const int64_t ids = std::max<int64_t>(2, std::min<int64_t>(h->hg.L[0].lcap, h->trav_rows));
    w.tag16 = pk::seen_tag16(ids, w.hlog2);
    w.idbits = std::max(pk::idbits_for(ids), w.hlog2 - 2);
    const int64_t qb = pk::trav_query_bytes(h->trav, h->trav_data_bytes);
    const int sl = pk::slot_class_width(cls >= 0 && cls < pk::kSlotClasses ? cls : pk::kSlotClasses - 1);
    w.smem = (size_t)w.wpb * pk::walk_layout(w.rb, trb, qb, w.hlog2, w.tag16, sl).total;
    while (w.wpb > 1 && w.smem > 200 * 1024) {
        w.wpb /= 2;
        w.smem = (size_t)w.wpb * pk::walk_layout(w.rb, trb, qb, w.hlog2, w.tag16, sl).total;
    }
    if (w.smem > 227 * 1024) return fail(PK_ERR_ARG, "walk working set exceeds shared memory: lower rows or filter bits");
    return PK_OK;
}

// One walk launch per list width: its shape, grid and visited tables in L2
// (one table per warp of every width's launch, since the launches run side
// by side; vt_off into one buffer of vt_total bytes, 0 with the tables off).
struct ClsPlan {
    WalkShape ws;
    int64_t grid = 0, vt_off = 0;
    int vt_log2 = 0;
};
int walk_plan(pk_index *h, int64_t nq, int slots, bool binned, int expand, ClsPlan *plan, int64_t &vt_total) {
    vt_total = 0;
    const int64_t ids0 = std::max<int64_t>(2, std::min<int64_t>(h->hg.L[0].lcap, h->trav_rows));
    for (int cls = 0; cls < pk::kSlotClasses && pk::slot_class_width(cls) <= slots; cls++) {
        const int sl = pk::slot_class_width(cls);
        if (!binned && sl != slots) continue;
        ClsPlan &P = plan[cls];
        PK_TRY(walk_shape(h, P.ws, cls));
        const int nb = pk::walk_blocks_per_sm(h->trav, sl, expand, P.ws.wpb, P.ws.smem);
        if (nb <= 0) return fail(PK_ERR_CUDA, "walk kernel cannot be resident");
        P.grid = std::min<int64_t>((int64_t)nb * h->num_sms, (nq + P.ws.wpb - 1) / P.ws.wpb);
        if (h->fast_vt >= 0 && h->cls_vt[cls] >= 0) {
            int l = h->fast_vt > 0 ? h->fast_vt : pk::visited_log2sets(sl, ids0);
            l = std::max(l, pk::idbits_for(ids0) - 15);
            P.vt_log2 = l;
            P.vt_off = vt_total;
            vt_total += P.grid * P.ws.wpb * ((int64_t)16 << l);
        }
    }
    return PK_OK;
}

// Low-precision walk, then exact re-rank of each query's final list.  Fully
// asynchronous on stream s.
// walk_only: the queries are padded device rows (row_bytes apart), and the
// call ends after the walk, leaving each query's candidate list in c.d_cand
// (no re-rank; k, k_arr, stride, ids and dists are unused).
int run_search_fast(pk_index *h, FastCtx &c, const void *queries, bool host_queries, int64_t nq, int32_t k,
                    int32_t ef, const int32_t *k_arr, const int32_t *ef_arr, int32_t stride, int32_t *ids,
                    float *dists, int32_t *counters, int32_t expand, cudaStream_t s, bool walk_only) {
    if (h->trav == 0) return fail(PK_ERR_STATE, "pk_index_prepare_fast has not been called");
    if (ef > pk::kFastMaxEf) return fail(PK_ERR_ARG, "ef too large for the fast path (max 1024)");
    PK_TRY(refresh_traversal(h));
    const int slots = pk::list_slots(ef);
    const int cs = 32 * slots;
    // per-query ef: queries are binned by list width and each width runs in
    // its own launch, so a query pays for the list it needs
    const bool binned = ef_arr != nullptr && slots > 1;
    WalkShape ws;
    PK_TRY(walk_shape(h, ws, pk::slot_class(ef)));
    PK_TRY(ensure_buf(h, &c.d_work, c.work_n, kWorkInts));
    PK_TRY(ensure_buf(h, &c.d_cand, c.cand_n, nq * cs));
    if (binned) PK_TRY(ensure_buf(h, &c.d_lists, c.lists_n, nq * pk::kSlotClasses));
    // exact queries (padded rows) and traversal queries
    const size_t w = (size_t)(h->dim * h->esz);
    const uint8_t *qx = static_cast<const uint8_t *>(queries);
    if (!walk_only && (host_queries || w != (size_t)h->row_bytes || ((uintptr_t)queries & 15) != 0)) {
        PK_TRY(ensure_buf(h, &c.d_fq, c.fq_n, nq * h->row_bytes));
        if (w != (size_t)h->row_bytes) PK_CUDA(cudaMemsetAsync(c.d_fq, 0, (size_t)(nq * h->row_bytes), s));
        PK_CUDA(cudaMemcpy2DAsync(c.d_fq, (size_t)h->row_bytes, queries, w, w, (size_t)nq,
                                  host_queries ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
        qx = c.d_fq;
    }
    const int64_t tq_rb = pk::trav_query_bytes(h->trav, h->trav_data_bytes);
    PK_TRY(ensure_buf(h, &c.d_tq, c.tq_n, nq * tq_rb));
    PK_TRY(ensure_buf(h, &c.d_qn, c.qn_n, nq));
    PK_CUDA(pk::launch_prep_queries(h->dtype, h->trav, qx, h->row_bytes, nq, (int)h->dim, h->d_scale, c.d_tq, tq_rb,
                                    h->trav_data_bytes, c.d_qn, s));
    PK_CUDA(cudaMemsetAsync(c.d_work, 0, sizeof(int32_t) * kWorkInts, s));
    if (binned) PK_CUDA(pk::launch_bin_by_slots(ef_arr, ef, nq, c.d_work + kWorkCounts, c.d_lists, s));
    pk::WalkArgs a{};
    a.nq = nq;
    a.ef = ef;
    a.expand = std::max(1, std::min(4, expand > 0 ? expand : 1));
    a.ef_arr = ef_arr;
    a.counters = counters;
    a.status = c.d_work + kWorkStatus;
    a.cand = c.d_cand;
    a.cand_stride = cs;
    a.tq_rows = c.d_tq;
    a.tq_row_bytes = tq_rb;
    a.qnorm = c.d_qn;
    a.trav = h->d_trav;
    a.trav_zero = h->d_trav_zero;
    a.trav_row_bytes = h->trav_row_bytes;
    a.trav_data_bytes = h->trav_data_bytes;
    a.trav_rows = h->trav_rows;
    ClsPlan plan[pk::kSlotClasses];
    int64_t vt_total = 0;
    PK_TRY(walk_plan(h, nq, slots, binned, a.expand, plan, vt_total));
    // the tables are scratch of the walk's own: if they cannot be had, the
    // walk runs with the shared-memory table alone (same results)
    if (vt_total > 0 && (vt_total > c.vt_n || !c.d_vt)) {
        if (c.vt_fixed || ensure_buf(h, &c.d_vt, c.vt_n, vt_total) != PK_OK) {
            if (!c.vt_fixed) c.vt_n = 0;
            vt_total = 0;
        }
    }
    const bool timed = h->fast_timing && &c == &h->fctx;
    if (timed) {
        for (cudaEvent_t &e : c.ev)
            if (!e) PK_CUDA(cudaEventCreate(&e));
        PK_CUDA(cudaEventRecord(c.ev[0], s));
        c.wend_mask = 0;
    }
    if (binned) {
        if (!c.fork) PK_CUDA(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
        PK_CUDA(cudaEventRecord(c.fork, s));
    }
    // the exact re-rank of the lists of cap entries (at most cand_stride) of
    // the queries in qlist (all queries when null), on stream ls
    auto rerank = [&](cudaStream_t ls, int cap, int32_t ef_bound, const int32_t *qlist, const int32_t *qcount,
                      int64_t nmax) -> int {
        int rwpb = 4;
        size_t rsmem = (size_t)rwpb * pk::rerank_layout(cap, h->row_bytes).total;
        while (rwpb > 1 && rsmem > 200 * 1024) {
            rwpb /= 2;
            rsmem = (size_t)rwpb * pk::rerank_layout(cap, h->row_bytes).total;
        }
        const int rnb = pk::rerank_blocks_per_sm(h->dtype, h->lc, rwpb, rsmem);
        if (rnb <= 0) return fail(PK_ERR_CUDA, "re-rank kernel cannot be resident");
        const int64_t rgrid = std::min<int64_t>((int64_t)rnb * h->num_sms, (nmax + rwpb - 1) / rwpb);
        pk::RerankArgs r{};
        r.nq = nq;
        r.k = k;
        r.ef = ef_bound;
        r.k_arr = k_arr;
        r.ef_arr = ef_arr;
        r.out_stride = stride;
        r.cand_stride = cs;
        r.cand_cap = cap;
        r.out_ids = ids;
        r.out_dists = dists;
        r.ext0 = h->hg.L[0].ext;
        r.cand = c.d_cand;
        r.status = c.d_work + kWorkStatus;
        r.queries = qx;
        r.row_bytes = h->row_bytes;
        r.qlist = qlist;
        r.qcount = qcount;
        PK_CUDA(pk::launch_rerank(h->dg, h->dtype, h->lc, r, (int)std::max<int64_t>(rgrid, 1), rwpb, rsmem, ls));
        return PK_OK;
    };
    // widest first: each launch fills the GPU and the next one's blocks take
    // the SMs its warps leave as its work runs out, so the launch that ends
    // the batch - whose tail nothing fills - is the one with the shortest
    // queries.  With per-query ef each width's re-rank follows its walk on
    // the width's own stream, so it overlaps the other widths' walks instead
    // of waiting for the last of them; its sort takes that width's lists only.
    for (int cls = pk::kSlotClasses - 1; cls >= 0; cls--) {
        const int sl = pk::slot_class_width(cls);
        if (sl > slots || (!binned && sl != slots)) continue;
        const ClsPlan &P = plan[cls];
        cudaStream_t ls = s;
        if (binned) {
            if (!c.aux[cls]) PK_CUDA(cudaStreamCreateWithFlags(&c.aux[cls], cudaStreamNonBlocking));
            if (!c.join[cls]) PK_CUDA(cudaEventCreateWithFlags(&c.join[cls], cudaEventDisableTiming));
            ls = c.aux[cls];
            PK_CUDA(cudaStreamWaitEvent(ls, c.fork, 0));
        }
        a.rb = P.ws.rb;
        a.hlog2 = P.ws.hlog2;
        a.tag16 = P.ws.tag16 ? 1 : 0;
        a.idbits = P.ws.idbits;
        a.vt = vt_total > 0 ? c.d_vt + P.vt_off : nullptr;
        a.vt_log2sets = P.vt_log2;
        const int vb = std::max(pk::idbits_for(std::max<int64_t>(2, std::min<int64_t>(h->hg.L[0].lcap, h->trav_rows))),
                                P.vt_log2);
        a.vt_tbits = vb - P.vt_log2;
        a.vt_bmask = vb >= 32 ? 0xffffffffu : (1u << vb) - 1u;
        a.merge_min = h->fast_merge < 0 ? (1 << 30) : h->fast_merge > 0 ? h->fast_merge : pk::merge_min_for(sl);
        a.work = c.d_work + kWorkCounters + cls;
        a.qlist = binned ? c.d_lists + cls * nq : nullptr;
        a.qcount = binned ? c.d_work + kWorkCounts + cls : nullptr;
        PK_CUDA(pk::launch_walk(h->dg, h->trav, sl, a, (int)P.grid, P.ws.wpb, P.ws.smem, ls));
        if (binned) {
            if (timed) {
                if (!c.wend[cls]) PK_CUDA(cudaEventCreate(&c.wend[cls]));
                PK_CUDA(cudaEventRecord(c.wend[cls], ls));
                c.wend_mask |= 1u << cls;
            }
            if (!walk_only)
                PK_TRY(rerank(ls, std::min(32 * sl, cs), std::min(ef, 32 * sl), a.qlist, a.qcount, nq));
            PK_CUDA(cudaEventRecord(c.join[cls], ls));
            PK_CUDA(cudaStreamWaitEvent(s, c.join[cls], 0));
        }
    }
    if (timed) PK_CUDA(cudaEventRecord(c.ev[1], s));
    if (walk_only) return PK_OK;
    if (!binned) PK_TRY(rerank(s, cs, ef, nullptr, nullptr, nq));
    if (timed) PK_CUDA(cudaEventRecord(c.ev[2], s));
    return PK_OK;
}

// After a synchronised fast search: the walk's status.
int fast_status(pk_index *h, FastCtx &c, cudaStream_t s) {
    int32_t st = 0;
    PK_CUDA(cudaMemcpyAsync(&st, c.d_work + kWorkStatus, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    if (st != 0) return fail(PK_ERR_TIMEOUT, "a row fetch of the fast search did not complete in time");
    return PK_OK;
}

// --------------------------------------------------------------- create -----

int init_handle(pk_index *h, int metric, int dtype, int64_t dim, int64_t M, int64_t efc) {
    if (metric != PK_METRIC_L2 && metric != PK_METRIC_IP) return fail(PK_ERR_ARG, "metric must be 1 (L2) or 2 (IP)");
    if (pk::elem_size(dtype) == 0) return fail(PK_ERR_ARG, "dtype must be 0..3");
    if (dim <= 0 || dim > 65536) return fail(PK_ERR_ARG, "dim out of range");
    if (M < 2 || M > 4096) return fail(PK_ERR_ARG, "M out of range");
    if (efc < 1 || efc > 20000) return fail(PK_ERR_ARG, "ef_construction out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(PK_ERR_NO_DEVICE, "no CUDA device");
    }
    PK_CUDA(cudaGetDevice(&h->device));
    PK_CUDA(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    h->metric = metric;
    h->dtype = dtype;
    h->dim = dim;
    h->M = M;
    h->efc = efc;
    h->esz = pk::elem_size(dtype);
    h->row_bytes = (dim * h->esz + 15) / 16 * 16;
    h->lc = pk::lane_config(h->row_bytes);
    PK_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    PK_TRY(dalloc(h, (void **)&h->dg, sizeof(pk::DevGraph)));
    PK_TRY(dalloc(h, (void **)&h->zero_row, (size_t)h->row_bytes));
    PK_CUDA(cudaMemset(h->zero_row, 0, (size_t)h->row_bytes));
    h->hg = pk::DevGraph{};
    h->hg.zero_row = h->zero_row;
    h->hg.row_bytes = h->row_bytes;
    h->hg.dim = (int32_t)dim;
    h->hg.dtype = dtype;
    h->hg.metric = metric;
    h->hg.enter_level = 0;
    // layer 0 always exists
    PK_TRY(ensure_layer(h, 0, 0, 2 * M));
    PK_TRY(ensure_vec(h, 16));
    PK_TRY(push_graph(h));
    return PK_OK;
}

void free_fast_ctx(pk_index *h, FastCtx &c) {
    release_ctx_sync(c);
    dfree(h, c.d_work, 4 * (size_t)c.work_n);
    dfree(h, c.d_cand, 4 * (size_t)c.cand_n);
    dfree(h, c.d_lists, 4 * (size_t)c.lists_n);
    dfree(h, c.d_fq, (size_t)c.fq_n);
    dfree(h, c.d_tq, (size_t)c.tq_n);
    dfree(h, c.d_qn, 4 * (size_t)c.qn_n);
    if (!c.vt_fixed) dfree(h, c.d_vt, (size_t)c.vt_n);
    c = FastCtx{};
}

void destroy_handle(pk_index *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int l = 0; l < h->num_layers; l++) {
        pk::DevLayer &L = h->hg.L[l];
        cudaFree(L.adj);
        cudaFree(L.dist);
        cudaFree(L.deg);
        cudaFree(L.heu);
        cudaFree(L.ext);
        cudaFree(L.vrow);
        cudaFree(L.down);
    }
    cudaFree((void *)h->hg.vec0);
    cudaFree(h->zero_row);
    cudaFree(h->dg);
    for (SearchScratch *s : {&h->qs, &h->bs}) {
        cudaFree(s->bitmap);
        cudaFree(s->vlist);
        cudaFree(s->cand_tail);
        cudaFree(s->work);
    }
    cudaFree(h->d_trav);
    cudaFree(h->d_trav_zero);
    cudaFree(h->d_scale);
    cudaFree(h->d_rownorm);
    free_fast_ctx(h, h->fctx);
    cudaFree(h->d_fids);
    cudaFree(h->d_fdists);
    cudaFree(h->d_karr);
    cudaFree(h->d_efarr);
    cudaFree(h->d_qstage);
    cudaFree(h->d_ids);
    cudaFree(h->d_dists);
    cudaFree(h->d_status);
    cudaFree(h->d_qlist);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

// ====================================================================== ABI ==

namespace {


static int pk_index_create_impl(pk_index **out, int metric, int dtype, int64_t dim, int64_t M, int64_t ef_construction) {
    if (!out) return fail(PK_ERR_ARG, "out is NULL");
    *out = nullptr;
    pk_index *h = new (std::nothrow) pk_index();
    if (!h) return fail(PK_ERR_OOM, "host allocation failed");
    int rc = init_handle(h, metric, dtype, dim, M, ef_construction);
    if (rc != PK_OK) {
        destroy_handle(h);
        return rc;
    }
    *out = h;
    return PK_OK;
}

static int pk_index_destroy_impl(pk_index *h) {
    destroy_handle(h);
    return PK_OK;
}

static int pk_index_set_seed_impl(pk_index *h, uint64_t seed) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (h->touched) return fail(PK_ERR_STATE, "seed must be set before the first insertion");
    h->seed = seed;
    return PK_OK;
}

static int pk_index_set_levels_impl(pk_index *h, const uint8_t *levels, int64_t n) {
    if (!h || (!levels && n > 0) || n < 0) return fail(PK_ERR_ARG, "bad arguments");
    if (h->touched) return fail(PK_ERR_STATE, "levels must be set before the first insertion");
    for (int64_t i = 0; i < n; i++)
        if (levels[i] >= pk::kMaxLayers) return fail(PK_ERR_ARG, "level too high");
    h->level_override.assign(levels, levels + n);
    return PK_OK;
}

static int pk_index_build_impl(pk_index *h, const void *data, int64_t n, const int32_t *ext_ids, int32_t max_batch) {
    if (!h || (!data && n > 0) || n < 0) return fail(PK_ERR_ARG, "bad arguments");
    if (h->n0() > 0) return fail(PK_ERR_STATE, "build needs an empty index");
    std::vector<int32_t> order(n);
    for (int64_t i = 0; i < n; i++) {
        order[i] = ext_ids ? ext_ids[i] : (int32_t)i;
        if (order[i] < 0 || order[i] >= n) return fail(PK_ERR_ARG, "external ids must lie in [0, n)");
    }
    // rows in insertion order: row i is data[order[i]]
    const size_t w = (size_t)(h->dim * h->esz);
    std::vector<uint8_t> rows;
    try {
        rows.resize((size_t)n * w);
    } catch (...) {
        return fail(PK_ERR_OOM, "host allocation failed");
    }
    const uint8_t *src = static_cast<const uint8_t *>(data);
    for (int64_t i = 0; i < n; i++) std::memcpy(rows.data() + (size_t)i * w, src + (size_t)order[i] * w, w);
    if (h->capacity < n) {
        h->capacity = n;
        h->ext_in0.resize(n, -1);
        h->ext_level.resize(n, 0);
    }
    return insert_rows(h, rows.data(), order.data(), n, max_batch);
}

static int pk_index_add_impl(pk_index *h, const void *rows, int64_t n, const int32_t *ext_ids, int32_t max_batch) {
    if (!h || ((!rows || !ext_ids) && n > 0) || n < 0) return fail(PK_ERR_ARG, "bad arguments");
    return insert_rows(h, static_cast<const uint8_t *>(rows), ext_ids, n, max_batch);
}

static int pk_index_search_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                    float *out_dists) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists) && nq > 0)) return fail(PK_ERR_ARG, "bad arguments");
    if (k < 1 || ef < 1) return fail(PK_ERR_ARG, "k and ef must be >= 1");
    if (nq == 0) return PK_OK;
    if (h->n0() == 0) {
        for (int64_t i = 0; i < nq * k; i++) {
            out_ids[i] = -1;
            out_dists[i] = FLT_MAX;
        }
        return PK_OK;
    }
    cudaStream_t s = h->stream;
    PK_TRY(stage_queries(h, queries, nq, cudaMemcpyHostToDevice, s));
    PK_TRY(ensure_buf(h, &h->d_ids, h->ids_n, nq * k));
    PK_TRY(ensure_buf(h, &h->d_dists, h->dists_n, nq * k));
    PK_TRY(run_search(h, h->d_qstage, nq, k, ef, nullptr, nullptr, k, h->d_ids, h->d_dists, nullptr, s));
    PK_CUDA(cudaMemcpyAsync(out_ids, h->d_ids, sizeof(int32_t) * nq * k, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaMemcpyAsync(out_dists, h->d_dists, sizeof(float) * nq * k, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    return PK_OK;
}

// Host buffers with a k and an ef per query (row i of the output holds
// k_per_query[i] results, then -1 / FLT_MAX up to out_stride).
static int pk_index_search_var_impl(pk_index *h, const void *queries, int64_t nq, const int32_t *k_per_query,
                                    const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids,
                                    float *out_dists) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists || !k_per_query || !ef_per_query) && nq > 0))
        return fail(PK_ERR_ARG, "bad arguments");
    if (nq == 0) return PK_OK;
    int32_t kmax = 0, efmax = 0;
    for (int64_t i = 0; i < nq; i++) {
        if (k_per_query[i] < 1 || ef_per_query[i] < 1) return fail(PK_ERR_ARG, "every k and ef must be >= 1");
        kmax = std::max(kmax, k_per_query[i]);
        efmax = std::max(efmax, ef_per_query[i]);
    }
    if (out_stride < kmax) return fail(PK_ERR_ARG, "out_stride below the largest k");
    if (h->n0() == 0) {
        for (int64_t i = 0; i < nq * out_stride; i++) {
            out_ids[i] = -1;
            out_dists[i] = FLT_MAX;
        }
        return PK_OK;
    }
    cudaStream_t s = h->stream;
    PK_TRY(stage_queries(h, queries, nq, cudaMemcpyHostToDevice, s));
    PK_TRY(ensure_buf(h, &h->d_ids, h->ids_n, nq * out_stride));
    PK_TRY(ensure_buf(h, &h->d_dists, h->dists_n, nq * out_stride));
    PK_TRY(ensure_buf(h, &h->d_karr, h->karr_n, nq));
    PK_TRY(ensure_buf(h, &h->d_efarr, h->efarr_n, nq));
    PK_CUDA(cudaMemcpyAsync(h->d_karr, k_per_query, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaMemcpyAsync(h->d_efarr, ef_per_query, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
    PK_CUDA(fill_i32(h->d_ids, nq * out_stride, -1, s));
    PK_CUDA(fill_f32(h->d_dists, nq * out_stride, FLT_MAX, s));
    PK_TRY(run_search(h, h->d_qstage, nq, kmax, efmax, h->d_karr, h->d_efarr, out_stride, h->d_ids, h->d_dists,
                      nullptr, s));
    PK_CUDA(cudaMemcpyAsync(out_ids, h->d_ids, sizeof(int32_t) * nq * out_stride, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaMemcpyAsync(out_dists, h->d_dists, sizeof(float) * nq * out_stride, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    return PK_OK;
}

static int pk_index_search_device_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                           const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride,
                           int32_t *out_ids, float *out_dists, int32_t *counters, void *stream) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists) && nq > 0)) return fail(PK_ERR_ARG, "bad arguments");
    if (k < 1 || ef < 1 || out_stride < k) return fail(PK_ERR_ARG, "need k >= 1, ef >= 1, out_stride >= k");
    if (nq == 0) return PK_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (h->n0() == 0) {
        PK_CUDA(fill_i32(out_ids, nq * out_stride, -1, s));
        PK_CUDA(fill_f32(out_dists, nq * out_stride, FLT_MAX, s));
        return PK_OK;
    }
    const size_t w = (size_t)(h->dim * h->esz);
    const uint8_t *q = static_cast<const uint8_t *>(queries);
    if (w != (size_t)h->row_bytes || ((uintptr_t)queries & 15) != 0) {
        PK_TRY(stage_queries(h, queries, nq, cudaMemcpyDeviceToDevice, s));
        q = h->d_qstage;
    }
    return run_search(h, q, nq, k, ef, k_per_query, ef_per_query, out_stride, out_ids, out_dists, counters, s);
}

static int pk_index_save_impl(const pk_index *hc, const char *path) {
    pk_index *h = const_cast<pk_index *>(hc);
    if (!h || !path) return fail(PK_ERR_ARG, "bad arguments");
    PK_CUDA(cudaStreamSynchronize(h->stream));
    pk::FileGraph g;
    g.metric = h->metric;
    g.dtype = h->dtype;
    g.dim = h->dim;
    g.max_degree = h->M;
    g.build_ef = h->efc;
    g.capacity = h->capacity;
    g.enter_level = h->hg.enter_level;
    const int nl = h->n0() > 0 ? h->num_layers : 0;
    g.layers.resize(nl);
    for (int l = 0; l < nl; l++) {
        const pk::DevLayer &L = h->hg.L[l];
        pk::FileLayer &F = g.layers[l];
        F.n = L.n;
        F.layer_capacity = std::max(L.lcap, L.n);
        F.cap = L.cap;
        F.ent = L.ent;
        F.ext.resize(F.n);
        std::vector<int32_t> deg(F.n), heu(F.n), vrow(F.n);
        F.adj.resize((size_t)(F.layer_capacity * F.cap));
        F.dist.resize((size_t)(F.layer_capacity * F.cap));
        PK_CUDA(cudaMemcpy(F.ext.data(), L.ext, 4 * F.n, cudaMemcpyDeviceToHost));
        PK_CUDA(cudaMemcpy(deg.data(), L.deg, 4 * F.n, cudaMemcpyDeviceToHost));
        PK_CUDA(cudaMemcpy(heu.data(), L.heu, 4 * F.n, cudaMemcpyDeviceToHost));
        PK_CUDA(cudaMemcpy(F.adj.data(), L.adj, 4 * F.adj.size(), cudaMemcpyDeviceToHost));
        PK_CUDA(cudaMemcpy(F.dist.data(), L.dist, 4 * F.dist.size(), cudaMemcpyDeviceToHost));
        if (l > 0) PK_CUDA(cudaMemcpy(vrow.data(), L.vrow, 4 * F.n, cudaMemcpyDeviceToHost));
        F.degree.resize(F.n);
        F.heuristic.resize(F.n);
        F.has_vector.resize(F.n);
        for (int64_t i = 0; i < F.n; i++) {
            F.degree[i] = (int16_t)deg[i];
            F.heuristic[i] = (int16_t)heu[i];
            F.has_vector[i] = l == 0 ? 1 : (vrow[i] >= 0 ? 1 : 0);
        }
    }
    const int64_t n0 = h->n0();
    const size_t w = (size_t)(h->dim * h->esz);
    g.vectors.resize((size_t)n0 * w);
    if (n0 > 0)
        PK_CUDA(cudaMemcpy2D(g.vectors.data(), w, h->hg.vec0, (size_t)h->row_bytes, w, (size_t)n0,
                             cudaMemcpyDeviceToHost));
    const int rc = pk::write_graph_file(path, g);
    if (rc != PK_OK) return fail(rc, std::string("cannot write ") + path);
    return PK_OK;
}

// Maps the file, checks it, and uploads each array from the mapping to the
// device (the large ones - adjacency, distances, vectors - with no host copy).
static int pk_index_load_impl(pk_index **out, const char *path) {
    if (!out || !path) return fail(PK_ERR_ARG, "bad arguments");
    *out = nullptr;
    pk::MappedGraph g;
    std::string err;
    int rc = pk::map_graph_file(path, g, err);
    if (rc != PK_OK) return fail(rc, err);
    const int nl = (int)g.layers.size();
    if (nl > pk::kMaxLayers) return fail(PK_ERR_FORMAT, "too many layers");
    // the small per-node arrays, read out of the (unaligned) mapping
    std::vector<std::vector<int32_t>> ext(nl), deg(nl), heu(nl);
    std::vector<std::vector<uint8_t>> hasv(nl);
    for (int l = 0; l < nl; l++) {
        const pk::MappedLayer &F = g.layers[l];
        ext[l].resize(F.n);
        deg[l].resize(F.n);
        heu[l].resize(F.n);
        hasv[l].resize(F.n);
        std::vector<int16_t> d16(F.n), h16(F.n);
        std::memcpy(ext[l].data(), F.ext, 4 * (size_t)F.n);
        std::memcpy(d16.data(), F.degree, 2 * (size_t)F.n);
        std::memcpy(h16.data(), F.heuristic, 2 * (size_t)F.n);
        std::memcpy(hasv[l].data(), F.has_vector, (size_t)F.n);
        // consistency checks the reference would trip over (ids, ranges)
        if (F.cap != (l == 0 ? 2 * g.max_degree : g.max_degree)) return fail(PK_ERR_FORMAT, "unexpected layer cap");
        if (F.n > 0 && (F.ent < 0 || F.ent >= F.layer_capacity)) return fail(PK_ERR_FORMAT, "bad entry id");
        for (int64_t i = 0; i < F.n; i++) {
            if (ext[l][i] < 0 || ext[l][i] >= g.capacity) return fail(PK_ERR_FORMAT, "external id out of range");
            if (d16[i] < 0 || h16[i] < 0) return fail(PK_ERR_FORMAT, "negative degree");
            deg[l][i] = d16[i];
            heu[l][i] = h16[i];
        }
    }
    pk_index *h = new (std::nothrow) pk_index();
    if (!h) return fail(PK_ERR_OOM, "host allocation failed");
    rc = init_handle(h, g.metric, g.dtype, g.dim, g.max_degree, g.build_ef);
    if (rc != PK_OK) {
        destroy_handle(h);
        return rc;
    }
    auto bail = [&](int code) {
        destroy_handle(h);
        return code;
    };
    h->touched = true;
    h->capacity = g.capacity;
    h->ext_in0.assign(g.capacity, -1);
    h->ext_level.assign(g.capacity, 0);
    std::vector<std::vector<int32_t>> ext2in(nl);
    for (int l = 0; l < nl; l++) {
        const pk::MappedLayer &F = g.layers[l];
        ext2in[l].assign(g.capacity, -1);
        for (int64_t i = 0; i < F.n; i++) {
            ext2in[l][ext[l][i]] = (int32_t)i;
            h->ext_level[ext[l][i]] = (uint8_t)l;
        }
    }
    if (nl > 0)
        for (int64_t i = 0; i < g.layers[0].n; i++) h->ext_in0[ext[0][i]] = (int32_t)i;
    for (int l = 0; l < nl; l++) {
        const pk::MappedLayer &F = g.layers[l];
        // spare rows after the last node so that a spilled list read past the
        // end meets -1 entries (skipped) rather than unallocated memory
        int64_t need = F.layer_capacity;
        for (int64_t i = 0; i < F.n; i++) need = std::max(need, (i * F.cap + deg[l][i] + F.cap - 1) / F.cap);
        if ((rc = ensure_layer(h, l, need, F.cap)) != PK_OK) return bail(rc);
        pk::DevLayer &L = h->hg.L[l];
        L.lcap = F.layer_capacity;
        L.n = F.n;
        L.ent = F.ent;
        std::vector<int32_t> vrow(F.n, -1), down(F.n, -1);
        if (l > 0)
            for (int64_t i = 0; i < F.n; i++) {
                vrow[i] = hasv[l][i] ? h->ext_in0[ext[l][i]] : -1;
                down[i] = ext2in[l - 1][ext[l][i]];
            }
        const size_t e = (size_t)(F.layer_capacity * F.cap);
        if (cudaMemcpy(L.ext, ext[l].data(), 4 * F.n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.deg, deg[l].data(), 4 * F.n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.heu, heu[l].data(), 4 * F.n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.adj, F.adj, 4 * e, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.dist, F.dist, 4 * e, cudaMemcpyHostToDevice) != cudaSuccess ||
            (l > 0 && cudaMemcpy(L.vrow, vrow.data(), 4 * F.n, cudaMemcpyHostToDevice) != cudaSuccess) ||
            (l > 0 && cudaMemcpy(L.down, down.data(), 4 * F.n, cudaMemcpyHostToDevice) != cudaSuccess))
            return bail(fail(PK_ERR_CUDA, "upload failed"));
    }
    const int64_t n0 = nl > 0 ? g.layers[0].n : 0;
    const int64_t lcap0 = nl > 0 ? g.layers[0].layer_capacity : 0;
    if ((rc = ensure_vec(h, std::max<int64_t>(lcap0, 1))) != PK_OK) return bail(rc);
    const size_t w = (size_t)(h->dim * h->esz);
    if (n0 > 0 && cudaMemcpy2D((void *)h->hg.vec0, (size_t)h->row_bytes, g.vectors, w, w, (size_t)n0,
                               cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(PK_ERR_CUDA, "vector upload failed"));
    h->hg.enter_level = nl > 0 ? g.enter_level : 0;
    if ((rc = push_graph(h)) != PK_OK) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(PK_ERR_CUDA, "sync failed"));
    *out = h;
    return PK_OK;
}

static int pk_index_info_impl(const pk_index *h, int64_t *out) {
    if (!h || !out) return fail(PK_ERR_ARG, "bad arguments");
    out[0] = h->n0();
    out[1] = h->n0() > 0 ? h->num_layers : 0;
    out[2] = h->hg.enter_level;
    out[3] = h->capacity;
    out[4] = h->dim;
    out[5] = h->M;
    out[6] = h->efc;
    out[7] = h->metric;
    out[8] = h->dtype;
    out[9] = (int64_t)h->dev_bytes;
    out[10] = 2 * h->M;
    out[11] = h->hg.L[0].ent;
    return PK_OK;
}

static int pk_index_layer_impl(const pk_index *hc, int level, int64_t *n, int64_t *layer_capacity, int64_t *cap, int32_t *ext,
                   int16_t *degree, int16_t *heuristic, uint8_t *has_vector, int32_t *adj, float *dist) {
    pk_index *h = const_cast<pk_index *>(hc);
    if (!h || !n || !layer_capacity || !cap) return fail(PK_ERR_ARG, "bad arguments");
    if (level < 0 || level >= h->num_layers) return fail(PK_ERR_ARG, "no such layer");
    PK_CUDA(cudaStreamSynchronize(h->stream));
    const pk::DevLayer &L = h->hg.L[level];
    *n = L.n;
    *layer_capacity = std::max(L.lcap, L.n);
    *cap = L.cap;
    const int64_t cnt = *layer_capacity * L.cap;
    if (ext) PK_CUDA(cudaMemcpy(ext, L.ext, 4 * L.n, cudaMemcpyDeviceToHost));
    std::vector<int32_t> tmp(L.n);
    if (degree) {
        PK_CUDA(cudaMemcpy(tmp.data(), L.deg, 4 * L.n, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < L.n; i++) degree[i] = (int16_t)tmp[i];
    }
    if (heuristic) {
        PK_CUDA(cudaMemcpy(tmp.data(), L.heu, 4 * L.n, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < L.n; i++) heuristic[i] = (int16_t)tmp[i];
    }
    if (has_vector) {
        if (level == 0) {
            for (int64_t i = 0; i < L.n; i++) has_vector[i] = 1;
        } else {
            PK_CUDA(cudaMemcpy(tmp.data(), L.vrow, 4 * L.n, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < L.n; i++) has_vector[i] = tmp[i] >= 0;
        }
    }
    if (adj) PK_CUDA(cudaMemcpy(adj, L.adj, 4 * cnt, cudaMemcpyDeviceToHost));
    if (dist) PK_CUDA(cudaMemcpy(dist, L.dist, 4 * cnt, cudaMemcpyDeviceToHost));
    return PK_OK;
}

}  // namespace

namespace {

static int pk_index_prepare_fast_impl(pk_index *h, int traversal) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (traversal != PK_TRAVERSAL_F16 && traversal != PK_TRAVERSAL_FP8)
        return fail(PK_ERR_ARG, "traversal must be PK_TRAVERSAL_F16 or PK_TRAVERSAL_FP8");
    return build_traversal(h, traversal == PK_TRAVERSAL_F16 ? pk::kTravF16 : pk::kTravE4M3);
}

// Times the walk + re-rank of this batch (uniform k and ef) for a grid of
// launch shapes (rows per fetch batch, visited-filter size, warps per block)
// and returns the fastest.  The result lists are the same for every shape;
// only the work and its overlap change, so the choice is by time alone.  The
// shapes are tried as the shape of ef's list-width class, which is left as it
// was.  reps = timed runs per shape (after one warm-up run); a shape's time is
// the fastest of them (the least disturbed by whatever else shares the GPU).
int tune_shape(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t expand, int reps,
               cudaStream_t s, int &brb, int &bh, int &bw, float &best, int &bvt) {
    PK_TRY(ensure_buf(h, &h->d_fids, h->fids_n, nq * k));
    PK_TRY(ensure_buf(h, &h->d_fdists, h->fdists_n, nq * k));
    const int cls = pk::slot_class(ef);
    const int keep_rb = h->cls_rb[cls], keep_h = h->cls_hlog2[cls], keep_w = h->cls_wpb[cls];
    const int keep_vt = h->cls_vt[cls];
    bvt = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PK_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PK_ERR_CUDA, "cudaEventCreate failed");
    }
    best = -1.f;
    brb = bh = bw = 0;
    int rc = PK_OK;
    // times one shape; false if it does not fit or a launch failed (rc set)
    auto time_shape = [&](int rb, int hl, int wp) -> bool {
        h->cls_rb[cls] = rb;
        h->cls_hlog2[cls] = hl;
        h->cls_wpb[cls] = wp;
        WalkShape ws;
        if (walk_shape(h, ws, cls) != PK_OK || ws.wpb != wp) return false;
        float ms = 0.f;
        for (int rep = 0; rep <= reps && rc == PK_OK; rep++) {
            if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(PK_ERR_CUDA, "cudaEventRecord failed");
            if (rc == PK_OK)
                rc = run_search_fast(h, h->fctx, queries, false, nq, k, ef, nullptr, nullptr, k, h->d_fids,
                                     h->d_fdists, nullptr, expand, s);
            if (rc == PK_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
                rc = fail(PK_ERR_CUDA, "tuning launch failed");
            float t = 0.f;
            if (rc == PK_OK && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
                rc = fail(PK_ERR_CUDA, "cudaEventElapsedTime failed");
            if (rep > 0) ms = rep == 1 ? t : std::min(ms, t);
        }
        // a walk that stopped early on a fetch timeout must not look fast
        if (rc == PK_OK) rc = fast_status(h, h->fctx, s);
        if (rc != PK_OK) return false;
        if (best < 0.f || ms < best) {
            best = ms;
            brb = rb;
            bh = hl;
            bw = wp;
        }
        return true;
    };
    // stage 1: visited-table size and warps per block at 16 and at 32 rows
    // per batch (the table trades re-fetched rows against occupancy, more so
    // as ef grows, and the staged rows share the same shared memory: large
    // rows at 32 per batch leave room only for small tables); stage 2: rows
    // per batch at the best triple
    // (with the visited tables in L2 behind it, small shared-memory tables
    // that leave room for more warps are often the fastest)
    const int hls[] = {6, 8, 9, 10, 11, 12, 13};
    h->cls_vt[cls] = 0;
    const int wps[] = {1, 2, 4};
    const int rbs1[] = {16, 32};
    for (int rb : rbs1)
        for (int hl : hls)
            for (int wp : wps)
                if (rc == PK_OK) time_shape(rb, hl, wp);
    const int r1 = brb, h1 = bh, w1 = bw;
    const int rbs[] = {8, 16, 24, 32, 48, 64};
    for (int rb : rbs)
        if (rc == PK_OK && best >= 0.f && rb != r1) time_shape(rb, h1, w1);
    // stage 3: the best shape without the visited tables in L2 (narrow lists
    // meet few nodes again, and the tables' round trip can cost more than
    // the rows they spare)
    if (rc == PK_OK && best >= 0.f && h->fast_vt >= 0) {
        const float with = best;
        h->cls_vt[cls] = -1;
        time_shape(brb, bh, bw);
        if (best < with) bvt = -1;
    }
    h->cls_vt[cls] = keep_vt;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->cls_rb[cls] = keep_rb;
    h->cls_hlog2[cls] = keep_h;
    h->cls_wpb[cls] = keep_w;
    if (rc == PK_OK) rc = fast_status(h, h->fctx, s);
    if (rc != PK_OK) return rc;
    if (best < 0.f) return fail(PK_ERR_ARG, "no launch shape fits this index");
    return PK_OK;
}

static int tune_check(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef) {
    if (!h || !queries || nq < 1 || k < 1 || ef < k) return fail(PK_ERR_ARG, "bad arguments");
    if (ef > pk::kFastMaxEf) return fail(PK_ERR_ARG, "ef too large for the fast path");
    if (h->trav == 0) return fail(PK_ERR_STATE, "pk_index_prepare_fast has not been called");
    if (h->n0() == 0) return fail(PK_ERR_STATE, "the index is empty");
    return PK_OK;
}

// Tunes at this batch's ef and keeps the winner as the handle's shape for
// every list width (the per-class shapes are cleared).
static int pk_index_tune_fast_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                                   int32_t expand, int32_t *out_shape, float *out_ms, void *stream) {
    PK_TRY(tune_check(h, queries, nq, k, ef));
    int rb = 0, hl = 0, wp = 0, vt = 0;
    float ms = 0.f;
    PK_TRY(tune_shape(h, queries, nq, k, ef, expand, 2, static_cast<cudaStream_t>(stream), rb, hl, wp, ms, vt));
    h->fast_rb = rb;
    h->fast_hlog2 = hl;
    h->fast_wpb = wp;
    // the tables' choice holds for the tuned ef's width only (wider lists
    // meet many more nodes again)
    for (int c = 0; c < pk::kSlotClasses; c++) {
        h->cls_rb[c] = h->cls_hlog2[c] = h->cls_wpb[c] = 0;
        h->cls_vt[c] = c == pk::slot_class(ef) ? vt : 0;
    }
    if (out_shape) {
        out_shape[0] = rb;
        out_shape[1] = hl;
        out_shape[2] = wp;
    }
    if (out_ms) *out_ms = ms;
    return PK_OK;
}

// Tunes every list-width class up to max_ef on this batch (each at the widest
// ef of its class, k = min(k, that ef)) and keeps one shape per class, for
// batches whose queries carry their own ef.
static int pk_index_tune_fast_classes_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t max_ef,
                                           int32_t expand, int32_t *out_shapes, float *out_ms, void *stream) {
    PK_TRY(tune_check(h, queries, nq, std::min(k, max_ef), max_ef));
    for (int c = 0; c < pk::kSlotClasses; c++) {
        if (out_shapes) out_shapes[3 * c] = out_shapes[3 * c + 1] = out_shapes[3 * c + 2] = 0;
        if (out_ms) out_ms[c] = 0.f;
        const int lo = c == 0 ? 1 : 32 * pk::slot_class_width(c - 1) + 1;
        if (lo > max_ef) continue;
        const int ef = std::min(32 * pk::slot_class_width(c), std::min(max_ef, pk::kFastMaxEf));
        int rb = 0, hl = 0, wp = 0, vt = 0;
        float ms = 0.f;
        PK_TRY(tune_shape(h, queries, nq, std::min(k, ef), ef, expand, 2, static_cast<cudaStream_t>(stream), rb, hl,
                          wp, ms, vt));
        h->cls_vt[c] = vt;
        h->cls_rb[c] = rb;
        h->cls_hlog2[c] = hl;
        h->cls_wpb[c] = wp;
        if (out_shapes) {
            out_shapes[3 * c] = rb;
            out_shapes[3 * c + 1] = hl;
            out_shapes[3 * c + 2] = wp;
        }
        if (out_ms) out_ms[c] = ms;
    }
    return PK_OK;
}

static int pk_index_search_fast_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                                     const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride,
                                     int32_t *out_ids, float *out_dists, int32_t *counters, int32_t expand,
                                     void *stream) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists) && nq > 0)) return fail(PK_ERR_ARG, "bad arguments");
    if (k < 1 || ef < 1 || out_stride < k) return fail(PK_ERR_ARG, "need k >= 1, ef >= 1, out_stride >= k");
    if (nq == 0) return PK_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (h->n0() == 0) {
        PK_CUDA(fill_i32(out_ids, nq * out_stride, -1, s));
        PK_CUDA(fill_f32(out_dists, nq * out_stride, FLT_MAX, s));
        return PK_OK;
    }
    return run_search_fast(h, h->fctx, queries, false, nq, k, ef, k_per_query, ef_per_query, out_stride, out_ids,
                           out_dists, counters, expand, s);
}

static int pk_index_search_fast_host_impl(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                                          int32_t *out_ids, float *out_dists, int32_t expand) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists) && nq > 0)) return fail(PK_ERR_ARG, "bad arguments");
    if (k < 1 || ef < 1) return fail(PK_ERR_ARG, "k and ef must be >= 1");
    if (nq == 0) return PK_OK;
    if (h->n0() == 0) {
        for (int64_t i = 0; i < nq * k; i++) {
            out_ids[i] = -1;
            out_dists[i] = FLT_MAX;
        }
        return PK_OK;
    }
    cudaStream_t s = h->stream;
    PK_TRY(ensure_buf(h, &h->d_fids, h->fids_n, nq * k));
    PK_TRY(ensure_buf(h, &h->d_fdists, h->fdists_n, nq * k));
    PK_TRY(run_search_fast(h, h->fctx, queries, true, nq, k, ef, nullptr, nullptr, k, h->d_fids, h->d_fdists,
                           nullptr, expand, s));
    PK_CUDA(cudaMemcpyAsync(out_ids, h->d_fids, sizeof(int32_t) * nq * k, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaMemcpyAsync(out_dists, h->d_fdists, sizeof(float) * nq * k, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    return fast_status(h, h->fctx, s);
}

static int pk_index_search_fast_host_var_impl(pk_index *h, const void *queries, int64_t nq,
                                              const int32_t *k_per_query, const int32_t *ef_per_query,
                                              int32_t out_stride, int32_t *out_ids, float *out_dists,
                                              int32_t expand) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists || !k_per_query || !ef_per_query) && nq > 0))
        return fail(PK_ERR_ARG, "bad arguments");
    if (nq == 0) return PK_OK;
    int32_t kmax = 0, efmax = 0;
    for (int64_t i = 0; i < nq; i++) {
        if (k_per_query[i] < 1 || ef_per_query[i] < 1) return fail(PK_ERR_ARG, "every k and ef must be >= 1");
        kmax = std::max(kmax, k_per_query[i]);
        efmax = std::max(efmax, ef_per_query[i]);
    }
    if (out_stride < kmax) return fail(PK_ERR_ARG, "out_stride below the largest k");
    if (h->n0() == 0) {
        for (int64_t i = 0; i < nq * out_stride; i++) {
            out_ids[i] = -1;
            out_dists[i] = FLT_MAX;
        }
        return PK_OK;
    }
    cudaStream_t s = h->stream;
    PK_TRY(ensure_buf(h, &h->d_fids, h->fids_n, nq * out_stride));
    PK_TRY(ensure_buf(h, &h->d_fdists, h->fdists_n, nq * out_stride));
    PK_TRY(ensure_buf(h, &h->d_karr, h->karr_n, nq));
    PK_TRY(ensure_buf(h, &h->d_efarr, h->efarr_n, nq));
    PK_CUDA(cudaMemcpyAsync(h->d_karr, k_per_query, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaMemcpyAsync(h->d_efarr, ef_per_query, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
    PK_CUDA(fill_i32(h->d_fids, nq * out_stride, -1, s));
    PK_CUDA(fill_f32(h->d_fdists, nq * out_stride, FLT_MAX, s));
    PK_TRY(run_search_fast(h, h->fctx, queries, true, nq, kmax, efmax, h->d_karr, h->d_efarr, out_stride, h->d_fids,
                           h->d_fdists, nullptr, expand, s));
    PK_CUDA(cudaMemcpyAsync(out_ids, h->d_fids, sizeof(int32_t) * nq * out_stride, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaMemcpyAsync(out_dists, h->d_fdists, sizeof(float) * nq * out_stride, cudaMemcpyDeviceToHost, s));
    PK_CUDA(cudaStreamSynchronize(s));
    return fast_status(h, h->fctx, s);
}

}  // namespace

// ---------------------------------------------------------------- server ----
// Continuous batching over the fast search.  A worker thread owns `slots`
// execution streams.  Requests (each a group of queries with one k and ef)
// wait in a FIFO; whenever a stream is free, the worker packs queued
// requests into a batch of up to max_batch queries as long as the batch's
// device buffers (queries, per-query k and ef, results, the walk's scratch,
// all sized from the batch's own nq, largest k and largest ef) fit the free
// part of the server's device-memory arena, carves them out of it, copies the
// batch in, launches the search with per-query k and ef, copies the results
// out and records an event.  Batches in flight overlap on the device; a
// finished batch returns its memory and its stream.  So the number of
// queries in flight follows the memory their k and ef need: many small
// requests run side by side, a large one waits until enough is free (counted
// as deferred for memory), and one larger than the whole arena is refused at
// submission.  A batch that has not completed within the watchdog period
// fails its requests with PK_ERR_TIMEOUT.
namespace {

using Clock = std::chrono::steady_clock;

struct SrvRequest {
    int64_t ticket = 0;
    int32_t nq = 0, k = 0, ef = 0;
    std::vector<uint8_t> q;
    std::vector<int32_t> ids;
    std::vector<float> dists;
    Clock::time_point t_submit, t_done;
    int status = 0;
    bool done = false;
    bool deferred = false;  // once found waiting for device memory
};

// Where a batch's device buffers sit in the server's arena (byte offsets).
struct SrvLayout {
    size_t q = 0, k = 0, ef = 0, ids = 0, d = 0, work = 0, cand = 0, lists = 0, fq = 0, tq = 0, qn = 0, total = 0;
    int64_t cand_n = 0, lists_n = 0, fq_n = 0, tq_n = 0, qn_n = 0;
};

struct SrvSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    FastCtx ctx;                   // points into the arena while a batch runs
    uint8_t *h_q = nullptr;
    int32_t *h_k = nullptr, *h_ef = nullptr, *h_ids = nullptr;
    float *h_d = nullptr;
    int32_t *h_status = nullptr;   // the walk's status, copied back with the results
    bool busy = false;
    std::vector<std::shared_ptr<SrvRequest>> reqs;
    std::vector<int32_t> offs;
    int32_t nq = 0, stride = 0;
    size_t chunk_off = 0, chunk_bytes = 0;  // the batch's arena chunk
    Clock::time_point t_launch;
    // the walk's visited tables in L2 for this slot's batches (outside the
    // arena; null = the walk runs with its shared-memory table alone)
    uint8_t *vt = nullptr;
    size_t vt_bytes = 0;
};

}  // namespace

struct pk_server {
    pk_index *h = nullptr;
    int32_t max_batch = 0, max_k = 0, max_ef = 0, expand = 1;
    double watchdog_s = 30.0;
    std::vector<SrvSlot> slots;
    // device memory: one arena, carved per batch (first fit); admission waits
    // while the queue's next request does not fit the free space
    uint8_t *arena = nullptr;
    size_t arena_bytes = 0, in_use = 0, peak_in_use = 0;
    std::vector<std::pair<size_t, size_t>> free_list;  // (offset, bytes), sorted by offset
    int64_t deferred_for_memory = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<SrvRequest>> queue;
    std::unordered_map<int64_t, std::shared_ptr<SrvRequest>> table;
    int64_t next_ticket = 1;
    bool stop = false;
    int error = 0;
    std::thread worker;
    // statistics
    int64_t batches = 0, queries = 0, max_inflight = 0;
};

namespace {

// Device bytes of a batch of nq queries whose largest k and ef are kmax and
// efmax: the server's copies of queries, k, ef and results, and what the
// fast search needs for them (pk_index_search_fast's scratch).
SrvLayout srv_layout(const pk_index *h, int64_t nq, int32_t kmax, int32_t efmax) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    SrvLayout L;
    const size_t w = (size_t)(h->dim * h->esz);
    const int64_t cs = 32 * pk::list_slots(std::min(efmax, pk::kFastMaxEf));
    const int64_t tq_rb = pk::trav_query_bytes(h->trav, h->trav_data_bytes);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += al(std::max<size_t>(bytes, 16));
        return at;
    };
    L.q = take(nq * w);
    L.k = take(4 * nq);
    L.ef = take(4 * nq);
    L.ids = take(4 * nq * kmax);
    L.d = take(4 * nq * kmax);
    L.work = take(4 * (size_t)kWorkInts);
    L.cand_n = nq * cs;
    L.cand = take(4 * L.cand_n);
    L.lists_n = nq * pk::kSlotClasses;
    L.lists = take(4 * L.lists_n);
    L.fq_n = w != (size_t)h->row_bytes ? nq * h->row_bytes : 0;
    L.fq = take((size_t)L.fq_n);
    L.tq_n = nq * tq_rb;
    L.tq = take((size_t)L.tq_n);
    L.qn_n = nq;
    L.qn = take(4 * nq);
    L.total = off;
    return L;
}

// First fit in the arena (caller holds S->mu); false if nothing fits.
bool arena_take(pk_server *S, size_t bytes, size_t &off) {
    for (size_t i = 0; i < S->free_list.size(); i++) {
        auto &f = S->free_list[i];
        if (f.second < bytes) continue;
        off = f.first;
        f.first += bytes;
        f.second -= bytes;
        if (f.second == 0) S->free_list.erase(S->free_list.begin() + (long)i);
        S->in_use += bytes;
        S->peak_in_use = std::max(S->peak_in_use, S->in_use);
        return true;
    }
    return false;
}

size_t arena_largest(const pk_server *S) {
    size_t m = 0;
    for (const auto &f : S->free_list) m = std::max(m, f.second);
    return m;
}

void arena_give(pk_server *S, size_t off, size_t bytes) {
    if (bytes == 0) return;
    auto &fl = S->free_list;
    auto it = std::lower_bound(fl.begin(), fl.end(), std::make_pair(off, (size_t)0));
    it = fl.insert(it, {off, bytes});
    // merge with the neighbours
    if (it + 1 != fl.end() && it->first + it->second == (it + 1)->first) {
        it->second += (it + 1)->second;
        fl.erase(it + 1);
    }
    if (it != fl.begin() && (it - 1)->first + (it - 1)->second == it->first) {
        (it - 1)->second += it->second;
        fl.erase(it);
    }
    S->in_use -= std::min(S->in_use, bytes);
}

void srv_fail_all(pk_server *S, int code) {
    // caller holds S->mu
    S->error = code;
    for (auto &kv : S->table)
        if (!kv.second->done) {
            kv.second->status = code;
            kv.second->done = true;
            kv.second->t_done = Clock::now();
        }
    S->cv_done.notify_all();
}

void srv_finish_slot(pk_server *S, SrvSlot &sl) {
    // caller holds S->mu
    arena_give(S, sl.chunk_off, sl.chunk_bytes);
    sl.chunk_bytes = 0;
    sl.reqs.clear();
    sl.offs.clear();
    sl.busy = false;
}

void srv_loop(pk_server *S) {
    pk_index *h = S->h;
    cudaSetDevice(h->device);
    const size_t w = (size_t)(h->dim * h->esz);
    for (;;) {
        bool did = false;
        // 1. completions
        for (SrvSlot &sl : S->slots) {
            if (!sl.busy) continue;
            // the watchdog looks first: a batch whose completion the host has
            // not observed within the period fails, finished or not
            double wd;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                wd = S->watchdog_s;
            }
            if (std::chrono::duration<double>(Clock::now() - sl.t_launch).count() > wd) {
                std::lock_guard<std::mutex> lk(S->mu);
                for (auto &r : sl.reqs) {
                    r->status = PK_ERR_TIMEOUT;
                    r->done = true;
                    r->t_done = Clock::now();
                }
                // the batch may still be running: its memory stays taken
                sl.chunk_bytes = 0;
                sl.reqs.clear();
                sl.offs.clear();
                srv_fail_all(S, PK_ERR_TIMEOUT);
                sl.busy = false;
                continue;
            }
            const cudaError_t e = cudaEventQuery(sl.ev);
            if (e == cudaErrorNotReady) continue;
            const auto now = Clock::now();
            const int code = e != cudaSuccess ? PK_ERR_CUDA : *sl.h_status != 0 ? PK_ERR_TIMEOUT : PK_OK;
            std::lock_guard<std::mutex> lk(S->mu);
            for (size_t i = 0; i < sl.reqs.size(); i++) {
                SrvRequest &r = *sl.reqs[i];
                if (code != PK_OK) {
                    r.status = code;
                } else {
                    r.ids.resize((size_t)r.nq * r.k);
                    r.dists.resize((size_t)r.nq * r.k);
                    for (int32_t j = 0; j < r.nq; j++) {
                        const int64_t row = sl.offs[i] + j;
                        std::memcpy(r.ids.data() + (size_t)j * r.k, sl.h_ids + row * sl.stride, 4 * (size_t)r.k);
                        std::memcpy(r.dists.data() + (size_t)j * r.k, sl.h_d + row * sl.stride, 4 * (size_t)r.k);
                    }
                }
                r.done = true;
                r.t_done = now;
            }
            if (code != PK_OK) srv_fail_all(S, code);
            srv_finish_slot(S, sl);
            did = true;
            S->cv_done.notify_all();
        }
        // 2. admissions into free streams, as far as the arena has room
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->stop) break;
            int inflight = 0;
            for (SrvSlot &sl : S->slots) inflight += sl.busy;
            for (SrvSlot &sl : S->slots) {
                if (sl.busy || S->queue.empty() || S->error) continue;
                const size_t room = arena_largest(S);
                int32_t nq = 0, kmax = 0, efmax = 0;
                size_t need = 0, count = 0;
                for (const auto &r : S->queue) {
                    if (nq + r->nq > S->max_batch) break;
                    const SrvLayout L = srv_layout(h, nq + r->nq, std::max(kmax, r->k), std::max(efmax, r->ef));
                    if (L.total > room) break;
                    nq += r->nq;
                    kmax = std::max(kmax, r->k);
                    efmax = std::max(efmax, r->ef);
                    need = L.total;
                    count++;
                }
                if (count == 0) {
                    // the head waits for device memory, not for a stream
                    if (!S->queue.front()->deferred) {
                        S->queue.front()->deferred = true;
                        S->deferred_for_memory++;
                    }
                    break;
                }
                size_t off = 0;
                if (!arena_take(S, need, off)) break;
                const SrvLayout L = srv_layout(h, nq, kmax, efmax);
                sl.chunk_off = off;
                sl.chunk_bytes = need;
                sl.stride = kmax;
                int32_t at = 0;
                for (size_t i = 0; i < count; i++) {
                    auto r = S->queue.front();
                    S->queue.pop_front();
                    sl.offs.push_back(at);
                    std::memcpy(sl.h_q + (size_t)at * w, r->q.data(), (size_t)r->nq * w);
                    for (int32_t j = 0; j < r->nq; j++) {
                        sl.h_k[at + j] = r->k;
                        sl.h_ef[at + j] = r->ef;
                    }
                    at += r->nq;
                    sl.reqs.push_back(std::move(r));
                }
                sl.nq = nq;
                uint8_t *base = S->arena + off;
                uint8_t *d_q = base + L.q;
                int32_t *d_k = reinterpret_cast<int32_t *>(base + L.k);
                int32_t *d_ef = reinterpret_cast<int32_t *>(base + L.ef);
                int32_t *d_ids = reinterpret_cast<int32_t *>(base + L.ids);
                float *d_d = reinterpret_cast<float *>(base + L.d);
                // the search's scratch, in the chunk (sized so that nothing grows)
                sl.ctx.d_work = reinterpret_cast<int32_t *>(base + L.work);
                sl.ctx.work_n = kWorkInts;
                sl.ctx.d_cand = reinterpret_cast<int32_t *>(base + L.cand);
                sl.ctx.cand_n = L.cand_n;
                sl.ctx.d_lists = reinterpret_cast<int32_t *>(base + L.lists);
                sl.ctx.lists_n = L.lists_n;
                sl.ctx.d_fq = L.fq_n ? base + L.fq : nullptr;
                sl.ctx.fq_n = L.fq_n;
                sl.ctx.d_tq = base + L.tq;
                sl.ctx.tq_n = L.tq_n;
                sl.ctx.d_qn = reinterpret_cast<float *>(base + L.qn);
                sl.ctx.qn_n = L.qn_n;
                lk.unlock();
                int rc = PK_OK;
                if (cudaMemcpyAsync(d_q, sl.h_q, (size_t)nq * w, cudaMemcpyHostToDevice, sl.stream) != cudaSuccess ||
                    cudaMemcpyAsync(d_k, sl.h_k, 4 * (size_t)nq, cudaMemcpyHostToDevice, sl.stream) != cudaSuccess ||
                    cudaMemcpyAsync(d_ef, sl.h_ef, 4 * (size_t)nq, cudaMemcpyHostToDevice, sl.stream) != cudaSuccess)
                    rc = PK_ERR_CUDA;
                if (rc == PK_OK)
                    rc = run_search_fast(h, sl.ctx, d_q, false, nq, kmax, efmax, d_k, d_ef, kmax, d_ids, d_d, nullptr,
                                         S->expand, sl.stream);
                if (rc == PK_OK &&
                    (cudaMemcpyAsync(sl.h_ids, d_ids, 4 * (size_t)nq * kmax, cudaMemcpyDeviceToHost, sl.stream) !=
                         cudaSuccess ||
                     cudaMemcpyAsync(sl.h_d, d_d, 4 * (size_t)nq * kmax, cudaMemcpyDeviceToHost, sl.stream) !=
                         cudaSuccess ||
                     cudaMemcpyAsync(sl.h_status, sl.ctx.d_work + kWorkStatus, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                     sl.stream) != cudaSuccess ||
                     cudaEventRecord(sl.ev, sl.stream) != cudaSuccess))
                    rc = PK_ERR_CUDA;
                lk.lock();
                if (rc != PK_OK) {
                    for (auto &r : sl.reqs) {
                        r->status = rc;
                        r->done = true;
                        r->t_done = Clock::now();
                    }
                    cudaStreamSynchronize(sl.stream);
                    srv_finish_slot(S, sl);
                    srv_fail_all(S, rc);
                    continue;
                }
                sl.busy = true;
                sl.t_launch = Clock::now();
                S->batches++;
                S->queries += nq;
                inflight++;
                S->max_inflight = std::max<int64_t>(S->max_inflight, inflight);
                did = true;
            }
            bool any_busy = false;
            for (SrvSlot &sl : S->slots) any_busy |= sl.busy;
            if (!did) {
                if (any_busy) {
                    lk.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(20));
                } else {
                    S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
                }
            }
        }
    }
}

void srv_free(pk_server *S) {
    for (SrvSlot &sl : S->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        // the slot's scratch lives in the arena: only its streams and events
        // are its own
        release_ctx_sync(sl.ctx);
        cudaFreeHost(sl.h_q);
        cudaFreeHost(sl.h_k);
        cudaFreeHost(sl.h_ef);
        cudaFreeHost(sl.h_ids);
        cudaFreeHost(sl.h_d);
        cudaFreeHost(sl.h_status);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.stream) cudaStreamDestroy(sl.stream);
        dfree(S->h, sl.vt, sl.vt_bytes);
    }
    if (S->arena) dfree(S->h, S->arena, S->arena_bytes);
    delete S;
}

int srv_create(pk_server **out, pk_index *h, int traversal, int nslots, int32_t max_batch, int32_t max_k,
               int32_t max_ef, int32_t expand, int64_t device_bytes) {
    if (!out || !h || nslots < 1 || nslots > 64 || max_batch < 1 || max_k < 1 || max_ef < max_k ||
        max_ef > pk::kFastMaxEf || device_bytes < 0)
        return fail(PK_ERR_ARG, "bad server arguments (need 1 <= slots <= 64, max_batch >= 1, "
                                "1 <= max_k <= max_ef <= 1024, device_bytes >= 0)");
    if (h->n0() == 0) return fail(PK_ERR_STATE, "the index is empty");
    if (h->trav != (traversal == PK_TRAVERSAL_F16 ? pk::kTravF16 : pk::kTravE4M3)) {
        int rc = pk_index_prepare_fast_impl(h, traversal);
        if (rc != PK_OK) return rc;
    }
    PK_TRY(refresh_traversal(h));
    auto *S = new (std::nothrow) pk_server();
    if (!S) return fail(PK_ERR_OOM, "host allocation failed");
    S->h = h;
    S->max_batch = max_batch;
    S->max_k = max_k;
    S->max_ef = max_ef;
    S->expand = std::max(1, expand);
    // the arena: as asked, else every stream's full batch at the largest k
    // and ef, but at most half of the device memory free now
    size_t bytes = (size_t)device_bytes;
    if (bytes == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            delete S;
            return fail(PK_ERR_CUDA, "cudaMemGetInfo failed");
        }
        bytes = std::min(srv_layout(h, max_batch, max_k, max_ef).total * (size_t)nslots, fr / 2);
    }
    bytes = (bytes + 255) & ~(size_t)255;
    if (dalloc(h, (void **)&S->arena, bytes) != PK_OK) {
        delete S;
        return fail(PK_ERR_OOM, "the server's device memory (" + std::to_string(bytes) + " bytes) is not free");
    }
    S->arena_bytes = bytes;
    S->free_list.push_back({0, bytes});
    S->slots.resize(nslots);
    const size_t w = (size_t)(h->dim * h->esz);
    for (SrvSlot &sl : S->slots) {
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_q, (size_t)max_batch * w) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_k, 4 * (size_t)max_batch) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_ef, 4 * (size_t)max_batch) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_ids, 4 * (size_t)max_batch * max_k) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_d, 4 * (size_t)max_batch * max_k) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_status, sizeof(int32_t)) != cudaSuccess) {
            cudaGetLastError();
            srv_free(S);
            return fail(PK_ERR_OOM, "server host buffers could not be allocated");
        }
    }
    // with the default arena, each slot also gets the walk's visited tables
    // for a full batch at the largest ef (a batch whose launch shapes need
    // more, or a slot whose tables could not be allocated, walks with the
    // shared-memory table alone: the same results); an explicit device_bytes
    // is all the device memory the server takes
    if (device_bytes == 0) {
        ClsPlan plan[pk::kSlotClasses];
        int64_t vt_total = 0;
        if (walk_plan(h, max_batch, pk::list_slots(max_ef), true, S->expand, plan, vt_total) == PK_OK &&
            vt_total > 0) {
            for (SrvSlot &sl : S->slots) {
                if (dalloc(h, (void **)&sl.vt, (size_t)vt_total) != PK_OK) break;
                sl.vt_bytes = (size_t)vt_total;
                sl.ctx.d_vt = sl.vt;
                sl.ctx.vt_n = vt_total;
            }
        }
        cudaGetLastError();
    }
    for (SrvSlot &sl : S->slots) sl.ctx.vt_fixed = true;
    S->worker = std::thread(srv_loop, S);
    *out = S;
    return PK_OK;
}

int srv_submit(pk_server *S, const void *queries, int32_t nq, int32_t k, int32_t ef, int64_t *ticket) {
    if (!S || !queries || nq < 1 || !ticket) return fail(PK_ERR_ARG, "bad arguments");
    if (nq > S->max_batch) return fail(PK_ERR_ARG, "request larger than the server's batch capacity");
    if (k < 1 || k > S->max_k || ef < k || ef > S->max_ef) return fail(PK_ERR_ARG, "k or ef outside the server's limits");
    const size_t need = srv_layout(S->h, nq, k, ef).total;
    if (need > S->arena_bytes)
        return fail(PK_ERR_CAPACITY, "request needs " + std::to_string(need) + " bytes of device memory; the server holds " +
                                         std::to_string(S->arena_bytes));
    auto r = std::make_shared<SrvRequest>();
    r->nq = nq;
    r->k = k;
    r->ef = ef;
    const size_t bytes = (size_t)nq * (size_t)(S->h->dim * S->h->esz);
    r->q.assign(static_cast<const uint8_t *>(queries), static_cast<const uint8_t *>(queries) + bytes);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->error) return fail(S->error, "the server has failed");
    r->ticket = S->next_ticket++;
    *ticket = r->ticket;
    S->table[r->ticket] = r;
    S->queue.push_back(std::move(r));
    S->cv_work.notify_one();
    return PK_OK;
}

int srv_wait(pk_server *S, int64_t ticket, int32_t *out_ids, float *out_dists, double *latency_ms,
             int32_t timeout_ms) {
    if (!S) return fail(PK_ERR_ARG, "NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->table.find(ticket);
    if (it == S->table.end()) return fail(PK_ERR_ARG, "unknown ticket");
    std::shared_ptr<SrvRequest> r = it->second;
    const auto pred = [&] { return r->done; };
    if (timeout_ms < 0) {
        S->cv_done.wait(lk, pred);
    } else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        return fail(PK_ERR_TIMEOUT, "request not finished within the timeout");
    }
    S->table.erase(ticket);
    if (r->status != PK_OK) return fail(r->status, "request failed");
    if (out_ids) std::memcpy(out_ids, r->ids.data(), 4 * r->ids.size());
    if (out_dists) std::memcpy(out_dists, r->dists.data(), 4 * r->dists.size());
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return PK_OK;
}

}  // namespace

namespace pk {
// Read-only view of a handle for entry points defined in other files.
IndexView index_view(const pk_index *h) {
    IndexView v{};
    v.device = h->device;
    v.num_sms = h->num_sms;
    v.dtype = h->dtype;
    v.dim = h->dim;
    v.esz = h->esz;
    v.row_bytes = h->row_bytes;
    v.lc = h->lc;
    v.dg = h->dg;
    v.ext0 = h->hg.L[0].ext;
    v.n0 = h->n0();
    v.lcap0 = h->hg.L[0].lcap;
    return v;
}
void set_error(const char *msg) { g_last_error = msg; }
}  // namespace pk

extern "C" {

const char *pk_last_error(void) { return g_last_error.c_str(); }

int pk_version(void) { return 100; }

int pk_index_create(pk_index **out, int metric, int dtype, int64_t dim, int64_t M, int64_t ef_construction) {
    try {
        return pk_index_create_impl(out, metric, dtype, dim, M, ef_construction);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_create: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_create: unknown exception");
    }
}

int pk_index_destroy(pk_index *h) {
    try {
        return pk_index_destroy_impl(h);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_destroy: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_destroy: unknown exception");
    }
}

int pk_index_set_seed(pk_index *h, uint64_t seed) {
    try {
        return pk_index_set_seed_impl(h, seed);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_set_seed: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_set_seed: unknown exception");
    }
}

int pk_index_set_levels(pk_index *h, const uint8_t *levels, int64_t n) {
    try {
        return pk_index_set_levels_impl(h, levels, n);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_set_levels: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_set_levels: unknown exception");
    }
}

int pk_index_build(pk_index *h, const void *data, int64_t n, const int32_t *ext_ids, int32_t max_batch) {
    try {
        return pk_index_build_impl(h, data, n, ext_ids, max_batch);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_build: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_build: unknown exception");
    }
}

int pk_index_add(pk_index *h, const void *rows, int64_t n, const int32_t *ext_ids, int32_t max_batch) {
    try {
        return pk_index_add_impl(h, rows, n, ext_ids, max_batch);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_add: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_add: unknown exception");
    }
}

int pk_index_search(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                    float *out_dists) {
    try {
        return pk_index_search_impl(h, queries, nq, k, ef, out_ids, out_dists);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_search: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search: unknown exception");
    }
}

int pk_index_search_device(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                           const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride,
                           int32_t *out_ids, float *out_dists, int32_t *counters, void *stream) {
    try {
        return pk_index_search_device_impl(h, queries, nq, k, ef, k_per_query, ef_per_query, out_stride, out_ids, out_dists, counters, stream);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_search_device: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_device: unknown exception");
    }
}

int pk_index_save(const pk_index *hc, const char *path) {
    try {
        return pk_index_save_impl(hc, path);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_save: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_save: unknown exception");
    }
}

int pk_index_load(pk_index **out, const char *path) {
    try {
        return pk_index_load_impl(out, path);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_load: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_load: unknown exception");
    }
}

int pk_index_info(const pk_index *h, int64_t *out) {
    try {
        return pk_index_info_impl(h, out);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_info: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_info: unknown exception");
    }
}

int pk_index_layer(const pk_index *hc, int level, int64_t *n, int64_t *layer_capacity, int64_t *cap, int32_t *ext,
                   int16_t *degree, int16_t *heuristic, uint8_t *has_vector, int32_t *adj, float *dist) {
    try {
        return pk_index_layer_impl(hc, level, n, layer_capacity, cap, ext, degree, heuristic, has_vector, adj, dist);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PK_ERR_STATE, std::string("pk_index_layer: ") + e.what());
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_layer: unknown exception");
    }
}

int pk_index_prepare_fast(pk_index *h, int traversal) {
    try {
        return pk_index_prepare_fast_impl(h, traversal);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_prepare_fast: unexpected exception");
    }
}

int pk_index_tune_fast(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t expand,
                       int32_t *out_shape, float *out_ms, void *stream) {
    try {
        return pk_index_tune_fast_impl(h, queries, nq, k, ef, expand, out_shape, out_ms, stream);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_tune_fast: unexpected exception");
    }
}

int pk_index_search_fast(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                         const int32_t *k_per_query, const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids,
                         float *out_dists, int32_t *counters, int32_t expand, void *stream) {
    try {
        return pk_index_search_fast_impl(h, queries, nq, k, ef, k_per_query, ef_per_query, out_stride, out_ids,
                                         out_dists, counters, expand, stream);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_fast: unexpected exception");
    }
}

int pk_index_set_fast_params(pk_index *h, int32_t rows_per_batch, int32_t filter_log2, int32_t warps_per_block) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (rows_per_batch < 0 || rows_per_batch > 256) return fail(PK_ERR_ARG, "rows_per_batch must be 0..256");
    if (filter_log2 != 0 && (filter_log2 < 5 || filter_log2 > 15))
        return fail(PK_ERR_ARG, "filter_log2 must be 0 or 5..15");
    if (warps_per_block < 0 || warps_per_block > 8) return fail(PK_ERR_ARG, "warps_per_block must be 0..8");
    h->fast_rb = rows_per_batch;
    h->fast_hlog2 = filter_log2;
    h->fast_wpb = warps_per_block;
    for (int c = 0; c < pk::kSlotClasses; c++) h->cls_rb[c] = h->cls_hlog2[c] = h->cls_wpb[c] = 0;
    return PK_OK;
}

int pk_index_set_fast_class_params(pk_index *h, int32_t width_class, int32_t rows_per_batch, int32_t filter_log2,
                                   int32_t warps_per_block) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (width_class < 0 || width_class >= pk::kSlotClasses) return fail(PK_ERR_ARG, "width_class must be 0..9");
    if (rows_per_batch < 0 || rows_per_batch > 256) return fail(PK_ERR_ARG, "rows_per_batch must be 0..256");
    if (filter_log2 != 0 && (filter_log2 < 5 || filter_log2 > 15))
        return fail(PK_ERR_ARG, "filter_log2 must be 0 or 5..15");
    if (warps_per_block < 0 || warps_per_block > 8) return fail(PK_ERR_ARG, "warps_per_block must be 0..8");
    if ((rows_per_batch == 0) != (filter_log2 == 0) || (rows_per_batch == 0) != (warps_per_block == 0))
        return fail(PK_ERR_ARG, "give all three values, or all three 0 to fall back to the handle's shape");
    h->cls_rb[width_class] = rows_per_batch;
    h->cls_hlog2[width_class] = filter_log2;
    h->cls_wpb[width_class] = warps_per_block;
    return PK_OK;
}

int pk_index_tune_fast_classes(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t max_ef,
                               int32_t expand, int32_t *out_shapes, float *out_ms, void *stream) {
    try {
        return pk_index_tune_fast_classes_impl(h, queries, nq, k, max_ef, expand, out_shapes, out_ms, stream);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_tune_fast_classes: unexpected exception");
    }
}

int pk_index_set_fast_visited(pk_index *h, int32_t log2_sets) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (log2_sets < -1 || log2_sets > 20) return fail(PK_ERR_ARG, "log2_sets must be -1, 0 or 1..20");
    h->fast_vt = log2_sets;
    for (int c = 0; c < pk::kSlotClasses; c++) h->cls_vt[c] = 0;  // the tuners' per-width choices
    return PK_OK;
}

int pk_index_set_build_walk(pk_index *h, int64_t min_batch) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (min_batch < 0) return fail(PK_ERR_ARG, "min_batch must be 0 (off) or positive");
    h->build_walk = min_batch;
    return PK_OK;
}

int pk_index_set_fast_merge(pk_index *h, int32_t min_winners) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    if (min_winners < -1 || min_winners > 32) return fail(PK_ERR_ARG, "min_winners must be -1, 0 or 1..32");
    h->fast_merge = min_winners;
    return PK_OK;
}

int pk_index_set_fast_timing(pk_index *h, int enable) {
    if (!h) return fail(PK_ERR_ARG, "NULL handle");
    h->fast_timing = enable != 0;
    return PK_OK;
}

int pk_index_fast_timing(pk_index *h, float *walk_ms, float *rerank_ms) {
    if (!h || !walk_ms || !rerank_ms) return fail(PK_ERR_ARG, "bad arguments");
    const FastCtx &c = h->fctx;
    if (!h->fast_timing || !c.ev[2]) return fail(PK_ERR_STATE, "no timed fast search has run");
    PK_CUDA(cudaEventSynchronize(c.ev[2]));
    if (c.wend_mask == 0) {
        PK_CUDA(cudaEventElapsedTime(walk_ms, c.ev[0], c.ev[1]));
        PK_CUDA(cudaEventElapsedTime(rerank_ms, c.ev[1], c.ev[2]));
        return PK_OK;
    }
    // per-width launches: the walks span from the start to the end of the
    // last width's walk; the re-ranks of the widths that ended earlier ran
    // inside that span, and what follows it is the last re-ranks' time
    float walk = 0.f, all = 0.f;
    for (int cls = 0; cls < pk::kSlotClasses; cls++) {
        if (!((c.wend_mask >> cls) & 1u)) continue;
        float t = 0.f;
        PK_CUDA(cudaEventElapsedTime(&t, c.ev[0], c.wend[cls]));
        walk = std::max(walk, t);
    }
    PK_CUDA(cudaEventElapsedTime(&all, c.ev[0], c.ev[2]));
    *walk_ms = walk;
    *rerank_ms = std::max(0.f, all - walk);
    return PK_OK;
}

int pk_index_search_fast_host(pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                              float *out_dists, int32_t expand) {
    try {
        return pk_index_search_fast_host_impl(h, queries, nq, k, ef, out_ids, out_dists, expand);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_fast_host: unexpected exception");
    }
}

int pk_index_search_var(pk_index *h, const void *queries, int64_t nq, const int32_t *k_per_query,
                        const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids, float *out_dists) {
    try {
        return pk_index_search_var_impl(h, queries, nq, k_per_query, ef_per_query, out_stride, out_ids, out_dists);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_var: unexpected exception");
    }
}

int pk_index_search_fast_host_var(pk_index *h, const void *queries, int64_t nq, const int32_t *k_per_query,
                                  const int32_t *ef_per_query, int32_t out_stride, int32_t *out_ids,
                                  float *out_dists, int32_t expand) {
    try {
        return pk_index_search_fast_host_var_impl(h, queries, nq, k_per_query, ef_per_query, out_stride, out_ids,
                                                  out_dists, expand);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_fast_host_var: unexpected exception");
    }
}

int pk_server_create(pk_server **out, pk_index *h, int traversal, int slots, int32_t max_batch, int32_t max_k,
                     int32_t max_ef, int32_t expand) {
    try {
        return srv_create(out, h, traversal, slots, max_batch, max_k, max_ef, expand, 0);
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_server_create: unexpected exception");
    }
}

int pk_server_create_with_memory(pk_server **out, pk_index *h, int traversal, int slots, int32_t max_batch,
                                 int32_t max_k, int32_t max_ef, int32_t expand, int64_t device_bytes) {
    try {
        return srv_create(out, h, traversal, slots, max_batch, max_k, max_ef, expand, device_bytes);
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_server_create_with_memory: unexpected exception");
    }
}

int pk_server_memory(pk_server *s, int64_t *out) {
    if (!s || !out) return fail(PK_ERR_ARG, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = (int64_t)s->arena_bytes;
    out[1] = (int64_t)s->in_use;
    out[2] = (int64_t)s->peak_in_use;
    out[3] = s->deferred_for_memory;
    return PK_OK;
}

int pk_server_request_bytes(pk_server *s, int32_t nq, int32_t k, int32_t ef, int64_t *bytes) {
    if (!s || !bytes || nq < 1 || k < 1 || ef < 1) return fail(PK_ERR_ARG, "bad arguments");
    *bytes = (int64_t)srv_layout(s->h, nq, k, std::min(ef, pk::kFastMaxEf)).total;
    return PK_OK;
}

int pk_server_submit(pk_server *s, const void *queries, int32_t nq, int32_t k, int32_t ef, int64_t *ticket) {
    try {
        return srv_submit(s, queries, nq, k, ef, ticket);
    } catch (const std::bad_alloc &) {
        return fail(PK_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_server_submit: unexpected exception");
    }
}

int pk_server_wait(pk_server *s, int64_t ticket, int32_t *out_ids, float *out_dists, double *latency_ms,
                   int32_t timeout_ms) {
    try {
        return srv_wait(s, ticket, out_ids, out_dists, latency_ms, timeout_ms);
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_server_wait: unexpected exception");
    }
}

int pk_server_stats(pk_server *s, int64_t *out) {
    if (!s || !out) return fail(PK_ERR_ARG, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = s->batches;
    out[1] = s->queries;
    out[2] = s->max_inflight;
    out[3] = (int64_t)s->queue.size();
    out[4] = s->error;
    return PK_OK;
}

int pk_server_replay(pk_server *s, const void *queries, int64_t n, const int32_t *nq, const double *arrival_us,
                     const int32_t *k, const int32_t *ef, int32_t *out_ids, float *out_dists, int32_t out_stride,
                     double *latency_ms) {
    if (!s || !queries || n < 0 || !nq || !arrival_us || !k || !ef || !latency_ms || out_stride < 1)
        return fail(PK_ERR_ARG, "bad arguments");
    try {
        const size_t w = (size_t)(s->h->dim * s->h->esz);
        std::vector<int64_t> tickets(n, 0), qoff(n + 1, 0);
        for (int64_t i = 0; i < n; i++) qoff[i + 1] = qoff[i] + nq[i];
        std::atomic<int64_t> submitted{0};
        std::atomic<int> rc_prod{PK_OK};
        const auto t0 = Clock::now();
        std::thread prod([&] {
            for (int64_t i = 0; i < n; i++) {
                const auto due = t0 + std::chrono::nanoseconds((int64_t)(arrival_us[i] * 1000.0));
                while (Clock::now() < due) {
                }
                const int rc = srv_submit(s, static_cast<const uint8_t *>(queries) + (size_t)qoff[i] * w, nq[i], k[i],
                                          ef[i], &tickets[i]);
                if (rc != PK_OK) {
                    rc_prod = rc;
                    break;
                }
                submitted.store(i + 1, std::memory_order_release);
            }
        });
        std::vector<int32_t> ids;
        std::vector<float> ds;
        int rc = PK_OK;
        for (int64_t i = 0; i < n && rc == PK_OK; i++) {
            while (submitted.load(std::memory_order_acquire) <= i && rc_prod == PK_OK) std::this_thread::yield();
            if (rc_prod != PK_OK) {
                rc = rc_prod;
                break;
            }
            ids.resize((size_t)nq[i] * k[i]);
            ds.resize((size_t)nq[i] * k[i]);
            rc = srv_wait(s, tickets[i], ids.data(), ds.data(), &latency_ms[i], -1);
            if (rc == PK_OK && out_ids && out_dists)
                for (int32_t j = 0; j < nq[i]; j++) {
                    std::memcpy(out_ids + (qoff[i] + j) * out_stride, ids.data() + (size_t)j * k[i], 4 * (size_t)k[i]);
                    std::memcpy(out_dists + (qoff[i] + j) * out_stride, ds.data() + (size_t)j * k[i],
                                4 * (size_t)k[i]);
                }
        }
        prod.join();
        return rc;
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_server_replay: unexpected exception");
    }
}

int pk_server_set_watchdog(pk_server *s, double seconds) {
    if (!s || !(seconds >= 0.0)) return fail(PK_ERR_ARG, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    s->watchdog_s = seconds;
    return PK_OK;
}

int pk_server_destroy(pk_server *s) {
    if (!s) return PK_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    srv_free(s);
    return PK_OK;
}

}  // extern "C"
