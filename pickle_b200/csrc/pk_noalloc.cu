// pk_index_search_noalloc: the exact device search with no device allocation.
//
// Some callers cannot let a library call cudaMalloc.  A serving loop that
// must keep its tail latency flat cannot afford the implicit device-wide
// synchronisation that cudaMalloc and cudaFree can bring, and a process whose
// device memory is already carved up by another allocator (a framework's
// caching pool that reserved most of the GPU) may find that a fresh
// cudaMalloc fails or eats memory promised elsewhere.  pk_index_search_device
// grows its scratch (visited tables, candidate-heap spill, query staging) on
// demand; this entry point instead runs the same search kernel with all of
// its scratch carved out of one fixed array that is part of the library
// image, so a call touches no allocator.
//
// Rules of use (also in include/pickle_b200.h):
//  * The array is kNoAllocScratchBytes (64 MiB) of device memory, held by
//    every GPU that loads the library until the process exits.
//  * Limits: nq <= kNoAllocMaxQueries, ef <= kNoAllocMaxEf; larger requests are
//    rejected with PK_ERR_ARG before anything runs.  A query that still
//    outgrows the fixed scratch is not retried: the call returns
//    PK_ERR_OVERFLOW and the caller can fall back to pk_index_search_device.
//  * The first call on a device looks up the array's device address there
//    (with that device current).  Every call waits for its own work on the
//    stream before it returns (it reads the overflow count back).
//  * Every call on a device shares the one array, which keeps the previous
//    call's contents.  What must start from zero is cleared by the call: the
//    work counters on every call, and the visited bitmaps, which sit at the
//    front of the array: a completed search leaves its bitmaps all-zero, so a
//    call clears only the part of its bitmap area that reaches beyond the area
//    the previous calls on this device left clean.  Calls that overlap on the
//    GPU (two streams, two threads, two indexes on the same device) race on
//    the array and give wrong results: serialise them.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "pk_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr int64_t kNoAllocMaxQueries = 65536;
constexpr int32_t kNoAllocMaxEf = 1024;
constexpr int kMaxDevices = 64;

// The scratch of every no-allocation search on this device.  In host code
// this name is only a stand-in for the symbol, not a device address: host
// code must use the address cudaGetSymbolAddress returned (g_scratch_addr).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};
// bytes at the front of the bitmap area known to be zero on each device
size_t g_clean_bytes[kMaxDevices] = {};

__global__ void noalloc_fill_kernel(int32_t *ids, float *d, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        ids[i] = -1;
        d[i] = FLT_MAX;
    }
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int fail(int code, const char *msg) {
    pk::set_error(msg);
    return code;
}

// Once per device, with that device current: the device address of the array.
int scratch_address(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(PK_ERR_ARG, "pk_index_search_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(PK_ERR_CUDA, "pk_index_search_noalloc: cudaGetSymbolAddress of the scratch array failed");
        }
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return PK_OK;
}

int search_noalloc(const pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef, int32_t *out_ids,
                   float *out_dists, void *stream) {
    if (!h || nq < 0 || ((!queries || !out_ids || !out_dists) && nq > 0))
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: bad arguments");
    if (k < 1 || ef < 1) return fail(PK_ERR_ARG, "pk_index_search_noalloc: k and ef must be >= 1");
    if (nq > kNoAllocMaxQueries)
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: nq exceeds the fixed-scratch limit of 65536 queries");
    if (ef > kNoAllocMaxEf)
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: ef exceeds the fixed-scratch limit of 1024");
    if (nq == 0) return PK_OK;
    const pk::IndexView v = pk::index_view(h);
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != v.device)
        return fail(PK_ERR_STATE, "pk_index_search_noalloc: the index's device must be the current device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (v.n0 == 0) {
        noalloc_fill_kernel<<<256, 256, 0, s>>>(out_ids, out_dists, nq * k);
        return cudaGetLastError() == cudaSuccess ? PK_OK : fail(PK_ERR_CUDA, "fill launch failed");
    }
    unsigned char *base = nullptr;
    int rc = scratch_address(v.device, &base);
    if (rc != PK_OK) return rc;

    // kernel shape, as pk_index_search_device chooses it
    const int wcap = ef + 2;
    int wpb = 4;
    size_t smem = (size_t)wpb * pk::search_smem_per_warp(wcap, v.row_bytes);
    while (wpb > 1 && smem > 200 * 1024) {
        wpb /= 2;
        smem = (size_t)wpb * pk::search_smem_per_warp(wcap, v.row_bytes);
    }
    if (smem > 220 * 1024)
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: ef and the row size need more shared memory than a block has");
    const int nb = pk::search_blocks_per_sm(v.dtype, v.lc, wpb, smem);
    if (nb <= 0) {
        cudaGetLastError();
        return fail(PK_ERR_CUDA, "pk_index_search_noalloc: search kernel cannot be resident");
    }
    const int64_t bm_words = (v.lcap0 + 31) / 32 + 1;
    const int64_t vl_cap = std::max<int64_t>(4096, 16LL * ef);
    const int64_t tail = std::max<int64_t>(4096, 32LL * ef);

    // carve the array: counters | bitmaps | status | staged queries | id lists | spills
    const bool stage = (v.dim * v.esz) != v.row_bytes || (reinterpret_cast<uintptr_t>(queries) & 15) != 0;
    const size_t bm_off = 256;  // after the work counters
    size_t fixed = align256((size_t)nq) + (stage ? align256((size_t)nq * (size_t)v.row_bytes) : 0) + 256 * 4;
    const size_t per_warp = (size_t)bm_words * 4 + (size_t)vl_cap * 4 + (size_t)tail * 8;
    if (bm_off + fixed >= kNoAllocScratchBytes)
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: the queries do not fit the fixed scratch");
    int64_t warps = (int64_t)((kNoAllocScratchBytes - bm_off - fixed) / per_warp);
    warps = std::min<int64_t>(warps, (int64_t)nb * v.num_sms * wpb);
    warps = std::min<int64_t>(warps, (nq + wpb - 1) / wpb * wpb);
    warps = warps / wpb * wpb;
    if (warps < wpb)
        return fail(PK_ERR_ARG, "pk_index_search_noalloc: the index or ef is too large for the fixed scratch");
    const size_t bm_bytes = (size_t)warps * (size_t)bm_words * 4;
    size_t off = align256(bm_off + bm_bytes);
    const size_t status_off = off;
    off = align256(off + (size_t)nq);
    const size_t qstage_off = off;
    if (stage) off = align256(off + (size_t)nq * (size_t)v.row_bytes);
    const size_t vl_off = off;
    off = align256(off + (size_t)warps * (size_t)vl_cap * 4);
    const size_t tail_off = off;
    off += (size_t)warps * (size_t)tail * 8;
    if (off > kNoAllocScratchBytes) return fail(PK_ERR_ARG, "pk_index_search_noalloc: scratch layout overflow");

    // what must start at zero: the counters, and the bitmaps beyond the part
    // that earlier calls left clean
    if (cudaMemsetAsync(base, 0, 256, s) != cudaSuccess) return fail(PK_ERR_CUDA, "memset of counters failed");
    {
        std::lock_guard<std::mutex> lock(g_mu);
        size_t &clean = g_clean_bytes[v.device];
        if (bm_bytes > clean) {
            if (cudaMemsetAsync(base + bm_off + clean, 0, bm_bytes - clean, s) != cudaSuccess)
                return fail(PK_ERR_CUDA, "pk_index_search_noalloc: clearing the visited bitmaps failed");
        }
        // after this call only its own bitmap area is known to be clean: the
        // regions behind it are overwritten by the lists, spills and staging
        clean = bm_bytes;
    }
    const uint8_t *q = static_cast<const uint8_t *>(queries);
    if (stage) {
        const size_t w = (size_t)(v.dim * v.esz);
        if (cudaMemsetAsync(base + qstage_off, 0, (size_t)nq * v.row_bytes, s) != cudaSuccess ||
            cudaMemcpy2DAsync(base + qstage_off, (size_t)v.row_bytes, queries, w, w, (size_t)nq,
                              cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return fail(PK_ERR_CUDA, "pk_index_search_noalloc: query staging failed");
        q = base + qstage_off;
    }

    pk::SearchArgs a{};
    a.queries = q;
    a.nq = nq;
    a.qlist = nullptr;
    a.k = k;
    a.ef = ef;
    a.k_arr = nullptr;
    a.ef_arr = nullptr;
    a.out_stride = k;
    a.out_ids = out_ids;
    a.out_dists = out_dists;
    a.ext0 = v.ext0;
    a.counters = nullptr;
    a.status = base + status_off;
    a.work = reinterpret_cast<int32_t *>(base);
    a.gs = pk::WarpGlobalScratch{reinterpret_cast<uint32_t *>(base + bm_off), bm_words,
                                 reinterpret_cast<int32_t *>(base + vl_off), (int32_t)vl_cap, base + tail_off,
                                 (int32_t)tail};
    a.wcap = wcap;
    // a search that did not complete may leave marks in its bitmaps: the next
    // call then clears the whole area again
    auto forget_clean = [&]() {
        std::lock_guard<std::mutex> lock(g_mu);
        g_clean_bytes[v.device] = 0;
    };
    cudaError_t e = pk::launch_search_exact(v.dg, v.dtype, v.lc, a, (int)(warps / wpb), wpb, smem, s);
    if (e != cudaSuccess) {
        forget_clean();
        return fail(PK_ERR_CUDA, "pk_index_search_noalloc: launch failed");
    }
    int32_t over = 0;
    if (cudaMemcpyAsync(&over, base + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        forget_clean();
        return fail(PK_ERR_CUDA, "pk_index_search_noalloc: kernel failed");
    }
    if (over != 0)
        return fail(PK_ERR_OVERFLOW,
                    "pk_index_search_noalloc: some queries outgrew the fixed scratch; use pk_index_search_device");
    return PK_OK;
}

}  // namespace

extern "C" int pk_index_search_noalloc(const pk_index *h, const void *queries, int64_t nq, int32_t k, int32_t ef,
                                       int32_t *out_ids, float *out_dists, void *stream) {
    try {
        return search_noalloc(h, queries, nq, k, ef, out_ids, out_dists, stream);
    } catch (...) {
        return fail(PK_ERR_STATE, "pk_index_search_noalloc: unexpected exception");
    }
}
