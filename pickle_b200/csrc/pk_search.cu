// Exact HNSW query kernel: one query per warp, persistent grid, work taken
// from a global counter (work stealing across warps).
//
// Per query it does what the reference's AnnSearch does (include/hnsw.hpp:509-525):
// SlideLayer from the top layer's entry down to layer 1, SearchLayerFast on
// layer 0 with the query's ef, then extractMinTopK and the mapping to external
// ids (include/hnsw.hpp:118-125, include/queue.hpp:265-286).  The building
// blocks are in pk_warp.cuh.  A query whose visited table or candidate heap
// outgrows the per-warp scratch is flagged (status 1) and rerun by the host
// with larger scratch, so results never depend on the scratch size.
#include "pk_warp.cuh"

namespace pk {

namespace {

using namespace dev;

template <int DT, int KMAX>
__global__ void __launch_bounds__(128, 6)
    search_exact_kernel(const DevGraph *__restrict__ gp, const LaneCfg lc, const SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int gwarp = blockIdx.x * wpb + wib;

    const int64_t row_bytes = gp->row_bytes;
    WarpScratch ws;
    unsigned char *my = smem + (size_t)wib * search_smem_per_warp(a.wcap, row_bytes);
    ws.wbuf = reinterpret_cast<Ent *>(my);
    ws.wcap = a.wcap;
    ws.ctop = ws.wbuf + a.wcap;
    ws.st = reinterpret_cast<Stage *>(my + search_stage_off(a.wcap));
    ws.rowbuf = reinterpret_cast<uint8_t *>(my + search_rowbuf_off(a.wcap));
    ws.bind(a.gs, gwarp);

    const VecView vv{gp->vec0, gp->zero_row, gp->row_bytes};
    const bool ip = gp->metric == PK_METRIC_IP;
    const int enter_level = gp->enter_level;
    const DevLayer L0 = gp->L[0];

    for (;;) {
        int qi = 0;
        if (lane == 0) qi = atomicAdd(&a.work[0], 1);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= a.nq) break;
        const int q = a.qlist ? a.qlist[qi] : qi;
        // per-query values are clamped to what the launch was sized for
        const int k = max(0, min(a.k_arr ? a.k_arr[q] : a.k, a.out_stride));
        const int ef = max(1, min(a.ef_arr ? a.ef_arr[q] : a.ef, a.ef));

        uint4 qr[KMAX];
        load_regs<KMAX>(qr, a.queries + (int64_t)q * vv.row_bytes, lc, lane, false);

        int32_t cnt[6] = {0, 0, 0, 0, 0, 0};
        bool full = false;

        int32_t enter = gp->L[enter_level].ent;
        for (int level = enter_level; level >= 1 && !full; --level) {
            const DevLayer L = gp->L[level];
            const int32_t c = slide_layer<DT, KMAX, false>(vv, lc, qr, ip, L, enter, ws, cnt, full, lane);
            // GetEntInID(GetExtID(c)) one level down (include/hnsw.hpp:515-519);
            // an unused slot has external id -1, which maps to the entry id
            const int32_t dn = L.down[c];
            enter = dn >= 0 ? dn : gp->L[level - 1].ent;
        }
        int wl = 0;
        if (!full) wl = search_layer<DT, KMAX, false>(vv, lc, qr, ip, L0, true, enter, ef, ws, cnt + 3, full, lane);

        int32_t *oid = a.out_ids + (int64_t)q * a.out_stride;
        float *od = a.out_dists + (int64_t)q * a.out_stride;
        if (full) {
            if (lane == 0) {
                a.status[q] = 1;
                atomicAdd(&a.work[1], 1);
            }
        } else {
            const int kk = k < wl ? k : wl;
            if (lane == 0) {
                // extractMinTopK on the result heap, then external ids
                MaxHeap W{ws.wbuf, wl};
                while (W.len > kk) W.pop();
                for (int i = 0; i < kk; i++) {
                    const Ent e = W.a[0];
                    W.pop();
                    oid[kk - 1 - i] = a.ext0[e.id];
                    od[kk - 1 - i] = e.d;
                }
                a.status[q] = 0;
            }
            for (int i = kk + lane; i < k; i += 32) {
                oid[i] = -1;
                od[i] = FLT_MAX;
            }
        }
        if (a.counters && lane == 0) {
            int32_t *cp = a.counters + (int64_t)q * 6;
#pragma unroll
            for (int i = 0; i < 6; i++) cp[i] = cnt[i];
        }
        __syncwarp();
    }
}

template <int DT>
void *pick_kernel(int kmax) {
    switch (kmax) {
        case 1: return (void *)search_exact_kernel<DT, 1>;
        case 2: return (void *)search_exact_kernel<DT, 2>;
        case 4: return (void *)search_exact_kernel<DT, 4>;
        case 8: return (void *)search_exact_kernel<DT, 8>;
        case 16: return (void *)search_exact_kernel<DT, 16>;
        case 32: return (void *)search_exact_kernel<DT, 32>;
        default: return nullptr;
    }
}

void *search_kernel_ptr(int dtype, int kmax) {
    switch (dtype) {
        case PK_DTYPE_U8: return pick_kernel<PK_DTYPE_U8>(kmax);
        case PK_DTYPE_I8: return pick_kernel<PK_DTYPE_I8>(kmax);
        case PK_DTYPE_F32: return pick_kernel<PK_DTYPE_F32>(kmax);
        case PK_DTYPE_F16: return pick_kernel<PK_DTYPE_F16>(kmax);
        default: return nullptr;
    }
}

}  // namespace

int search_blocks_per_sm(int dtype, const LaneCfg &lc, int wpb, size_t smem) {
    void *fn = search_kernel_ptr(dtype, lc.KMAX);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, wpb * 32, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_search_exact(const DevGraph *g, int dtype, const LaneCfg &lc, const SearchArgs &a, int grid, int wpb,
                                size_t smem, cudaStream_t s) {
    void *fn = search_kernel_ptr(dtype, lc.KMAX);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void *args[] = {(void *)&g, (void *)&lc, (void *)&a};
    return cudaLaunchKernel(fn, dim3(grid), dim3(wpb * 32), args, smem, s);
}

}  // namespace pk
