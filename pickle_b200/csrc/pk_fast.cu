// Batched low-precision HNSW search with exact re-ranking.
//
// The exact kernel (pk_search.cu) replays the reference's binary heaps with
// one lane, which is what makes its ids bit-identical to the reference's but
// also what bounds it.  This kernel answers the same question - the k nearest
// neighbours found by a best-first walk of the HNSW graph with a result set
// of ef entries (include/hnsw.hpp:373-444) - with data structures suited to a
// warp, and is judged by recall:
//   * traversal distances come from a low-precision copy of the vectors:
//     FP16, or FP8 E4M3 scaled per dimension (a query is scaled by the same
//     per-dimension factors; for L2 a per-row norm of the scaled copy turns
//     the distance into a dot product), always accumulated in FP32;
//   * the result set is a sorted list of ef slots in shared memory (distance,
//     id, expanded flag) instead of two heaps; each iteration expands the P
//     best unexpanded entries at once, marks their neighbours in the exact
//     visited bitmap, stages the new rows with cp.async, sorts the new
//     candidates with a warp bitonic sort and merges them into the list;
//   * the walk ends when every listed entry is expanded; the listed entries
//     (the top ef) are then re-ranked with exact distances from the original
//     vectors and the k best are written, closest first (ties by id).
// Upper layers are descended greedily as in SlideLayer (include/hnsw.hpp:446-494),
// with traversal distances.  Queries run one per warp with work stealing and
// may have different k and ef.  There is no host round trip, so a batch can
// be captured in a CUDA graph.
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "pk_fast.h"
#include "pk_warp.cuh"

namespace pk {

namespace {

using namespace dev;

constexpr uint32_t kExpanded = 0x80000000u;

// ------------------------------------------------------- traversal distances
// Lane layout for traversal rows: CT 16-byte chunks per row, GT lanes per row
// (power of two >= CT, at most 32), KT chunks per lane.

struct TravCfg {
    int GT, KT, CT;
};

// F16 traversal: the query is held as halves, accumulated in FP32 (Acc<F16>).
// E4M3 traversal: the query is held as 16 floats per chunk (pre-scaled).
template <int TRAV, int KT>
struct TravQuery;

template <int KT>
struct TravQuery<kTravF16, KT> {
    uint4 q[KT];
    __device__ __forceinline__ float dot_or_l2(const uint4 &r, int k, bool ip) const {
        float a = 0.f;
        Acc<PK_DTYPE_F16>::add(a, q[k], r, ip);
        return a;
    }
};

template <int KT>
struct TravQuery<kTravE4M3, KT> {
    float q[KT][16];
    __device__ __forceinline__ float dot_or_l2(const uint4 &r, int k, bool) const {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
        float a = 0.f;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const __nv_fp8x2_storage_t lo = (__nv_fp8x2_storage_t)(w[i] & 0xffffu);
            const __nv_fp8x2_storage_t hi = (__nv_fp8x2_storage_t)(w[i] >> 16);
            const __half2 h0 = __half2(__nv_cvt_fp8x2_to_halfraw2(lo, __NV_E4M3));
            const __half2 h1 = __half2(__nv_cvt_fp8x2_to_halfraw2(hi, __NV_E4M3));
            const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
            a = fmaf(q[k][4 * i + 0], f0.x, a);
            a = fmaf(q[k][4 * i + 1], f0.y, a);
            a = fmaf(q[k][4 * i + 2], f1.x, a);
            a = fmaf(q[k][4 * i + 3], f1.y, a);
        }
        return a;
    }
};

struct TravView {
    const uint8_t *rows;      // traversal copy, row_bytes apart
    const uint8_t *zero_row;
    int64_t row_bytes;
    const float *rownorm;     // E4M3 + L2: sum_d (s_d x_d)^2 of the stored row
    __device__ __forceinline__ const uint8_t *row(int32_t r) const {
        return r >= 0 ? rows + (int64_t)r * row_bytes : zero_row;
    }
};

// Traversal distance of nrows rows (<= 32) staged kStageRows at a time.
template <int TRAV, int KT>
__device__ __forceinline__ void trav_dist_rows(const TravView &tv, const TravCfg &tc, const TravQuery<TRAV, KT> &tq,
                                               bool ip, float qnorm, const int32_t *rows, float *outd, int nrows,
                                               uint8_t *rowbuf, int lane) {
    const int G = tc.GT, R = 32 / G, grp = lane / G, gl = lane % G;
    for (int b0 = 0; b0 < nrows; b0 += kStageRows) {
        const int nb = min(kStageRows, nrows - b0);
        for (int t = grp; t < nb; t += R) {
            const uint8_t *src = tv.row(rows[b0 + t]);
            uint8_t *dst = rowbuf + (int64_t)t * tv.row_bytes;
#pragma unroll
            for (int k = 0; k < KT; k++) {
                const int c = gl + k * G;
                if (c < tc.CT) cp_async16(dst + c * 16, src + c * 16);
            }
        }
        cp_async_wait_all();
        for (int base = 0; base < nb; base += R) {
            const int t = base + grp;
            float acc = 0.f;
            if (t < nb) {
                const uint8_t *row = rowbuf + (int64_t)t * tv.row_bytes;
#pragma unroll
                for (int k = 0; k < KT; k++) {
                    const int c = gl + k * G;
                    if (c < tc.CT) acc += tq.dot_or_l2(*reinterpret_cast<const uint4 *>(row + c * 16), k, ip);
                }
            }
            for (int off = G >> 1; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
            if (gl == 0 && t < nb) {
                float d;
                if constexpr (TRAV == kTravF16) {
                    d = ip ? -acc : acc;
                } else {
                    const int32_t r = rows[b0 + t];
                    d = ip ? -acc : qnorm - 2.f * acc + (r >= 0 ? tv.rownorm[r] : 0.f);
                }
                outd[b0 + t] = d;
            }
        }
    }
}

// ------------------------------------------------------------ sorted list --
// Entries order by (distance, id), the expanded flag masked off.
__device__ __forceinline__ bool ent_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (da == db && (ia & ~kExpanded) < (ib & ~kExpanded));
}

// Bitonic sort of one (d, id) pair per lane, ascending across the warp.
__device__ __forceinline__ void warp_sort32(float &d, uint32_t &id, int lane) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const float od = __shfl_xor_sync(kFull, d, stride);
            const uint32_t oi = __shfl_xor_sync(kFull, id, stride);
            const bool up = ((lane & size) == 0);
            const bool lower = (lane & stride) == 0;
            // the lower lane keeps the smaller entry in an ascending run
            const bool take_other = lower == up ? ent_less(od, oi, d, id) : ent_less(d, id, od, oi);
            if (take_other) {
                d = od;
                id = oi;
            }
        }
    }
}

struct ListBuf {
    float *d;
    uint32_t *id;
};

// Merge up to 32 sorted new entries (one per lane: nd/nid, +inf padded) into
// the sorted list src[0..cnt), writing the first L of the union to dst.
// Returns the new count.  newd/newid: shared scratch of 32 entries.
__device__ __forceinline__ int merge_into(const ListBuf &src, const ListBuf &dst, int cnt, int L, float nd,
                                          uint32_t nid, int m, float *newd, uint32_t *newid, int lane) {
    newd[lane] = nd;
    newid[lane] = nid;
    __syncwarp();
    // list entries: new position = i + #new entries before them
    for (int i = lane; i < cnt; i += 32) {
        const float d = src.d[i];
        const uint32_t id = src.id[i];
        int lo = 0, hi = m;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ent_less(newd[mid], newid[mid], d, id)) lo = mid + 1;
            else hi = mid;
        }
        const int p = i + lo;
        if (p < L) {
            dst.d[p] = d;
            dst.id[p] = id;
        }
    }
    // new entries: position = lane + #list entries before them
    if (lane < m) {
        int lo = 0, hi = cnt;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ent_less(src.d[mid], src.id[mid], nd, nid)) lo = mid + 1;
            else hi = mid;
        }
        const int p = lane + lo;
        if (p < L) {
            dst.d[p] = nd;
            dst.id[p] = nid;
        }
    }
    __syncwarp();
    return min(L, cnt + m);
}

// Bitonic sort of n (power of two, <= 2*list size) entries in shared memory.
__device__ __forceinline__ void smem_sort(float *d, uint32_t *id, int n, int lane) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < n / 2; i += 32) {
                const int lo = 2 * i - (i & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const float dl = d[lo], dh = d[hi];
                const uint32_t il = id[lo], ih = id[hi];
                const bool swap = up ? ent_less(dh, ih, dl, il) : ent_less(dl, il, dh, ih);
                if (swap) {
                    d[lo] = dh;
                    d[hi] = dl;
                    id[lo] = ih;
                    id[hi] = il;
                }
            }
            __syncwarp();
        }
    }
}

template <int DT, int KMAX, int TRAV, int KT>
__global__ void __launch_bounds__(128, 6)
    search_fast_kernel(const DevGraph *__restrict__ gp, const LaneCfg lc, const TravCfg tc, const FastArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * wpb + wib;
    const int Lmax = a.list_cap;
    unsigned char *my = smem + (size_t)wib * fast_smem_per_warp(Lmax, a.rowbuf_bytes);
    ListBuf A{reinterpret_cast<float *>(my), reinterpret_cast<uint32_t *>(my) + Lmax};
    ListBuf B{reinterpret_cast<float *>(my) + 2 * Lmax, reinterpret_cast<uint32_t *>(my) + 3 * Lmax};
    float *newd = reinterpret_cast<float *>(my) + 4 * Lmax;
    uint32_t *newid = reinterpret_cast<uint32_t *>(newd + 32);
    Stage *st = reinterpret_cast<Stage *>(newid + 32);
    uint8_t *rowbuf = reinterpret_cast<uint8_t *>(st + 1);

    WarpScratch ws;
    ws.st = st;
    ws.rowbuf = rowbuf;
    ws.bind(a.gs, gwarp);

    const VecView vv{gp->vec0, gp->zero_row, gp->row_bytes};
    const TravView tv{a.trav, a.trav_zero, a.trav_row_bytes, a.rownorm};
    const bool ip = gp->metric == PK_METRIC_IP;
    const int enter_level = gp->enter_level;
    const DevLayer L0 = gp->L[0];

    for (;;) {
        int qi = 0;
        if (lane == 0) qi = atomicAdd(a.work, 1);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= a.nq) break;
        const int q = qi;
        const int k = max(0, min(a.k_arr ? a.k_arr[q] : a.k, a.out_stride));
        const int ef = max(1, min(a.ef_arr ? a.ef_arr[q] : a.ef, Lmax));
        const int L = ef;

        // traversal query: lane-local chunks of the query in the traversal format
        TravQuery<TRAV, KT> tq;
        float qnorm = 0.f;
        {
            const int G = tc.GT, gl = lane % G;
            const uint8_t *qrow = a.tq_rows + (int64_t)q * a.tq_row_bytes;
#pragma unroll
            for (int kk = 0; kk < KT; kk++) {
                const int c = gl + kk * G;
                if constexpr (TRAV == kTravF16) {
                    tq.q[kk] = c < tc.CT ? ld16(qrow + c * 16) : make_uint4(0, 0, 0, 0);
                } else {
#pragma unroll
                    for (int e = 0; e < 16; e++) tq.q[kk][e] = 0.f;
                    if (c < tc.CT) {
                        const float *qf = reinterpret_cast<const float *>(qrow) + c * 16;
#pragma unroll
                        for (int e = 0; e < 16; e++) tq.q[kk][e] = qf[e];
                    }
                }
            }
            if (TRAV == kTravE4M3) qnorm = a.qnorm[q];
        }

        int32_t cnt[6] = {0, 0, 0, 0, 0, 0};
        // ---- upper layers: greedy descent with traversal distances ----
        int32_t enter = gp->L[enter_level].ent;
        for (int level = enter_level; level >= 1; --level) {
            const DevLayer Ly = gp->L[level];
            if (lane == 0) st->row[0] = Ly.vrow[enter];
            __syncwarp();
            trav_dist_rows<TRAV, KT>(tv, tc, tq, ip, qnorm, st->row, st->d, 1, rowbuf, lane);
            __syncwarp();
            float cd = st->d[0];
            __syncwarp();
            int32_t c = enter;
            if (lane == 0) ws.mark_one(enter);
            ws.vl_n++;
            __syncwarp();
            bool updated;
            int64_t rounds = 0;
            do {
                updated = false;
                const int32_t cur = c;
                const int64_t base = (int64_t)cur * Ly.cap;
                const int deg = Ly.deg[cur];
                cnt[0]++;
                cnt[2] += deg;
                for (int j0 = 0; j0 < deg; j0 += 32) {
                    const int nn = take_new(Ly, false, base, j0, deg, ws, lane, false, 0);
                    trav_dist_rows<TRAV, KT>(tv, tc, tq, ip, qnorm, st->row, st->d, nn, rowbuf, lane);
                    __syncwarp();
                    for (int t = 0; t < nn; t++) {
                        const float d = st->d[t];
                        if (d < cd) {
                            cd = d;
                            c = st->id[t];
                            updated = true;
                        }
                    }
                    cnt[1] += nn;
                    __syncwarp();
                }
            } while (updated && ++rounds <= Ly.lcap);
            ws.end_layer(lane);
            const int32_t dn = Ly.down[c];
            enter = dn >= 0 ? dn : gp->L[level - 1].ent;
        }

        // ---- layer 0: best-first walk over a sorted list of ef slots ----
        int count = 0;
        {
            if (lane == 0) st->row[0] = enter;
            __syncwarp();
            trav_dist_rows<TRAV, KT>(tv, tc, tq, ip, qnorm, st->row, st->d, 1, rowbuf, lane);
            __syncwarp();
            if (lane == 0) {
                A.d[0] = st->d[0];
                A.id[0] = (uint32_t)enter;
                ws.mark_one(enter);
            }
            ws.vl_n++;
            count = 1;
            __syncwarp();
        }
        int64_t iters = 0;
        for (;;) {
            // the P best unexpanded entries, in list order
            int picked[4] = {-1, -1, -1, -1};
            int np = 0;
            for (int base = 0; base < count && np < a.expand; base += 32) {
                const int i = base + lane;
                const bool un = i < count && !(A.id[i] & kExpanded);
                unsigned m = __ballot_sync(kFull, un);
                while (m && np < a.expand) {
                    const int b = __ffs(m) - 1;
                    picked[np++] = base + b;
                    m &= m - 1;
                }
            }
            if (np == 0 || ++iters > L0.lcap) break;
            // the ids now: a merge below moves entries to the other buffer
            int32_t cids[4];
#pragma unroll
            for (int p = 0; p < 4; p++) cids[p] = p < np ? (int32_t)(A.id[picked[p]] & ~kExpanded) : -1;
            __syncwarp();
            if (lane == 0)
                for (int p = 0; p < np; p++) A.id[picked[p]] |= kExpanded;
            __syncwarp();
            for (int p = 0; p < np; p++) {
                const int32_t cid = cids[p];
                const int64_t base = (int64_t)cid * L0.cap;
                const int32_t pre = lane < L0.cap ? L0.adj[base + lane] : -1;
                const int deg = L0.deg[cid];
                cnt[3]++;
                cnt[5] += deg;
                for (int j0 = 0; j0 < deg; j0 += 32) {
                    const int nn = take_new(L0, true, base, j0, deg, ws, lane, j0 == 0 && L0.cap >= 32, pre);
                    cnt[4] += nn;
                    if (nn == 0) continue;
                    trav_dist_rows<TRAV, KT>(tv, tc, tq, ip, qnorm, st->row, st->d, nn, rowbuf, lane);
                    __syncwarp();
                    // keep what beats the worst listed entry once the list is full
                    float nd = FLT_MAX;
                    uint32_t nid = 0x7fffffffu;
                    if (lane < nn) {
                        nd = st->d[lane];
                        nid = (uint32_t)st->id[lane];
                        if (count >= L && !ent_less(nd, nid, A.d[count - 1], A.id[count - 1])) {
                            nd = FLT_MAX;
                            nid = 0x7fffffffu;
                        }
                    }
                    const unsigned keep = __ballot_sync(kFull, nd != FLT_MAX);
                    const int m = __popc(keep);
                    if (m == 0) continue;
                    if (m <= 4) {
                        // a few survivors: insert each by shifting the list
                        // tail one slot (lanes own list slots i = lane + 32j)
                        unsigned left = keep;
                        while (left) {
                            const int src = __ffs(left) - 1;
                            left &= left - 1;
                            const float cd = __shfl_sync(kFull, nd, src);
                            const uint32_t ci = __shfl_sync(kFull, nid, src);
                            if (count >= L && !ent_less(cd, ci, A.d[count - 1], A.id[count - 1])) continue;
                            int pos = 0;
                            for (int b = 0; b < count; b += 32) {
                                const int i = b + lane;
                                pos += __popc(__ballot_sync(kFull, i < count && ent_less(A.d[i], A.id[i], cd, ci)));
                            }
                            const int last = min(count, L - 1);  // slot the tail moves into
                            // move [pos, last) up by one, from the top down
                            for (int b = ((last - 1) / 32) * 32; b >= 0 && last > pos; b -= 32) {
                                const int i = b + lane;
                                float vd = 0.f;
                                uint32_t vi = 0;
                                const bool mv = i >= pos && i < last;
                                if (mv) {
                                    vd = A.d[i];
                                    vi = A.id[i];
                                }
                                __syncwarp();
                                if (mv) {
                                    A.d[i + 1] = vd;
                                    A.id[i + 1] = vi;
                                }
                                __syncwarp();
                            }
                            if (lane == 0) {
                                A.d[pos] = cd;
                                A.id[pos] = ci;
                            }
                            count = min(count + 1, L);
                            __syncwarp();
                        }
                    } else {
                        warp_sort32(nd, nid, lane);
                        count = merge_into(A, B, count, L, nd, nid, m, newd, newid, lane);
                        const ListBuf T = A;
                        A = B;
                        B = T;
                    }
                }
            }
        }
        ws.end_layer(lane);

        // ---- re-rank the listed entries with exact distances ----
        uint4 qr[KMAX];
        load_regs<KMAX>(qr, a.queries + (int64_t)q * vv.row_bytes, lc, lane, false);
        const int R = count;
        for (int b0 = 0; b0 < R; b0 += 32) {
            const int nn = min(32, R - b0);
            if (lane < nn) st->row[lane] = (int32_t)(A.id[b0 + lane] & ~kExpanded);
            __syncwarp();
            dist_rows_staged<DT, KMAX>(vv, lc, qr, ip, st->row, st->d, nn, rowbuf, lane);
            __syncwarp();
            if (lane < nn) {
                B.d[b0 + lane] = st->d[lane];
                B.id[b0 + lane] = A.id[b0 + lane] & ~kExpanded;
            }
            __syncwarp();
        }
        int n2 = 1;
        while (n2 < R) n2 <<= 1;
        for (int i = R + lane; i < n2; i += 32) {
            B.d[i] = FLT_MAX;
            B.id[i] = 0x7fffffffu;
        }
        __syncwarp();
        smem_sort(B.d, B.id, n2, lane);
        int32_t *oid = a.out_ids + (int64_t)q * a.out_stride;
        float *od = a.out_dists + (int64_t)q * a.out_stride;
        for (int i = lane; i < k; i += 32) {
            if (i < R) {
                oid[i] = a.ext0[B.id[i]];
                od[i] = B.d[i];
            } else {
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

template <int DT, int KMAX, int TRAV>
void *pick_kt(int kt) {
    switch (kt) {
        case 1: return (void *)search_fast_kernel<DT, KMAX, TRAV, 1>;
        case 2: return (void *)search_fast_kernel<DT, KMAX, TRAV, 2>;
        case 4: return (void *)search_fast_kernel<DT, KMAX, TRAV, 4>;
        default: return nullptr;
    }
}
template <int DT, int KMAX>
void *pick_trav(int trav, int kt) {
    return trav == kTravF16 ? pick_kt<DT, KMAX, kTravF16>(kt) : pick_kt<DT, KMAX, kTravE4M3>(kt);
}
template <int DT>
void *pick_kmax(int kmax, int trav, int kt) {
    switch (kmax) {
        case 1: return pick_trav<DT, 1>(trav, kt);
        case 2: return pick_trav<DT, 2>(trav, kt);
        case 4: return pick_trav<DT, 4>(trav, kt);
        case 8: return pick_trav<DT, 8>(trav, kt);
        default: return nullptr;
    }
}
void *fast_kernel_ptr(int dtype, int kmax, int trav, int kt) {
    switch (dtype) {
        case PK_DTYPE_U8: return pick_kmax<PK_DTYPE_U8>(kmax, trav, kt);
        case PK_DTYPE_I8: return pick_kmax<PK_DTYPE_I8>(kmax, trav, kt);
        case PK_DTYPE_F32: return pick_kmax<PK_DTYPE_F32>(kmax, trav, kt);
        case PK_DTYPE_F16: return pick_kmax<PK_DTYPE_F16>(kmax, trav, kt);
        default: return nullptr;
    }
}

// ------------------------------------------------- traversal-copy kernels --

// Per-dimension max |x| over rows [0, n) (atomicMax on the float bits of
// non-negative values orders them like the values).
template <int DT>
__global__ void absmax_kernel(const uint8_t *vec0, int64_t row_bytes, int64_t n, int dim, uint32_t *out) {
    for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
        const uint8_t *row = vec0 + r * row_bytes;
        for (int d = threadIdx.x; d < dim; d += blockDim.x) {
            float v;
            if (DT == PK_DTYPE_F32) v = reinterpret_cast<const float *>(row)[d];
            else if (DT == PK_DTYPE_F16) v = __half2float(reinterpret_cast<const __half *>(row)[d]);
            else if (DT == PK_DTYPE_U8) v = (float)row[d];
            else v = (float)reinterpret_cast<const int8_t *>(row)[d];
            atomicMax(out + d, __float_as_uint(fabsf(v)));
        }
    }
}

template <int DT>
__device__ __forceinline__ float elem(const uint8_t *row, int d) {
    if (DT == PK_DTYPE_F32) return reinterpret_cast<const float *>(row)[d];
    if (DT == PK_DTYPE_F16) return __half2float(reinterpret_cast<const __half *>(row)[d]);
    if (DT == PK_DTYPE_U8) return (float)row[d];
    return (float)reinterpret_cast<const int8_t *>(row)[d];
}

// Rows [r0, r1) of vec0 into the traversal copy (and, for E4M3, the per-row
// norm of the scaled stored values).  One block per row.
template <int DT, int TRAV>
__global__ void convert_rows_kernel(const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1, int dim,
                                    const float *scale, uint8_t *trav, int64_t trav_row_bytes, float *rownorm) {
    __shared__ float red[32];
    for (int64_t r = r0 + blockIdx.x; r < r1; r += gridDim.x) {
        const uint8_t *row = vec0 + r * row_bytes;
        uint8_t *out = trav + r * trav_row_bytes;
        float part = 0.f;
        for (int d = threadIdx.x; d < dim; d += blockDim.x) {
            const float v = elem<DT>(row, d);
            if constexpr (TRAV == kTravF16) {
                reinterpret_cast<__half *>(out)[d] = __float2half_rn(v);
            } else {
                const __nv_fp8_storage_t x = __nv_cvt_float_to_fp8(v / scale[d], __NV_SATFINITE, __NV_E4M3);
                out[d] = x;
                const float back = __half2float(__half(__nv_cvt_fp8_to_halfraw(x, __NV_E4M3))) * scale[d];
                part += back * back;
            }
        }
        if (TRAV == kTravE4M3) {
            for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(kFull, part, off);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
            __syncthreads();
            if (threadIdx.x == 0) {
                float s = 0.f;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
                rownorm[r] = s;
            }
            __syncthreads();
        }
    }
}

// Queries into the traversal format: F16 rows of halves (padded), or E4M3
// rows of floats pre-multiplied by the per-dimension scales (padded to a
// multiple of 16 elements) plus sum_d q_d^2 for L2.
template <int DT, int TRAV>
__global__ void prep_queries_kernel(const uint8_t *q, int64_t row_bytes, int64_t nq, int dim, const float *scale,
                                    uint8_t *out, int64_t out_row_bytes, float *qnorm) {
    __shared__ float red[32];
    for (int64_t r = blockIdx.x; r < nq; r += gridDim.x) {
        const uint8_t *row = q + r * row_bytes;
        uint8_t *o = out + r * out_row_bytes;
        float part = 0.f;
        const int padded = TRAV == kTravF16 ? (int)(out_row_bytes / 2) : (int)(out_row_bytes / 4);
        for (int d = threadIdx.x; d < padded; d += blockDim.x) {
            const float v = d < dim ? elem<DT>(row, d) : 0.f;
            if constexpr (TRAV == kTravF16) {
                reinterpret_cast<__half *>(o)[d] = __float2half_rn(v);
            } else {
                reinterpret_cast<float *>(o)[d] = d < dim ? v * scale[d] : 0.f;
                part += v * v;
            }
        }
        if (TRAV == kTravE4M3) {
            for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(kFull, part, off);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
            __syncthreads();
            if (threadIdx.x == 0) {
                float s = 0.f;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
                qnorm[r] = s;
            }
            __syncthreads();
        }
    }
}

}  // namespace

TravCfgHost trav_config(int64_t trav_row_bytes, int trav) {
    TravCfgHost t;
    t.CT = (int)(trav_row_bytes / 16);
    // FP16: groups of G lanes with up to 4 chunks each (as the exact path);
    // E4M3: a chunk holds 16 elements, whose query part is 16 floats, so a
    // lane keeps one chunk
    const int want = trav == kTravF16 ? (t.CT + 3) / 4 : t.CT;
    int G = trav == kTravF16 ? 2 : 1;
    while (G < want && G < 32) G *= 2;
    t.GT = G;
    t.KT = (t.CT + G - 1) / G;
    int kt = 1;
    while (kt < t.KT) kt *= 2;
    t.KTMAX = kt;
    return t;
}

int fast_blocks_per_sm(int dtype, const LaneCfg &lc, int trav, const TravCfgHost &tc, int wpb, size_t smem) {
    void *fn = fast_kernel_ptr(dtype, lc.KMAX, trav, tc.KTMAX);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, wpb * 32, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_search_fast(const DevGraph *g, int dtype, const LaneCfg &lc, int trav, const TravCfgHost &tch,
                               const FastArgs &a, int grid, int wpb, size_t smem, cudaStream_t s) {
    void *fn = fast_kernel_ptr(dtype, lc.KMAX, trav, tch.KTMAX);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    TravCfg tc{tch.GT, tch.KT, tch.CT};
    void *args[] = {(void *)&g, (void *)&lc, (void *)&tc, (void *)&a};
    return cudaLaunchKernel(fn, dim3(grid), dim3(wpb * 32), args, smem, s);
}

cudaError_t launch_absmax(int dtype, const uint8_t *vec0, int64_t row_bytes, int64_t n, int dim, uint32_t *out,
                          cudaStream_t s) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(n, 1), 4096);
    switch (dtype) {
        case PK_DTYPE_U8: absmax_kernel<PK_DTYPE_U8><<<grid, 128, 0, s>>>(vec0, row_bytes, n, dim, out); break;
        case PK_DTYPE_I8: absmax_kernel<PK_DTYPE_I8><<<grid, 128, 0, s>>>(vec0, row_bytes, n, dim, out); break;
        case PK_DTYPE_F32: absmax_kernel<PK_DTYPE_F32><<<grid, 128, 0, s>>>(vec0, row_bytes, n, dim, out); break;
        case PK_DTYPE_F16: absmax_kernel<PK_DTYPE_F16><<<grid, 128, 0, s>>>(vec0, row_bytes, n, dim, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int DT>
static void conv(int trav, const uint8_t *vec0, int64_t rb, int64_t r0, int64_t r1, int dim, const float *scale,
                 uint8_t *t, int64_t trb, float *rn, cudaStream_t s) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(r1 - r0, 1), 8192);
    if (trav == kTravF16)
        convert_rows_kernel<DT, kTravF16><<<grid, 128, 0, s>>>(vec0, rb, r0, r1, dim, scale, t, trb, rn);
    else
        convert_rows_kernel<DT, kTravE4M3><<<grid, 128, 0, s>>>(vec0, rb, r0, r1, dim, scale, t, trb, rn);
}

cudaError_t launch_convert_rows(int dtype, int trav, const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1,
                                int dim, const float *scale, uint8_t *trav_rows, int64_t trav_row_bytes,
                                float *rownorm, cudaStream_t s) {
    if (r1 <= r0) return cudaSuccess;
    switch (dtype) {
        case PK_DTYPE_U8: conv<PK_DTYPE_U8>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, rownorm, s); break;
        case PK_DTYPE_I8: conv<PK_DTYPE_I8>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, rownorm, s); break;
        case PK_DTYPE_F32: conv<PK_DTYPE_F32>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, rownorm, s); break;
        case PK_DTYPE_F16: conv<PK_DTYPE_F16>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, rownorm, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int DT>
static void prep(int trav, const uint8_t *q, int64_t rb, int64_t nq, int dim, const float *scale, uint8_t *out,
                 int64_t orb, float *qn, cudaStream_t s) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(nq, 1), 8192);
    if (trav == kTravF16)
        prep_queries_kernel<DT, kTravF16><<<grid, 128, 0, s>>>(q, rb, nq, dim, scale, out, orb, qn);
    else
        prep_queries_kernel<DT, kTravE4M3><<<grid, 128, 0, s>>>(q, rb, nq, dim, scale, out, orb, qn);
}

cudaError_t launch_prep_queries(int dtype, int trav, const uint8_t *q, int64_t row_bytes, int64_t nq, int dim,
                                const float *scale, uint8_t *out, int64_t out_row_bytes, float *qnorm,
                                cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    switch (dtype) {
        case PK_DTYPE_U8: prep<PK_DTYPE_U8>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, qnorm, s); break;
        case PK_DTYPE_I8: prep<PK_DTYPE_I8>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, qnorm, s); break;
        case PK_DTYPE_F32: prep<PK_DTYPE_F32>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, qnorm, s); break;
        case PK_DTYPE_F16: prep<PK_DTYPE_F16>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, qnorm, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pk
