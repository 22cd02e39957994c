// Warp-level building blocks of the exact HNSW path, shared by the query
// kernel (pk_search.cu) and the insertion kernels (pk_build.cu).
//
// Reference behaviour reproduced here (juelinl/pickle):
//   Distance         include/distance.hpp:10-20, include/distance/avx512.hpp
//   EntryHeap        include/queue.hpp:99-289  (push / pop / tie order)
//   ByteMap          include/visited.hpp:540-589 (exact visited set)
//   SlideLayer       include/hnsw.hpp:446-494
//   SearchLayer(Fast) include/hnsw.hpp:304-444
//
// A warp works on one query (or one node being inserted).  Work that does not
// depend on heap state runs on all 32 lanes: reading an adjacency list, the
// visited test, and the distances of a hop's new neighbours.  The heaps are
// replayed by lane 0 in the reference's order, because the reference's
// results depend on its heaps' tie order.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_fp16.h>

#include "pk_internal.h"

namespace pk {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;

struct Ent {
    float d;
    int32_t id;
};
static_assert(sizeof(Ent) == 8, "entry layout");

__device__ __forceinline__ uint4 ld16(const uint8_t *p) { return __ldg(reinterpret_cast<const uint4 *>(p)); }
// Coherent 16-byte load, for rows written earlier in the same kernel.
__device__ __forceinline__ uint4 ld16c(const uint8_t *p) { return *reinterpret_cast<const uint4 *>(p); }

// ---------------------------------------------------------------- distances --
// Per-lane partial sums over 16-byte chunks.  Integer types accumulate exactly
// in 32 bits, as the reference does (include/distance/avx512.hpp:14-149);
// float16 is widened to float32; float types use fused multiply-adds.

template <int DT>
struct Acc;

template <>
struct Acc<PK_DTYPE_F32> {
    typedef float T;
    static __device__ __forceinline__ void add(T &a, const uint4 &q, const uint4 &r, bool ip) {
        const float qf[4] = {__uint_as_float(q.x), __uint_as_float(q.y), __uint_as_float(q.z), __uint_as_float(q.w)};
        const float rf[4] = {__uint_as_float(r.x), __uint_as_float(r.y), __uint_as_float(r.z), __uint_as_float(r.w)};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (ip) {
                a = fmaf(qf[i], rf[i], a);
            } else {
                const float d = qf[i] - rf[i];
                a = fmaf(d, d, a);
            }
        }
    }
    static __device__ __forceinline__ T shfl(T a, int off) { return __shfl_xor_sync(kFull, a, off); }
    static __device__ __forceinline__ float finish(T a, bool ip) { return ip ? -a : a; }
};

template <>
struct Acc<PK_DTYPE_F16> {
    typedef float T;
    static __device__ __forceinline__ void add(T &a, const uint4 &q, const uint4 &r, bool ip) {
        const uint32_t qw[4] = {q.x, q.y, q.z, q.w}, rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 qf = __half22float2(*reinterpret_cast<const __half2 *>(&qw[i]));
            const float2 rf = __half22float2(*reinterpret_cast<const __half2 *>(&rw[i]));
            if (ip) {
                a = fmaf(qf.x, rf.x, a);
                a = fmaf(qf.y, rf.y, a);
            } else {
                const float d0 = qf.x - rf.x, d1 = qf.y - rf.y;
                a = fmaf(d0, d0, a);
                a = fmaf(d1, d1, a);
            }
        }
    }
    static __device__ __forceinline__ T shfl(T a, int off) { return __shfl_xor_sync(kFull, a, off); }
    static __device__ __forceinline__ float finish(T a, bool ip) { return ip ? -a : a; }
};

template <>
struct Acc<PK_DTYPE_U8> {
    typedef int32_t T;
    static __device__ __forceinline__ void add(T &a, const uint4 &q, const uint4 &r, bool ip) {
        const uint32_t qw[4] = {q.x, q.y, q.z, q.w}, rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (ip) {
                a = (int32_t)__dp4a(qw[i], rw[i], (uint32_t)a);
            } else {
                const uint32_t d = __vabsdiffu4(qw[i], rw[i]);
                a = (int32_t)__dp4a(d, d, (uint32_t)a);
            }
        }
    }
    static __device__ __forceinline__ T shfl(T a, int off) { return __shfl_xor_sync(kFull, a, off); }
    static __device__ __forceinline__ float finish(T a, bool ip) {
        const float f = __int2float_rn(a);
        return ip ? -f : f;
    }
};

template <>
struct Acc<PK_DTYPE_I8> {
    typedef int32_t T;
    static __device__ __forceinline__ void add(T &a, const uint4 &q, const uint4 &r, bool ip) {
        const uint32_t qw[4] = {q.x, q.y, q.z, q.w}, rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (ip) {
                a = __dp4a((int)qw[i], (int)rw[i], a);
            } else {
                const uint32_t d = __vabsdiffs4(qw[i], rw[i]);  // |a - b| per byte, 0..255
                a = (int32_t)__dp4a(d, d, (uint32_t)a);
            }
        }
    }
    static __device__ __forceinline__ T shfl(T a, int off) { return __shfl_xor_sync(kFull, a, off); }
    static __device__ __forceinline__ float finish(T a, bool ip) {
        const float f = __int2float_rn(a);
        return ip ? -f : f;
    }
};

struct VecView {
    const uint8_t *vec0;      // layer-0 rows
    const uint8_t *zero_row;  // a row of zeros
    int64_t row_bytes;
    __device__ __forceinline__ const uint8_t *row(int32_t r) const {
        return r >= 0 ? vec0 + (int64_t)r * row_bytes : zero_row;
    }
};

// Each lane holds the chunks gl, gl + G, ... of a row ("the query").
template <int KMAX>
__device__ __forceinline__ void load_regs(uint4 (&qr)[KMAX], const uint8_t *row, const LaneCfg &lc, int lane,
                                          bool coherent) {
    const int gl = lane % lc.G;
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
        const int c = gl + k * lc.G;
        const bool ok = k < lc.K && c < lc.C;
        qr[k] = ok ? (coherent ? ld16c(row + c * 16) : ld16(row + c * 16)) : make_uint4(0, 0, 0, 0);
    }
}

// Distances from the row held in qr to nrows rows (layer-0 row indices in
// rows[], -1 = zero row), written to outd[] by each group's first lane.  All
// 32 lanes must call it.  Each group keeps U rows in flight per step.
template <int DT, int KMAX, bool COHERENT>
__device__ __forceinline__ void dist_rows(const VecView &g, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip,
                                          const int32_t *rows, float *outd, int nrows, int lane) {
    typedef Acc<DT> A;
    constexpr int U = KMAX <= 1 ? 4 : KMAX <= 2 ? 2 : 1;
    const int G = lc.G, R = 32 / G, grp = lane / G, gl = lane % G;
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (int base = 0; base < nrows; base += U * R) {
        const uint8_t *p[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = base + u * R + grp;
            p[u] = t < nrows ? g.row(rows[t]) : nullptr;
        }
        uint4 b[U][KMAX];
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
            const int c = gl + k * G;
            const bool ok = k < lc.K && c < lc.C;
#pragma unroll
            for (int u = 0; u < U; u++)
                b[u][k] = (ok && p[u]) ? (COHERENT ? ld16c(p[u] + c * 16) : ld16(p[u] + c * 16)) : z;
        }
        typename A::T acc[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            acc[u] = 0;
#pragma unroll
            for (int k = 0; k < KMAX; k++) A::add(acc[u], qr[k], b[u][k], ip);
        }
        for (int off = G >> 1; off > 0; off >>= 1) {
#pragma unroll
            for (int u = 0; u < U; u++) acc[u] += A::shfl(acc[u], off);
        }
        if (gl == 0) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = base + u * R + grp;
                if (t < nrows) outd[t] = A::finish(acc[u], ip);
            }
        }
    }
}

// ------------------------------------------------------------- visited set --
// Open addressing over 64-bit slots (epoch << 32 | id): a slot whose epoch is
// not the current one is empty, so a new layer search only bumps the epoch.
// The inserting lanes hold distinct ids, so a lost compare-and-swap only means
// the slot was taken by a neighbour lane.
// Returns 1 if v was inserted (not visited before), 0 if present, 2 if full.
__device__ __forceinline__ int vis_insert(unsigned long long *vis, uint32_t mask, int shift, uint32_t epoch,
                                          int32_t v) {
    uint32_t h = ((uint32_t)v * 2654435761u) >> shift;
    const unsigned long long mine = ((unsigned long long)epoch << 32) | (uint32_t)v;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        unsigned long long s = vis[h];
        for (;;) {
            if ((uint32_t)(s >> 32) != epoch) {
                const unsigned long long old = atomicCAS(vis + h, s, mine);
                if (old == s) return 1;
                s = old;
                continue;
            }
            if ((uint32_t)s == (uint32_t)v) return 0;
            break;
        }
        h = (h + 1) & mask;
    }
    return 2;
}

// ------------------------------------------------------------------- heaps --
// The reference's EntryHeap: a push moves the new entry up while its parent
// compares strictly before it (queue.hpp:119-125; std::push_heap in
// queue.hpp:204-216 does the same); a pop moves the last entry to the root and
// sifts it down, taking the left child if it compares strictly before the
// entry and then the right child if it compares strictly before the better of
// the two (queue.hpp:127-150, :230-236).  Comparators read the distance only.

// MinFirst heap (top = smallest) whose first kCandTop entries live in shared
// memory and the rest in a global spill.
struct MinHeap {
    Ent *top;
    Ent *tail;
    int len;
    int cap;
    __device__ __forceinline__ Ent &at(int i) { return i < kCandTop ? top[i] : tail[i - kCandTop]; }
    __device__ __forceinline__ void push(Ent e) {
        int i = len++;
        while (i > 0) {
            const int p = (i - 1) >> 1;
            const Ent pe = at(p);
            if (!(pe.d > e.d)) break;
            at(i) = pe;
            i = p;
        }
        at(i) = e;
    }
    __device__ __forceinline__ Ent pop() {
        const Ent t = at(0);
        const Ent last = at(len - 1);
        len--;
        if (len > 0) {
            int i = 0;
            for (;;) {
                const int l = 2 * i + 1, r = l + 1;
                int best = i;
                Ent be = last;
                if (l < len) {
                    const Ent le = at(l);
                    if (be.d > le.d) { best = l; be = le; }
                }
                if (r < len) {
                    const Ent re = at(r);
                    if (be.d > re.d) { best = r; be = re; }
                }
                if (best == i) break;
                at(i) = be;
                i = best;
            }
            at(i) = last;
        }
        return t;
    }
};

// MinFirst heap held entirely in one array (shared memory).
struct SmallMinHeap {
    Ent *a;
    int len;
    __device__ __forceinline__ void push(Ent e) {
        int i = len++;
        while (i > 0) {
            const int p = (i - 1) >> 1;
            if (!(a[p].d > e.d)) break;
            a[i] = a[p];
            i = p;
        }
        a[i] = e;
    }
    __device__ __forceinline__ Ent pop() {
        const Ent t = a[0];
        const Ent last = a[len - 1];
        len--;
        if (len > 0) {
            int i = 0;
            for (;;) {
                const int l = 2 * i + 1, r = l + 1;
                int best = i;
                Ent be = last;
                if (l < len && be.d > a[l].d) { best = l; be = a[l]; }
                if (r < len && be.d > a[r].d) { best = r; be = a[r]; }
                if (best == i) break;
                a[i] = be;
                i = best;
            }
            a[i] = last;
        }
        return t;
    }
};

// MaxFirst heap (top = largest) in shared memory: the result set W.
struct MaxHeap {
    Ent *a;
    int len;
    __device__ __forceinline__ void push(Ent e) {
        int i = len++;
        while (i > 0) {
            const int p = (i - 1) >> 1;
            if (!(a[p].d < e.d)) break;
            a[i] = a[p];
            i = p;
        }
        a[i] = e;
    }
    __device__ __forceinline__ void pop() {
        const Ent last = a[len - 1];
        len--;
        if (len == 0) return;
        int i = 0;
        for (;;) {
            const int l = 2 * i + 1, r = l + 1;
            int best = i;
            Ent be = last;
            if (l < len && be.d < a[l].d) { best = l; be = a[l]; }
            if (r < len && be.d < a[r].d) { best = r; be = a[r]; }
            if (best == i) break;
            a[i] = be;
            i = best;
        }
        a[i] = last;
    }
};

struct Stage {
    int32_t id[32];
    int32_t row[32];
    float d[32];
};
static_assert(sizeof(Stage) == kStageBytes, "staging layout");

// Per-warp working memory of a layer search.
struct WarpScratch {
    unsigned long long *vis;  // visited table (global)
    uint32_t vmask;
    int vshift;
    uint32_t vlimit;          // entries allowed before the table counts as full
    uint32_t epoch;
    Ent *wbuf;                // result heap (shared), wcap entries
    int wcap;
    Ent *ctop;                // candidate heap, shared part
    Ent *ctail;               // candidate heap, global part
    int ccap;
    Stage *st;

    __device__ __forceinline__ void next_epoch(int lane) {
        epoch++;
        if (epoch == 0) {  // wrapped: clear the table once
            for (uint32_t i = lane; i <= vmask; i += 32) vis[i] = 0ull;
            __syncwarp();
            epoch = 1;
        }
    }
};

// One chunk (<= 32 entries) of an adjacency list: find the entries that are
// in range, first within the chunk and not yet visited; mark them; stage ids
// and vector rows.  Returns the count (warp-uniform).  Ids outside [0, lcap)
// are skipped (the reference would index its visited table out of range).
__device__ __forceinline__ int take_new(const DevLayer &L, bool layer0, int64_t base, int j0, int deg, WarpScratch &ws,
                                        int lane, bool &full) {
    const int j = j0 + lane;
    int32_t v = -1;
    if (j < deg) v = L.adj[base + j];
    const bool valid = j < deg && v >= 0 && (int64_t)v < L.lcap;
    const int key = valid ? v : -1 - lane;
    const unsigned peers = __match_any_sync(kFull, key);
    const bool first = valid && (__ffs(peers) - 1) == lane;
    int r = 0;
    if (first) r = vis_insert(ws.vis, ws.vmask, ws.vshift, ws.epoch, v);
    const bool is_new = r == 1;
    const unsigned nm = __ballot_sync(kFull, is_new);
    if (__any_sync(kFull, r == 2)) full = true;
    if (is_new) {
        const int pos = __popc(nm & ((1u << lane) - 1));
        ws.st->id[pos] = v;
        ws.st->row[pos] = layer0 ? v : L.vrow[v];
    }
    __syncwarp();
    return __popc(nm);
}

// Distance from the row in qr to node `id` of layer L (warp-uniform result).
template <int DT, int KMAX, bool COH>
__device__ __forceinline__ float dist_one(const VecView &vv, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip,
                                          int32_t row, WarpScratch &ws, int lane) {
    if (lane == 0) ws.st->row[0] = row;
    __syncwarp();
    dist_rows<DT, KMAX, COH>(vv, lc, qr, ip, ws.st->row, ws.st->d, 1, lane);
    __syncwarp();
    const float d = ws.st->d[0];
    __syncwarp();
    return d;
}

// SlideLayer (include/hnsw.hpp:446-494): greedy descent with strict '<', each
// round scanning the whole list of the node the round started from.
// cnt[0..2] += hops, distance evaluations, neighbours scanned.
template <int DT, int KMAX, bool COH>
__device__ int32_t slide_layer(const VecView &vv, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip,
                               const DevLayer &L, int32_t enter, WarpScratch &ws, int32_t *cnt, bool &full, int lane) {
    ws.next_epoch(lane);
    float cd = dist_one<DT, KMAX, COH>(vv, lc, qr, ip, L.vrow[enter], ws, lane);
    int32_t c = enter;
    uint32_t nvis = 1;
    if (lane == 0) vis_insert(ws.vis, ws.vmask, ws.vshift, ws.epoch, enter);
    __syncwarp();
    bool updated;
    int64_t rounds = 0;
    do {
        updated = false;
        const int32_t cur = c;
        const int deg = L.deg[cur];
        const int64_t base = (int64_t)cur * L.cap;
        cnt[0]++;
        cnt[2] += deg;
        for (int j0 = 0; j0 < deg && !full; j0 += 32) {
            const int nn = take_new(L, false, base, j0, deg, ws, lane, full);
            dist_rows<DT, KMAX, COH>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, lane);
            __syncwarp();
            // list order, strict '<': the first occurrence of the minimum wins
            for (int t = 0; t < nn; t++) {
                const float d = ws.st->d[t];
                if (d < cd) {
                    cd = d;
                    c = ws.st->id[t];
                    updated = true;
                }
            }
            cnt[1] += nn;
            nvis += nn;
            if (nvis > ws.vlimit) full = true;
            __syncwarp();
        }
    } while (updated && !full && ++rounds <= L.lcap);
    return c;
}

// SearchLayer / SearchLayerFast (include/hnsw.hpp:304-444).  Leaves the
// result heap W in ws.wbuf and returns its length (warp-uniform).
// cnt[0..2] += hops, distance evaluations, neighbours scanned.
template <int DT, int KMAX, bool COH>
__device__ int search_layer(const VecView &vv, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip, const DevLayer &L,
                            bool layer0, int32_t enter, int ef, WarpScratch &ws, int32_t *cnt, bool &full, int lane) {
    ws.next_epoch(lane);
    const float ed = dist_one<DT, KMAX, COH>(vv, lc, qr, ip, layer0 ? enter : L.vrow[enter], ws, lane);
    MaxHeap W{ws.wbuf, 0};
    MinHeap C{ws.ctop, ws.ctail, 0, ws.ccap};
    if (lane == 0) {
        const Ent e{ed, enter};
        W.push(e);
        C.push(e);
        vis_insert(ws.vis, ws.vmask, ws.vshift, ws.epoch, enter);
    }
    __syncwarp();
    uint32_t nvis = 1;
    int64_t hops = 0;
    for (;;) {
        int32_t cid = -1;
        if (lane == 0 && C.len > 0) {
            const Ent c = C.pop();
            if (!(c.d > W.a[0].d)) cid = c.id;
        }
        cid = __shfl_sync(kFull, cid, 0);
        if (cid < 0) break;
        const int deg = L.deg[cid];
        const int64_t base = (int64_t)cid * L.cap;
        cnt[0]++;
        cnt[2] += deg;
        for (int j0 = 0; j0 < deg && !full; j0 += 32) {
            const int nn = take_new(L, layer0, base, j0, deg, ws, lane, full);
            dist_rows<DT, KMAX, COH>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, lane);
            __syncwarp();
            int over = 0;
            if (lane == 0) {
                for (int t = 0; t < nn; t++) {
                    const float d = ws.st->d[t];
                    if (W.len < ef || W.a[0].d > d) {
                        if (C.len >= C.cap || W.len >= ws.wcap) {
                            over = 1;
                            break;
                        }
                        const Ent e{d, ws.st->id[t]};
                        W.push(e);
                        C.push(e);
                        if (W.len > ef) W.pop();
                    }
                }
            }
            if (__shfl_sync(kFull, over, 0)) full = true;
            cnt[1] += nn;
            nvis += nn;
            if (nvis > ws.vlimit) full = true;
            __syncwarp();
        }
        if (full || ++hops > L.lcap) {
            full = true;
            break;
        }
    }
    int wl = W.len;
    wl = __shfl_sync(kFull, wl, 0);
    return wl;
}

}  // namespace dev
}  // namespace pk
