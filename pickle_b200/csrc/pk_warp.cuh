// Warp-level building blocks of the exact HNSW path, shared by the query
// kernel (pk_search.cu) and the insertion kernels (pk_build.cu).
//
// Reference behaviour reproduced here (juelinl/pickle):
//   Distance         include/distance.hpp:10-20, include/distance/avx512.hpp
//   EntryHeap        include/queue.hpp:99-289  (push / pop / tie order)
//   ByteMap          include/visited.hpp:248-297 (exact visited set)
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

// 16-byte asynchronous copy global -> shared (LDGSTS), bypassing L1.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Distances from the query in qr to nrows (<= 32) rows, staged through
// shared memory kStageRows rows at a time: every lane first issues
// asynchronous copies of exactly the chunks it will read (its group's rows,
// its chunk columns), so a batch of rows arrives in one memory round trip;
// then each group reduces its rows.  rowbuf holds kStageRows rows of
// row_bytes.  All lanes call it.
template <int DT, int KMAX>
__device__ __forceinline__ void dist_rows_staged(const VecView &g, const LaneCfg &lc, const uint4 (&qr)[KMAX],
                                                 bool ip, const int32_t *rows, float *outd, int nrows,
                                                 uint8_t *rowbuf, int lane) {
    typedef Acc<DT> A;
    const int G = lc.G, R = 32 / G, grp = lane / G, gl = lane % G;
    const int64_t rb = g.row_bytes;
    for (int b0 = 0; b0 < nrows; b0 += kStageRows) {
        const int nb = min(kStageRows, nrows - b0);
        for (int t = grp; t < nb; t += R) {
            const uint8_t *src = g.row(rows[b0 + t]);
            uint8_t *dst = rowbuf + (int64_t)t * rb;
#pragma unroll
            for (int k = 0; k < KMAX; k++) {
                const int c = gl + k * G;
                if (k < lc.K && c < lc.C) cp_async16(dst + c * 16, src + c * 16);
            }
        }
        cp_async_wait_all();
        for (int base = 0; base < nb; base += R) {
            const int t = base + grp;
            typename A::T acc = 0;
            if (t < nb) {
                const uint8_t *row = rowbuf + (int64_t)t * rb;
#pragma unroll
                for (int k = 0; k < KMAX; k++) {
                    const int c = gl + k * G;
                    if (k < lc.K && c < lc.C) A::add(acc, qr[k], *reinterpret_cast<const uint4 *>(row + c * 16), ip);
                }
            }
            for (int off = G >> 1; off > 0; off >>= 1) acc += A::shfl(acc, off);
            if (gl == 0 && t < nb) outd[b0 + t] = A::finish(acc, ip);
        }
    }
}

// ------------------------------------------------------------- visited set --
// An exact visited set per warp: a bitmap over the layer's node ids in global
// memory.  atomicOr marks a node and tells, in one round trip, whether it was
// marked before.  The ids marked during a layer search are listed, and the
// words they touched are zeroed when the search ends, so the next search
// starts from an empty set without clearing the whole bitmap (a list that
// overflowed clears the whole bitmap instead).

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
    uint32_t *bm;             // visited bitmap (global), bm_words words
    int64_t bm_words;
    int32_t *vlist;           // ids marked in the current layer search (global)
    int vl_cap;
    int vl_n;
    Ent *wbuf;                // result heap (shared), wcap entries
    int wcap;
    Ent *ctop;                // candidate heap, shared part
    Ent *ctail;               // candidate heap, global part
    int ccap;
    Stage *st;
    uint8_t *rowbuf;          // shared staging of 32 rows

    __device__ __forceinline__ void bind(const WarpGlobalScratch &g, int64_t gwarp) {
        bm = g.bitmap + gwarp * g.bm_words;
        bm_words = g.bm_words;
        vlist = g.vlist + gwarp * g.vl_cap;
        vl_cap = g.vl_cap;
        vl_n = 0;
        ctail = reinterpret_cast<Ent *>(g.cand_tail) + gwarp * g.cand_tail_cap;
        ccap = kCandTop + g.cand_tail_cap;
    }

    // One lane marks v (the entry of a layer search).
    __device__ __forceinline__ void mark_one(int32_t v) {
        atomicOr(bm + (v >> 5), 1u << (v & 31));
        if (vl_n < vl_cap) vlist[vl_n] = v;
    }

    // End of a layer search: unmark what was marked.  All lanes call it.
    __device__ __forceinline__ void end_layer(int lane) {
        __syncwarp();
        if (vl_n <= vl_cap) {
            for (int i = lane; i < vl_n; i += 32) bm[vlist[i] >> 5] = 0u;
        } else {
            for (int64_t i = lane; i < bm_words; i += 32) bm[i] = 0u;
        }
        vl_n = 0;
        __threadfence();
        __syncwarp();
    }
};

// One chunk (<= 32 entries) of an adjacency list: find the entries that are
// in range, first within the chunk and not yet visited; mark them; stage ids
// and vector rows.  Returns the count (warp-uniform).  Ids outside [0, lcap)
// are skipped (the reference would index its visited table out of range).
// v_pre: this lane's entry, already loaded (pass have_pre = true).
__device__ __forceinline__ int take_new(const DevLayer &L, bool layer0, int64_t base, int j0, int deg, WarpScratch &ws,
                                        int lane, bool have_pre, int32_t v_pre) {
    const int j = j0 + lane;
    int32_t v = -1;
    if (j < deg) v = have_pre ? v_pre : L.adj[base + j];
    const bool valid = j < deg && v >= 0 && (int64_t)v < L.lcap;
    const int key = valid ? v : -1 - lane;
    const unsigned peers = __match_any_sync(kFull, key);
    const bool first = valid && (__ffs(peers) - 1) == lane;
    bool is_new = false;
    if (first) {
        const uint32_t bit = 1u << (v & 31);
        is_new = (atomicOr(ws.bm + (v >> 5), bit) & bit) == 0;
    }
    const unsigned nm = __ballot_sync(kFull, is_new);
    if (is_new) {
        const int pos = __popc(nm & ((1u << lane) - 1));
        ws.st->id[pos] = v;
        ws.st->row[pos] = layer0 ? v : L.vrow[v];
        if (ws.vl_n + pos < ws.vl_cap) ws.vlist[ws.vl_n + pos] = v;
    }
    ws.vl_n += __popc(nm);
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
    float cd = dist_one<DT, KMAX, COH>(vv, lc, qr, ip, L.vrow[enter], ws, lane);
    int32_t c = enter;
    if (lane == 0) ws.mark_one(enter);
    ws.vl_n++;
    __syncwarp();
    bool updated;
    int64_t rounds = 0;
    do {
        updated = false;
        const int32_t cur = c;
        const int64_t base = (int64_t)cur * L.cap;
        const int32_t pre = lane < L.cap ? L.adj[base + lane] : -1;  // issued with the degree load
        const int deg = L.deg[cur];
        cnt[0]++;
        cnt[2] += deg;
        for (int j0 = 0; j0 < deg; j0 += 32) {
            const int nn = take_new(L, false, base, j0, deg, ws, lane, j0 == 0 && L.cap >= 32, pre);
            dist_rows_staged<DT, KMAX>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, ws.rowbuf, lane);
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
            __syncwarp();
        }
    } while (updated && ++rounds <= L.lcap);
    if (rounds > L.lcap) full = true;
    ws.end_layer(lane);
    return c;
}

// SearchLayer / SearchLayerFast (include/hnsw.hpp:304-444).  Leaves the
// result heap W in ws.wbuf and returns its length (warp-uniform).
// cnt[0..2] += hops, distance evaluations, neighbours scanned.
template <int DT, int KMAX, bool COH>
__device__ int search_layer(const VecView &vv, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip, const DevLayer &L,
                            bool layer0, int32_t enter, int ef, WarpScratch &ws, int32_t *cnt, bool &full, int lane) {
    const float ed = dist_one<DT, KMAX, COH>(vv, lc, qr, ip, layer0 ? enter : L.vrow[enter], ws, lane);
    MaxHeap W{ws.wbuf, 0};
    MinHeap C{ws.ctop, ws.ctail, 0, ws.ccap};
    if (lane == 0) {
        const Ent e{ed, enter};
        W.push(e);
        C.push(e);
        ws.mark_one(enter);
    }
    ws.vl_n++;
    __syncwarp();
    int64_t hops = 0;
    for (;;) {
        int32_t cid = -1;
        if (lane == 0 && C.len > 0) {
            const Ent c = C.pop();
            if (!(c.d > W.a[0].d)) cid = c.id;
        }
        cid = __shfl_sync(kFull, cid, 0);
        if (cid < 0) break;
        const int64_t base = (int64_t)cid * L.cap;
        const int32_t pre = lane < L.cap ? L.adj[base + lane] : -1;  // issued with the degree load
        const int deg = L.deg[cid];
        cnt[0]++;
        cnt[2] += deg;
        for (int j0 = 0; j0 < deg && !full; j0 += 32) {
            const int nn = take_new(L, layer0, base, j0, deg, ws, lane, j0 == 0 && L.cap >= 32, pre);
            dist_rows_staged<DT, KMAX>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, ws.rowbuf, lane);
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
            __syncwarp();
        }
        if (full || ++hops > L.lcap) {
            full = true;
            break;
        }
    }
    ws.end_layer(lane);
    int wl = W.len;
    wl = __shfl_sync(kFull, wl, 0);
    return wl;
}

}  // namespace dev
}  // namespace pk
