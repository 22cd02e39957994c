// Batched low-precision HNSW search with exact re-ranking.
//
// The exact kernel (pk_search.cu) replays the reference's binary heaps with
// one lane, which is what makes its ids bit-identical to the reference's but
// also what bounds it.  These kernels answer the same question - the k
// nearest neighbours found by a best-first walk of the HNSW graph with a
// result set of ef entries (include/hnsw.hpp:373-444) - with data structures
// suited to a warp, and are judged by recall.  Two kernels, a walk then a
// re-rank (with per-query ef: one of each per list width, on that width's
// own stream):
//
// walk_kernel (one query per warp, work stealing, per-query ef):
//   * traversal distances come from a low-precision copy of the vectors,
//     FP16 or FP8 E4M3 scaled per dimension (a query is scaled by the same
//     per-dimension factors), as dot products on the tensor cores; for L2
//     the row's norm turns the distance into a dot product (E4M3 rows carry
//     it after their values, FP16 rows get it from the same tensor-core
//     steps as the Gram diagonal of the staged rows);
//   * upper layers are descended greedily as in SlideLayer
//     (include/hnsw.hpp:446-494);
//   * on layer 0 the result set is a sorted list of ef entries held in
//     registers (lane l owns entries l*S .. l*S+S-1); each iteration expands
//     the `expand` best unexpanded entries, filters their neighbours through
//     a table of recently seen ids in shared memory (exact 16-bit tags in
//     4-way sets where the ids allow, least recently inserted out) and then,
//     for what that table does not hold, through a larger per-warp table in
//     global memory that stays in L2 (exact 16-bit tags in 8-way sets),
//     fetches the new rows with one bulk copy (cp.async.bulk) per row onto a
//     per-warp mbarrier, and inserts what beats the worst listed entry;
//   * the walk ends when the first ef entries are all expanded, and their
//     ids are written out.
//   The visited tables forget ids on collisions, which costs a recomputed
//   distance but never a duplicate: an insertion of an id the list holds is
//   dropped, and a node that left the list (or was turned away) cannot come
//   back, since the worst listed distance never rises.  So the list after
//   each step - the best ef of what was listed and what was met - does not
//   depend on the tables' sizes (or on whether the L2 table is used at all)
//   or on the batch order.
//
// rerank_kernel (one query per warp; all queries, or one list width's):
// exact distances from the original vectors for the ef listed ids, sorted by
// (distance, id); the k best are written with their external ids.
//
// There is no host round trip, so a batch can be captured in a CUDA graph.
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "pk_fast.h"
#include "pk_warp.cuh"

namespace pk {

namespace {

using namespace dev;


// ------------------------------------------------------- traversal distances
// Traversal formats; both walk with tensor-core dot products (trav_dist_buf)
// and stage the query in shared memory.
// FP16: rows and queries are stored divided by one power of two that brings
// the largest stored magnitude into [4, 8) (a power of two changes no
// rounding and no order of distances).
// FP8 E4M3: rows are stored divided by per-dimension scales (largest
// magnitude onto 448); a query is multiplied by the same scales, brought into
// E4M3's range by a power of two, and stored as two E4M3 parts - its rounding
// and the rounding of the remainder - which together recover a component to
// 0.04% (median; 0.2% at worst) where one part alone is off by 2%; the power
// of two is undone after the product.

struct TravView {
    const uint8_t *rows;      // traversal copy, row_bytes apart
    const uint8_t *zero_row;
    int32_t row_bytes;
    __device__ __forceinline__ const uint8_t *row(int32_t r) const {
        return r >= 0 ? rows + (int64_t)r * row_bytes : zero_row;
    }
};

// ------------------------------------------------------ asynchronous rows --
// Rows move from global to shared memory with one bulk copy per row, issued
// by as many lanes as there are rows and completing on a per-warp mbarrier
// that counts the bytes, with an L2 evict-first hint.  A warp waits once per
// batch of rows.

// Bound on the wait for one batch of rows: 2 s of the global timer (a batch
// lands in microseconds), checked every 64 polls.
constexpr uint64_t kWaitNs = 2000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_poll(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

struct RowFetch {
    uint8_t *buf;    // row t lands at buf + t * stride
    int32_t stride;
    uint64_t *bar;
    uint32_t parity;
};

// Copies rows[0..n) of the traversal copy (n >= 1; each a row index below the
// copy's row count, or -1 for the zero row) into f.buf.  All lanes call.  Returns false on
// every lane if the copies did not land within the time bound; the copies are
// then given one more bounded wait before returning.
__device__ __forceinline__ bool fetch_rows(RowFetch &f, const TravView &tv, const int32_t *rows, int n, int lane) {
    __syncwarp();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(f.bar)),
                     "r"((uint32_t)(n * tv.row_bytes))
                     : "memory");
    __syncwarp();
    // rows are read once per visit: marked first to leave L2, so that the
    // walks' visited tables (and the hot adjacency rows) stay there longer
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    for (int t = lane; t < n; t += 32) {
        const int32_t r = rows[t];
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
            "%4;" ::"r"(smem_u32(f.buf + t * f.stride)),
            "l"(tv.row(r)), "r"((uint32_t)tv.row_bytes), "r"(smem_u32(f.bar)), "l"(pol)
            : "memory");
    }
    bool ok = mbar_poll(f.bar, f.parity);
    if (!ok) {
        const uint64_t t0 = global_ns();
        for (int i = 1; !ok; i++) {
            ok = mbar_poll(f.bar, f.parity);
            if (!ok && (i & 63) == 0 && global_ns() - t0 > kWaitNs) break;
        }
    }
    const bool all = __all_sync(kFull, ok);
    if (!all && !ok) {
        const uint64_t t0 = global_ns();
        for (int i = 1; !ok; i++) {
            ok = mbar_poll(f.bar, f.parity);
            if (!ok && (i & 63) == 0 && global_ns() - t0 > kWaitNs) break;
        }
    }
    f.parity ^= 1u;
    __syncwarp();
    return all;
}

// One tensor-core step: the 16 staged rows' fragment a times the query's
// fragment (b0, b1), accumulated into c.  FP16: k = 16 elements; E4M3: k = 32.
template <int TRAV>
__device__ __forceinline__ void mma_step(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    if constexpr (TRAV == kTravF16)
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    else
        asm volatile(
            "mma.sync.aligned.m16n8k32.row.col.f32.e4m3.e4m3.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Traversal distances of the n staged rows to the query, into cd[t].  A row's
// values take data_bytes (whole 32-byte steps); for L2 in E4M3 its stored
// norm (float) follows them.  All lanes call.
//
// Sixteen staged rows at a time are the A operand of mma.m16n8k16 (FP16) or
// mma.m16n8k32 (E4M3): ldmatrix takes one row address per lane, so gathered
// rows need no particular layout, and a 32-byte step of a row is one k-step
// in both formats.  The query is column 0 of B (lanes 0-3 hold its fragment;
// B's other columns are zero), and column 0 of the FP32 accumulator holds the
// 16 dot products.  E4M3 puts the query's second part (data_bytes into the
// staged query) in column 1 (lanes 4-7), so one product per k-step yields
// both; a row's dot product is columns 0 + 1, scaled by qfac.
// L2 = |q|^2 + |x|^2 - 2 q.x.  E4M3 rows carry their norm (per-dimension
// scales make it no function of the stored codes alone).  FP16 rows are the
// values divided by one power of two, so |x|^2 in those units is the Gram
// diagonal of the staged rows: the A fragment registers of rows 0-7 (a[0],
// a[2]) and of rows 8-15 (a[1], a[3]) are, as they sit, the B fragments of
// those rows' transposes, and two more products per k-step give A A[0:8]^T
// and A A[8:16]^T, whose diagonals are the 16 norms - no norm bytes in the
// row and no extra load.
template <int TRAV>
__device__ __forceinline__ void trav_dist_buf(bool ip, float qnorm,
                                              float qfac, const RowFetch &f, int32_t data_bytes, const uint8_t *qbuf,
                                              float *cd, int n, int lane) {
    auto xnorm = [&](int t) { return *reinterpret_cast<const float *>(f.buf + t * f.stride + data_bytes); };
    const int ks = (int)(data_bytes / 32);
    const uint32_t *qw = reinterpret_cast<const uint32_t *>(qbuf);
    const int low = (int)(data_bytes / 4);  // E4M3: first word of the query's second part
    const bool gram = TRAV == kTravF16 && !ip;
    for (int t0 = 0; t0 < n; t0 += 16) {
        const int r = min(t0 + (lane & 15), n - 1);
        const uint32_t arow = smem_u32(f.buf + r * f.stride) + (uint32_t)(lane >> 4) * 16u;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        float g0[4] = {0.f, 0.f, 0.f, 0.f}, g1[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kk = 0; kk < ks; kk++) {
            uint32_t a[4];
            asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                         : "r"(arow + (uint32_t)kk * 32u)
                         : "memory");
            uint32_t b0 = 0, b1 = 0;
            if (TRAV == kTravF16 ? lane < 4 : lane < 8) {
                const int w = (TRAV == kTravE4M3 && lane >= 4 ? low : 0) + kk * 8 + (lane & 3);
                b0 = qw[w];
                b1 = qw[w + 4];
            }
            mma_step<TRAV>(c, a, b0, b1);
            if (gram) {
                mma_step<TRAV>(g0, a, a[0], a[2]);
                mma_step<TRAV>(g1, a, a[1], a[3]);
            }
        }
        // lane 4g + e of quad g holds columns 2e, 2e + 1 of rows g (c[0],
        // c[1]) and g + 8 (c[2], c[3]): the query's column 0 is at lane 4g;
        // the Gram diagonal of row g is column g of g0 (lane 4g + g/2,
        // element g % 2) and of row g + 8 column g of g1 (same lane, element
        // 2 + g % 2)
        const int g = lane >> 2;
        float na = 0.f, nb = 0.f;
        if (gram) {
            const float va = (g & 1) ? g0[1] : g0[0];
            const float vb = (g & 1) ? g1[3] : g1[2];
            na = __shfl_sync(kFull, va, 4 * g + (g >> 1));
            nb = __shfl_sync(kFull, vb, 4 * g + (g >> 1));
        }
        if ((lane & 3) == 0) {
            const int ra = t0 + g, rb = ra + 8;
            const float da = TRAV == kTravE4M3 ? (c[0] + c[1]) * qfac : c[0];
            const float db = TRAV == kTravE4M3 ? (c[2] + c[3]) * qfac : c[2];
            if (ra < n) cd[ra] = ip ? -da : qnorm + (gram ? na : xnorm(ra)) - 2.f * da;
            if (rb < n) cd[rb] = ip ? -db : qnorm + (gram ? nb : xnorm(rb)) - 2.f * db;
        }
    }
    __syncwarp();
}

// Appends this warp's new entries (lanes with ok, in lane order) to the
// pending batch crow/cid at n, flushing the batch whenever rb entries wait.
// Returns false if a flush failed.
template <class Flush>
__device__ __forceinline__ bool append_pending(bool ok, int32_t id, int32_t row, int32_t *crow, int32_t *cid, int &n,
                                               int rb, int lane, Flush &flush) {
    const unsigned m = __ballot_sync(kFull, ok);
    const int total = __popc(m);
    const int rank = __popc(m & ((1u << lane) - 1u));
    int done = 0;
    while (done < total) {
        if (n == rb) {
            __syncwarp();
            if (!flush(n)) return false;
            n = 0;
        }
        const int take = min(rb - n, total - done);
        if (ok && rank >= done && rank < done + take) {
            crow[n + rank - done] = row;
            cid[n + rank - done] = id;
        }
        n += take;
        done += take;
    }
    __syncwarp();
    return true;
}

// ----------------------------------------------------- recently-seen ids --
// Per-warp table in shared memory of 2^hlog2 id slots.  Exact 16-bit tags
// where they fit: the id is scrambled by a bijection of [0, 2^B) (odd
// multiplier, B = the ids' bits), the top bits pick a 4-way set of 8 bytes and
// the remaining B - (hlog2 - 2) <= 15 bits, plus one, are the tag - distinct
// ids never share a (set, tag), so a hit is always a real revisit.  Larger id
// spaces use 2-way sets of 32-bit ids.  Either way the most recent id goes
// first and the oldest of a full set is forgotten.
struct SeenTable {
    uint32_t *w;
    int words;        // 32-bit words of the table
    bool tag16;
    uint32_t bmask;   // tag16: 2^B - 1
    int tshift;       // tag16: B - set bits (the tag's width)
    int sshift;       // 32-bit ids: 33 - hlog2

    __device__ __forceinline__ void clear(int lane) {
        const int4 fill = tag16 ? make_int4(0, 0, 0, 0) : make_int4(-1, -1, -1, -1);
        for (int i = lane * 4; i < words; i += 128) *reinterpret_cast<int4 *>(w + i) = fill;
    }

    // Marks v as seen; true if it was not in the table.
    __device__ __forceinline__ bool test_and_mark(int32_t v) {
        if (tag16) {
            const uint32_t h = ((uint32_t)v * 2654435761u) & bmask;
            uint2 *set = reinterpret_cast<uint2 *>(w) + (h >> tshift);
            const uint32_t tag = (h & ((1u << tshift) - 1u)) + 1u;
            const uint2 x = *set;
            const uint32_t t2 = tag * 0x10001u;
            if ((__vcmpeq2(x.x, t2) | __vcmpeq2(x.y, t2)) != 0u) return false;
            *set = make_uint2((x.x << 16) | tag, (x.y << 16) | (x.x >> 16));
            return true;
        }
        int2 *set = reinterpret_cast<int2 *>(w) + (((uint32_t)v * 2654435769u) >> sshift);
        const int2 x = *set;
        if (x.x == v || x.y == v) return false;
        *set = make_int2(v, x.x);
        return true;
    }
};

// ------------------------------------------------------ visited ids in L2 --
// Second level of the visited filter, for ids the shared-memory table does
// not hold: a per-warp table in global memory of 2^log2sets sets of eight
// 16-bit tags (16 bytes, one load), cleared at the start of each query and
// sized by the list width to hold the ids a walk of that width meets (a few
// to a few tens of KB per warp: the resident warps' tables stay in L2).  Tags
// are exact as in the shared-memory table: the scrambled id's top bits pick
// the set and its remaining tbits (<= 15), plus one, are the tag, so a hit is
// always a real revisit; a full set forgets its oldest id.  Lanes of a warp
// that update one set at once may lose one of the two ids (a recomputed
// distance later, never a wrong answer).
struct L2Seen {
    uint4 *sets;      // this warp's table, or null
    int nsets;
    uint32_t bmask;
    int tbits;

    // the set index of v, and its tag
    __device__ __forceinline__ uint32_t set_of(int32_t v, uint32_t &tag) const {
        const uint32_t h = ((uint32_t)v * 2654435761u) & bmask;
        tag = (h & ((1u << tbits) - 1u)) + 1u;
        return h >> tbits;
    }
};

__device__ __forceinline__ uint4 ld_cg4(const uint4 *p) {
    uint4 r;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p)
                 : "memory");
    return r;
}
__device__ __forceinline__ void st_cg4(uint4 *p, uint4 v) {
    asm volatile("st.global.cg.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}
__device__ __forceinline__ bool set_has(uint4 x, uint32_t tag) {
    const uint32_t t2 = tag * 0x10001u;
    return (__vcmpeq2(x.x, t2) | __vcmpeq2(x.y, t2) | __vcmpeq2(x.z, t2) | __vcmpeq2(x.w, t2)) != 0u;
}
// the newest tag first; the oldest of eight falls off
__device__ __forceinline__ uint4 set_push(uint4 x, uint32_t tag) {
    return make_uint4((x.x << 16) | tag, __funnelshift_l(x.x, x.y, 16), __funnelshift_l(x.y, x.z, 16),
                      __funnelshift_l(x.z, x.w, 16));
}

// Two candidates per lane that passed the shared-memory table (ids >= 0; -1 =
// none): both sets are loaded before either is tested, so the warp waits for
// one round trip.  An id the table holds already becomes -1; the others are
// added to it.
__device__ __forceinline__ void l2_filter2(const L2Seen &vt, int32_t &va, int32_t &vb) {
    uint32_t ta = 0, tb = 0, ia = 0, ib = 0xffffffffu;
    uint4 xa = make_uint4(0, 0, 0, 0), xb = xa;
    if (va >= 0) {
        ia = vt.set_of(va, ta);
        xa = ld_cg4(vt.sets + ia);
    }
    if (vb >= 0) {
        ib = vt.set_of(vb, tb);
        xb = ld_cg4(vt.sets + ib);
    }
    if (va >= 0) {
        if (set_has(xa, ta)) {
            va = -1;
        } else {
            xa = set_push(xa, ta);
            st_cg4(vt.sets + ia, xa);
            if (ib == ia) xb = xa;  // b's set is the one just written
        }
    }
    if (vb >= 0) {
        if (set_has(xb, tb)) vb = -1;
        else st_cg4(vt.sets + ib, set_push(xb, tb));
    }
}

// ------------------------------------------------------------ result list --
// The ef best entries found so far, sorted by (distance, id), in registers:
// lane l holds positions l*S .. l*S+S-1 of 32*S, and the list takes the last
// ef of them, so that its ef-th entry - the bar a candidate must beat - is
// always lane 31's last slot.  A distance is held as an unsigned key of the
// same order (dist_key), so that (distance, id) compares as one 64-bit
// integer.  The positions before the list hold key 0 (below every distance):
// they count into each rank and never move.  Empty slots of the list hold
// (kEmpty, kEmpty), above every entry.  Bit s of a lane's mask xm is set when
// slot s cannot be expanded: its entry was expanded already, or the slot is
// empty or before the list.  Keeping the marks in one word per lane (not in
// the ids) makes finding the next entry to expand two bit operations and a
// ballot, and leaves the ids as they are for the compares.

constexpr uint32_t kEmpty = 0xffffffffu;
__device__ __forceinline__ bool key_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (da == db && ia < ib);
}

// A finite or infinite distance as an unsigned key in the same order, -0
// taken as +0 (the two compare equal as floats): positive values gain the top
// bit, negative ones are inverted.  Keys of distances lie in
// [0x007fffff, 0xff800000]: 0 and kEmpty stay free for the list's bounds.
__device__ __forceinline__ uint32_t dist_key(float d) {
    uint32_t u = __float_as_uint(d);
    u = u == 0x80000000u ? 0u : u;
    return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);
}

__device__ __forceinline__ uint64_t pack_key(uint32_t key, uint32_t id) { return ((uint64_t)key << 32) | id; }

template <int S>
struct RegList {
    static constexpr uint32_t kSlots = S >= 32 ? 0xffffffffu : (1u << S) - 1u;
    uint32_t k[S];
    uint32_t id[S];
    uint32_t xm;

    // An empty list of the last L of the 32*S positions.
    __device__ __forceinline__ void clear(int L, int lane) {
        const int p0 = 32 * S - L;
#pragma unroll
        for (int s = 0; s < S; s++) {
            k[s] = lane * S + s < p0 ? 0u : kEmpty;
            id[s] = kEmpty;
        }
        xm = kSlots;
    }

    // The first position of an empty list of L: the entry point (not yet
    // expanded).  The slot is chosen at run time, so every slot is written
    // through a mask: a branch on (s == slot) lets the compiler fold the
    // unrolled writes back into one store at a run-time index, which moves
    // the whole list out of registers into local memory.
    __device__ __forceinline__ void put_first(int L, uint32_t nk, uint32_t nid, int lane) {
        const int p0 = 32 * S - L;
        if (lane == p0 / S) {
#pragma unroll
            for (int s = 0; s < S; s++) {
                const uint32_t m = 0u - (uint32_t)(s == p0 % S);
                k[s] ^= (k[s] ^ nk) & m;
                id[s] ^= (id[s] ^ nid) & m;
            }
            xm &= ~(1u << (p0 % S));
        }
    }

    // Inserts (nk, nid) at its rank, unexpanded, unless the list holds nid
    // already; the last entry of the 32*S falls off.
    __device__ __forceinline__ void insert(uint32_t nk, uint32_t nid, int lane) {
        const uint64_t x = pack_key(nk, nid);
        // one bit per slot below the new entry (a prefix: the slots are
        // sorted) and per slot holding its id, folded by OR trees so that
        // the rank is a popcount, not a chain of S dependent adds
        uint32_t lt[S], eq[S];
#pragma unroll
        for (int s = 0; s < S; s++) {
            lt[s] = pack_key(k[s], id[s]) < x ? (1u << s) : 0u;
            eq[s] = id[s] == nid ? 1u : 0u;
        }
#pragma unroll
        for (int w = 1; w < S; w <<= 1)
#pragma unroll
            for (int s = 0; s + w < S; s += 2 * w) {
                lt[s] |= lt[s + w];
                eq[s] |= eq[s + w];
            }
        if (__any_sync(kFull, eq[0] != 0u)) return;
        const int c = __popc(lt[0]);
        // sorted: lanes before the rank have c == S, lanes after it c == 0
        const uint32_t pk = __shfl_up_sync(kFull, k[S - 1], 1);
        const uint32_t pi = __shfl_up_sync(kFull, id[S - 1], 1);
        const int pc = __shfl_up_sync(kFull, c, 1);
        const uint32_t pb = __shfl_up_sync(kFull, xm >> (S - 1), 1) & 1u;
        const bool here = c > 0 || lane == 0 || pc == S;  // the new entry lands in slot c of this lane
        const uint32_t ck = here ? nk : pk, ci = here ? nid : pi;
        // slots above c shift up one, slot c takes the entry; a lane with
        // c == S keeps all its slots
#pragma unroll
        for (int s = S - 1; s >= 0; s--) {
            if (s > 0 && s > c) {
                k[s] = k[s - 1];
                id[s] = id[s - 1];
            } else if (s == c) {
                k[s] = ck;
                id[s] = ci;
            }
        }
        // the marks move with their entries: slots below c stay, slots above
        // shift up one, slot c takes the new entry's (clear) or the previous
        // lane's last mark
        const uint32_t bitc = c < 32 ? 1u << c : 0u;
        const uint32_t low = bitc - 1u;
        xm = ((xm & low) | ((xm << 1) & ~(low | bitc)) | (here || pb == 0u ? 0u : bitc)) & kSlots;
    }

    // Merges a chunk's winners - the lanes with win, each (nk, nid) below the
    // list's last entry when the chunk was taken - into the list at once.
    // The list after it is the one inserting them one by one would leave:
    // the best 32*S of the list and the winners, an entry the list holds
    // already (same id, hence the same traversal distance and key) taken
    // once with its expanded mark, new entries unexpanded.
    //   1. the winners are sorted across the lanes (bitonic, 64-bit keys);
    //   2. the list is staged in shared memory (position p = l*S + s at
    //      s*32 + l: consecutive lanes, consecutive words) with its marks;
    //   3. each winner finds its rank r in the list by binary search, and is
    //      dropped if the entry at r is itself (or the previous winner is);
    //   4. the j-th kept winner lands at r + j; each lane gathers its S new
    //      slots: a winner's destination takes that winner, any other slot o
    //      the list entry at o minus the winners landed before o.
    // sm: walk_merge_bytes(S) bytes of shared memory, free during the call.
    __device__ __forceinline__ void merge(bool win, uint32_t nk, uint32_t nid, unsigned char *sm, int lane) {
        uint64_t *lst = reinterpret_cast<uint64_t *>(sm);  // 32 * S
        uint64_t *wv = lst + 32 * S;                       // 32 winners
        uint32_t *dm = reinterpret_cast<uint32_t *>(wv + 32);  // destination masks
        uint32_t *mk = dm + 32;                             // expanded marks
        uint64_t x = win ? pack_key(nk, nid) : ~0ull;
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                const uint64_t y = __shfl_xor_sync(kFull, x, j);
                const bool lower = (lane & j) == 0, up = (lane & kk) == 0;
                x = (lower == up) == (y < x) ? y : x;
            }
        }
        const int w = __popc(__ballot_sync(kFull, win));
#pragma unroll
        for (int s = 0; s < S; s++) lst[s * 32 + lane] = pack_key(k[s], id[s]);
        mk[lane] = xm;
        dm[lane] = 0u;
        const uint64_t prev = __shfl_up_sync(kFull, x, 1);
        __syncwarp();
        bool keep = lane < w && (lane == 0 || prev != x);
        int r = 0;
        if (keep) {
            int lo = 0, hi = 32 * S;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (lst[(mid % S) * 32 + mid / S] < x) lo = mid + 1;
                else hi = mid;
            }
            r = lo;
            if (r < 32 * S && lst[(r % S) * 32 + r / S] == x) keep = false;
        }
        const unsigned km = __ballot_sync(kFull, keep);
        if (km == 0u) return;
        const int dst = r + __popc(km & ((1u << lane) - 1u));
        if (keep) {
            wv[__popc(km & ((1u << lane) - 1u))] = x;
            if (dst < 32 * S) atomicOr(dm + dst / S, 1u << (dst % S));
        }
        __syncwarp();
        const uint32_t my = dm[lane];
        // winners landing before this lane's first slot
        int before = __popc(my);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, before, o);
            if (lane >= o) before += t;
        }
        before -= __popc(my);
        uint32_t nm = 0u;
#pragma unroll
        for (int s = 0; s < S; s++) {
            uint64_t v;
            uint32_t mark;
            if ((my >> s) & 1u) {
                v = wv[before];
                mark = 0u;
                before++;
            } else {
                const int p = lane * S + s - before;
                v = lst[(p % S) * 32 + p / S];
                mark = (mk[p / S] >> (p % S)) & 1u;
            }
            k[s] = (uint32_t)(v >> 32);
            id[s] = (uint32_t)v;
            nm |= mark << s;
        }
        xm = nm & kSlots;
        __syncwarp();
    }

    // Marks the first expandable entry as expanded and returns its id, or -1
    // if there is none.
    __device__ __forceinline__ int32_t take_first(int lane) {
        const unsigned un = ~xm & kSlots;
        const unsigned b = __ballot_sync(kFull, un != 0);
        if (b == 0) return -1;
        const int fl = __ffs(b) - 1;
        int32_t v = 0;
        if (lane == fl) {
            const int fs = __ffs(un) - 1;
            // masked, like put_first: no read at a run-time index
#pragma unroll
            for (int s = 0; s < S; s++) v |= (int32_t)(id[s] & (0u - (uint32_t)(s == fs)));
            xm |= 1u << fs;
        }
        return __shfl_sync(kFull, v, fl);
    }

    // The list's last entry (its ef-th) as a packed key.
    __device__ __forceinline__ uint64_t last() const {
        return pack_key(__shfl_sync(kFull, k[S - 1], 31), __shfl_sync(kFull, id[S - 1], 31));
    }
};

// Argmin over (cd[t], t), t < n: the first of the smallest distances.
__device__ __forceinline__ void warp_argmin(const float *cd, int n, float &bd, int &bt, int lane) {
    float d = __int_as_float(0x7f800000);
    int t = 0x7fffffff;
    for (int i = lane; i < n; i += 32) {
        const float x = cd[i];
        if (x < d) {
            d = x;
            t = i;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float od = __shfl_xor_sync(kFull, d, off);
        const int ot = __shfl_xor_sync(kFull, t, off);
        if (od < d || (od == d && ot < t)) {
            d = od;
            t = ot;
        }
    }
    bd = d;
    bt = t;
}

// ------------------------------------------------------------------ walk ---
// Registers per thread that each instantiation is compiled for: 80 (24 warps
// per SM) up to 8 slots per lane (ef <= 256) except FP8 with four parents,
// where the list and the rest fit without spills (ptxas -v); 128 (16 warps)
// for wider lists.  At 12 and 16 slots the 80-register build spills, and 128
// registers measured 11-15% faster than 80 on 2M x 128 FP16 rows (ef = 384,
// 512) and 2-10% faster than 88 or 96 (which fit without spills, 20-22 warps).
constexpr int walk_max_regs(int trav, int s, int exp) {
    return s <= 4 ? 80 : (s <= 8 && (trav == kTravF16 || exp == 1)) ? 80 : 128;
}

// EXP bounds the parents expanded per step: the walk with one parent per
// step (the default) has its own instantiation, a quarter of the layer-0
// loop's code of the one that takes up to four.
template <int TRAV, int S, int EXP>
__global__ void __maxnreg__(walk_max_regs(TRAV, S, EXP))
    walk_kernel(const DevGraph *__restrict__ gp, const WalkArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const WalkLayout lay = walk_layout(a.rb, a.trav_row_bytes, a.tq_row_bytes, a.hlog2, a.tag16 != 0, S);
    unsigned char *my = smem + (size_t)wib * lay.total;
    SeenTable seen;
    seen.w = reinterpret_cast<uint32_t *>(my + lay.tab);
    seen.tag16 = a.tag16 != 0;
    seen.words = seen.tag16 ? (1 << (a.hlog2 - 1)) : (1 << a.hlog2);
    seen.bmask = a.idbits >= 32 ? 0xffffffffu : (1u << a.idbits) - 1u;
    seen.tshift = a.idbits - (a.hlog2 - 2);
    seen.sshift = 33 - a.hlog2;
    int32_t *crow = reinterpret_cast<int32_t *>(my + lay.crow);
    int32_t *cid = reinterpret_cast<int32_t *>(my + lay.cid);
    float *cd = reinterpret_cast<float *>(my + lay.cd);
    uint64_t *bar = reinterpret_cast<uint64_t *>(my + lay.bar);
    if (lane == 0) mbar_init(bar);
    __syncwarp();
    uint8_t *qbuf = my + lay.qbuf;
    RowFetch f{my + lay.rowbuf, (int32_t)lay.stride, bar, 0u};
    L2Seen vt;
    vt.nsets = 1 << a.vt_log2sets;
    vt.sets = a.vt ? reinterpret_cast<uint4 *>(a.vt) +
                         ((int64_t)(blockIdx.x * (blockDim.x >> 5) + wib) << a.vt_log2sets)
                   : nullptr;
    vt.bmask = a.vt_bmask;
    vt.tbits = a.vt_tbits;

    const TravView tv{a.trav, a.trav_zero, (int32_t)a.trav_row_bytes};
    const bool ip = gp->metric == PK_METRIC_IP;
    const int32_t tdb = (int32_t)a.trav_data_bytes;
    const int enter_level = gp->enter_level;
    const int rb = a.rb;
    const int expand = max(1, min(a.expand, EXP));
    const DevLayer L0 = gp->L[0];
    const int32_t lim0 = (int32_t)min(L0.lcap, a.trav_rows);
    const int32_t cap0 = (int32_t)L0.cap;
    const float kInf = __int_as_float(0x7f800000);

    const int64_t nlim = a.qcount ? (int64_t)*a.qcount : a.nq;
    for (;;) {
        int qi = 0;
        if (lane == 0) qi = atomicAdd(a.work, 1);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= nlim) break;
        const int64_t q = a.qlist ? a.qlist[qi] : qi;
        const int L = max(1, min(a.ef_arr ? a.ef_arr[q] : a.ef, 32 * S));

        // the query in the traversal format, staged in shared memory
        const float qnorm = ip ? 0.f : a.qnorm[q];
        float qfac = 1.f;
        {
            const uint8_t *qrow = a.tq_rows + q * a.tq_row_bytes;
            for (int c = lane; c < (int)(a.tq_row_bytes / 16); c += 32)
                reinterpret_cast<uint4 *>(qbuf)[c] = ld16(qrow + c * 16);
            __syncwarp();
            if (TRAV == kTravE4M3) qfac = *reinterpret_cast<const float *>(qbuf + 2 * a.trav_data_bytes);
        }

        int32_t cnt[6] = {0, 0, 0, 0, 0, 0};
        bool failed = false;

        // ---- upper layers: greedy descent with traversal distances ----
        int32_t enter = gp->L[enter_level].ent;
        for (int level = enter_level; level >= 1 && !failed; --level) {
            const DevLayer Ly = gp->L[level];
            auto vrow = [&](int32_t v) -> int32_t {
                const int32_t r = Ly.vrow[v];
                return r < a.trav_rows ? r : -1;
            };
            if (lane == 0) crow[0] = vrow(enter);
            if (!fetch_rows(f, tv, crow, 1, lane)) {
                failed = true;
                break;
            }
            trav_dist_buf<TRAV>(ip, qnorm, qfac, f, tdb, qbuf, cd, 1, lane);
            float best = cd[0];
            int32_t c = enter;
            bool moved = false;
            auto flush_up = [&](int nn) -> bool {
                if (!fetch_rows(f, tv, crow, nn, lane)) return false;
                trav_dist_buf<TRAV>(ip, qnorm, qfac, f, tdb, qbuf, cd, nn, lane);
                float bd;
                int bt;
                warp_argmin(cd, nn, bd, bt, lane);
                if (bd < best) {
                    best = bd;
                    c = cid[bt];
                    moved = true;
                }
                cnt[1] += nn;
                __syncwarp();
                return true;
            };
            for (int64_t round = 0; round <= Ly.lcap; round++) {
                const int64_t base = (int64_t)c * Ly.cap;
                const int deg = Ly.deg[c];
                cnt[0]++;
                cnt[2] += deg;
                moved = false;
                int n = 0;
                for (int j0 = 0; j0 < deg && !failed; j0 += 32) {
                    const int j = j0 + lane;
                    const int32_t v = j < deg ? Ly.adj[base + j] : -1;
                    const bool ok = v >= 0 && v < Ly.lcap;
                    const int32_t r = ok ? vrow(v) : -1;
                    if (!append_pending(ok, v, r, crow, cid, n, rb, lane, flush_up)) failed = true;
                }
                if (!failed && n > 0 && !flush_up(n)) failed = true;
                if (failed || !moved) break;
            }
            const int32_t dn = Ly.down[c];
            enter = dn >= 0 ? dn : gp->L[level - 1].ent;
        }

        // the upper layers' counters go out now: fewer registers live below
        if (a.counters && lane == 0) {
            int32_t *cp = a.counters + q * 6;
            cp[0] = cnt[0];
            cp[1] = cnt[1];
            cp[2] = cnt[2];
        }

        // ---- layer 0: best-first walk over the register list ----
        RegList<S> list;
        list.clear(L, lane);
        uint64_t wk = pack_key(kEmpty, kEmpty);
        if (!failed) {
            seen.clear(lane);
            if (vt.sets)
                for (int i = lane; i < vt.nsets; i += 32) st_cg4(vt.sets + i, make_uint4(0, 0, 0, 0));
            __syncwarp();
            if (enter < 0 || enter >= lim0) enter = 0;
            if (lane == 0) crow[0] = enter;
            if (!fetch_rows(f, tv, crow, 1, lane)) failed = true;
        }
        if (!failed) {
            trav_dist_buf<TRAV>(ip, qnorm, qfac, f, tdb, qbuf, cd, 1, lane);
            const float d0 = cd[0];
            list.put_first(L, dist_key(d0), (uint32_t)enter, lane);
            if (lane == 0) {
                seen.test_and_mark(enter);
                if (vt.sets) {
                    uint32_t tag;
                    uint4 *p = vt.sets + vt.set_of(enter, tag);
                    st_cg4(p, set_push(ld_cg4(p), tag));
                }
            }
            __syncwarp();
            wk = list.last();
        }
        auto flush0 = [&](int nn) -> bool {
            if (!fetch_rows(f, tv, crow, nn, lane)) return false;
            trav_dist_buf<TRAV>(ip, qnorm, qfac, f, tdb, qbuf, cd, nn, lane);
            cnt[4] += nn;
            for (int i0 = 0; i0 < nn; i0 += 32) {
                const int i = i0 + lane;
                uint32_t nk = kEmpty, nid = kEmpty;
                bool ok = false;
                if (i < nn) {
                    const float nd = cd[i];
                    nk = dist_key(nd);
                    nid = (uint32_t)crow[i];
                    ok = nd < kInf;
                }
                unsigned m = __ballot_sync(kFull, ok && pack_key(nk, nid) < wk);
                if constexpr (S >= kMergeMinSlots) {
                    if (__popc(m) >= a.merge_min) {
                        list.merge((m >> lane) & 1u, nk, nid, f.buf, lane);
                        wk = list.last();
                        m = 0u;
                    }
                }
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t xk = __shfl_sync(kFull, nk, src);
                    const uint32_t xi = __shfl_sync(kFull, nid, src);
                    if (!(pack_key(xk, xi) < wk)) continue;
                    list.insert(xk, xi, lane);
                    wk = list.last();
                }
            }
            __syncwarp();
            return true;
        };
        int32_t iters = 0;
        while (!failed) {
            int32_t pc[4];
#pragma unroll
            for (int p = 0; p < 4; p++) pc[p] = p < EXP && p < expand ? list.take_first(lane) : -1;
            if (pc[0] < 0 || ++iters > lim0) break;
            // degrees and the first 64 slots of each parent's list, all in flight
            int pdeg[4];
            int32_t pa0[4], pa1[4];
#pragma unroll
            for (int p = 0; p < EXP; p++) {
                pdeg[p] = 0;
                pa0[p] = -1;
                pa1[p] = -1;
                if (pc[p] >= 0) {
                    const int64_t base = (int64_t)pc[p] * cap0;
                    pdeg[p] = L0.deg[pc[p]];
                    if (lane < cap0) pa0[p] = L0.adj[base + lane];
                    if (32 + lane < cap0) pa1[p] = L0.adj[base + 32 + lane];
                }
            }
            int n = 0;
#pragma unroll
            for (int p = 0; p < EXP; p++) {
                if (pc[p] < 0 || failed) continue;
                const int deg = pdeg[p];
                const int64_t base = (int64_t)pc[p] * cap0;
                cnt[3]++;
                cnt[5] += deg;
                // 64 neighbour slots at a time, two per lane: the shared-memory
                // table first, then (for what it does not hold) the table in
                // L2, both sets loaded before either is tested
                for (int j0 = 0; j0 < deg; j0 += 64) {
                    const int ja = j0 + lane, jb = ja + 32;
                    int32_t va = -1, vb = -1;
                    if (ja < deg) va = (j0 == 0 && ja < cap0) ? pa0[p] : L0.adj[base + ja];
                    if (jb < deg) vb = (j0 == 0 && jb < cap0) ? pa1[p] : L0.adj[base + jb];
                    if (!(va >= 0 && va < lim0 && seen.test_and_mark(va))) va = -1;
                    if (!(vb >= 0 && vb < lim0 && seen.test_and_mark(vb))) vb = -1;
                    if (vt.sets) l2_filter2(vt, va, vb);
                    // one site appends (and flushes) both halves: the flush's
                    // code is inlined once here
#pragma unroll 1
                    for (int h2 = 0; h2 < 2 && j0 + 32 * h2 < deg; h2++) {
                        const int32_t v = h2 == 0 ? va : vb;
                        if (!append_pending(v >= 0, v, v, crow, cid, n, rb, lane, flush0)) {
                            failed = true;
                            break;
                        }
                    }
                    if (failed) break;
                }
            }
            if (!failed && n > 0 && !flush0(n)) failed = true;
        }
        if (failed) {
            if (lane == 0) atomicExch(a.status, 1);
            return;
        }

        int32_t *out = a.cand + q * a.cand_stride;
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int i = lane * S + s - (32 * S - L);
            if (i >= 0) out[i] = list.id[s] == kEmpty ? -1 : (int32_t)list.id[s];
        }
        if (a.counters && lane == 0) {
            int32_t *cp = a.counters + q * 6;
            cp[3] = cnt[3];
            cp[4] = cnt[4];
            cp[5] = cnt[5];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- rerank ---
// Bitonic sort of n (power of two) entries in shared memory by (distance, id).
__device__ __forceinline__ void smem_sort(float *d, uint32_t *id, int n, int lane) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < n / 2; i += 32) {
                const int lo = 2 * i - (i & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const float dl = d[lo], dh = d[hi];
                const uint32_t il = id[lo], ih = id[hi];
                const bool swap = up ? key_less(dh, ih, dl, il) : key_less(dl, il, dh, ih);
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

template <int DT, int KMAX>
__global__ void __launch_bounds__(128)
    rerank_kernel(const DevGraph *__restrict__ gp, const LaneCfg lc, const RerankArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int cap = a.cand_cap > 0 ? a.cand_cap : a.cand_stride;
    const RerankLayout lay = rerank_layout(cap, a.row_bytes);
    unsigned char *my = smem + (size_t)wib * lay.total;
    Stage *st = reinterpret_cast<Stage *>(my);
    float *sd = reinterpret_cast<float *>(my + lay.sd);
    uint32_t *sid = reinterpret_cast<uint32_t *>(my + lay.sid);
    uint8_t *rowbuf = my + lay.rowbuf;
    const VecView vv{gp->vec0, gp->zero_row, gp->row_bytes};
    const bool ip = gp->metric == PK_METRIC_IP;
    const bool walk_failed = *a.status != 0;
    const int64_t nlim = a.qcount ? (int64_t)*a.qcount : a.nq;
    for (int64_t i = (int64_t)blockIdx.x * wpb + wib; i < nlim; i += (int64_t)gridDim.x * wpb) {
        const int64_t q = a.qlist ? a.qlist[i] : i;
        const int k = max(0, min(a.k_arr ? a.k_arr[q] : a.k, a.out_stride));
        const int L = max(1, min(a.ef_arr ? a.ef_arr[q] : a.ef, cap));
        int32_t *oid = a.out_ids + q * a.out_stride;
        float *od = a.out_dists + q * a.out_stride;
        if (walk_failed) {
            // no result rather than a stale one
            for (int i = lane; i < k; i += 32) {
                oid[i] = -1;
                od[i] = FLT_MAX;
            }
            continue;
        }
        uint4 qr[KMAX];
        load_regs<KMAX>(qr, a.queries + q * vv.row_bytes, lc, lane, false);
        const int32_t *cl = a.cand + q * a.cand_stride;
        for (int b0 = 0; b0 < L; b0 += 32) {
            const int nn = min(32, L - b0);
            int32_t r = -1;
            if (lane < nn) {
                r = cl[b0 + lane];
                st->row[lane] = r;
            }
            __syncwarp();
            dist_rows_staged<DT, KMAX>(vv, lc, qr, ip, st->row, st->d, nn, rowbuf, lane);
            __syncwarp();
            if (lane < nn) {
                sd[b0 + lane] = r >= 0 ? st->d[lane] : FLT_MAX;
                sid[b0 + lane] = r >= 0 ? (uint32_t)r : 0x7fffffffu;
            }
            __syncwarp();
        }
        int n2 = 1;
        while (n2 < L) n2 <<= 1;
        for (int i = L + lane; i < n2; i += 32) {
            sd[i] = FLT_MAX;
            sid[i] = 0x7fffffffu;
        }
        __syncwarp();
        smem_sort(sd, sid, n2, lane);
        for (int i = lane; i < k; i += 32) {
            const bool have = i < L && sid[i] != 0x7fffffffu;
            oid[i] = have ? a.ext0[sid[i]] : -1;
            od[i] = have ? sd[i] : FLT_MAX;
        }
        __syncwarp();
    }
}

// Queries by list slots per lane: a walk launch per class then pays for the
// list width its queries need, not the batch's widest.
__global__ void bin_by_slots_kernel(const int32_t *ef_arr, int32_t ef_bound, int64_t nq, int32_t *counts,
                                    int32_t *lists) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (int64_t)gridDim.x * blockDim.x) {
        const int ef = max(1, min(ef_arr[q], ef_bound));
        const int c = slot_class(ef);
        const int pos = atomicAdd(counts + c, 1);
        lists[(int64_t)c * nq + pos] = (int32_t)q;
    }
}

// ------------------------------------------------------------ dispatch -----
template <int TRAV, int EXP>
void *walk_pick_s(int s) {
    switch (s) {
        case 1: return (void *)walk_kernel<TRAV, 1, EXP>;
        case 2: return (void *)walk_kernel<TRAV, 2, EXP>;
        case 3: return (void *)walk_kernel<TRAV, 3, EXP>;
        case 4: return (void *)walk_kernel<TRAV, 4, EXP>;
        case 6: return (void *)walk_kernel<TRAV, 6, EXP>;
        case 8: return (void *)walk_kernel<TRAV, 8, EXP>;
        case 12: return (void *)walk_kernel<TRAV, 12, EXP>;
        case 16: return (void *)walk_kernel<TRAV, 16, EXP>;
        case 24: return (void *)walk_kernel<TRAV, 24, EXP>;
        case 32: return (void *)walk_kernel<TRAV, 32, EXP>;
        default: return nullptr;
    }
}
void *walk_kernel_ptr(int trav, int s, int expand) {
    if (trav == kTravF16) return expand > 1 ? walk_pick_s<kTravF16, 4>(s) : walk_pick_s<kTravF16, 1>(s);
    if (trav == kTravE4M3) return expand > 1 ? walk_pick_s<kTravE4M3, 4>(s) : walk_pick_s<kTravE4M3, 1>(s);
    return nullptr;
}

template <int DT>
void *rerank_pick(int kmax) {
    switch (kmax) {
        case 1: return (void *)rerank_kernel<DT, 1>;
        case 2: return (void *)rerank_kernel<DT, 2>;
        case 4: return (void *)rerank_kernel<DT, 4>;
        case 8: return (void *)rerank_kernel<DT, 8>;
        default: return nullptr;
    }
}
void *rerank_kernel_ptr(int dtype, int kmax) {
    switch (dtype) {
        case PK_DTYPE_U8: return rerank_pick<PK_DTYPE_U8>(kmax);
        case PK_DTYPE_I8: return rerank_pick<PK_DTYPE_I8>(kmax);
        case PK_DTYPE_F32: return rerank_pick<PK_DTYPE_F32>(kmax);
        case PK_DTYPE_F16: return rerank_pick<PK_DTYPE_F16>(kmax);
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

// Rows [r0, r1) of vec0 into the traversal copy (divided by the scales) and
// the per-row sum of squares of the stored values (into rownorm and, with
// norm_off >= 0, into the row at that byte).  One block per row.
template <int DT, int TRAV>
__global__ void convert_rows_kernel(const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1, int dim,
                                    const float *scale, uint8_t *trav, int64_t trav_row_bytes, int64_t norm_off,
                                    float *rownorm) {
    __shared__ float red[32];
    for (int64_t r = r0 + blockIdx.x; r < r1; r += gridDim.x) {
        const uint8_t *row = vec0 + r * row_bytes;
        uint8_t *out = trav + r * trav_row_bytes;
        float part = 0.f;
        for (int d = threadIdx.x; d < dim; d += blockDim.x) {
            const float v = elem<DT>(row, d);
            float back;
            if constexpr (TRAV == kTravF16) {
                const __half h = __float2half_rn(v / scale[d]);
                reinterpret_cast<__half *>(out)[d] = h;
                back = __half2float(h);
            } else {
                const __nv_fp8_storage_t x = __nv_cvt_float_to_fp8(v / scale[d], __NV_SATFINITE, __NV_E4M3);
                out[d] = x;
                back = __half2float(__half(__nv_cvt_fp8_to_halfraw(x, __NV_E4M3))) * scale[d];
            }
            part += back * back;
        }
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(kFull, part, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            float sum = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += red[w];
            rownorm[r] = sum;
            if (norm_off >= 0) *reinterpret_cast<float *>(out + norm_off) = sum;
        }
        __syncthreads();
    }
}

// Queries into the traversal format (rows of out_row_bytes; data_bytes of
// values) and their sums of squares.  FP16: halves divided by the scale
// (clamped to 64 scaled units: the copy's rows stay within 32), zero padded;
// qnorm = sum of the stored halves' squares.  E4M3: q_d * scale_d times a
// power of two p bringing the largest magnitude into [128, 256), stored as
// its E4M3 rounding (bytes [0, data_bytes)) and the E4M3 rounding of the
// remainder (bytes [data_bytes, 2 data_bytes)), then the float 1/p; qnorm =
// sum of q_d^2.
template <int DT, int TRAV>
__global__ void prep_queries_kernel(const uint8_t *q, int64_t row_bytes, int64_t nq, int dim, const float *scale,
                                    uint8_t *out, int64_t out_row_bytes, int64_t data_bytes, float *qnorm) {
    __shared__ float red[32];
    __shared__ float pmul;
    for (int64_t r = blockIdx.x; r < nq; r += gridDim.x) {
        const uint8_t *row = q + r * row_bytes;
        uint8_t *o = out + r * out_row_bytes;
        float part = 0.f;
        if constexpr (TRAV == kTravF16) {
            const int padded = (int)(data_bytes / 2);
            for (int d = threadIdx.x; d < padded; d += blockDim.x) {
                const float v = d < dim ? elem<DT>(row, d) : 0.f;
                const __half h = __float2half_rn(d < dim ? fminf(fmaxf(v / scale[d], -64.f), 64.f) : 0.f);
                reinterpret_cast<__half *>(o)[d] = h;
                const float b = __half2float(h);
                part += b * b;
            }
        } else {
            // largest |q_d * scale_d| of the query, then the power of two
            float mx = 0.f;
            for (int d = threadIdx.x; d < dim; d += blockDim.x) mx = fmaxf(mx, fabsf(elem<DT>(row, d) * scale[d]));
            for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, off));
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
            __syncthreads();
            if (threadIdx.x == 0) {
                float m = 0.f;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
                int e = 0;
                if (m > 0.f && isfinite(m)) frexpf(m, &e);  // m = f * 2^e, f in [0.5, 1)
                pmul = (m > 0.f && isfinite(m)) ? ldexpf(1.f, 8 - e) : 1.f;  // m * pmul in [128, 256)
            }
            __syncthreads();
            const float pm = pmul;
            for (int d = threadIdx.x; d < (int)data_bytes; d += blockDim.x) {
                const float v = d < dim ? elem<DT>(row, d) : 0.f;
                const float x = d < dim ? v * scale[d] * pm : 0.f;
                const __nv_fp8_storage_t hi = __nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
                const float back = __half2float(__half(__nv_cvt_fp8_to_halfraw(hi, __NV_E4M3)));
                o[d] = hi;
                o[data_bytes + d] = __nv_cvt_float_to_fp8(x - back, __NV_SATFINITE, __NV_E4M3);
                part += v * v;
            }
            if (threadIdx.x == 0) *reinterpret_cast<float *>(o + 2 * data_bytes) = 1.f / pm;
        }
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(kFull, part, off);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            float sum = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += red[w];
            qnorm[r] = sum;
        }
        __syncthreads();
    }
}

}  // namespace

int walk_blocks_per_sm(int trav, int slots, int expand, int wpb, size_t smem) {
    void *fn = walk_kernel_ptr(trav, slots, expand);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, wpb * 32, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_walk(const DevGraph *g, int trav, int slots, const WalkArgs &a, int grid, int wpb, size_t smem,
                        cudaStream_t s) {
    void *fn = walk_kernel_ptr(trav, slots, a.expand);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void *args[] = {(void *)&g, (void *)&a};
    return cudaLaunchKernel(fn, dim3(grid), dim3(wpb * 32), args, smem, s);
}

cudaError_t launch_bin_by_slots(const int32_t *ef_arr, int32_t ef_bound, int64_t nq, int32_t *counts,
                                int32_t *lists, cudaStream_t s) {
    const int grid = (int)std::min<int64_t>((nq + 255) / 256, 1024);
    bin_by_slots_kernel<<<std::max(grid, 1), 256, 0, s>>>(ef_arr, ef_bound, nq, counts, lists);
    return cudaGetLastError();
}

int rerank_blocks_per_sm(int dtype, const LaneCfg &lc, int wpb, size_t smem) {
    void *fn = rerank_kernel_ptr(dtype, lc.KMAX);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, wpb * 32, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_rerank(const DevGraph *g, int dtype, const LaneCfg &lc, const RerankArgs &a, int grid, int wpb,
                          size_t smem, cudaStream_t s) {
    void *fn = rerank_kernel_ptr(dtype, lc.KMAX);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void *args[] = {(void *)&g, (void *)&lc, (void *)&a};
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
                 uint8_t *t, int64_t trb, int64_t noff, float *rn, cudaStream_t s) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(r1 - r0, 1), 8192);
    if (trav == kTravF16)
        convert_rows_kernel<DT, kTravF16><<<grid, 128, 0, s>>>(vec0, rb, r0, r1, dim, scale, t, trb, noff, rn);
    else
        convert_rows_kernel<DT, kTravE4M3><<<grid, 128, 0, s>>>(vec0, rb, r0, r1, dim, scale, t, trb, noff, rn);
}

cudaError_t launch_convert_rows(int dtype, int trav, const uint8_t *vec0, int64_t row_bytes, int64_t r0, int64_t r1,
                                int dim, const float *scale, uint8_t *trav_rows, int64_t trav_row_bytes,
                                int64_t norm_off, float *rownorm, cudaStream_t s) {
    if (r1 <= r0) return cudaSuccess;
    switch (dtype) {
        case PK_DTYPE_U8: conv<PK_DTYPE_U8>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, norm_off, rownorm, s); break;
        case PK_DTYPE_I8: conv<PK_DTYPE_I8>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, norm_off, rownorm, s); break;
        case PK_DTYPE_F32: conv<PK_DTYPE_F32>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, norm_off, rownorm, s); break;
        case PK_DTYPE_F16: conv<PK_DTYPE_F16>(trav, vec0, row_bytes, r0, r1, dim, scale, trav_rows, trav_row_bytes, norm_off, rownorm, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int DT>
static void prep(int trav, const uint8_t *q, int64_t rb, int64_t nq, int dim, const float *scale, uint8_t *out,
                 int64_t orb, int64_t db, float *qn, cudaStream_t s) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(nq, 1), 8192);
    if (trav == kTravF16)
        prep_queries_kernel<DT, kTravF16><<<grid, 128, 0, s>>>(q, rb, nq, dim, scale, out, orb, db, qn);
    else
        prep_queries_kernel<DT, kTravE4M3><<<grid, 128, 0, s>>>(q, rb, nq, dim, scale, out, orb, db, qn);
}

cudaError_t launch_prep_queries(int dtype, int trav, const uint8_t *q, int64_t row_bytes, int64_t nq, int dim,
                                const float *scale, uint8_t *out, int64_t out_row_bytes, int64_t data_bytes,
                                float *qnorm, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    switch (dtype) {
        case PK_DTYPE_U8: prep<PK_DTYPE_U8>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, data_bytes, qnorm, s); break;
        case PK_DTYPE_I8: prep<PK_DTYPE_I8>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, data_bytes, qnorm, s); break;
        case PK_DTYPE_F32: prep<PK_DTYPE_F32>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, data_bytes, qnorm, s); break;
        case PK_DTYPE_F16: prep<PK_DTYPE_F16>(trav, q, row_bytes, nq, dim, scale, out, out_row_bytes, data_bytes, qnorm, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pk
