// Host-side checks of the fast walk's launch arithmetic (pickle_b200/csrc/pk_fast.h):
// list-width classes, the per-warp shared-memory layout of the walk and of the
// re-rank, and the recently-seen table's tag width.  These are the sizes every
// walk and re-rank launch is computed from; a wrong one would let a kernel
// index past its shared memory, so they are checked exhaustively on the CPU.
// Prints "ok" and exits 0, or prints the first violated property and exits 1.
#include <cstdio>

#include "pk_fast.h"

#define CHECK(cond, ...)                          \
    do {                                          \
        if (!(cond)) {                            \
            std::printf("FAIL %s: ", #cond);      \
            std::printf(__VA_ARGS__);             \
            std::printf("\n");                    \
            return 1;                             \
        }                                         \
    } while (0)

int main() {
    using namespace pk;
    // widths: increasing, the widest holds kFastMaxEf
    for (int c = 1; c < kSlotClasses; c++)
        CHECK(slot_class_width(c) > slot_class_width(c - 1), "class %d", c);
    CHECK(32 * slot_class_width(kSlotClasses - 1) == kFastMaxEf, "widest %d", slot_class_width(kSlotClasses - 1));

    // every ef takes the narrowest width that holds it: at most twice ef up to
    // 64, at most half again as wide above
    for (int ef = 1; ef <= kFastMaxEf; ef++) {
        const int c = slot_class(ef), w = slot_class_width(c);
        CHECK(32 * w >= ef, "ef %d width %d", ef, w);
        CHECK(c == 0 || 32 * slot_class_width(c - 1) < ef, "ef %d not the narrowest (class %d)", ef, c);
        CHECK(list_slots(ef) == w, "ef %d", ef);
        if (ef > 32) CHECK(32 * w <= 2 * ef, "ef %d width %d", ef, w);
        if (ef > 64) CHECK(2 * 32 * w <= 3 * ef, "ef %d width %d", ef, w);
    }

    // re-rank: the bitonic sort buffers hold the padded power of two of every
    // list width, and the layout's regions follow one another on 16-byte bounds
    for (int c = 0; c < kSlotClasses; c++) {
        const int cs = 32 * slot_class_width(c);
        const int cap = pow2_at_least(cs);
        CHECK(cap >= cs && (cap & (cap - 1)) == 0 && cap < 2 * cs, "cand_stride %d cap %d", cs, cap);
        for (int64_t rb : {16, 48, 144, 528, 1552}) {
            const RerankLayout r = rerank_layout(cs, rb);
            CHECK(r.sd >= kStageBytes && r.sd % 16 == 0, "sd %d", r.sd);
            CHECK(r.sid >= r.sd + 4 * cap && r.sid % 16 == 0, "sid %d", r.sid);
            CHECK(r.rowbuf >= r.sid + 4 * cap && r.rowbuf % 16 == 0, "rowbuf %d", r.rowbuf);
            CHECK(r.total >= r.rowbuf + kStageRows * rb && r.total % 16 == 0, "total %d", r.total);
        }
    }

    // walk: staged rows at an odd number of 16-byte chunks, then the query, the
    // table, the pending batch and the mbarrier, each on a 16-byte boundary and
    // clear of the previous region
    for (int trav : {kTravF16, kTravE4M3}) {
        for (int64_t tdb = 32; tdb <= 2048; tdb += 32) {
            for (int norm : {0, 32}) {
                const int64_t trb = tdb + norm;
                const int64_t qb = trav_query_bytes(trav, tdb);
                CHECK(qb >= (trav == kTravF16 ? tdb : 2 * tdb + 4), "query bytes %lld", (long long)qb);
                const int64_t st = stage_stride(trb);
                CHECK(st >= trb && st % 16 == 0 && (st / 16) % 2 == 1, "stride %lld for row %lld", (long long)st,
                      (long long)trb);
                for (int rb : {1, 8, 16, 24, 32, 48, 64, 256}) {
                    for (int hl = 5; hl <= 15; hl++) {
                        for (bool t16 : {false, true}) {
                          for (int c = 0; c < kSlotClasses; c++) {
                            const int sl = slot_class_width(c);
                            const WalkLayout w = walk_layout(rb, trb, qb, hl, t16, sl);
                            CHECK(w.stride == st, "stride");
                            CHECK(w.qbuf >= rb * st && w.qbuf % 16 == 0, "qbuf %d", w.qbuf);
                            // the merge's working space (list, winners, masks,
                            // marks) fits in the staged rows' region
                            CHECK(w.qbuf >= walk_merge_bytes(sl), "merge space %d for %d slots", w.qbuf, sl);
                            CHECK(sl < kMergeMinSlots || walk_merge_bytes(sl) >= 8 * 32 * sl + 8 * 32 + 8 * 32,
                                  "merge bytes %lld", (long long)walk_merge_bytes(sl));
                            CHECK(w.tab >= w.qbuf + qb && w.tab % 16 == 0, "tab %d", w.tab);
                            CHECK(w.crow >= w.tab + ((t16 ? 2 : 4) << hl) && w.crow % 16 == 0, "crow %d", w.crow);
                            CHECK(w.cid >= w.crow + 4 * rb && w.cid % 16 == 0, "cid %d", w.cid);
                            CHECK(w.cd >= w.cid + 4 * rb && w.cd % 16 == 0, "cd %d", w.cd);
                            CHECK(w.bar >= w.cd + 4 * rb && w.bar % 16 == 0, "bar %d", w.bar);
                            CHECK(w.total >= w.bar + 8, "total %d", w.total);
                          }
                        }
                    }
                }
            }
        }
    }

    // recently-seen table: where 16-bit tags are chosen, an id's bits beyond
    // the set index fit the 15 tag bits (tag + 1 never wraps to the empty 0)
    for (int hl = 5; hl <= 15; hl++) {
        for (int64_t n : {2LL, 1000LL, 1LL << 16, 1000000LL, 10000000LL, 1LL << 28, 1LL << 31}) {
            const int b = idbits_for(n) > hl - 2 ? idbits_for(n) : hl - 2;
            CHECK(((int64_t)1 << idbits_for(n)) >= n, "idbits %d for %lld", idbits_for(n), (long long)n);
            if (seen_tag16(n, hl)) CHECK(b - (hl - 2) <= 15, "tag bits %d (n %lld, hlog2 %d)", b - (hl - 2),
                                         (long long)n, hl);
        }
    }
    // visited tables in L2: exact tags (the id's bits beyond the set index fit
    // 15 bits, so tag + 1 fits 16), at most about twice the ids, and room
    // for what a walk of the width meets
    for (int c = 0; c < kSlotClasses; c++) {
        const int sl = slot_class_width(c);
        for (int64_t n : {2LL, 100LL, 3000LL, 1LL << 16, 1000000LL, 10000000LL, 1LL << 28, 1LL << 31}) {
            const int l = visited_log2sets(sl, n);
            const int b = idbits_for(n) > l ? idbits_for(n) : l;
            CHECK(l >= 0 && l <= 20, "log2 sets %d", l);
            CHECK(b - l <= 15, "tag bits %d (n %lld, slots %d)", b - l, (long long)n, sl);
            CHECK(((int64_t)8 << l) >= ((1536 + 16 * 32 * (int64_t)sl) * 5 / 4 < 2 * n ? (1536 + 16 * 32 * sl) * 5 / 4 : 2 * n),
                  "table too small: 2^%d sets (n %lld, slots %d)", l, (long long)n, sl);
            CHECK(l == 0 || ((int64_t)8 << (l - 1)) < 2 * n || b - (l - 1) > 15, "table larger than needed");
        }
    }
    for (int s = 1; s <= 32; s++) CHECK(merge_min_for(s) >= 1 && merge_min_for(s) <= 32, "merge_min %d", s);
    std::printf("ok\n");
    return 0;
}
