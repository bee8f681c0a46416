// Host checks of the construction's memory plan (sadcs_b200/csrc/sadcs_gpu.cu, included whole so
// that the checks run the library's own planning code) for CPU tests: a batch's placement, and that
// the slab a context allocates for (capacity, texts) holds the layout of every batch it admits.
// Test infrastructure only.
#include "../sadcs_b200/csrc/sadcs_gpu.cu"

namespace {

int checkPlacement(const Batch& b, const uint64_t* lengths, uint32_t count, int64_t* detail) {
    uint64_t outputs = 0, live = 0;
    for (uint32_t j = 0; j < count; j++) {
        detail[0] = j;
        if (b.start[j] % kV != 0) return 2;                       // every text starts on a period
        if (b.end[j] - b.start[j] != lengths[j]) return 3;          // and holds its bytes
        if (j > 0 && b.start[j] < b.end[j - 1]) return 4;           // after the previous one
        if (b.outBase[j] != outputs || b.sampleBase[j] != live) return 5;
        outputs += lengths[j];
        live += sampleSize(lengths[j]);
    }
    if (b.outBase[count] != outputs || b.outputs != outputs || b.live != live) return 6;
    if (b.span % kV != 0 || (count > 0 && b.span < b.end[count - 1])) return 7;
    uint64_t classTotal = 0;
    for (int d = 0; d < kClasses; d++) classTotal += b.classes.start[d + 1] - b.classes.start[d];
    if (classTotal != outputs || b.classes.start[1] != live) return 8;  // classes partition the positions
    detail[0] = b.merge.top;
    detail[1] = b.merge.start[b.merge.top][kClasses];
    if (detail[1] > static_cast<int64_t>(mergeCap(kMergeRMin))) return 9;  // the top merge level fits one tile
    return 0;
}

}  // namespace

// 0 when every check passes, else the number of the first failed check; detail[0..2] say where.
extern "C" int plan_check(const uint64_t* lengths, uint32_t count, uint64_t capacity, uint32_t texts, int64_t* detail) {
    Batch b;
    if (!planBatch(lengths, count, b)) return 1;
    if (const int failed = checkPlacement(b, lengths, count, detail); failed) return failed;
    const Extent a = extentOf(b), x = extentBound(capacity, texts);
    const uint64_t actual[] = {a.span, a.slots, a.live, a.outputs, a.largestClass, a.splitterWords, a.rows, a.count};
    const uint64_t bound[] = {x.span, x.slots, x.live, x.outputs, x.largestClass, x.splitterWords, x.rows, x.count};
    for (int f = 0; f < 8; f++) {
        if (actual[f] > bound[f]) {
            detail[0] = f;
            detail[1] = static_cast<int64_t>(actual[f]);
            detail[2] = static_cast<int64_t>(bound[f]);
            return 10 + f;
        }
    }
    for (int sa = 0; sa < 2; sa++) {
        for (int bwt = 0; bwt < 2; bwt++) {
            // a one-text context from the carry threshold on plans room for carried words; its
            // constructions use it
            const bool carry = planCarry(capacity, texts);
            const size_t need = planLayout(a, sa, bwt, carry).peak, have = planLayout(x, sa, bwt, carry).peak;
            if (need > have) {
                detail[0] = 2 * sa + bwt;
                detail[1] = static_cast<int64_t>(need);
                detail[2] = static_cast<int64_t>(have);
                return 20;
            }
        }
    }
    if (planLayout(a, true, true, planCarry(capacity, texts)).peak > contextBytes(static_cast<int64_t>(capacity), texts)) {
        return 21;
    }
    return 0;
}

// The planned peak of a construction of these texts (SA and BWT inside the slab).
extern "C" uint64_t plan_peak(const uint64_t* lengths, uint32_t count) {
    Batch b;
    if (!planBatch(lengths, count, b)) return 0;
    return planLayout(extentOf(b), true, true, planCarry(b.outputs, count)).peak;
}

// The first output any tile from this row on can own (merge.cuh: tileOutputBound, the bound the
// overlapped download of the last merge level copies up to). row: list (or -1 for the level's
// start) then 7 counts; start: the 8 list offsets of the level.
extern "C" uint64_t plan_tile_bound(const uint32_t* row, const uint32_t* start) {
    MergeRow r;
    r.list = row[0];
    for (int b = 0; b < kClasses; b++) r.c[b] = row[1 + b];
    return tileOutputBound(r, start);
}
