// server_policy.h - which queued requests a free worker of the serving loop (server.cuh) takes
// next, and whether it may start them. Plain host C++ with no CUDA, so that the policy is tested
// on its own.
//
// Grouping: requests are taken in arrival order. A request larger than smallLimit bytes is taken
// alone when it is at the head of the queue; otherwise the worker takes the head and the small
// requests behind it while they fit one batch (at most batchBytes bytes of text together and at
// most batchTexts texts), stopping at the first one that does not fit or is large.
// Small lane: with two workers or more, worker 0 takes small requests only. Its group starts at
// the first small request in the queue (the large ones before it wait for the other workers), so a
// run of large requests never holds every worker while small ones queue behind them.
// Admission: a group whose construction needs `need` bytes of device memory starts when it fits
// the budget beside the constructions running (inUse bytes), or when nothing is running (a request
// alone on an idle device is always admitted: its allocation then is the budget check).
#pragma once

#include <cstddef>
#include <cstdint>

namespace sadcs {

// lengthAt(k): the length of the k-th queued request, k < count. Returns how many to take from the
// head (at least 1 when count > 0).
template <class LengthAt>
inline size_t serverGroupSize(size_t count, LengthAt lengthAt, uint64_t smallLimit, uint64_t batchBytes,
                              uint32_t batchTexts) {
    size_t take = 0;
    uint64_t bytes = 0;
    for (size_t k = 0; k < count; k++) {
        const uint64_t n = lengthAt(k);
        const bool small = n <= smallLimit;
        if (take == 0) {
            bytes = n;
            take = 1;
            if (!small) break;
            continue;
        }
        if (!small || bytes + n > batchBytes || take >= batchTexts) break;
        bytes += n;
        take++;
    }
    return take;
}

// The queue index a worker's group starts at: 0, or for the small lane the first small request
// (count if there is none: the lane waits).
template <class LengthAt>
inline size_t serverGroupStart(size_t count, LengthAt lengthAt, uint64_t smallLimit, bool smallLane) {
    if (!smallLane) return 0;
    for (size_t k = 0; k < count; k++) {
        if (lengthAt(k) <= smallLimit) return k;
    }
    return count;
}

inline bool serverIsSmallLane(int worker, int workers) {
    return workers >= 2 && worker == 0;
}

inline bool serverAdmits(uint64_t need, uint64_t inUse, uint64_t budget) {
    return need + inUse <= budget || inUse == 0;
}

}  // namespace sadcs
