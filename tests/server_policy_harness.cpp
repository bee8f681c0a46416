// Host build of the serving loop's grouping and admission policy (sadcs_b200/csrc/server_policy.h)
// for CPU tests. Test infrastructure only.
#include <cstddef>
#include <cstdint>

#include "../sadcs_b200/csrc/server_policy.h"

extern "C" size_t policy_group_size(const uint64_t* lengths, size_t count, uint64_t small_limit, uint64_t batch_bytes,
                                    uint32_t batch_texts) {
    return sadcs::serverGroupSize(count, [lengths](size_t k) { return lengths[k]; }, small_limit, batch_bytes,
                                  batch_texts);
}

extern "C" int policy_admits(uint64_t need, uint64_t in_use, uint64_t budget) {
    return sadcs::serverAdmits(need, in_use, budget) ? 1 : 0;
}

extern "C" size_t policy_group_start(const uint64_t* lengths, size_t count, uint64_t small_limit, int small_lane) {
    return sadcs::serverGroupStart(count, [lengths](size_t k) { return lengths[k]; }, small_limit, small_lane != 0);
}

extern "C" int policy_is_small_lane(int worker, int workers) {
    return sadcs::serverIsSmallLane(worker, workers) ? 1 : 0;
}
