// Host build of the LCP array's per-thread bodies (sadcs_b200/csrc/lcp.cuh) for CPU tests: the
// same functions the kernels call, run over every thread index in the order the kernels' launches
// run, with a warp step emulated as the minimum over its 32 lanes and the max-scan as a running
// maximum. Every text read is checked against the text's end. Test infrastructure only.
#include <cstdint>
#include <cstring>
#include <vector>

static uint64_t gTextSize = 0;
static uint64_t gBadRead = 0;  // end of the first read past the text, 0 if none
// nvcc also compiles the kernels for the device, where the check has nothing to record.
#ifdef __CUDA_ARCH__
#define SADCS_LCP_TEXT_READ(end) ((void)0)
#else
#define SADCS_LCP_TEXT_READ(end)                                                        \
    do {                                                                                \
        if (static_cast<uint64_t>(end) > gTextSize && !gBadRead) gBadRead = (end);      \
    } while (0)
#endif

#include "../sadcs_b200/csrc/lcp.cuh"

using namespace sadcs::lcp;

namespace {

template <bool kAligned>
void run(const uint8_t* text, uint32_t n, const uint32_t* sa, uint32_t* out, uint32_t fill, int64_t* unfinishedCount) {
    std::vector<uint32_t> phiV(n, fill);  // what the device scratch held before
    for (uint32_t r = 0; r < n; r++) phiAt(sa, n, r, phiV.data());
    const uint32_t words = sadcs::ceilDiv(n, 32);
    std::vector<uint32_t> mask(words, 0);
    int64_t unfinishedTotal = 0;
    for (uint32_t p = 0; p < n; p++) {
        bool unfinished = false;
        const uint32_t v = shortValue<kAligned>(text, n, p, phiV[p], unfinished);
        if (unfinished) {
            mask[p >> 5] |= 1u << (p & 31);
            unfinishedTotal++;
        } else {
            phiV[p] = v;
        }
    }
    for (uint32_t w = 0; w < words; w++) {
        uint32_t bits = mask[w];
        while (bits) {
            const uint32_t p = 32 * w + static_cast<uint32_t>(__builtin_ctz(bits));
            bits &= bits - 1;
            const uint32_t q = phiV[p];
            uint32_t m = kNone;
            for (uint64_t off = kThreadBytes; m == kNone; off += kWarpStepBytes) {
                uint32_t warpMin = kNone;
                for (uint32_t lane = 0; lane < 32; lane++) {
                    const uint32_t l = laneMismatch<kAligned>(text, n, p, q, off, lane);
                    warpMin = l < warpMin ? l : warpMin;
                }
                m = warpMin;
            }
            phiV[p] = p + m;
        }
    }
    uint32_t running = 0;
    for (uint32_t p = 0; p < n; p++) {
        running = phiV[p] > running ? phiV[p] : running;
        phiV[p] = running;
    }
    for (uint32_t r = 0; r < n; r++) out[r] = gatherAt(sa, phiV.data(), n, r);
    *unfinishedCount = unfinishedTotal;
}

}  // namespace

// The LCP array of sa into out (out may be sa). aligned: run the word-load bodies on an 8-byte
// aligned copy of the text; otherwise the byte-load bodies on a copy at an odd address. fill: the
// scratch's contents before the first pass (they matter only where sa is not a permutation).
// Returns the end of the first text read past n (0 if none) in *bad_read and the number of
// comparisons handed to the warp pass in *unfinished.
extern "C" int lcp_emulate(const uint8_t* text, int64_t n, const uint32_t* sa, uint32_t* out, int aligned,
                           uint32_t fill, int64_t* bad_read, int64_t* unfinished) {
    std::vector<uint64_t> storage(static_cast<size_t>(n) / 8 + 2, 0);
    uint8_t* copy = reinterpret_cast<uint8_t*>(storage.data()) + (aligned ? 0 : 3);
    if (n > 0) std::memcpy(copy, text, static_cast<size_t>(n));
    gTextSize = static_cast<uint64_t>(n);
    gBadRead = 0;
    if (aligned)
        run<true>(copy, static_cast<uint32_t>(n), sa, out, fill, unfinished);
    else
        run<false>(copy, static_cast<uint32_t>(n), sa, out, fill, unfinished);
    *bad_read = static_cast<int64_t>(gBadRead);
    return 0;
}
