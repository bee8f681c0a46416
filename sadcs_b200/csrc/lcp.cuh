// lcp.cuh - the longest-common-prefix (LCP) array of a suffix array on the device:
// lcp[0] = 0 and lcp[r] = the length of the longest common prefix of suffixes sa[r - 1] and sa[r].
// The reference computes no LCP array; this is the usual consumer of a suffix array, built from
// the SA and the text alone.
//
// Method: the permuted LCP array of Kärkkäinen, Manzini and Puglisi ("Permuted Longest-Common-
// Prefix Array", CPM 2009), reshaped so that every step is a data-parallel pass:
//   Phi[sa[r]] = sa[r - 1]: the suffix just before p in suffix order (none for sa[0]).
//   PLCP[p] = lcp(p, Phi[p]) in text order. PLCP[p] >= PLCP[p - 1] - 1 (Kasai et al.), so
//   V[p] = p + PLCP[p] never decreases along the text. Position p is reducible when
//   T[p - 1] == T[Phi[p] - 1]: then Phi[p - 1] = Phi[p] - 1 and V[p] = V[p - 1] exactly. Only the
//   irreducible positions compare characters (their LCPs sum to at most 2 n log n, against the
//   O(n^2) of comparing every neighbouring pair on a text of runs), and an inclusive max-scan of V
//   with the reducible entries set to 0 gives V everywhere: PLCP[p] = scan(V)[p] - p.
//   lcp[r] = PLCP[sa[r]].
// Passes (one u32 scratch entry per position, Phi then V in place):
//   lcpPhi      reads sa (coalesced, 8 B/entry), writes Phi at random (4 B/entry)
//   lcpShort    reads Phi, T[p - 1] (coalesced) and T[Phi[p] - 1] (random); at irreducible
//               positions one thread compares up to kThreadBytes characters by 8-byte windows;
//               writes V, and one bit per position marks comparisons left unfinished
//   lcpLong     one warp per unfinished comparison: 32 lanes x kWarpWindows windows (1 KiB) per
//               step, the first mismatch by a warp minimum; a single long common prefix (a text
//               of runs) costs length / 1 KiB warp steps
//   max-scan    V in place (primitives.cuh)
//   lcpGather   lcp[r] = V[sa[r]] - sa[r]: reads sa (coalesced) and V (random), writes lcp
// Text reads go through textWord/textByte and never touch a byte at or past n: the caller's text
// needs no padding. Word loads need an 8-byte aligned text; an unaligned one is read byte by byte.
// Entries of sa that are >= n (not a suffix array) give an unspecified result but no access out
// of bounds; so does an sa that is not a permutation (Phi entries then stay unwritten and are
// guarded as "none" only when >= n, so their values are unspecified, never their addresses).
#pragma once

#include <algorithm>

#include "common.cuh"
#include "primitives.cuh"

// Checks of text reads for a host build of these bodies (the CPU test harness defines it to
// record a read at or past the end); empty in the library.
#ifndef SADCS_LCP_TEXT_READ
#define SADCS_LCP_TEXT_READ(end) ((void)0)
#endif

namespace sadcs {
namespace lcp {

constexpr uint32_t kNone = 0xFFFFFFFFu;  // Phi of the smallest suffix; "no mismatch found yet"
constexpr uint32_t kThreadBytes = 256;   // characters one thread compares before handing over
constexpr uint32_t kWarpWindows = 4;     // 8-byte windows per lane per warp step
constexpr uint32_t kWarpStepBytes = 8 * 32 * kWarpWindows;
static_assert(kThreadBytes % 8 == 0, "whole windows");

__host__ __device__ __forceinline__ uint32_t firstSetByte(uint64_t x) {  // x != 0
#ifdef __CUDA_ARCH__
    return static_cast<uint32_t>(__ffsll(static_cast<long long>(x)) - 1) >> 3;
#else
    return static_cast<uint32_t>(__builtin_ctzll(x)) >> 3;
#endif
}

// Text bytes 8w .. 8w + 7 as a little-endian word; bytes at n and past it read as 0 and are not
// loaded.
template <bool kAligned>
__host__ __device__ __forceinline__ uint64_t textWord(const uint8_t* __restrict__ text, uint64_t n, uint64_t w) {
    const uint64_t first = 8 * w;
    if (kAligned && first + 8 <= n) {
        SADCS_LCP_TEXT_READ(first + 8);
        return reinterpret_cast<const uint64_t*>(text)[w];
    }
    uint64_t v = 0;
    for (uint32_t i = 0; i < 8; i++) {
        if (first + i < n) {
            SADCS_LCP_TEXT_READ(first + i + 1);
            v |= static_cast<uint64_t>(text[first + i]) << (8 * i);
        }
    }
    return v;
}

__host__ __device__ __forceinline__ uint8_t textByte(const uint8_t* __restrict__ text, uint64_t i) {
    SADCS_LCP_TEXT_READ(i + 1);
    return text[i];
}

// Text bytes pos .. pos + 7 (byte j in bits 8j); zeros at n and past it.
template <bool kAligned>
__host__ __device__ __forceinline__ uint64_t textBytes(const uint8_t* __restrict__ text, uint64_t n, uint64_t pos) {
    const uint64_t w = pos >> 3;
    const uint32_t shift = static_cast<uint32_t>(pos & 7) * 8;
    const uint64_t lo = textWord<kAligned>(text, n, w);
    return shift ? (lo >> shift) | (textWord<kAligned>(text, n, w + 1) << (64 - shift)) : lo;
}

// Suffixes p and q compared over [off, off + 8), where limit = n - max(p, q) characters of both
// exist: the first offset at which they differ, limit if one of them ends first within or before
// the window, or kNone if all 8 agree and both go on past the window. limit <= n < 2^32 - 1, so a
// result other than kNone fits and differs from kNone.
template <bool kAligned>
__host__ __device__ __forceinline__ uint32_t windowMismatch(const uint8_t* __restrict__ text, uint64_t n, uint64_t p,
                                                            uint64_t q, uint64_t off, uint64_t limit) {
    if (off >= limit) return static_cast<uint32_t>(limit);
    const uint64_t x = textBytes<kAligned>(text, n, p + off) ^ textBytes<kAligned>(text, n, q + off);
    const uint64_t m = x ? off + firstSetByte(x) : off + 8;
    if (m >= limit) return static_cast<uint32_t>(limit);
    return x ? static_cast<uint32_t>(m) : kNone;
}

// Phi at sa[r].
__host__ __device__ __forceinline__ void phiAt(const uint32_t* __restrict__ sa, uint32_t n, uint32_t r,
                                               uint32_t* __restrict__ phi) {
    const uint32_t p = sa[r];
    if (p < n) phi[p] = r ? sa[r - 1] : kNone;
}

// V at position p from q = Phi[p]: p + PLCP[p] at an irreducible position whose comparison ends
// within kThreadBytes characters, 0 at a reducible one (the max-scan carries V[p - 1] there). An
// unfinished comparison sets unfinished and returns q, which stays in place for lcpLong.
template <bool kAligned>
__host__ __device__ __forceinline__ uint32_t shortValue(const uint8_t* __restrict__ text, uint32_t n, uint32_t p,
                                                        uint32_t q, bool& unfinished) {
    unfinished = false;
    if (q >= n) return p;  // sa[0] (or an entry that is not a position): PLCP = 0
    if (p > 0 && q > 0 && textByte(text, p - 1) == textByte(text, q - 1)) return 0;
    const uint64_t limit = static_cast<uint64_t>(n) - (p > q ? p : q);
    for (uint32_t off = 0; off < kThreadBytes; off += 8) {
        const uint32_t m = windowMismatch<kAligned>(text, n, p, q, off, limit);
        if (m != kNone) return p + m;
    }
    unfinished = true;
    return q;
}

// One lane's part of a warp step of lcpLong at offset off: the smallest result of its windows
// off + 8 (lane + 32 u), u < kWarpWindows. The warp's minimum over lanes is the comparison's
// result once it is not kNone.
template <bool kAligned>
__host__ __device__ __forceinline__ uint32_t laneMismatch(const uint8_t* __restrict__ text, uint32_t n, uint32_t p,
                                                          uint32_t q, uint64_t off, uint32_t lane) {
    const uint64_t limit = static_cast<uint64_t>(n) - (p > q ? p : q);
    uint32_t best = kNone;
#pragma unroll
    for (uint32_t u = 0; u < kWarpWindows; u++) {
        const uint32_t m = windowMismatch<kAligned>(text, n, p, q, off + 8 * (lane + 32 * u), limit);
        best = m < best ? m : best;
    }
    return best;
}

// lcp[r] from the scanned V. sa is not restrict: the output may be sa itself.
__host__ __device__ __forceinline__ uint32_t gatherAt(const uint32_t* sa, const uint32_t* __restrict__ v, uint32_t n,
                                                      uint32_t r) {
    if (r == 0) return 0;
    const uint32_t p = sa[r];
    return p < n ? v[p] - p : 0;
}

// ---- kernels ----------------------------------------------------------------------------------

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) lcpPhi(const uint32_t* __restrict__ sa, uint32_t n,
                                                    uint32_t* __restrict__ phi) {
    const uint64_t r = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    if (r < n) phiAt(sa, n, static_cast<uint32_t>(r), phi);
}

// One thread per position, a warp per 32 positions: the warp's ballot of unfinished comparisons is
// word p / 32 of the mask (every word is written, none needs clearing).
template <bool kAligned>
__global__ void __launch_bounds__(kThreads) lcpShort(const uint8_t* __restrict__ text, uint32_t n,
                                                      uint32_t* __restrict__ phiV, uint32_t* __restrict__ mask) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    bool unfinished = false;
    if (i < n) {
        const uint32_t p = static_cast<uint32_t>(i);
        const uint32_t v = shortValue<kAligned>(text, n, p, phiV[p], unfinished);
        if (!unfinished) phiV[p] = v;
    }
    const uint32_t bits = __ballot_sync(0xffffffffu, unfinished);  // every lane reaches it
    if ((threadIdx.x & 31) == 0 && (i >> 5) < ceilDiv(n, 32)) mask[i >> 5] = bits;
}

// Warps stride over the mask words; for each set bit the whole warp finishes that comparison. The
// word, p, q and the warp minimum are the same in every lane, so every loop is warp-uniform; the
// step loop ends once the offset passes limit (at most n / kWarpStepBytes + 1 steps).
template <bool kAligned>
__global__ void __launch_bounds__(kThreads) lcpLong(const uint8_t* __restrict__ text, uint32_t n,
                                                     const uint32_t* __restrict__ mask, uint32_t words,
                                                     uint32_t* __restrict__ phiV) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (kThreads / 32);
    for (uint32_t w = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); w < words; w += warps) {
        uint32_t bits = mask[w];
        while (bits) {
            const uint32_t p = 32 * w + static_cast<uint32_t>(__ffs(static_cast<int>(bits)) - 1);
            bits &= bits - 1;
            const uint32_t q = phiV[p];
            uint32_t m = kNone;
            for (uint64_t off = kThreadBytes; m == kNone; off += kWarpStepBytes)
                m = __reduce_min_sync(0xffffffffu, laneMismatch<kAligned>(text, n, p, q, off, lane));
            __syncwarp();  // every lane has read phiV[p] before it is overwritten
            if (lane == 0) phiV[p] = p + m;
        }
    }
}

__global__ void __launch_bounds__(kThreads) lcpGather(const uint32_t* sa, const uint32_t* __restrict__ v, uint32_t n,
                                                       uint32_t* out) {
    const uint64_t r = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    if (r < n) out[r] = gatherAt(sa, v, n, static_cast<uint32_t>(r));
}

// Scratch words of lcpArray for n positions: Phi/V, the mask, the scan's scratch.
inline size_t scratchWords(uint64_t n) {
    return n + (ceilDiv(n, 32) + 63) / 64 * 64 + scanScratchWords(n);
}

// The LCP array of sa (n entries, n <= 2^32 - 256) into out, on stream; out may be sa itself (each
// entry is read before it is written, by the same thread). scratch: scratchWords(n) words.
inline cudaError_t lcpArray(const uint8_t* text, uint32_t n, const uint32_t* sa, uint32_t* out, uint32_t* scratch,
                            cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    uint32_t* phiV = scratch;
    const uint32_t words = ceilDiv(n, 32);
    uint32_t* mask = scratch + n;
    uint32_t* scan = mask + (words + 63) / 64 * 64;
    const uint32_t blocks = ceilDiv(n, kThreads);
    const uint32_t longBlocks = std::min<uint32_t>(ceilDiv(words, kThreads / 32), 148u * 8);
    const bool aligned = (reinterpret_cast<uintptr_t>(text) & 7) == 0;
    SADCS_TRY(launch(lcpPhi, blocks, kThreads, 0, stream, sa, n, phiV));
    if (aligned) {
        SADCS_TRY(launch(lcpShort<true>, blocks, kThreads, 0, stream, text, n, phiV, mask));
        SADCS_TRY(launch(lcpLong<true>, longBlocks, kThreads, 0, stream, text, n, mask, words, phiV));
    } else {
        SADCS_TRY(launch(lcpShort<false>, blocks, kThreads, 0, stream, text, n, phiV, mask));
        SADCS_TRY(launch(lcpLong<false>, longBlocks, kThreads, 0, stream, text, n, mask, words, phiV));
    }
    SADCS_TRY((deviceScan<OpMax, true>(phiV, phiV, n, scan, nullptr, stream)));
    SADCS_TRY(launch(lcpGather, blocks, kThreads, 0, stream, sa, phiV, n, out));
    return cudaSuccess;
}

}  // namespace lcp
}  // namespace sadcs
