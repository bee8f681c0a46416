// common.cuh - what every phase of the device construction shares.
//
// The difference cover modulo 32, D = {0, 1, 3, 8, 12, 19, 25} (the cover of the reference's GPU
// path, src/common/differencecover.h:29-31 and src/cuda/devicecommon.cuh:31-36), with its lookup
// tables generated at compile time from D and placed in __constant__ memory by static
// initialisation, so every device that loads the module has them without an upload.
//
// Text layout in HBM: the text bytes, 8-byte aligned, followed by kTextPad zero bytes, so that a
// 16-byte window at any position <= n + 31 stays inside the buffer and reads zeros past the end.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

namespace sadcs {

constexpr int kV = 32;        // cover period
constexpr int kK = 7;         // cover size (sample positions per period)
constexpr int kClasses = 7;   // distance to the next sample position: 0 (the sample) .. 6
constexpr uint32_t kTextPad = 128;
constexpr uint32_t kRankPad = 16;  // zero rank entries past the sample: a 7-rank window at any p <= n stays inside

// The square tables come first and 16-byte aligned: kernels copy them to shared memory as words.
struct alignas(16) Cover {
    alignas(16) uint8_t tie[kV][kV];   // smallest k with a + k and b + k both sampled
    alignas(16) uint8_t slot[kV][kV];  // [a][k]: index of sample a + k among the samples in [a, a + 32)
    uint8_t below[kV];                 // cover residues below r
    uint8_t classOf[kV];               // distance from residue r to the next cover residue
    uint8_t residue[kK];
};
static_assert(offsetof(Cover, tie) % 16 == 0 && offsetof(Cover, slot) % 16 == 0, "word copies of the tables");

constexpr bool coverHas(int r) {
    constexpr int d[kK] = {0, 1, 3, 8, 12, 19, 25};
    for (int i = 0; i < kK; i++) {
        if (d[i] == (r & (kV - 1))) return true;
    }
    return false;
}

constexpr Cover makeCover() {
    Cover c{};
    int k = 0;
    for (int r = 0; r < kV; r++) {
        if (coverHas(r)) c.residue[k++] = static_cast<uint8_t>(r);
    }
    for (int r = 0; r < kV; r++) {
        int below = 0;
        for (int q = 0; q < r; q++) below += coverHas(q) ? 1 : 0;
        c.below[r] = static_cast<uint8_t>(below);
        int d = 0;
        while (!coverHas(r + d)) d++;
        c.classOf[r] = static_cast<uint8_t>(d);
    }
    for (int a = 0; a < kV; a++) {
        for (int b = 0; b < kV; b++) {
            int t = 0;
            while (!coverHas(a + t) || !coverHas(b + t)) t++;
            c.tie[a][b] = static_cast<uint8_t>(t);
        }
        for (int t = 0; t < kV; t++) {
            // samples in [a, a + t) = pack(a + t) - pack(a), with pack over absolute positions
            int count = 0;
            for (int q = a; q < a + t; q++) count += coverHas(q) ? 1 : 0;
            c.slot[a][t] = static_cast<uint8_t>(count);
        }
    }
    return c;
}

constexpr Cover kCoverTables = makeCover();

// The cover as a bit mask (bit r set for r in D) and its rotations: bit t of coverRotation(a) is
// set when a + t is sampled. The tie offset of residues a, b is the lowest bit set in both
// rotations, and the slot of sample a + k among the samples of [a, a + 32) is the number of bits
// of coverRotation(a) below k: two register instructions each instead of table lookups.
constexpr uint32_t coverMask() {
    uint32_t m = 0;
    for (int r = 0; r < kV; r++) m |= coverHas(r) ? (1u << r) : 0u;
    return m;
}
constexpr uint32_t kCoverMask = coverMask();
static_assert(kCoverMask == 0x0208110Bu, "cover mask");

__device__ __forceinline__ uint32_t coverRotation(uint32_t p) {
    return __funnelshift_r(kCoverMask, kCoverMask, p);  // rotate right by p mod 32
}

__device__ __forceinline__ uint32_t tieOffset(uint32_t rotA, uint32_t rotB) {
    return static_cast<uint32_t>(__ffs(rotA & rotB)) - 1;
}

__device__ __forceinline__ uint32_t sampleSlot(uint32_t rotA, uint32_t k) {
    return static_cast<uint32_t>(__popc(rotA & ((1u << k) - 1)));
}
static_assert(kCoverTables.classOf[2] == 1 && kCoverTables.classOf[26] == 6, "cover tables");

__constant__ Cover cCover = makeCover();

// Number of sample positions below p: a sample position's index in the compact rank array.
inline uint64_t packHost(uint64_t p) {
    return (p / kV) * kK + kCoverTables.below[p % kV];
}

// The cover's residues as 5-bit fields of one word, in increasing order.
constexpr uint64_t coverResidues() {
    uint64_t packed = 0;
    for (int k = 0; k < kK; k++) packed |= static_cast<uint64_t>(kCoverTables.residue[k]) << (5 * k);
    return packed;
}
constexpr uint64_t kCoverResidues = coverResidues();

// Device lookups of the cover by register arithmetic on its mask: a warp indexes them with
// different residues, which a __constant__ table would serve one address at a time.
__device__ __forceinline__ uint32_t pack(uint32_t p) {
    return (p / kV) * kK + static_cast<uint32_t>(__popc(kCoverMask & ((1u << (p % kV)) - 1)));
}

__device__ __forceinline__ uint32_t samplePosition(uint32_t t) {
    return (t / kK) * kV + static_cast<uint32_t>((kCoverResidues >> (5 * (t % kK))) & 31);
}

// Distance from residue r to the next sampled residue: its class.
__device__ __forceinline__ uint32_t classOfResidue(uint32_t r) {
    return static_cast<uint32_t>(__ffs(__funnelshift_r(kCoverMask, kCoverMask, r))) - 1;
}

inline uint64_t sampleSize(uint64_t n) {
    return n == 0 ? 0 : packHost(n);
}

// Positions below n in class d.
inline uint64_t classSize(uint64_t n, int d) {
    uint64_t size = 0;
    for (int r = 0; r < kV; r++) {
        if (kCoverTables.classOf[r] == d) size += n / kV + (static_cast<uint64_t>(r) < n % kV ? 1 : 0);
    }
    return size;
}

__device__ __forceinline__ uint64_t byteSwap64(uint64_t x) {
    const uint32_t lo = static_cast<uint32_t>(x), hi = static_cast<uint32_t>(x >> 32);
    return (static_cast<uint64_t>(__byte_perm(lo, 0, 0x0123)) << 32) | __byte_perm(hi, 0, 0x0123);
}

// The 8 text bytes from p as a big-endian word (integer order = byte-string order); zeros past n.
__device__ __forceinline__ uint64_t load8(const uint8_t* __restrict__ text, uint32_t p) {
    const uint64_t* words = reinterpret_cast<const uint64_t*>(text);
    const uint32_t w = p >> 3, shift = (p & 7) * 8;
    const uint64_t lo = __ldg(words + w);
    const uint64_t hi = __ldg(words + w + 1);
    return byteSwap64(shift ? (lo >> shift) | (hi << (64 - shift)) : lo);
}

// 16 bytes from p as two big-endian words.
__device__ __forceinline__ void load16(const uint8_t* __restrict__ text, uint32_t p, uint64_t& a, uint64_t& b) {
    const uint64_t* words = reinterpret_cast<const uint64_t*>(text);
    const uint32_t w = p >> 3, shift = (p & 7) * 8;
    const uint64_t w0 = __ldg(words + w), w1 = __ldg(words + w + 1), w2 = __ldg(words + w + 2);
    if (shift) {
        a = byteSwap64((w0 >> shift) | (w1 << (64 - shift)));
        b = byteSwap64((w1 >> shift) | (w2 << (64 - shift)));
    } else {
        a = byteSwap64(w0);
        b = byteSwap64(w1);
    }
}

__host__ __device__ __forceinline__ uint32_t ceilDiv(uint64_t a, uint64_t b) {
    return static_cast<uint32_t>((a + b - 1) / b);
}

// The texts of one construction, concatenated in HBM. Text j occupies [start[j], end[j]), start[j]
// a multiple of 32 so every position has the same residue modulo the cover period in its text and
// in the concatenation; the bytes between texts are zero. blockText[p / 32] is the text whose range
// contains or precedes block p / 32. With one text, blockText is null and its end is oneEnd.
struct TextSet {
    const uint32_t* blockText;
    const uint32_t* start;
    const uint32_t* end;
    uint32_t count;
    uint32_t oneEnd;
    // The packed code stream (alphabet.cuh), its shape, and code -> byte.
    const uint64_t* packed;
    const uint8_t* decode;
    uint32_t bits;       // per character
    uint32_t keyChars;   // characters per ranking key
    uint32_t tagBits;    // length tag bits of a ranking key
    __device__ __forceinline__ uint32_t textOf(uint32_t p) const { return blockText ? __ldg(blockText + (p >> 5)) : 0; }
    __device__ __forceinline__ uint32_t endOf(uint32_t p) const {
        return blockText ? __ldg(end + __ldg(blockText + (p >> 5))) : oneEnd;
    }
    __device__ __forceinline__ uint32_t startOf(uint32_t text) const { return blockText ? __ldg(start + text) : 0; }
    __device__ __forceinline__ uint32_t endOfText(uint32_t text) const { return blockText ? __ldg(end + text) : oneEnd; }
};

// Kernels launched by this thread since it last read the counter (reported in the stats).
inline thread_local uint64_t tLaunches = 0;

// Every kernel of the library is launched through here, so launches are counted.
template <typename... Params, typename... Args>
inline cudaError_t launch(void (*kernel)(Params...), dim3 grid, dim3 block, size_t shared, cudaStream_t stream,
                          Args&&... args) {
    if (grid.x == 0) return cudaSuccess;
    kernel<<<grid, block, shared, stream>>>(std::forward<Args>(args)...);
    ++tLaunches;
    return cudaGetLastError();
}

// Runs set() (a kernel's function attributes) the first time a call site meets the current device;
// `configured` is the call site's set of devices done. The server's worker threads reach the same
// call sites at once, so the set is atomic; two threads may both run set(), which is harmless (the
// attributes are the same), and a thread sees a device as done only after its set() returned.
template <class Set>
inline cudaError_t configureOnce(std::atomic<uint64_t>& configured, Set set) {
    int device = 0;
    cudaError_t error = cudaGetDevice(&device);
    if (error != cudaSuccess) return error;
    const uint64_t bit = uint64_t(1) << (device & 63);
    if (configured.load(std::memory_order_acquire) & bit) return cudaSuccess;
    if ((error = set()) != cudaSuccess) return error;
    configured.fetch_or(bit, std::memory_order_acq_rel);
    return cudaSuccess;
}

// Asynchronous copies from global to shared memory (completed by cpAsyncWaitAll in the issuing
// thread, then visible to the block after a barrier).
__device__ __forceinline__ void cpAsync8(void* sharedDst, const void* globalSrc) {
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(sharedDst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(globalSrc) : "memory");
}

__device__ __forceinline__ void cpAsync4(void* sharedDst, const void* globalSrc) {
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(sharedDst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(globalSrc) : "memory");
}

__device__ __forceinline__ void cpAsyncWaitAll() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

}  // namespace sadcs

#define SADCS_TRY(call)                                 \
    do {                                                \
        const cudaError_t sadcsError_ = (call);         \
        if (sadcsError_ != cudaSuccess) return sadcsError_; \
    } while (0)
