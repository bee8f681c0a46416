// primitives.cuh - device-wide scans and stable LSD radix passes, written for sm_100a.
//
// Scan: reduce-then-scan over tiles of 4096 u32 (256 threads x 16), recursive on the tile
// aggregates. Loads and stores are striped across the block (coalesced 128-byte lines); the scan
// inside a tile runs through shared memory with warp shuffles.
//
// Radix pass: one stable counting pass on an 8-bit digit. Upsweep counts digits per tile (warp
// ballots aggregate equal digits before a shared-memory add, so skewed digits do not serialise);
// the per-tile counts, digit-major, are scanned into global offsets; downsweep ranks each tile's
// elements stably (warp match on the digit + per-warp counters), stages them by digit in shared
// memory and writes each digit's run contiguously. Elements reach the kernels through a Loader
// (which may filter them out) and leave through a Storer, so the same kernels serve the sample
// sorts and the filtered class passes.
#pragma once

#include "common.cuh"

namespace sadcs {

// ---- scan ------------------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

struct OpSum {
    static __device__ __forceinline__ uint32_t apply(uint32_t a, uint32_t b) { return a + b; }
    static constexpr uint32_t identity = 0;
};
struct OpMax {
    static __device__ __forceinline__ uint32_t apply(uint32_t a, uint32_t b) { return a > b ? a : b; }
    static constexpr uint32_t identity = 0;
};

// Inclusive scan of v across the block; total gets the block aggregate. 256 threads.
template <class Op>
__device__ __forceinline__ uint32_t blockInclusiveScan(uint32_t v, uint32_t* warpTotals, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= static_cast<uint32_t>(d)) v = Op::apply(u, v);
    }
    if (lane == 31) warpTotals[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? warpTotals[lane] : Op::identity;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= static_cast<uint32_t>(d)) w = Op::apply(u, w);
        }
        if (lane < (blockDim.x >> 5)) warpTotals[lane] = w;
    }
    __syncthreads();
    total = warpTotals[(blockDim.x >> 5) - 1];
    const uint32_t result = warp ? Op::apply(warpTotals[warp - 1], v) : v;
    __syncthreads();
    return result;
}

template <class Op>
__global__ void __launch_bounds__(kScanThreads) scanReduceKernel(const uint32_t* __restrict__ in, uint32_t count,
                                                                 uint32_t* __restrict__ partials) {
    __shared__ uint32_t warpTotals[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    uint32_t acc = Op::identity;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint64_t i = base + j * kScanThreads + threadIdx.x;
        if (i < count) acc = Op::apply(acc, in[i]);
    }
    uint32_t total;
    blockInclusiveScan<Op>(acc, warpTotals, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Scans each tile with carry = carries[blockIdx.x] (exclusive-scanned aggregates) or the identity.
// The shared tile is padded by one word per 32 so the per-thread runs of 16 avoid bank conflicts.
__device__ __forceinline__ uint32_t scanPad(uint32_t i) { return i + (i >> 5); }

template <class Op, bool kInclusive>
__global__ void __launch_bounds__(kScanThreads) scanDownKernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                               uint32_t count, const uint32_t* __restrict__ carries,
                                                               uint32_t* __restrict__ totalOut) {
    __shared__ uint32_t tile[kScanTile + kScanTile / 32];
    __shared__ uint32_t warpTotals[32];
    __shared__ uint32_t threadInclusive[kScanThreads];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t k = j * kScanThreads + threadIdx.x;
        const uint64_t i = base + k;
        tile[scanPad(k)] = i < count ? in[i] : Op::identity;
    }
    __syncthreads();
    uint32_t local[kScanItems];
    uint32_t acc = Op::identity;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        local[j] = tile[scanPad(threadIdx.x * kScanItems + j)];
        acc = Op::apply(acc, local[j]);
    }
    uint32_t blockTotal;
    const uint32_t inclusive = blockInclusiveScan<Op>(acc, warpTotals, blockTotal);
    const uint32_t carry = carries ? carries[blockIdx.x] : Op::identity;
    threadInclusive[threadIdx.x] = inclusive;
    __syncthreads();
    uint32_t start = threadIdx.x ? Op::apply(carry, threadInclusive[threadIdx.x - 1]) : carry;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t next = Op::apply(start, local[j]);
        tile[scanPad(threadIdx.x * kScanItems + j)] = kInclusive ? next : start;
        start = next;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t k = j * kScanThreads + threadIdx.x;
        const uint64_t i = base + k;
        if (i < count) out[i] = tile[scanPad(k)];
    }
    if (totalOut && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *totalOut = Op::apply(carry, blockTotal);
}

// Words of scratch a scan of count elements needs.
inline size_t scanScratchWords(uint64_t count) {
    size_t words = 0;
    uint64_t c = count;
    while (c > kScanTile) {
        c = (c + kScanTile - 1) / kScanTile;
        words += c + 64;
    }
    return words + 64;
}

// out may equal in. totalOut (device, optional) gets the reduction of all elements.
template <class Op, bool kInclusive>
cudaError_t deviceScan(const uint32_t* in, uint32_t* out, uint32_t count, uint32_t* scratch, uint32_t* totalOut,
                       cudaStream_t stream) {
    if (count == 0) {
        if (totalOut) SADCS_TRY(cudaMemsetAsync(totalOut, 0, sizeof(uint32_t), stream));
        return cudaSuccess;
    }
    const uint32_t blocks = ceilDiv(count, kScanTile);
    if (blocks == 1) {
        scanDownKernel<Op, kInclusive><<<1, kScanThreads, 0, stream>>>(in, out, count, nullptr, totalOut);
        return cudaGetLastError();
    }
    uint32_t* partials = scratch;
    scanReduceKernel<Op><<<blocks, kScanThreads, 0, stream>>>(in, count, partials);
    SADCS_TRY(cudaGetLastError());
    SADCS_TRY((deviceScan<Op, false>(partials, partials, blocks, scratch + blocks + 64, nullptr, stream)));
    scanDownKernel<Op, kInclusive><<<blocks, kScanThreads, 0, stream>>>(in, out, count, partials, totalOut);
    return cudaGetLastError();
}

// ---- radix pass ------------------------------------------------------------------------------

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;
constexpr uint32_t kNoDigit = 0x100;

// Shared memory of radixDownsweep for a staged key of KeyBytes bytes.
constexpr size_t radixSharedBytes(size_t keyBytes) {
    return kSortTile * keyBytes + kSortTile * 4 + kSortTile + (kSortWarps * 256 + 256 + 256 + 32) * 4 + 64;
}

template <class Loader>
__global__ void __launch_bounds__(kSortThreads) radixUpsweep(Loader ld, uint32_t count, uint32_t tiles,
                                                             uint32_t* __restrict__ hist) {
    __shared__ uint32_t counts[kSortWarps][256];
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&counts[0][0])[i] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kSortItems; j++) {
        const uint64_t i = base + j * kSortThreads + threadIdx.x;
        uint32_t d = kNoDigit;
        if (i < count && !ld.digit(static_cast<uint32_t>(i), d)) d = kNoDigit;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d != kNoDigit && (peers & ((1u << lane) - 1)) == 0) counts[warp][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) s += counts[w][d];
        hist[static_cast<size_t>(d) * tiles + blockIdx.x] = s;
    }
}

template <class Key, class Loader, class Storer>
__global__ void __launch_bounds__(kSortThreads, 2) radixDownsweep(Loader ld, Storer st, uint32_t count, uint32_t tiles,
                                                                  const uint32_t* __restrict__ offsets) {
    extern __shared__ __align__(16) unsigned char smem[];
    Key* sKeys = reinterpret_cast<Key*>(smem);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(sKeys + kSortTile);
    uint8_t* sDig = reinterpret_cast<uint8_t*>(sVals + kSortTile);
    uint32_t* warpCount = reinterpret_cast<uint32_t*>(sDig + kSortTile);
    uint32_t* digitStart = warpCount + kSortWarps * 256;
    uint32_t* digitGlobal = digitStart + 256;
    uint32_t* warpTotals = digitGlobal + 256;

    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) warpCount[i] = 0;
    for (int d = threadIdx.x; d < 256; d += kSortThreads) digitGlobal[d] = offsets[static_cast<size_t>(d) * tiles + blockIdx.x];
    __syncthreads();

    const uint64_t warpBase = static_cast<uint64_t>(blockIdx.x) * kSortTile + warp * (kSortItems * 32);
    uint32_t* myCount = warpCount + warp * 256;
    const uint32_t lt = (1u << lane) - 1;
    Key keys[kSortItems];
    uint32_t vals[kSortItems];
    uint32_t rankDigit[kSortItems];  // (rank within warp << 9) | digit

#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        const uint64_t i = warpBase + j * 32 + lane;
        uint32_t d = kNoDigit;
        if (!(i < count && ld.load(static_cast<uint32_t>(i), keys[j], vals[j], d))) d = kNoDigit;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = 0;
        if (d != kNoDigit) before = myCount[d];
        __syncwarp();
        if (d != kNoDigit && (peers & lt) == 0) myCount[d] = before + __popc(peers);
        __syncwarp();
        rankDigit[j] = ((before + __popc(peers & lt)) << 9) | d;
    }
    __syncthreads();

    // Per digit: exclusive prefix over the warps, then the tile's digit starts.
    uint32_t digitTotal = 0;
    {
        const uint32_t d = threadIdx.x;  // kSortThreads == 256
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) {
            const uint32_t c = warpCount[w * 256 + d];
            warpCount[w * 256 + d] = s;
            s += c;
        }
        digitTotal = s;
    }
    uint32_t tileTotal;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(digitTotal, warpTotals, tileTotal);
    digitStart[threadIdx.x] = inclusive - digitTotal;
    __syncthreads();

#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        const uint32_t d = rankDigit[j] & 0x1FF;
        if (d != kNoDigit) {
            const uint32_t pos = digitStart[d] + warpCount[warp * 256 + d] + (rankDigit[j] >> 9);
            sKeys[pos] = keys[j];
            sVals[pos] = vals[j];
            sDig[pos] = static_cast<uint8_t>(d);
        }
    }
    __syncthreads();

    for (uint32_t i = threadIdx.x; i < tileTotal; i += kSortThreads) {
        const uint32_t d = sDig[i];
        st.store(digitGlobal[d] + i - digitStart[d], sKeys[i], sVals[i]);
    }
}

// Keys and values of a sort pass.
template <class Key>
struct SortLoader {
    const Key* __restrict__ keys;
    const uint32_t* __restrict__ vals;
    int shift;
    __device__ __forceinline__ bool digit(uint32_t i, uint32_t& d) const {
        d = static_cast<uint32_t>(keys[i] >> shift) & 0xFF;
        return true;
    }
    __device__ __forceinline__ bool load(uint32_t i, Key& k, uint32_t& v, uint32_t& d) const {
        k = keys[i];
        v = vals[i];
        d = static_cast<uint32_t>(k >> shift) & 0xFF;
        return true;
    }
};

template <class Key>
struct SortStorer {
    Key* __restrict__ keys;
    uint32_t* __restrict__ vals;
    __device__ __forceinline__ void store(uint32_t pos, Key k, uint32_t v) const {
        keys[pos] = k;
        vals[pos] = v;
    }
};

// Words of scratch one radix pass over count elements needs (histograms + their scan).
inline size_t radixScratchWords(uint64_t count) {
    const uint64_t tiles = (count + kSortTile - 1) / kSortTile;
    return static_cast<size_t>(tiles * 256) + scanScratchWords(tiles * 256) + 64;
}

template <class Key, class Loader, class Storer>
cudaError_t radixPass(const Loader& ld, const Storer& st, uint32_t count, uint32_t* scratch, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t tiles = ceilDiv(count, kSortTile);
    uint32_t* hist = scratch;
    uint32_t* scanScratch = scratch + static_cast<size_t>(tiles) * 256 + 32;
    radixUpsweep<Loader><<<tiles, kSortThreads, 0, stream>>>(ld, count, tiles, hist);
    SADCS_TRY(cudaGetLastError());
    SADCS_TRY((deviceScan<OpSum, false>(hist, hist, tiles * 256u, scanScratch, nullptr, stream)));
    constexpr size_t shared = radixSharedBytes(sizeof(Key));
    // The opt-in above 48 KiB of dynamic shared memory is per function and per device.
    static uint64_t configured = 0;
    int device = 0;
    SADCS_TRY(cudaGetDevice(&device));
    if (!(configured >> (device & 63) & 1)) {
        SADCS_TRY(cudaFuncSetAttribute(radixDownsweep<Key, Loader, Storer>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shared)));
        configured |= uint64_t(1) << (device & 63);
    }
    radixDownsweep<Key, Loader, Storer><<<tiles, kSortThreads, shared, stream>>>(ld, st, count, tiles, hist);
    return cudaGetLastError();
}

// Stable LSD sort of (keys, vals) over bits [beginBit, endBit), ping-ponging with the alternates.
// On return keys/vals point at the sorted data (swapped with the alternates if the pass count is odd).
template <class Key>
cudaError_t radixSortPairs(Key*& keys, Key*& keysAlt, uint32_t*& vals, uint32_t*& valsAlt, uint32_t count,
                           int beginBit, int endBit, uint32_t* scratch, cudaStream_t stream) {
    for (int bit = beginBit; bit < endBit; bit += 8) {
        SortLoader<Key> ld{keys, vals, bit};
        SortStorer<Key> st{keysAlt, valsAlt};
        SADCS_TRY((radixPass<Key>(ld, st, count, scratch, stream)));
        Key* k = keys;
        keys = keysAlt;
        keysAlt = k;
        uint32_t* v = vals;
        vals = valsAlt;
        valsAlt = v;
    }
    return cudaSuccess;
}

}  // namespace sadcs
