// classes.cuh - the sorted list of every class (the reference's step 3, src/cuda/classsort.cuh:1-20).
//
// Class d holds the positions whose next sample position is d characters ahead; class 0 is the
// sample, ordered by its ranks. For i in class d >= 1, i + 1 is in class d - 1, so suffix i is
// ordered by (T[i], suffix i + 1): class d is class d - 1 walked in order with n (the empty suffix,
// smallest) in front, keeping the predecessors that fall in class d, stably sorted by their first
// character. Position n - 1 comes from the prepended n and so leads its character bucket, as the
// one-character suffix must.
//
// B200 shape: the walk, the filter, the character gather and the stable counting sort are one
// radix pass (upsweep + scan + downsweep) through a filtering Loader, writing each class straight
// into its slice of the concatenated lists.
#pragma once

#include "common.cuh"
#include "primitives.cuh"

namespace sadcs {

struct ClassLayout {
    uint32_t start[kClasses + 1];
};

inline ClassLayout classLayout(uint64_t n) {
    ClassLayout c{};
    for (int d = 0; d < kClasses; d++) c.start[d + 1] = c.start[d] + static_cast<uint32_t>(classSize(n, d));
    return c;
}

__global__ void classScatterSample(const uint32_t* __restrict__ ranks, uint32_t m, uint32_t* __restrict__ list) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) list[ranks[t]] = samplePosition(t);
}

// Element k of class d - 1 with n prepended; keeps p - 1 if it is in class d, keyed by T[p - 1].
struct ClassLoader {
    const uint32_t* __restrict__ previous;
    const uint8_t* __restrict__ text;
    uint32_t n;
    uint32_t d;
    __device__ __forceinline__ bool pick(uint32_t k, uint32_t& q) const {
        const uint32_t p = k == 0 ? n : previous[k - 1];
        if (p == 0 || cCover.classOf[(p - 1) % kV] != d) return false;
        q = p - 1;
        return true;
    }
    __device__ __forceinline__ bool digit(uint32_t k, uint32_t& dig) const {
        uint32_t q;
        if (!pick(k, q)) return false;
        dig = text[q];
        return true;
    }
    __device__ __forceinline__ bool load(uint32_t k, uint8_t& key, uint32_t& v, uint32_t& dig) const {
        uint32_t q;
        if (!pick(k, q)) return false;
        dig = text[q];
        key = static_cast<uint8_t>(dig);
        v = q;
        return true;
    }
};

struct ClassStorer {
    uint32_t* __restrict__ out;
    __device__ __forceinline__ void store(uint32_t pos, uint8_t, uint32_t v) const { out[pos] = v; }
};

// Fills lists (n entries, laid out by classLayout(n)) from the sample ranks.
inline cudaError_t sortClasses(const uint8_t* text, uint32_t n, const uint32_t* ranks, uint32_t* lists,
                               uint32_t* scratch, cudaStream_t stream) {
    const ClassLayout layout = classLayout(n);
    const uint32_t m = layout.start[1];
    if (m > 0) {
        classScatterSample<<<(m + 255) / 256, 256, 0, stream>>>(ranks, m, lists);
        SADCS_TRY(cudaGetLastError());
    }
    for (int d = 1; d < kClasses; d++) {
        if (layout.start[d + 1] == layout.start[d]) continue;
        const uint32_t previousCount = layout.start[d] - layout.start[d - 1];
        ClassLoader ld{lists + layout.start[d - 1], text, n, static_cast<uint32_t>(d)};
        ClassStorer st{lists + layout.start[d]};
        SADCS_TRY((radixPass<uint8_t>(ld, st, previousCount + 1, scratch, stream)));
    }
    return cudaSuccess;
}

}  // namespace sadcs
