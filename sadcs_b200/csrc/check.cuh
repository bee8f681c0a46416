// check.cuh - suffix array and BWT checks on the device (the reference's checker,
// src/common/checker.cpp:53-109 and :196-245, restated as data-parallel kernels).
//
// Suffix array (Burkhardt-Karkkainen): SA is a permutation (every entry in range, inverse SA
// written by scatter, each slot owned by exactly one entry), and every neighbour pair is in order
// by (T[SA[i]], ISA[SA[i] + 1]) with the empty suffix's rank -1.
//
// BWT: the LF mapping of the BWT (a stable counting pass on its bytes, the sentinel's row first)
// must be one cycle that, followed from the sentinel's row, spells the text backwards. The walk is
// sequential in the reference; here every row's text position is found by pointer jumping along
// LF (log2 n rounds), and then each row's byte is compared with the text byte before its position.
#pragma once

#include "common.cuh"

namespace sadcs {

constexpr uint64_t kNoFailure = ~uint64_t(0);

__global__ void checkScatter(const uint32_t* __restrict__ sa, uint32_t n, uint32_t* __restrict__ isa,
                             unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = sa[i];
    if (p >= n) {
        atomicMin(firstBad, static_cast<unsigned long long>(i));
    } else {
        isa[p] = static_cast<uint32_t>(i);
    }
}

__global__ void checkDuplicates(const uint32_t* __restrict__ sa, uint32_t n, const uint32_t* __restrict__ isa,
                                unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (isa[sa[i]] != i) atomicMin(firstBad, static_cast<unsigned long long>(i));
}

__global__ void checkOrder(const uint8_t* __restrict__ text, const uint32_t* __restrict__ sa, uint32_t n,
                           const uint32_t* __restrict__ isa, unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i + 1 >= n) return;
    const uint32_t l = sa[i], r = sa[i + 1];
    bool ok = text[l] < text[r];
    if (text[l] == text[r]) {
        const int64_t ln = l + 1 < n ? static_cast<int64_t>(isa[l + 1]) : -1;
        const int64_t rn = r + 1 < n ? static_cast<int64_t>(isa[r + 1]) : -1;
        ok = ln < rn;
    }
    if (!ok) atomicMin(firstBad, static_cast<unsigned long long>(i));
}

}  // namespace sadcs
