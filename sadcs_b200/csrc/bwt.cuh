// bwt.cuh - the SA-to-BWT gather: BWT[0, n) from a device suffix array, in the convention of
// src/cli/selftest.cpp:141-159 of the reference (row of suffix 0 left out, primary = its row + 1,
// byte 0 = T[n - 1], the sentinel's row). The merge writes the BWT directly as it places each
// suffix; this gather serves callers that hold a suffix array already.
#pragma once

#include "common.cuh"

namespace sadcs {

__global__ void bwtFindZero(const uint32_t* __restrict__ sa, uint32_t n, uint32_t* row0) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n && sa[r] == 0) *row0 = r;
}

__global__ void bwtGather(const uint8_t* __restrict__ text, const uint32_t* __restrict__ sa, uint32_t n,
                          const uint32_t* __restrict__ row0Ptr, uint8_t* __restrict__ bwt) {
    const uint32_t row0 = *row0Ptr;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) bwt[0] = text[n - 1];
    if (r >= n) return;
    const uint32_t p = sa[r];
    if (p != 0 && p < n && row0 < n) bwt[r < row0 ? r + 1 : r] = text[p - 1];
}

inline cudaError_t bwtFromSa(const uint8_t* text, uint32_t n, const uint32_t* sa, uint8_t* bwt, uint32_t* row0Device,
                             uint32_t* hostWord, cudaStream_t stream, uint32_t* row0) {
    if (n == 0) {
        *row0 = 0;
        return cudaSuccess;
    }
    SADCS_TRY(cudaMemsetAsync(row0Device, 0, sizeof(uint32_t), stream));
    SADCS_TRY(launch(bwtFindZero, (n + 255) / 256, 256, 0, stream, sa, n, row0Device));
    SADCS_TRY(launch(bwtGather, (n + 255) / 256, 256, 0, stream, text, sa, n, row0Device, bwt));
    SADCS_TRY(cudaMemcpyAsync(hostWord, row0Device, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    *row0 = *hostWord;
    return cudaSuccess;
}

}  // namespace sadcs
