// ref_gpu_capi.cpp - C entry points over the reference's own CUDA build (src/cuda/gpusa.h,
// gpusa.cu of the reference, compiled unchanged by the Makefile target ref-gpu). Test
// infrastructure: the reference's GPU construction on the same device, as a timed comparison and
// as a second parity source. Statuses are the reference's GpuStatus values (0 Ok, 1 Unavailable,
// 2 NotEnoughMemory, 3 Failed).
#include <cstddef>
#include <cstdint>

#include "gpusa.h"

extern "C" {

int ref_gpu_create_context(int32_t capacity, void** context) {
    GpuContext* c = nullptr;
    const GpuStatus status = gpuCreateContext(capacity, c);
    *context = c;
    return static_cast<int>(status);
}

void ref_gpu_destroy_context(void* context) { gpuDestroyContext(static_cast<GpuContext*>(context)); }

int ref_gpu_suffix_array(void* context, const uint8_t* text, int32_t n, int32_t* sa, double* deviceSeconds) {
    GpuStats stats{};
    const GpuStatus status = gpuSuffixArray(static_cast<GpuContext*>(context), text, n, sa, &stats);
    if (deviceSeconds) *deviceSeconds = stats.deviceSeconds;
    return static_cast<int>(status);
}

int ref_gpu_bwt(void* context, const uint8_t* text, int32_t n, uint8_t* bwt, int32_t* primary,
                double* deviceSeconds) {
    GpuStats stats{};
    int32_t p = 0;
    const GpuStatus status = gpuBwt(static_cast<GpuContext*>(context), text, n, bwt, p, &stats);
    *primary = p;
    if (deviceSeconds) *deviceSeconds = stats.deviceSeconds;
    return static_cast<int>(status);
}

void* ref_gpu_allocate_pinned(size_t bytes) { return gpuAllocatePinned(bytes); }

void ref_gpu_free_pinned(void* pointer) { gpuFreePinned(pointer); }

const char* ref_gpu_last_error() { return gpuLastError(); }

}  // extern "C"
