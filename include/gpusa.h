/*
 * gpusa.h - the reference's GPU interface (src/cuda/gpusa.h:22-123 of acesds/sadcs), declaration
 * for declaration, implemented inline over the C ABI of libsadcs_gpu.so (sadcs_gpu.h).
 *
 * A drop-in: code written against the reference's gpusa.h (its CLI, src/cli/main.cpp, and its
 * selftest, src/cli/selftest.cpp) compiles unchanged against this header and links with
 * -lsadcs_gpu instead of the reference's gpusa.cu. Put this directory first on the include path.
 *
 * GpuCover is DifferenceCover<32> when the reference's differencecover.h is on the include path
 * (as when building its sources); otherwise an equivalent cover mod 32 defined here.
 */
#pragma once

#include <cstddef>
#include <cstdint>

#include "sadcs_gpu.h"

#if defined(__has_include)
#if __has_include("differencecover.h")
#include "differencecover.h"
#define SADCS_HAVE_DIFFERENCE_COVER 1
#endif
#endif

enum class GpuStatus {
    Ok = SADCS_OK,
    Unavailable = SADCS_UNAVAILABLE,
    NotEnoughMemory = SADCS_NOT_ENOUGH_MEMORY,
    Failed = SADCS_FAILED,
};

struct GpuDevice {
    char name[256];
    int computeMajor;
    int computeMinor;
    int64_t totalBytes;
    int64_t freeBytes;
};

struct GpuStats {
    int64_t deviceBytes = 0;
    int64_t rankingBytes = 0;
    int64_t classSortBytes = 0;
    int64_t mergeBytes = 0;
    bool pinned = false;
    double setupSeconds = 0.0;
    double uploadSeconds = 0.0;
    double deviceSeconds = 0.0;
    double rankingSeconds = 0.0;
    double classSortSeconds = 0.0;
    double mergeSeconds = 0.0;
    double bwtSeconds = 0.0;
    double downloadSeconds = 0.0;
    int32_t characterPasses = 0;
    int32_t doublingRounds = 0;
};

#ifdef SADCS_HAVE_DIFFERENCE_COVER
using GpuCover = DifferenceCover<32>;
#else
// The cover {0, 1, 3, 8, 12, 19, 25} modulo 32: membership and the packed sample index.
struct GpuCover {
    static constexpr int kSize = 7;
    static constexpr bool isSample(int32_t position) {
        return (0x0208110Bu >> (position & 31)) & 1u;
    }
    static constexpr int32_t pack(int32_t position) {
        return (position >> 5) * kSize + static_cast<int32_t>(__builtin_popcount(0x0208110Bu & ((1u << (position & 31)) - 1u)));
    }
};
#endif

inline int64_t gpuSampleSize(int32_t n) {
    return GpuCover::pack(n);
}

inline void gpuSampleRanksFromSuffixArray(const int32_t* sa, int32_t n, uint32_t* ranks) {
    uint32_t rank = 0;
    for (int32_t i = 0; i < n; i++) {
        if (GpuCover::isSample(sa[i])) {
            ranks[GpuCover::pack(sa[i])] = rank++;
        }
    }
}

namespace sadcs_gpusa_detail {
inline void copyStats(const sadcs_gpu_stats& in, GpuStats* out) {
    if (!out) return;
    out->deviceBytes = in.device_bytes;
    out->rankingBytes = in.ranking_bytes;
    out->classSortBytes = in.class_sort_bytes;
    out->mergeBytes = in.merge_bytes;
    out->pinned = in.pinned != 0;
    out->setupSeconds = in.setup_seconds;
    out->uploadSeconds = in.upload_seconds;
    out->deviceSeconds = in.device_seconds;
    out->rankingSeconds = in.ranking_seconds;
    out->classSortSeconds = in.class_sort_seconds;
    out->mergeSeconds = in.merge_seconds;
    out->bwtSeconds = in.bwt_seconds;
    out->downloadSeconds = in.download_seconds;
    out->characterPasses = in.character_passes;
    out->doublingRounds = in.doubling_rounds;
}
}  // namespace sadcs_gpusa_detail

inline GpuStatus gpuQueryDevice(GpuDevice& device) {
    sadcs_gpu_device d{};
    const int status = sadcs_gpu_query_device(&d);
    if (status == SADCS_OK) {
        for (size_t i = 0; i < sizeof device.name; i++) device.name[i] = d.name[i];
        device.computeMajor = d.compute_major;
        device.computeMinor = d.compute_minor;
        device.totalBytes = d.total_bytes;
        device.freeBytes = d.free_bytes;
    }
    return static_cast<GpuStatus>(status);
}

inline int64_t gpuRequiredBytes(int32_t n) {
    return sadcs_gpu_required_bytes(n);
}

constexpr int64_t kGpuMemoryReserve = int64_t(256) << 20;

struct GpuContext;

inline GpuStatus gpuCreateContext(int32_t capacity, GpuContext*& context) {
    sadcs_gpu_context* c = nullptr;
    const int status = sadcs_gpu_create_context(capacity, &c);
    context = reinterpret_cast<GpuContext*>(c);
    return static_cast<GpuStatus>(status);
}

inline void gpuDestroyContext(GpuContext* context) {
    sadcs_gpu_destroy_context(reinterpret_cast<sadcs_gpu_context*>(context));
}

inline GpuStatus gpuSuffixArray(GpuContext* context, const uint8_t* text, int32_t n, int32_t* sa,
                                GpuStats* stats = nullptr) {
    sadcs_gpu_stats s{};
    const int status = sadcs_gpu_suffix_array(reinterpret_cast<sadcs_gpu_context*>(context), text, n, sa, &s);
    if (stats) *stats = GpuStats{};
    sadcs_gpusa_detail::copyStats(s, stats);
    return static_cast<GpuStatus>(status);
}

inline GpuStatus gpuSuffixArray(const uint8_t* text, int32_t n, int32_t* sa, GpuStats* stats = nullptr) {
    return gpuSuffixArray(nullptr, text, n, sa, stats);
}

inline GpuStatus gpuBwt(GpuContext* context, const uint8_t* text, int32_t n, uint8_t* bwt, int32_t& primary,
                        GpuStats* stats = nullptr) {
    sadcs_gpu_stats s{};
    const int status = sadcs_gpu_bwt(reinterpret_cast<sadcs_gpu_context*>(context), text, n, bwt, &primary, &s);
    if (stats) *stats = GpuStats{};
    sadcs_gpusa_detail::copyStats(s, stats);
    return static_cast<GpuStatus>(status);
}

inline GpuStatus gpuBwt(const uint8_t* text, int32_t n, uint8_t* bwt, int32_t& primary, GpuStats* stats = nullptr) {
    return gpuBwt(nullptr, text, n, bwt, primary, stats);
}

inline GpuStatus gpuRankSample(const uint8_t* text, int32_t n, uint32_t* ranks, GpuStats* stats = nullptr) {
    sadcs_gpu_stats s{};
    const int status = sadcs_gpu_rank_sample(text, n, ranks, &s);
    if (stats) *stats = GpuStats{};
    sadcs_gpusa_detail::copyStats(s, stats);
    return static_cast<GpuStatus>(status);
}

inline void* gpuAllocatePinned(size_t bytes) {
    return sadcs_gpu_allocate_pinned(bytes);
}

inline void gpuFreePinned(void* pointer) {
    sadcs_gpu_free_pinned(pointer);
}

inline const char* gpuLastError() {
    return sadcs_gpu_last_error();
}
