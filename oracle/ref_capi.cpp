/*
 * ref_capi.cpp - A C entry point over the reference's CPU construction and checker.
 *
 * Test infrastructure only: compiled by oracle/Makefile together with the reference's own CPU
 * sources into oracle/_ref/libsadcs_ref.so, so that the tests can compare against the
 * reference's output and bench.py can time the reference's CPU variant. Nothing in the
 * product links it.
 *
 * Wraps (file:line in acesds/sadcs):
 *   buildSuffixArray   src/cpu/dcsort.h:34   (cover 64, 128 or 256; text followed by 64 zero bytes)
 *   buildBwt           src/cpu/dcsort.h:40   (divsufsort convention; returns the primary index)
 *   checkSuffixArray   src/common/checker.h:25
 *   checkBwt           src/common/checker.h:28
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>
#include "checker.h"
#include "dcsort.h"
#include "simd.h"

namespace {
    // The reference reads up to kTextPadding bytes past the text; copy into a padded buffer.
    std::vector<uint8_t> padded(const uint8_t* text, int32_t n) {
        std::vector<uint8_t> buffer(static_cast<size_t>(n) + kTextPadding, 0);
        if (n > 0) {
            memcpy(buffer.data(), text, static_cast<size_t>(n));
        }
        return buffer;
    }
}

extern "C" {

int ref_text_padding(void) {
    return kTextPadding;
}

long long ref_max_text_size(void) {
    return kMaxTextSize;
}

void ref_set_threads(int threads) {
    omp_set_num_threads(threads);
}

int ref_max_threads(void) {
    return omp_get_max_threads();
}

/* text must already carry ref_text_padding() zero bytes after n; returns 1 on success. */
int ref_build_sa_padded(const uint8_t* text, int32_t n, int32_t* sa, int cover) {
    return buildSuffixArray(text, n, sa, cover) ? 1 : 0;
}

int ref_build_sa(const uint8_t* text, int32_t n, int32_t* sa, int cover) {
    const std::vector<uint8_t> buffer = padded(text, n);
    return buildSuffixArray(buffer.data(), n, sa, cover) ? 1 : 0;
}

/* bwt gets n bytes; returns the primary index, or -1. sa is n entries of scratch. */
int32_t ref_build_bwt_padded(const uint8_t* text, int32_t n, uint8_t* bwt, int32_t* sa, int cover) {
    return buildBwt(text, n, bwt, sa, cover);
}

int32_t ref_build_bwt(const uint8_t* text, int32_t n, uint8_t* bwt, int cover) {
    const std::vector<uint8_t> buffer = padded(text, n);
    std::vector<int32_t> sa(static_cast<size_t>(n > 0 ? n : 1));
    return buildBwt(buffer.data(), n, bwt, sa.data(), cover);
}

/* mode: 0 fast, 1 low memory, 2 naive. Returns 1 if ok; *index gets the failing SA index. */
int ref_check_sa(const uint8_t* text, int32_t n, const int32_t* sa, int mode, long long* index) {
    const std::vector<uint8_t> buffer = padded(text, n);
    const CheckMode modes[] = {CheckMode::Fast, CheckMode::LowMemory, CheckMode::Naive};
    const CheckResult result = checkSuffixArray(buffer.data(), n, sa, modes[mode < 0 || mode > 2 ? 0 : mode]);
    if (index) {
        *index = result.index;
    }
    return result.ok ? 1 : 0;
}

int ref_check_bwt(const uint8_t* text, int32_t n, const uint8_t* bwt, int32_t primary, long long* index) {
    const CheckResult result = checkBwt(text, n, bwt, primary);
    if (index) {
        *index = result.index;
    }
    return result.ok ? 1 : 0;
}

}
