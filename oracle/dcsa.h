/*
 * dcsa.h - CPU restatement of the reference's GPU suffix-array/BWT path. TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg call it,
 * and only as the checker. The product (libsadcs_gpu.so) never links or calls it.
 *
 * Positions are uint32 (n < 2^32), so the 3 GiB genome-like workload, which the reference's int32
 * API cannot index, is covered too; sizes are int64.
 *
 * What each function restates (file:line in acesds/sadcs):
 *   oracle_cover_*             src/common/differencecover.h:29-31,154-194 (cover mod 32, pack, tieOffset,
 *                              nextSampleDistance) and src/cuda/devicecommon.cuh:53-115 (class tables)
 *   oracle_dc_sample_ranks     src/cuda/samplerank.cuh:1-20 (ranks of the sample suffixes; prefix doubling
 *                              over groups sharing a prefix of a multiple of 32 characters)
 *   oracle_dc_class_lists      src/cuda/classsort.cuh:1-20,100-123 (class d from class d-1 with n prepended,
 *                              stable by one character)
 *   oracle_dc_merge            src/cuda/merge.cuh:53-71 (lessGlobal, the O(1) difference-cover comparison)
 *                              applied as a plain 7-way merge
 *   oracle_naive_sa            src/cli/selftest.cpp:114-125 (std::sort with a memcmp-style comparison)
 *   oracle_doubling_sa         an independent prefix-doubling construction (not in the reference)
 *   oracle_bwt_from_sa         src/cli/selftest.cpp:141-159 (the BWT convention)
 *   oracle_sample_ranks_from_sa src/cuda/gpusa.h:65-73
 *   oracle_check_sa            src/common/checker.cpp:53-109 (checkFast), in 64-bit arithmetic
 *   oracle_check_bwt           src/common/checker.cpp:196-245 (LF inversion), in 64-bit arithmetic
 *   oracle_lcp                 no counterpart (the reference computes no LCP array): Kasai, Lee,
 *                              Arimura, Arikawa and Park's linear-time LCP, in the Phi-array
 *                              formulation (Karkkainen, Manzini and Puglisi), pinned by the definition
 *                              (tests/test_oracle.py compares it with direct comparison of neighbours)
 *
 * Parity pinning: tests/golden/ holds outputs of the reference's own CPU build (oracle/_ref), made by
 * tests/golden/make_golden.py; tests/test_oracle.py checks every function here against them.
 */
#ifndef SADCS_ORACLE_DCSA_H
#define SADCS_ORACLE_DCSA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cover mod 32: D = {0,1,3,8,12,19,25}. */
int64_t oracle_sample_size(int64_t n);
void oracle_cover_tables(uint8_t below[32], uint8_t tie_offset[32 * 32], uint8_t class_of[32]);

/* All return 0 on success, nonzero on a failed allocation or a size out of range. */
int oracle_naive_sa(const uint8_t* text, int64_t n, uint32_t* sa);
int oracle_doubling_sa(const uint8_t* text, int64_t n, uint32_t* sa);

int oracle_dc_sample_ranks(const uint8_t* text, int64_t n, uint32_t* ranks);
/* lists: n entries, the 7 classes one after another; start[0..7]. */
int oracle_dc_class_lists(const uint8_t* text, int64_t n, const uint32_t* ranks, uint32_t* lists, int64_t* start);
int oracle_dc_merge(const uint8_t* text, int64_t n, const uint32_t* ranks, const uint32_t* lists,
                    const int64_t* start, uint32_t* sa);
int oracle_dc_sa(const uint8_t* text, int64_t n, uint32_t* sa);

void oracle_sample_ranks_from_sa(const uint32_t* sa, int64_t n, uint32_t* ranks);
/* bwt gets n bytes; returns the primary index (0 for n == 0). */
int64_t oracle_bwt_from_sa(const uint8_t* text, int64_t n, const uint32_t* sa, uint8_t* bwt);

/* Return 1 if correct; *index gets the first failing SA index (or text position for the BWT), -1 if ok. */
int oracle_check_sa(const uint8_t* text, int64_t n, const uint32_t* sa, int64_t* index);
int oracle_check_bwt(const uint8_t* text, int64_t n, const uint8_t* bwt, int64_t primary, int64_t* index);

/* lcp[0] = 0 and lcp[r] = the length of the longest common prefix of suffixes sa[r - 1] and sa[r]
 * (r >= 1), for the suffix array sa of text. Returns 0 if memory runs out. */
int oracle_lcp(const uint8_t* text, int64_t n, const uint32_t* sa, uint32_t* lcp);

#ifdef __cplusplus
}
#endif

#endif
