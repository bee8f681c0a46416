/*
 * sadcs_gpu.h - C ABI of libsadcs_gpu.so: suffix array and BWT construction on one NVIDIA B200
 * (sm_100a), entirely in hand-written CUDA kernels.
 *
 * Every entry point here replaces one declaration of the reference's GPU interface,
 * src/cuda/gpusa.h of acesds/sadcs (cited per function), with plain C types: no references,
 * overloads, default arguments or enum classes, so cgo, JNI, ctypes or a C++ shim can bind it.
 * include/gpusa.h is that C++ shim: the reference's exact declarations, inline over these.
 *
 * Conventions shared with the reference:
 *   - The suffix array is divsufsort's: SA[i] is the start of the i-th smallest suffix, byte-wise
 *     lexicographic, a suffix that is a prefix of another being the smaller.
 *   - The BWT is divsufsort's/libsais's (src/cpu/dcsort.h:36-40): the BWT of text plus a sentinel,
 *     without the sentinel; primary is the sentinel's row (row of suffix 0, plus one).
 *   - Host buffers may be pageable or page-locked (sadcs_gpu_allocate_pinned); page-locked ones
 *     are copied directly at full link speed.
 *   - Status codes are GpuStatus's values (gpusa.h:22-27); the message of the last failure on the
 *     calling thread is sadcs_gpu_last_error().
 *   - A context serves one thread at a time (gpusa.h:91); different threads use different contexts.
 *     Contexts are bound to the device that was current when they were created.
 *
 * Extensions (marked "no counterpart"): 64-bit sizes with uint32 suffix arrays for texts of 2 GiB
 * and more (up to 2^32 - 256 bytes), SA and BWT from one construction, device-resident inputs and
 * outputs on a caller's stream, and the SA-to-BWT gather.
 */
#ifndef SADCS_GPU_H
#define SADCS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GpuStatus, gpusa.h:22-27. */
enum {
    SADCS_OK = 0,
    SADCS_UNAVAILABLE = 1,        /* no CUDA device or no usable driver */
    SADCS_NOT_ENOUGH_MEMORY = 2,  /* the input does not fit in free device memory / the context */
    SADCS_FAILED = 3              /* a CUDA call failed or an argument is invalid; see sadcs_gpu_last_error() */
};

/* GpuDevice, gpusa.h:29-35. */
typedef struct sadcs_gpu_device {
    char name[256];
    int32_t compute_major;
    int32_t compute_minor;
    int64_t total_bytes;
    int64_t free_bytes;
} sadcs_gpu_device;

/* GpuStats, gpusa.h:37-53 (same fields and meaning; bool pinned as int32). Seconds are host
 * wall-clock around each phase, as in the reference; device_* are CUDA-event times on the stream. */
typedef struct sadcs_gpu_stats {
    int64_t device_bytes;       /* peak device memory of the construction */
    int64_t ranking_bytes;
    int64_t class_sort_bytes;
    int64_t merge_bytes;
    int32_t pinned;             /* the transfers were direct copies of page-locked buffers */
    int32_t character_passes;
    int32_t doubling_rounds;
    int32_t reserved;
    double setup_seconds;
    double upload_seconds;
    double device_seconds;
    double ranking_seconds;
    double class_sort_seconds;
    double merge_seconds;
    double bwt_seconds;
    double download_seconds;
    /* No counterpart: CUDA-event times on the construction's stream, and the kernels it launched. */
    double ranking_device_ms;
    double class_sort_device_ms;
    double merge_device_ms;
    double merge_kernel_ms;     /* the final merge kernel alone (the level that writes the SA/BWT) */
    int64_t kernel_launches;
} sadcs_gpu_stats;

typedef struct sadcs_gpu_context sadcs_gpu_context;

/* kGpuMemoryReserve, gpusa.h:82: device memory left free when admitting a construction. */
int64_t sadcs_gpu_memory_reserve(void);

/* gpuSampleSize, gpusa.h:57-60: sample positions (cover mod 32) in a text of n bytes. */
int64_t sadcs_gpu_sample_size(int64_t n);

/* gpuQueryDevice, gpusa.h:76: the current CUDA device and its memory. */
int sadcs_gpu_query_device(sadcs_gpu_device* device);

/* gpuRequiredBytes, gpusa.h:79: peak device memory of a construction of n bytes, -1 if n is out of
 * range: about 11n, and 19n from the carry threshold on (256 MiB, or SADCS_CARRY_MIN_BYTES), where a
 * one-text context keeps room for the code words its class passes hand to the merge. */
int64_t sadcs_gpu_required_bytes(int64_t n);

/* gpuCreateContext, gpusa.h:93: device memory for inputs of up to capacity bytes, reserved once.
 * Refuses with SADCS_NOT_ENOUGH_MEMORY, allocating nothing, if the peak plus the reserve exceeds
 * the free device memory. */
int sadcs_gpu_create_context(int64_t capacity, sadcs_gpu_context** context);

/* gpuDestroyContext, gpusa.h:96. NULL is ignored. */
void sadcs_gpu_destroy_context(sadcs_gpu_context* context);

/* gpuSuffixArray, gpusa.h:102-103: the suffix array of text[0, n) into sa[0, n) (int32, so
 * n <= 2^31 - 1025 as in the reference, src/cpu/dcsort.h:21). context may be NULL: a temporary one
 * is created. With a context, n above its capacity is refused with SADCS_NOT_ENOUGH_MEMORY and the
 * context stays usable. stats may be NULL. */
int sadcs_gpu_suffix_array(sadcs_gpu_context* context, const uint8_t* text, int64_t n, int32_t* sa,
                           sadcs_gpu_stats* stats);

/* gpuBwt, gpusa.h:108-109: the BWT of text[0, n) into bwt[0, n) and its primary index.
 * bwt may equal text. */
int sadcs_gpu_bwt(sadcs_gpu_context* context, const uint8_t* text, int64_t n, uint8_t* bwt, int32_t* primary,
                  sadcs_gpu_stats* stats);

/* gpuRankSample, gpusa.h:115: ranks[pack(p)] of every sample position p (sadcs_gpu_sample_size(n)
 * entries): the number of sample suffixes smaller than suffix p. */
int sadcs_gpu_rank_sample(const uint8_t* text, int64_t n, uint32_t* ranks, sadcs_gpu_stats* stats);

/* gpuAllocatePinned / gpuFreePinned, gpusa.h:120-121. */
void* sadcs_gpu_allocate_pinned(size_t bytes);
void sadcs_gpu_free_pinned(void* pointer);

/* gpuLastError, gpusa.h:124: the last failure on this thread, "" if none. */
const char* sadcs_gpu_last_error(void);

/* ---- extensions -------------------------------------------------------------------------------- */

/* No counterpart: the suffix array (uint32) and/or the BWT of text[0, n) from ONE construction,
 * host to host, for n up to 2^32 - 256. sa or bwt may be NULL (not both). */
int sadcs_gpu_build(sadcs_gpu_context* context, const uint8_t* text, int64_t n, uint32_t* sa, uint8_t* bwt,
                    int64_t* primary, sadcs_gpu_stats* stats);

/* No counterpart: the same with device-resident buffers, on the caller's stream (a cudaStream_t,
 * NULL for the legacy default stream). d_text holds n bytes; d_sa (4n bytes) and d_bwt (n bytes) are
 * device outputs, either may be NULL (not both). Returns once the results are complete. */
int sadcs_gpu_build_device(sadcs_gpu_context* context, const uint8_t* d_text, int64_t n, uint32_t* d_sa,
                           uint8_t* d_bwt, int64_t* primary, void* stream, sadcs_gpu_stats* stats);

/* No counterpart (the SA-to-BWT gather): d_bwt[0, n) from a device suffix array, in the BWT
 * convention above; *primary gets the sentinel's row. Device buffers, caller's stream. */
int sadcs_gpu_bwt_from_sa(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, uint8_t* d_bwt,
                          int64_t* primary, void* stream);

/* No counterpart: peak device memory of a batch context for `texts` texts of `total` bytes together. */
int64_t sadcs_gpu_required_bytes_batch(int64_t total, int64_t texts);

/* No counterpart: a context for batches of up to max_texts texts of up to capacity bytes together. */
int sadcs_gpu_create_batch_context(int64_t capacity, int64_t max_texts, sadcs_gpu_context** context);

/* No counterpart: the SA (uint32, text-local positions) and/or BWT of `count` texts in ONE
 * construction. texts: the texts back to back (text j at the sum of the lengths before it);
 * outputs likewise back to back: text j's SA at sa + (sum of lengths before j), its BWT at the
 * same offset in bwt; primaries[j] gets text j's primary index (0 for an empty text). Each text's
 * SA and BWT are exactly what its own construction gives. */
int sadcs_gpu_build_batch(sadcs_gpu_context* context, const uint8_t* texts, const int64_t* lengths, int64_t count,
                          uint32_t* sa, uint8_t* bwt, int64_t* primaries, sadcs_gpu_stats* stats);

/* No counterpart: the same with device-resident texts and outputs on the caller's stream (lengths
 * and primaries are host arrays). */
int sadcs_gpu_build_batch_device(sadcs_gpu_context* context, const uint8_t* d_texts, const int64_t* lengths,
                                 int64_t count, uint32_t* d_sa, uint8_t* d_bwt, int64_t* primaries, void* stream,
                                 sadcs_gpu_stats* stats);

/* No counterpart: the reference checker's fast mode (src/common/checker.cpp:53-109) on the device.
 * Device buffers: d_text (n bytes), d_sa (n uint32 entries). *bad_index gets -1 if the suffix array
 * is correct, else the first failing SA index; *reason (if not NULL) a static description. Uses 4n
 * bytes of temporary device memory. Returns SADCS_OK whenever the check ran. */
int sadcs_gpu_check_suffix_array(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, int64_t* bad_index,
                                 const char** reason, void* stream);

/* No counterpart in the reference (its checker is CPU code that allocates host memory): the check
 * of sadcs_gpu_check_suffix_array, same arguments and results, allocating nothing - no device
 * memory, no page-locked host memory, no library routine that allocates. It is for callers that
 * must not allocate: code running beside a serving loop (sadcs_gpu_server_*) whose memory budget is
 * already promised to admitted constructions, where a new allocation could fail or take memory a
 * construction was admitted against; and code on a latency-critical path, where page-locking host
 * memory and growing a stream-ordered pool cost time and can fail.
 * Its scratch is one fixed array in the library's device code (4 MiB: the inverse suffix array of
 * up to SADCS_GPU_STATIC_CHECK_MAX entries, plus three result words). n above that limit is rejected
 * with SADCS_FAILED and a message naming the limit; nothing is launched.
 * The first call on each device looks up the array's address (cudaGetSymbolAddress), which may load
 * the library's device code: make that first call before capturing any stream. The address is kept
 * for the life of the process, so do not call this entry point again on a device after
 * cudaDeviceReset (the reset unloads the device code, and the array may come back elsewhere).
 * Initial values: the array keeps whatever the last call left; each call sets what must start
 * known before its kernels run: its three result words to all ones and the first n words of the
 * inverse suffix array to zero.
 * All calls on one device share that one array: calls that overlap in time (on other streams or
 * from other threads) race on it and their verdicts are undefined - serialise them. */
#define SADCS_GPU_STATIC_CHECK_MAX 1048576
int sadcs_gpu_check_suffix_array_static(const uint8_t* d_text, int64_t n, const uint32_t* d_sa,
                                        int64_t* bad_index, const char** reason, void* stream);

/* ---- serving (no counterpart) --------------------------------------------------------------------
 * A request loop on the current device: requests are submitted at any time and complete
 * asynchronously; queued small requests (up to small_limit bytes) are merged into one batched
 * construction of up to batch_bytes / batch_texts; a construction starts when its planned peak fits
 * memory_budget (<= 0: free memory minus the reserve) beside those running; `workers` threads with
 * their own streams overlap their constructions on the device. Each result equals the result of the
 * request's text built alone. text/sa/bwt stay owned by the caller until the request is waited for. */
typedef struct sadcs_gpu_server sadcs_gpu_server;
int sadcs_gpu_server_create(int64_t memory_budget, int32_t workers, int64_t small_limit, int64_t batch_bytes,
                            int32_t batch_texts, sadcs_gpu_server** server);
int sadcs_gpu_server_submit(sadcs_gpu_server* server, const uint8_t* text, int64_t n, uint32_t* sa, uint8_t* bwt,
                            uint64_t* ticket);
/* Blocks until the request is done (timeout_seconds < 0: no limit); latency gets queued, device and
 * total seconds; batch_size the number of requests built together with it. A ticket is waited for
 * once, by one thread: the wait that returns its result also forgets it. */
int sadcs_gpu_server_wait(sadcs_gpu_server* server, uint64_t ticket, double timeout_seconds, int64_t* primary,
                          double* latency, int32_t* batch_size);
void sadcs_gpu_server_counters(sadcs_gpu_server* server, int64_t* constructions, int64_t* launches);
/* Cancels a request that no worker has taken yet: returns SADCS_OK, and its wait returns SADCS_FAILED
 * with "cancelled". A request already being built or done, or an unknown ticket, gives SADCS_FAILED
 * and the request is left as it is. */
int sadcs_gpu_server_cancel(sadcs_gpu_server* server, uint64_t ticket);
/* Fault injection for tests of the error path: the next `count` constructions fail their device
 * allocation as the memory pool does when it is out of memory (a fake of cudaMallocFromPoolAsync
 * returning cudaErrorMemoryAllocation; nothing is allocated). Their requests complete with
 * SADCS_NOT_ENOUGH_MEMORY and the server goes on serving the others. */
void sadcs_gpu_server_fail_allocations(sadcs_gpu_server* server, int64_t count);
void sadcs_gpu_server_destroy(sadcs_gpu_server* server);

/* No counterpart: the reference's BWT check (src/common/checker.cpp:196-245) on the device: inverts
 * d_bwt (n bytes, primary) and compares with d_text. *bad_index = -1 if correct, else the first text
 * position that differs (0 if the BWT does not invert at all). Uses about 25n bytes of temporary
 * device memory. */
int sadcs_gpu_check_bwt(const uint8_t* d_text, int64_t n, const uint8_t* d_bwt, int64_t primary, int64_t* bad_index,
                        void* stream);

/* checkSuffixArray in fast mode (src/common/checker.h:24, checker.cpp:53-109) with host buffers, for
 * n up to 2^32 - 256 (uint32 entries; the reference's int32 array views the same bytes): text (n
 * bytes, no padding needed) and sa (n entries) are copied to the device and checked there by
 * sadcs_gpu_check_suffix_array. *bad_index and *reason as there (CheckResult's index and reason).
 * Uses 9n bytes of temporary device memory. Returns SADCS_OK whenever the check ran. */
int sadcs_gpu_check_suffix_array_host(const uint8_t* text, int64_t n, const uint32_t* sa, int64_t* bad_index,
                                      const char** reason);

/* checkBwt (src/common/checker.h:29, checker.cpp:196-245) with host buffers: text and bwt (n bytes
 * each) and primary, checked on the device by sadcs_gpu_check_bwt. *bad_index = -1 if the BWT
 * inverts to the text, else the first text position where it does not (0 if it does not invert).
 * Uses about 27n bytes of temporary device memory. */
int sadcs_gpu_check_bwt_host(const uint8_t* text, int64_t n, const uint8_t* bwt, int64_t primary, int64_t* bad_index);

/* No counterpart: the inverse BWT (unbwt) on the device: d_text (n bytes) from d_bwt and primary.
 * Returns SADCS_FAILED if d_bwt is not a valid BWT. */
int sadcs_gpu_inverse_bwt(const uint8_t* d_bwt, int64_t n, int64_t primary, uint8_t* d_text, void* stream);

/* No counterpart (the reference computes no LCP array): the longest-common-prefix array of a suffix
 * array on the device. lcp[0] = 0 and lcp[r] = the length of the longest common prefix of suffixes
 * d_sa[r - 1] and d_sa[r], for d_sa (n uint32 entries) the suffix array of d_text (n bytes, no
 * padding needed), n up to 2^32 - 256. d_lcp gets n uint32 entries and may be d_sa itself (the
 * suffix array is then replaced by its LCP array). Uses about 4.13n bytes of temporary device memory;
 * returns when the array is complete. A d_sa that is not the suffix array of d_text gives an
 * unspecified d_lcp, never a read outside the buffers. */
int sadcs_gpu_lcp(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, uint32_t* d_lcp, void* stream);

/* No counterpart: a test of the failure path of the radix passes' bounded wait (the decoupled
 * look-back, which every construction's sorts use). Runs one radix pass on a stream of its own in
 * which the only block waits on a predecessor tile that is never taken, so that nothing ever
 * publishes the status it waits for; after limit_cycles SM cycles (1 to 4e9) of waiting the block
 * gives up as a construction's pass would: it sets the pass's error word and stores nothing, and the
 * kernel returns. *error_word gets the error word. Returns SADCS_FAILED with the message of the
 * time-out when that happened (the expected outcome), SADCS_OK if the pass did not wait, and
 * SADCS_FAILED with a CUDA error's message otherwise. Uses about 100 KB of temporary device memory. */
int sadcs_gpu_test_lookback_timeout(int64_t limit_cycles, uint32_t* error_word);

/* No counterpart: the capacity (bytes of text) of a context. */
int64_t sadcs_gpu_context_capacity(const sadcs_gpu_context* context);

#ifdef __cplusplus
}
#endif

#endif
