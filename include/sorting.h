/*
 * sorting.h — key/permutation radix sort of the B200 Barnes-Hut engine.
 *
 * Drop-in counterpart of the reference's sorting.h (sorting.h:12-23), which
 * wraps CUB's DeviceRadixSort::SortPairs (sorting.cu:15-92).  Here the sort is
 * this library's own onesweep LSD radix sort for sm_100a (8-bit digits,
 * decoupled look-back); the semantics are the reference's: a STABLE ascending
 * sort of (uint64 key, uint32 value) pairs, inputs left untouched, results in
 * separate output buffers.
 *
 * Two forms of each entry point:
 *   - the reference's names and argument meaning; on an error they print a
 *     message and call exit(-1), as the reference does (sorting.cu:16-20,
 *     73-76, 84-87);
 *   - `bh_*` variants that return a bh_status code instead.
 * All device pointers are caller-allocated device memory.
 */
#ifndef BH_SORTING_H
#define BH_SORTING_H

#include <stdint.h>
#include <driver_types.h> /* cudaStream_t */
#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces sorterCreate (sorting.h:14, sorting.cu:15-63): a sorter able to
 * sort up to maxCount pairs.  Allocates its scratch once. */
radixSorter* sorterCreate(int maxCount);

/* Replaces radixSortPairs (sorting.h:16-18, sorting.cu:65-79): stable sort of
 * numCount pairs by all 64 key bits, on the legacy default stream. */
void radixSortPairs(radixSorter* sorter, const uint64_t* keysIn, uint64_t* keysOut,
                    const uint32_t* valsIn, uint32_t* valsOut, int numCount);

/* Replaces sorterDestroyer (sorting.h:20, sorting.cu:81-92). */
void sorterDestroyer(radixSorter* sorter);

/* Replaces the reorderParticles kernel (sorting.h:12, sorting.cu:99-107):
 * posOut[i] = posIn[originalIndex[i]], velOut[i] = velIn[originalIndex[i]].
 * A launcher: the reference's `<<<g,b>>>` becomes a call with a stream. */
void reorderParticles(const float4* posMassValsIn, const float3* velValsIn,
                      float4* posMassValsOut, float3* velValsOut,
                      uint32_t* originalIndex, int starCount, cudaStream_t stream);

/* Status-returning variants (bh_status codes, see bh_api.h). keyBits limits
 * the sort to the low keyBits bits (ceil(keyBits/8) digit passes); 64 gives
 * the reference's full-width sort. */
int bh_sorter_create(radixSorter** out, int maxCount);
int bh_radix_sort_pairs(radixSorter* sorter, const uint64_t* keysIn, uint64_t* keysOut,
                        const uint32_t* valsIn, uint32_t* valsOut, int numCount,
                        int keyBits, cudaStream_t stream);
int bh_sorter_destroy(radixSorter* sorter);

/* No counterpart in the reference (CUB reports no device-side errors).  The
 * passes' look-back waits are bounded: a wait that gives up sets
 * BH_ERR_TIMEOUT in the sorter's device error word instead of hanging, and
 * the bh_radix_sort_pairs() call has already returned BH_OK by then.  This
 * reads that word after the work queued on `stream` (it waits for it),
 * returns the lowest error as a bh_status, stores the raw bits in *errorBits
 * (optional) and clears the word; call it outside a stream capture.
 * radixSortPairs() does this itself after every sort and exits on an error. */
int bh_sorter_errors(radixSorter* sorter, int* errorBits, cudaStream_t stream);

/* Self-test of the error path above, with no fault: runs the look-back wait
 * on the sorter's own status words with a predecessor that never publishes,
 * so that the wait gives up (about a second) and bh_sorter_errors() then
 * returns BH_ERR_TIMEOUT.  The sorter stays usable. */
int bh_selftest_sorter_timeout(radixSorter* sorter, cudaStream_t stream);

/* Most pairs bh_radix_sort_pairs_noalloc() sorts: the size of its static
 * scratch (about 3.6 MB of device memory per GPU that loads the library). */
#define BH_NOALLOC_SORT_MAX 262144

/* No counterpart in the reference.  The same stable sort as
 * bh_radix_sort_pairs(), for callers that cannot allocate device memory where
 * they sort: code that must not stall the device (cudaFree synchronises it),
 * or a plugin whose host framework's allocator has already reserved the
 * device memory.  It allocates nothing: the scratch is a statically allocated
 * array inside the library, shared by all calls.
 *   - numCount must be 1..BH_NOALLOC_SORT_MAX; larger inputs are rejected
 *     with BH_ERR_INVALID (use a sorter from bh_sorter_create instead);
 *   - the first call on a device resolves the array's address on that device:
 *     make it before any stream capture;
 *   - calls that overlap on the GPU race on the shared array: order them
 *     (one stream, or events between streams);
 *   - inputs are left untouched; results go to keysOut/valsOut;
 *   - the return code covers the arguments and the launches; a look-back
 *     wait that gives up on the device is reported by
 *     bh_radix_sort_noalloc_errors(). */
int bh_radix_sort_pairs_noalloc(const uint64_t* keysIn, uint64_t* keysOut, const uint32_t* valsIn,
                                uint32_t* valsOut, int numCount, int keyBits, cudaStream_t stream);

/* The device error word of the last bh_radix_sort_pairs_noalloc() on the
 * current device (it lives in the same static array), read after the work
 * queued on `stream` (it waits for it): BH_OK, or BH_ERR_TIMEOUT when a
 * look-back wait gave up; raw bits in *errorBits (optional).  Read it before
 * the next call, which clears it, and outside a stream capture (it waits for
 * the stream).  Allocates nothing. */
int bh_radix_sort_noalloc_errors(int* errorBits, cudaStream_t stream);

/* Self-test of that error path, with no fault: the look-back wait run on the
 * static array's status words with a predecessor that never publishes; it
 * gives up, and bh_radix_sort_noalloc_errors() then returns BH_ERR_TIMEOUT.
 * The next sort clears the word. */
int bh_selftest_noalloc_timeout(cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* BH_SORTING_H */
