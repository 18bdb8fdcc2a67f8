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

#ifdef __cplusplus
}
#endif

#endif /* BH_SORTING_H */
