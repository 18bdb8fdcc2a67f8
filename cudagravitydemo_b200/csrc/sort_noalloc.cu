// sort_noalloc.cu — the key/permutation radix sort without any allocation.
//
// bh_radix_sort_pairs() needs a sorter, whose scratch (temporary key and
// value buffers, digit histograms, look-back status words) comes from
// cudaMalloc.  Some callers cannot allocate at the point where they sort:
// code that must not stall the device (cudaFree synchronises it), or a
// plugin running inside a host framework whose own allocator has already
// reserved the device memory.  For them,
// bh_radix_sort_pairs_noalloc() sorts with scratch that lives in this file's
// statically allocated device array instead.
//
// The first call on a device resolves the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before capturing any stream.  Later calls outside a stream capture resolve
// it again (cheap), so a device reset between calls is followed.  A
// look-back wait that gives up leaves BH_ERR_TIMEOUT in the array's error
// word; bh_radix_sort_noalloc_errors() reads it.  The array holds the scratch
// for at most BH_NOALLOC_SORT_MAX pairs and is part of the library image:
// every GPU that loads the library holds it (about 3.6 MB) until the process
// exits.  All calls share it, and each call leaves
// its contents behind; everything the sort needs zeroed is cleared at the
// start of every call.  Calls that overlap on the GPU (different streams, or
// different host threads without ordering between them) race on the array.
#include <mutex>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"
#include "sorting.h"

namespace {

constexpr int kMaxPairs = BH_NOALLOC_SORT_MAX;
constexpr int kPasses = 8;  // up to 64 key bits
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Layout of the scratch array (byte offsets).
constexpr size_t kTileCount(int tile) { return (size_t)(kMaxPairs + tile - 1) / tile; }
constexpr size_t kKeysOff = 0;
constexpr size_t kValsOff = align256(kKeysOff + sizeof(uint64_t) * kMaxPairs);
constexpr size_t kHistOff = align256(kValsOff + sizeof(uint32_t) * kMaxPairs);
constexpr size_t kStatusOff = align256(kHistOff + sizeof(uint32_t) * kPasses * 256);
constexpr int kSortTile = 4096;  // keys per tile of k_sort_pass (radix_sort.cu)
constexpr size_t kStatusWords = 256 + (size_t)kPasses * kTileCount(kSortTile) * 256;
constexpr size_t kErrOff = align256(kStatusOff + sizeof(uint32_t) * kStatusWords);
constexpr size_t kScratchBytes = align256(kErrOff + sizeof(int));

// The scratch itself: file-scope, statically allocated device memory.
static __device__ __align__(256) unsigned char g_sortScratch[kScratchBytes];

// Device address of g_sortScratch, resolved once per device.  In host code
// the name g_sortScratch is only a host-side stand-in for the symbol, never a
// device address, so kernels get the resolved pointer.
constexpr int kMaxDevices = 64;
unsigned char* g_scratchAddr[kMaxDevices] = {};
std::mutex g_setupMutex;

// s: the stream the caller will use; while it is being captured, the cached
// address is used as it is (no runtime call that capture could object to).
int scratch_for_current_device(cudaStream_t s, unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    if (dev < 0 || dev >= kMaxDevices) return BH_ERR_INVALID;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (cap != cudaStreamCaptureStatusNone) {
        if (!g_scratchAddr[dev]) return BH_ERR_INVALID;  // set-up must come before capture
        *out = g_scratchAddr[dev];
        return BH_OK;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sortScratch);  // with `dev` current
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    if (g_scratchAddr[dev] != p) {
        // first call on this device (or the module was reloaded): the
        // digit-pass kernel needs its dynamic shared-memory limit raised on
        // this device (a function attribute, not an allocation)
        e = bh_sort_init();
        if (e != cudaSuccess) return bh_note_cuda_error(e);
        g_scratchAddr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratchAddr[dev];
    return BH_OK;
}

int sort_noalloc(const uint64_t* keysIn, uint64_t* keysOut, const uint32_t* valsIn, uint32_t* valsOut, int n,
                 int keyBits, cudaStream_t s) {
    if (!keysIn || !keysOut || !valsIn || !valsOut || keyBits < 1 || keyBits > 64) return BH_ERR_INVALID;
    if (n <= 0 || n > kMaxPairs) return BH_ERR_INVALID;  // beyond the static scratch
    if (bh_sort_tile() != kSortTile) return BH_ERR_INTERNAL;
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(s, &base);
    if (rc) return rc;
    uint64_t* keysTmp = reinterpret_cast<uint64_t*>(base + kKeysOff);
    uint32_t* valsTmp = reinterpret_cast<uint32_t*>(base + kValsOff);
    uint32_t* hist = reinterpret_cast<uint32_t*>(base + kHistOff);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kStatusOff);
    int* err = reinterpret_cast<int*>(base + kErrOff);

    const int npass = (keyBits + 7) / 8;
    const int tiles = (n + kSortTile - 1) / kSortTile;
    // what must start at zero: histograms, tile counters, look-back words,
    // the error word (a previous call leaves them dirty)
    BH_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * npass * 256, s));
    BH_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(uint32_t) * (256 + (size_t)npass * tiles * 256), s));
    BH_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
    BH_CUDA_TRY(bh_launch_sort_histogram(keysIn, n, hist, npass, s));
    const uint64_t* ksrc = keysIn;
    const uint32_t* vsrc = valsIn;
    for (int p = 0; p < npass; p++) {
        const bool toOut = ((npass - 1 - p) % 2) == 0;
        uint64_t* kdst = toOut ? keysOut : keysTmp;
        uint32_t* vdst = toOut ? valsOut : valsTmp;
        BH_CUDA_TRY(bh_launch_sort_pass(ksrc, vsrc, kdst, vdst, n, 8 * p, hist + 256 * p,
                                        status + 256 + (size_t)p * tiles * 256, reinterpret_cast<int*>(status) + p,
                                        err, 0, s));
        ksrc = kdst;
        vsrc = vdst;
    }
    return BH_OK;
}

}  // namespace

extern "C" int bh_radix_sort_pairs_noalloc(const uint64_t* keysIn, uint64_t* keysOut, const uint32_t* valsIn,
                                           uint32_t* valsOut, int n, int keyBits, cudaStream_t s) {
    return bh_record_status(sort_noalloc(keysIn, keysOut, valsIn, valsOut, n, keyBits, s));
}

// The error word of the last bh_radix_sort_pairs_noalloc() on the current
// device, read after the work queued on `s` (the stream of that call).  The
// next call clears it.
extern "C" int bh_radix_sort_noalloc_errors(int* errorBits, cudaStream_t s) {
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(s, &base);
    if (rc) return bh_record_status(rc);
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, base + kErrOff, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bh_record_status(bh_note_cuda_error(e));
    if (errorBits) *errorBits = h;
    return bh_record_status(bh_status_from_bits(h));
}

// Failure detection without a fault: the look-back wait run against the
// array's own status words, with a predecessor tile that never publishes.  It
// gives up and leaves BH_ERR_TIMEOUT in the array's error word, where
// bh_radix_sort_noalloc_errors() must find it.
extern "C" int bh_selftest_noalloc_timeout(cudaStream_t s) {
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(s, &base);
    if (rc) return bh_record_status(rc);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kStatusOff);
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t) * 2 * 256, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + kErrOff, 0, sizeof(int), s);
    if (e == cudaSuccess) e = bh_launch_lookback_selftest(status, reinterpret_cast<int*>(base + kErrOff), s);
    return bh_record_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}
