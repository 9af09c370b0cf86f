// cn_noalloc.cu -- the broadphase cell-key sort for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc while they step: code running inside an
// engine whose device memory is owned by its own pool or arena (a renderer or RL environment
// that hands out sub-allocations and forbids foreign allocations), frame loops that must not hit
// the allocator's implicit device synchronisation, and real-time callers that pre-reserve every
// byte at start-up.  cn_sort_cell_keys_noalloc gives them the stable (cellKey, particleIndex) sort
// of the broadphase without any allocation: its scratch (digit histograms, look-back flags and the
// ping-pong key/index arrays) lives in one file-scope device array, sized for at most
// kNoAllocMaxKeys keys, that every GPU loading the library holds until the process exits.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_device.h"
#include "cn_internal.h"

namespace {

constexpr uint32_t kNoAllocMaxKeys = 1u << 20;               // 1,048,576 keys
constexpr size_t kMetaWords = size_t(1) << 19;               // 2 MiB: histograms, tile counters, look-back
constexpr size_t kScratchWords = kMetaWords + 2 * size_t(kNoAllocMaxKeys) + 64; // + ping-pong keys/indices
// ~10 MiB per device.  Shared by every call: the sort clears its histogram / look-back region at
// the start of each call; the ping-pong arrays need no clearing.
static __device__ __align__(256) uint32_t g_noAllocSortScratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
uint32_t *g_scratchPtr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code the array's name is
// only a host-side stand-in, so the address must come from cudaGetSymbolAddress, once per device
// with that device current.  The address is cached for the life of the process: after
// cudaDeviceReset (which unloads the module and may place the array elsewhere) the cached address
// is stale, so this entry point must not be called on a device that has been reset.
cn_status scratchForCurrentDevice(uint32_t **out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return cn::setError(CN_ERR_NO_DEVICE, std::string("cn_sort_cell_keys_noalloc: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices)
        return cn::setError(CN_ERR_UNSUPPORTED, "cn_sort_cell_keys_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchPtr[device]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noAllocSortScratch);
        if (e != cudaSuccess || ptr == nullptr)
            return cn::setError(CN_ERR_CUDA, std::string("cn_sort_cell_keys_noalloc: cudaGetSymbolAddress: ") +
                                                 cudaGetErrorString(e));
        g_scratchPtr[device] = static_cast<uint32_t *>(ptr);
    }
    *out = g_scratchPtr[device];
    return CN_OK;
}

} // namespace

extern "C" {

CN_API cn_status cn_sort_cell_keys_noalloc(const uint32_t *keys, uint32_t *sorted_keys, uint32_t *sorted_indices,
                                           uint32_t count, uint32_t *out_timeouts, void *stream)
{
    if (count > kNoAllocMaxKeys)
        return cn::setError(CN_ERR_CAPACITY, "cn_sort_cell_keys_noalloc: " + std::to_string(count) +
                                                 " keys exceed the allocation-free limit of 1048576");
    if (count == 0) {
        if (out_timeouts)
            return cudaMemsetAsync(out_timeouts, 0, sizeof(uint32_t), static_cast<cudaStream_t>(stream)) == cudaSuccess
                       ? CN_OK
                       : cn::setError(CN_ERR_CUDA, "cn_sort_cell_keys_noalloc: cudaMemsetAsync failed");
        return CN_OK;
    }
    if (!keys || !sorted_keys || !sorted_indices)
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_sort_cell_keys_noalloc: null device pointer");
    // The sort works in place on (sorted_keys, sorted_indices) after copying the keys there, so an
    // output that is the input would sort `keys` in place, and the two outputs must be distinct.
    if (sorted_keys == keys || sorted_indices == keys || sorted_indices == sorted_keys)
        return cn::setError(CN_ERR_INVALID_ARGUMENT,
                            "cn_sort_cell_keys_noalloc: keys, sorted_keys and sorted_indices must not alias");
    if (cn::radixSortScratchBytes(count) > kMetaWords * sizeof(uint32_t))
        return cn::setError(CN_ERR_CAPACITY, "cn_sort_cell_keys_noalloc: sort metadata exceeds its reserved region");
    uint32_t *scratch = nullptr;
    const cn_status st = scratchForCurrentDevice(&scratch);
    if (st != CN_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t *meta = scratch;
    uint32_t *keysB = scratch + kMetaWords;
    uint32_t *valsB = keysB + kNoAllocMaxKeys;
    uint32_t *timeouts = valsB + kNoAllocMaxKeys;
    // The sort runs in place on (sorted_keys, sorted_indices) with the scratch arrays as the
    // ping-pong pair; it zeroes its histogram and look-back words itself.
    // The timeout word counts look-back waits that gave up during this call; it starts at zero.
    cudaError_t e = cudaMemsetAsync(timeouts, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sorted_keys, keys, size_t(count) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess)
        return cn::setError(CN_ERR_CUDA, std::string("cn_sort_cell_keys_noalloc: ") + cudaGetErrorString(e));
    cn::radixSortPairs(sorted_keys, sorted_indices, keysB, valsB, count, meta, timeouts, s);
    // A nonzero count means a tile stopped waiting for an earlier tile's digit counts, so its
    // offsets (and the output permutation) are wrong; the caller reads it once `stream` is done.
    if (out_timeouts)
        cudaMemcpyAsync(out_timeouts, timeouts, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cn::setError(CN_ERR_CUDA, std::string("cn_sort_cell_keys_noalloc: ") + cudaGetErrorString(e));
    return CN_OK;
}

} // extern "C"
