// cn_sort.cu -- stable radix sort of the broadphase (cellKey, particleIndex) pairs and a
// device-wide exclusive scan.
//
// The reference sorts with 32 one-bit split passes, each classify -> exclusive scan ->
// finalize -> scatter (src/physics/physics_pass_dispatcher.cpp:3963-4057,
// assets/shaders/physics/shared/physics_radix_{classify,finalize,scatter}.cs.hlsl).  Any stable
// LSD sort yields the same permutation, so this file sorts 8 bits per pass in 4 "onesweep"
// passes: one kernel per pass ranks its 4096-key tile with warp match/ballot digit ranking,
// publishes per-digit tile counts, resolves its global digit offsets by decoupled look-back
// over earlier tiles and scatters through shared memory so that global writes are contiguous
// per digit run.  Every look-back spin is bounded; a spin that gives up bumps a timeout
// counter (read back through cn_solver_validate_meta) instead of hanging the GPU.
#include <cstdint>
#include <cuda_runtime.h>

#include "cn_device.h"

namespace cn {
namespace {

constexpr int kRadix = 256;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kSortThreads * kItems; // 4096 keys
constexpr int kWarpTile = 32 * kItems;       // 512 keys per warp

constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagInclusive = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;

struct SortScratch {
    uint32_t *hist;      // [4][256] digit counts, then exclusive offsets
    uint32_t *counters;  // [4] tile counters
    uint32_t *lookback;  // [4][tiles][256]
};

__host__ __device__ inline uint32_t numTiles(uint32_t n) { return (n + kTile - 1) / kTile; }

SortScratch carve(void *scratch, uint32_t n)
{
    uint8_t *p = static_cast<uint8_t *>(scratch);
    SortScratch s;
    s.hist = reinterpret_cast<uint32_t *>(p);
    p += 4 * kRadix * sizeof(uint32_t);
    s.counters = reinterpret_cast<uint32_t *>(p);
    p += 64;
    s.lookback = reinterpret_cast<uint32_t *>(p);
    return s;
}

// One pass over the keys builds all four digit histograms.
__device__ __forceinline__ uint32_t liveCount(uint32_t n, const uint32_t *count)
{
    return count ? min(n, *count) : n;
}

__global__ void __launch_bounds__(256) k_radixHistogram(const uint32_t *__restrict__ keys, uint32_t capacity,
                                                        const uint32_t *__restrict__ count,
                                                        uint32_t *__restrict__ hist)
{
    const uint32_t n = liveCount(capacity, count);
    __shared__ uint32_t sh[4][kRadix];
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t k = keys[i];
        atomicAdd(&sh[0][k & 255u], 1u);
        atomicAdd(&sh[1][(k >> 8) & 255u], 1u);
        atomicAdd(&sh[2][(k >> 16) & 255u], 1u);
        atomicAdd(&sh[3][k >> 24], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) {
        const uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Exclusive scan of each 256-bucket histogram (one block of 256 threads, 4 digits).
__global__ void __launch_bounds__(256) k_radixHistogramScan(uint32_t *hist)
{
    __shared__ uint32_t sh[kRadix];
    for (int d = 0; d < 4; ++d) {
        const uint32_t v = hist[d * kRadix + threadIdx.x];
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < kRadix; off <<= 1) {
            const uint32_t t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0u;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        hist[d * kRadix + threadIdx.x] = sh[threadIdx.x] - v;
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t ldVolatile(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void stRelease(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One onesweep pass over digit `shift`.  firstPass: the value of each key is its input index.
template <bool kFirstPass>
__global__ void __launch_bounds__(kSortThreads) k_onesweep(const uint32_t *__restrict__ keysIn,
                                                           const uint32_t *__restrict__ valsIn,
                                                           uint32_t *__restrict__ keysOut,
                                                           uint32_t *__restrict__ valsOut, uint32_t capacity,
                                                           const uint32_t *__restrict__ count, uint32_t shift,
                                                           const uint32_t *__restrict__ digitOffsets,
                                                           uint32_t *lookback, uint32_t *tileCounter,
                                                           uint32_t *waitTimeouts)
{
    __shared__ uint32_t warpHist[kSortWarps][kRadix];
    __shared__ uint32_t tileDigitStart[kRadix];
    __shared__ uint32_t digitGlobal[kRadix];
    __shared__ uint32_t stageKeys[kTile];
    __shared__ uint32_t stageVals[kTile];
    __shared__ uint32_t tileId;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) tileId = atomicAdd(tileCounter, 1u);
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&warpHist[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t tile = tileId;
    const uint32_t n = liveCount(capacity, count);
    // Tiles past a device-side count have nothing to sort.  Tickets are handed out in order, so
    // every tile a live tile looks back on is live too.
    if (tile >= numTiles(n)) return;
    const uint32_t warpBase = tile * kTile + warp * kWarpTile;

    uint32_t key[kItems], val[kItems], rnk[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t idx = warpBase + j * 32 + lane;
        if (idx < n) {
            key[j] = keysIn[idx];
            val[j] = kFirstPass ? idx : valsIn[idx];
        } else {
            key[j] = 0xffffffffu; // padding sorts behind every valid key of digit 255
            val[j] = 0xffffffffu;
        }
    }
    const uint32_t lanesBelow = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t d = (key[j] >> shift) & 255u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t below = __popc(peers & lanesBelow);
        const int leader = __ffs(peers) - 1;
        const uint32_t base = warpHist[warp][d];
        __syncwarp();
        if (lane == leader) warpHist[warp][d] = base + __popc(peers);
        __syncwarp();
        rnk[j] = base + below;
    }
    __syncthreads();

    // Exclusive prefix of each digit across warps (warp order is input order).
    const uint32_t t = threadIdx.x; // one thread per digit
    uint32_t tileCount = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = warpHist[w][t];
        warpHist[w][t] = tileCount;
        tileCount += c;
    }

    // Publish this tile's digit count, then resolve the exclusive prefix over earlier tiles.
    uint32_t *myLook = lookback + size_t(tile) * kRadix + t;
    if (tile == 0) {
        stRelease(myLook, kFlagInclusive | tileCount);
        digitGlobal[t] = digitOffsets[t];
    } else {
        stRelease(myLook, kFlagAggregate | tileCount);
        uint32_t exclusive = 0;
        int32_t k = int32_t(tile) - 1;
        uint32_t spins = 0;
        while (k >= 0) {
            const uint32_t v = ldVolatile(lookback + size_t(k) * kRadix + t);
            const uint32_t flag = v & ~kValueMask;
            if (flag == 0u) {
                if (++spins > kSpinLimit) {
                    atomicAdd(waitTimeouts, 1u);
                    break;
                }
                continue;
            }
            exclusive += v & kValueMask;
            if (flag == kFlagInclusive) break;
            --k;
        }
        stRelease(myLook, kFlagInclusive | (exclusive + tileCount));
        digitGlobal[t] = digitOffsets[t] + exclusive;
    }

    // Tile-local digit starts (exclusive scan of tileCount over digits).
    tileDigitStart[t] = tileCount;
    __syncthreads();
    for (int off = 1; off < kRadix; off <<= 1) {
        const uint32_t v = t >= uint32_t(off) ? tileDigitStart[t - off] : 0u;
        __syncthreads();
        tileDigitStart[t] += v;
        __syncthreads();
    }
    const uint32_t inclusiveStart = tileDigitStart[t];
    __syncthreads();
    tileDigitStart[t] = inclusiveStart - tileCount;
    __syncthreads();

    // Stage the tile in digit order, then write contiguous runs.
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t d = (key[j] >> shift) & 255u;
        const uint32_t local = tileDigitStart[d] + warpHist[warp][d] + rnk[j];
        stageKeys[local] = key[j];
        stageVals[local] = val[j];
    }
    __syncthreads();
    const uint32_t tileBase = tile * kTile;
    const uint32_t valid = n > tileBase ? min(uint32_t(kTile), n - tileBase) : 0u;
#pragma unroll 4
    for (int i = threadIdx.x; i < kTile; i += kSortThreads) {
        if (uint32_t(i) >= valid) break;
        const uint32_t k = stageKeys[i];
        const uint32_t d = (k >> shift) & 255u;
        const uint32_t dst = digitGlobal[d] + (uint32_t(i) - tileDigitStart[d]);
        keysOut[dst] = k;
        valsOut[dst] = stageVals[i];
    }
}

// ---- exclusive scan (reduce, scan of partials, down-sweep) ----
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t &total)
{
    __shared__ uint32_t warpSums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warpSums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warpSums[lane] = w;
    }
    __syncthreads();
    const uint32_t warpPrefix = warp > 0 ? warpSums[warp - 1] : 0u;
    total = warpSums[kScanThreads / 32 - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scanReduce(const uint32_t *__restrict__ in, uint32_t n,
                                                             uint32_t *__restrict__ partials)
{
    const uint32_t base = blockIdx.x * kScanChunk;
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t idx = base + i * kScanThreads + threadIdx.x;
        if (idx < n) sum += in[idx];
    }
    uint32_t total;
    blockExclusiveScan(sum, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scanPartials(uint32_t *partials, uint32_t count,
                                                               uint32_t *total)
{
    uint32_t carry = 0;
    for (uint32_t base = 0; base < count; base += kScanThreads) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t v = idx < count ? partials[idx] : 0u;
        uint32_t t;
        const uint32_t ex = blockExclusiveScan(v, t);
        if (idx < count) partials[idx] = carry + ex;
        carry += t;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scanDown(const uint32_t *__restrict__ in, uint32_t n,
                                                           const uint32_t *__restrict__ partials,
                                                           uint32_t *__restrict__ out)
{
    // Blocked layout: thread t owns kScanItems consecutive elements of the chunk.
    const uint32_t base = blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    uint32_t vals[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t idx = base + i;
        vals[i] = idx < n ? in[idx] : 0u;
        sum += vals[i];
    }
    uint32_t total;
    uint32_t prefix = blockExclusiveScan(sum, total) + partials[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t idx = base + i;
        if (idx < n) out[idx] = prefix;
        prefix += vals[i];
    }
}

// Small inputs (at most kScanSingleMax elements): one CTA walks the chunks with a running carry,
// the same integers in one launch instead of three.
constexpr uint32_t kScanSingleMax = 8u * kScanChunk;
__global__ void __launch_bounds__(kScanThreads) k_scanSingle(const uint32_t *__restrict__ in, uint32_t n,
                                                             uint32_t *__restrict__ out, uint32_t *total)
{
    uint32_t carry = 0;
    for (uint32_t chunk = 0; chunk < n; chunk += kScanChunk) {
        const uint32_t base = chunk + threadIdx.x * kScanItems;
        uint32_t vals[kScanItems];
        uint32_t sum = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const uint32_t idx = base + i;
            vals[i] = idx < n ? in[idx] : 0u;
            sum += vals[i];
        }
        uint32_t t;
        uint32_t prefix = blockExclusiveScan(sum, t) + carry;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const uint32_t idx = base + i;
            if (idx < n) out[idx] = prefix;
            prefix += vals[i];
        }
        carry += t;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

} // namespace

size_t radixSortScratchBytes(uint32_t n)
{
    return 4 * kRadix * sizeof(uint32_t) + 64 + size_t(4) * numTiles(n) * kRadix * sizeof(uint32_t);
}

void radixSortPairs(uint32_t *keysA, uint32_t *valsA, uint32_t *keysB, uint32_t *valsB, uint32_t n,
                    void *scratch, uint32_t *waitTimeouts, cudaStream_t st, const uint32_t *count)
{
    if (n == 0) return;
    const SortScratch s = carve(scratch, n);
    const uint32_t tiles = numTiles(n);
    cudaMemsetAsync(scratch, 0, radixSortScratchBytes(n), st);
    const uint32_t histBlocks = min(tiles * 4u, 148u * 4u);
    k_radixHistogram<<<histBlocks, 256, 0, st>>>(keysA, n, count, s.hist);
    k_radixHistogramScan<<<1, 256, 0, st>>>(s.hist);
    uint32_t *kin = keysA, *vin = valsA, *kout = keysB, *vout = valsB;
    for (int pass = 0; pass < 4; ++pass) {
        uint32_t *look = s.lookback + size_t(pass) * tiles * kRadix;
        if (pass == 0)
            k_onesweep<true><<<tiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, count, 0u, s.hist, look,
                                                             s.counters + 0, waitTimeouts);
        else
            k_onesweep<false><<<tiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, count, 8u * pass,
                                                              s.hist + pass * kRadix, look,
                                                              s.counters + pass, waitTimeouts);
        uint32_t *tk = kin, *tv = vin;
        kin = kout; vin = vout; kout = tk; vout = tv;
    }
    // After four passes the result is back in (keysA, valsA); with a count, only [0, count).
}

size_t scanScratchBytes(uint32_t n)
{
    const uint32_t blocks = (n + kScanChunk - 1) / kScanChunk;
    return size_t(blocks + 1) * sizeof(uint32_t);
}

void exclusiveScan(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *total, void *scratch,
                   cudaStream_t st)
{
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    if (n <= kScanSingleMax) {
        k_scanSingle<<<1, kScanThreads, 0, st>>>(in, n, out, total);
        return;
    }
    uint32_t *partials = static_cast<uint32_t *>(scratch);
    const uint32_t blocks = (n + kScanChunk - 1) / kScanChunk;
    k_scanReduce<<<blocks, kScanThreads, 0, st>>>(in, n, partials);
    k_scanPartials<<<1, kScanThreads, 0, st>>>(partials, blocks, total);
    k_scanDown<<<blocks, kScanThreads, 0, st>>>(in, n, partials, out);
}

} // namespace cn
