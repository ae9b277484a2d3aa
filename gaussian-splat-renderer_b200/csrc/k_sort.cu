// Sorting the (tile | depth) list, the tile ranges, and the standalone prefix-sum primitive.
//
// The sort is a stable LSD radix sort over 8-bit digits in the onesweep form (Adinets and
// Merrill, 2022): one histogram kernel computes the digit counts of every pass in a single
// read of the keys, then each pass is ONE kernel whose blocks (ordered by a ticket) rank their
// 4096-key tile locally with warp-level multisplit (match.any), publish per-digit counts, get
// their global digit offsets by a decoupled look-back over the earlier tiles, and scatter
// through shared memory. Ties keep their input order (warp order, then lane/item order).
//
// Key shortening: the list key is (tile << 32 | depth bits). All depth bits above the highest
// bit where the frame's smallest and largest depth differ are equal for every key, and so are
// the tile bits above the largest tile id; the sort therefore orders the "virtual key"
// (tile << W | depth & (2^W - 1)) with W = bit_width(depthMin ^ depthMax), which is the same
// order with fewer passes (the reference's radixSortPairs skips constant digits in the same
// spirit, src/splat/depth_sort.cpp:53-56). Passes whose digit is constant over all keys are
// skipped as well. The reference's GPU sort sorts all keyBits = 32 + tileBits bits
// (gpu_radix_sort.cpp); the result of a stable sort is the same either way.
#include "gsr_device.cuh"
#include "kernels.cuh"

namespace gsr {

namespace {

__device__ __forceinline__ uint32_t bitWidth(uint32_t x) { return x ? 32u - __clz(x) : 0u; }

__device__ __forceinline__ uint64_t virtualKey(uint64_t key, uint32_t lowBits, uint64_t keyMask) {
    const uint64_t low = lowBits >= 32 ? (key & 0xFFFFFFFFull) : (key & ((1ull << lowBits) - 1ull));
    const uint64_t hi = key >> 32;
    return ((lowBits >= 64 ? 0ull : (hi << lowBits)) | low) & keyMask;
}

__device__ __forceinline__ uint64_t maskOf(uint32_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1ull); }

__device__ __forceinline__ uint32_t laneMaskLt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Block-wide exclusive scan of one value per thread (256 threads); returns the exclusive
// prefix, *total = the sum.
__device__ __forceinline__ uint32_t blockExclusiveScan256(uint32_t v, uint32_t* sWarp, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= uint32_t(d)) incl += o;
    }
    if (lane == 31) sWarp[warp] = incl;
    __syncthreads();
    uint32_t base = 0, sum = 0;
#pragma unroll
    for (uint32_t w = 0; w < 8; ++w) {
        const uint32_t t = sWarp[w];
        if (w < warp) base += t;
        sum += t;
    }
    __syncthreads();
    *total = sum;
    return base + incl - v;
}

// ---- histogram of every pass's digit + the plan ---------------------------------------------
__global__ void __launch_bounds__(256) sortHistKernel(const __grid_constant__ SortArgs a) {
    __shared__ uint32_t sHist[kMaxSortPasses][256];
    __shared__ uint32_t sWarp[8];
    __shared__ uint32_t sLast;
    __shared__ uint32_t sAny;
    DeviceControl* ctl = a.ctl;
    const uint32_t entries = ctl->c.entries;
    uint32_t lowBits, keyBits, packed = 0, indexBits = 0;
    if (a.frameMode) {
        const KeyLayout lay = keyLayout(ctl, a.tileCount, a.count);
        lowBits = lay.lowBits;
        packed = lay.packed;
        indexBits = lay.indexBits;
        keyBits = bitWidth(ctl->c.tile_max) + lowBits;
    } else {
        lowBits = a.fixedLowBits;
        keyBits = a.fixedKeyBits;
    }
    uint32_t passes = entries ? (keyBits + 7) / 8 : 0;
    if (passes > a.passesLaunched) {  // planned for fewer bits than the keys carry: report
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_KEY_RANGE));
        passes = a.passesLaunched;
    }
    const uint64_t keyMask = maskOf(keyBits);
    for (uint32_t j = threadIdx.x; j < kMaxSortPasses * 256; j += 256) (&sHist[0][0])[j] = 0;
    __syncthreads();
    const uint64_t* keys = a.keys[0];
    for (uint32_t k = blockIdx.x * 256 + threadIdx.x; k < entries; k += gridDim.x * 256) {
        const uint64_t key = __ldg(&keys[k]);
        const uint64_t v = packed ? (key >> indexBits) : virtualKey(key, lowBits, keyMask);
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sHist[p][uint32_t(v >> (8 * p)) & 0xFFu], 1u);
    }
    __syncthreads();
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t c = sHist[p][threadIdx.x];
        if (c) atomicAdd(&a.plan->hist[p][threadIdx.x], c);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sLast = atomicAdd(&ctl->histDone, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!sLast) return;
    __threadfence();
    // the last block: per-pass activity, digit bases, buffer parity
    SortPlan* plan = a.plan;
    uint32_t activeCount = 0;
    for (uint32_t p = 0; p < kMaxSortPasses; ++p) {
        const uint32_t c = p < passes ? ldAcquire32(&plan->hist[p][threadIdx.x]) : 0;
        if (threadIdx.x == 0) sAny = 0;
        __syncthreads();
        if (p < passes && c == entries) sAny = 1;  // one digit holds every key: constant
        __syncthreads();
        const bool active = p < passes && !sAny;
        uint32_t total;
        const uint32_t excl = blockExclusiveScan256(c, sWarp, &total);
        plan->digitBase[p][threadIdx.x] = excl;
        if (threadIdx.x == 0) {
            plan->active[p] = active ? 1u : 0u;
            plan->inBuffer[p] = activeCount & 1u;
        }
        activeCount += active ? 1u : 0u;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        plan->passes = passes;
        plan->lowBits = lowBits;
        plan->keyBits = keyBits;
        plan->packed = packed;
        plan->indexBits = indexBits;
        ctl->c.packed_entries = packed;
        ctl->c.index_bits = indexBits;
        ctl->c.sort_passes = activeCount;
        ctl->c.sorted_buffer = activeCount & 1u;
        ctl->c.key_bits = keyBits;
        ctl->c.depth_low_bits = lowBits;
        ctl->c.visible = ctl->c.cull_counts[0];
    }
}

// ---- one onesweep pass ------------------------------------------------------------------------
constexpr int kSortSmemBytes = kSortTile * 12 + 8 * 256 * 4;

// Three blocks per SM (<= 85 registers): the digits are recomputed from the keys instead of
// being kept, and the warp ranks (< 512) are packed two per register. PACKED: the entries are
// single words (vkey << indexBits | index) and no value array moves; the frame launches both
// instantiations and the one that does not match the plan's layout returns at once.
template <bool PACKED>
__global__ void __launch_bounds__(kSortThreads, PACKED ? 4 : 3) sortPassKernel(const __grid_constant__ SortArgs a,
                                                                                uint32_t p) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sKeys = reinterpret_cast<uint64_t*>(smem);
    uint32_t* sWarpHist = reinterpret_cast<uint32_t*>(smem + kSortTile * 8);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(smem + kSortTile * 8 + 8 * 256 * 4);
    __shared__ uint32_t sDigitStart[256], sGlobalBase[256], sWarp[8], sTile;
    const SortPlan* plan = a.plan;
    if (!plan->active[p] || (plan->packed != 0) != PACKED) return;
    DeviceControl* ctl = a.ctl;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t entries = ctl->c.entries;
    if (tid == 0) sTile = atomicAdd(&ctl->tickets[1 + p], 1u);
#pragma unroll
    for (int j = 0; j < 8; ++j) sWarpHist[j * 256 + tid] = 0;
    __syncthreads();
    const uint32_t t = sTile;
    const uint32_t tileBase = t * kSortTile;
    if (tileBase >= entries || t >= a.maxTiles) return;
    const uint32_t in = plan->inBuffer[p];
    const uint64_t* keysIn = a.keys[in];
    const uint32_t* valsIn = a.values[in];
    uint64_t* keysOut = a.keys[in ^ 1u];
    uint32_t* valsOut = a.values[in ^ 1u];
    const uint32_t lowBits = plan->lowBits;
    const uint64_t keyMask = maskOf(plan->keyBits);
    const uint32_t shift = 8 * p + (PACKED ? plan->indexBits : 0u);

    const uint32_t itemBase = tileBase + warp * (32 * kSortItems) + lane;
    // digit of a key; past the end: 0x100, ranked nowhere
    auto digit = [&](uint64_t k) -> uint32_t {
        return PACKED ? uint32_t(k >> shift) & 0xFFu : uint32_t(virtualKey(k, lowBits, keyMask) >> shift) & 0xFFu;
    };
    auto digitOf = [&](uint64_t k, uint32_t idx) -> uint32_t { return idx < entries ? digit(k) : 0x100u; };
    uint64_t key[kSortItems];
    uint32_t val[PACKED ? 1 : kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t idx = itemBase + j * 32;
        key[j] = idx < entries ? keysIn[idx] : 0ull;
        if (!PACKED) val[PACKED ? 0 : j] = idx < entries ? valsIn[idx] : 0u;
    }
    // warp-level multisplit: rank of each item among the warp's earlier items of its digit
    uint32_t* wh = sWarpHist + warp * 256;
    const uint32_t ltMask = laneMaskLt();
    uint32_t rank[kSortItems / 2];  // two 16-bit ranks per word
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t d = digitOf(key[j], itemBase + j * 32);
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t below = peers & ltMask;
        const uint32_t pre = d < 256 ? wh[d] : 0u;
        __syncwarp();
        if (d < 256 && below == 0) wh[d] = pre + __popc(peers);
        __syncwarp();
        const uint32_t r = pre + __popc(below);
        if (j & 1) rank[j >> 1] |= r << 16;
        else rank[j >> 1] = r;
    }
    __syncthreads();
    // digit tid: warp offsets (exclusive over warps) and the block's count
    const uint32_t d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const uint32_t c = sWarpHist[w * 256 + d];
        sWarpHist[w * 256 + d] = run;
        run += c;
    }
    const uint32_t blockCount = run;
    const uint32_t epoch = ctl->c.epoch;
    uint64_t* status = a.status + (size_t(p) * a.maxTiles) * 256;
    stRelease(&status[size_t(t) * 256 + d], packStatus(epoch, t == 0 ? kFlagInclusive : kFlagAggregate, blockCount));
    uint32_t total;
    sDigitStart[d] = blockExclusiveScan256(blockCount, sWarp, &total);
    // decoupled look-back for digit d over the earlier tiles of this pass
    uint32_t exclusive = 0;
    if (t > 0) {
        const uint32_t forced = ctl->forceTimeout;
        uint32_t spins = 0;
        int q = int(t) - 1;
        while (q >= 0) {
            const uint64_t s = ldAcquire(&status[size_t(q) * 256 + d]);
            bool ready = statusReady(s, epoch);
            if (forced && spins < forced) ready = false;
            if (!ready) {
                if (++spins >= kSpinLimit || (forced && spins >= forced)) {
                    reportTimeout(ctl, kWaitSort);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            exclusive += uint32_t(s);
            if (statusFlag(s) == kFlagInclusive) break;
            --q;
        }
        stRelease(&status[size_t(t) * 256 + d], packStatus(epoch, kFlagInclusive, exclusive + blockCount));
    }
    sGlobalBase[d] = plan->digitBase[p][d] + exclusive;
    __syncthreads();
    // local stable order in shared memory
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t dj = digitOf(key[j], itemBase + j * 32);
        if (dj < 256) {
            const uint32_t r = (j & 1) ? (rank[j >> 1] >> 16) : (rank[j >> 1] & 0xFFFFu);
            const uint32_t pos = sDigitStart[dj] + sWarpHist[warp * 256 + dj] + r;
            sKeys[pos] = key[j];
            if (!PACKED) sVals[pos] = val[PACKED ? 0 : j];
        }
    }
    __syncthreads();
    const uint32_t n = entries - tileBase < uint32_t(kSortTile) ? entries - tileBase : uint32_t(kSortTile);
    for (uint32_t k = tid; k < n; k += kSortThreads) {
        const uint64_t kk = sKeys[k];
        const uint32_t dk = digit(kk);
        const uint32_t g = sGlobalBase[dk] + (k - sDigitStart[dk]);
        if (g < entries) {
            keysOut[g] = kk;
            if (!PACKED) valsOut[g] = sVals[k];
        } else {
            atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
        }
    }
}

// ---- one onesweep pass over packed entries: 12288-key tiles, 768 threads ----------------------
// The frame's usual layout. One block per SM: the first wave of a pass is ~148 tiles deep
// instead of ~600, so the decoupled look-back chains stay short. Each tile publishes its
// per-digit counts as soon as its keys are loaded (a shared-memory histogram), ranks them with
// warp-level multisplit meanwhile, then looks back 8 predecessors per round trip.
constexpr int kBigThreads = 768;
constexpr int kBigTile = kBigThreads * kSortItems;  // 12288 keys
constexpr int kBigWarps = kBigThreads / 32;
constexpr int kBigSmemBytes = kBigTile * 8 + kBigWarps * 256 * 4;
static_assert(kBigWarps * 256 == 8 * kBigThreads, "the warp histograms are zeroed 8 words per thread");

__global__ void __launch_bounds__(kBigThreads, 1) sortPassPackedKernel(const __grid_constant__ SortArgs a, uint32_t p) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sKeys = reinterpret_cast<uint64_t*>(smem);
    uint32_t* sWarpHist = reinterpret_cast<uint32_t*>(smem + kBigTile * 8);  // [kBigWarps][256]
    __shared__ uint32_t sBlockHist[256], sDigitStart[256], sGlobalBase[256], sWarp[8], sTile;
    const SortPlan* plan = a.plan;
    if (!plan->active[p] || !plan->packed) return;
    DeviceControl* ctl = a.ctl;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t entries = ctl->c.entries;
    if (tid == 0) sTile = atomicAdd(&ctl->tickets[1 + p], 1u);
#pragma unroll
    for (int j = 0; j < 8; ++j) sWarpHist[j * kBigThreads + tid] = 0;
    if (tid < 256) sBlockHist[tid] = 0;
    __syncthreads();
    const uint32_t t = sTile;
    const uint32_t tileBase = t * kBigTile;
    if (tileBase >= entries) return;
    const uint32_t in = plan->inBuffer[p];
    const uint64_t* keysIn = a.keys[in];
    uint64_t* keysOut = a.keys[in ^ 1u];
    const uint32_t shift = 8 * p + plan->indexBits;
    const uint32_t itemBase = tileBase + warp * (32 * kSortItems) + lane;
    auto digitOf = [&](uint64_t k, uint32_t idx) -> uint32_t {
        return idx < entries ? uint32_t(k >> shift) & 0xFFu : 0x100u;
    };
    uint64_t key[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t idx = itemBase + j * 32;
        key[j] = idx < entries ? keysIn[idx] : 0ull;
    }
    // 1) the tile's digit counts, published at once (aggregate; inclusive for the first tile)
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t d = digitOf(key[j], itemBase + j * 32);
        if (d < 256) atomicAdd(&sBlockHist[d], 1u);
    }
    __syncthreads();
    const uint32_t epoch = ctl->c.epoch;
    uint64_t* status = a.status + (size_t(p) * a.maxTiles) * 256;
    uint32_t blockCount = 0;
    if (tid < 256) {
        blockCount = sBlockHist[tid];
        stRelease(&status[size_t(t) * 256 + tid], packStatus(epoch, t == 0 ? kFlagInclusive : kFlagAggregate, blockCount));
    }
    // 2) warp-level multisplit ranks
    uint32_t* wh = sWarpHist + warp * 256;
    const uint32_t ltMask = laneMaskLt();
    uint32_t rank[kSortItems / 2];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t d = digitOf(key[j], itemBase + j * 32);
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t below = peers & ltMask;
        const uint32_t pre = d < 256 ? wh[d] : 0u;
        __syncwarp();
        if (d < 256 && below == 0) wh[d] = pre + __popc(peers);
        __syncwarp();
        const uint32_t r = pre + __popc(below);
        if (j & 1) rank[j >> 1] |= r << 16;
        else rank[j >> 1] = r;
    }
    __syncthreads();
    // 3) digit d = tid < 256: warp offsets, the tile's digit starts, and the look-back
    if (tid < 256) {
        const uint32_t d = tid;
        uint32_t run = 0;
        for (int w = 0; w < kBigThreads / 32; ++w) {
            const uint32_t c = sWarpHist[w * 256 + d];
            sWarpHist[w * 256 + d] = run;
            run += c;
        }
        // block-wide exclusive scan of the 256 counts (warps 0-7)
        uint32_t incl = blockCount;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= uint32_t(o)) incl += v;
        }
        if (lane == 31) sWarp[warp] = incl;
    }
    __syncthreads();
    if (tid < 256) {
        const uint32_t d = tid;
        uint32_t base = 0;
        for (uint32_t w = 0; w < warp; ++w) base += sWarp[w];
        uint32_t incl = blockCount;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= uint32_t(o)) incl += v;
        }
        sDigitStart[d] = base + incl - blockCount;
    }
    __syncthreads();
    // 4) local order in shared memory (before the look-back: the keys leave the registers)
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint32_t dj = digitOf(key[j], itemBase + j * 32);
        if (dj < 256) {
            const uint32_t r = (j & 1) ? (rank[j >> 1] >> 16) : (rank[j >> 1] & 0xFFFFu);
            sKeys[sDigitStart[dj] + sWarpHist[warp * 256 + dj] + r] = key[j];
        }
    }
    if (tid < 256) {
        const uint32_t d = tid;
        // 5) windowed look-back: 8 predecessors per round trip
        uint32_t exclusive = 0;
        if (t > 0) {
            const uint32_t forced = ctl->forceTimeout;
            uint32_t spins = 0;
            int q = int(t) - 1;
            bool found = false;
            while (!found && q >= 0) {
                uint64_t w[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    w[j] = q - j >= 0 ? ldAcquire(&status[size_t(q - j) * 256 + d]) : packStatus(epoch, kFlagInclusive, 0);
                int used = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (found || used != j) continue;
                    bool ready = statusReady(w[j], epoch);
                    if (forced && spins < forced) ready = false;
                    if (!ready) continue;
                    exclusive += uint32_t(w[j]);
                    ++used;
                    if (statusFlag(w[j]) == kFlagInclusive) found = true;
                }
                if (found) break;
                q -= used;
                if (used < 8) {
                    if (++spins >= kSpinLimit || (forced && spins >= forced)) {
                        reportTimeout(ctl, kWaitSort);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            stRelease(&status[size_t(t) * 256 + d], packStatus(epoch, kFlagInclusive, exclusive + blockCount));
        }
        sGlobalBase[d] = plan->digitBase[p][d] + exclusive;
    }
    __syncthreads();
    // 6) coalesced runs to the global positions
    const uint32_t n = entries - tileBase < uint32_t(kBigTile) ? entries - tileBase : uint32_t(kBigTile);
    for (uint32_t k = tid; k < n; k += kBigThreads) {
        const uint64_t kk = sKeys[k];
        const uint32_t dk = uint32_t(kk >> shift) & 0xFFu;
        const uint32_t g = sGlobalBase[dk] + (k - sDigitStart[dk]);
        if (g < entries) keysOut[g] = kk;
        else atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
    }
}

// The gaussian index and the tile of sorted entry k in either layout.
__device__ __forceinline__ uint32_t entryTile(const uint64_t* keys, uint32_t k, const SortPlan* plan) {
    const uint64_t key = keys[k];
    return plan->packed ? uint32_t(key >> (plan->indexBits + plan->lowBits)) : uint32_t(key >> 32);
}

// ---- tile ranges (tile_ranges.comp:22-44) -----------------------------------------------------
__global__ void rangesKernel(const __grid_constant__ RenderArgs a) {
    const DeviceControl* ctl = a.ctl;
    const uint32_t n = ctl->c.entries;
    const uint64_t* keys = a.keys[ctl->c.sorted_buffer & 1u];
    const uint32_t tileCount = a.tilesX * a.tilesY;
    uint2* ranges = reinterpret_cast<uint2*>(a.ranges);
    const SortPlan* plan = a.plan;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t tile = entryTile(keys, k, plan);
        if (tile >= tileCount) {
            // the sentinel tile (sorted last) closes the last real tile's range
            if (k > 0) {
                const uint32_t prev = entryTile(keys, k - 1, plan);
                if (prev < tileCount) ranges[prev].y = k;
            }
            continue;
        }
        if (k == 0) {
            ranges[tile].x = 0;
        } else {
            const uint32_t prev = entryTile(keys, k - 1, plan);
            if (prev != tile) {
                if (prev < tileCount) ranges[prev].y = k;
                ranges[tile].x = k;
            }
        }
        if (k == n - 1) ranges[tile].y = n;
    }
}

// ---- standalone exclusive scan (GpuScan plain / kNonZero / kGather) ---------------------------
constexpr int kScanItems = 8;
__global__ void __launch_bounds__(256) scanKernel(const uint32_t* __restrict__ in, const uint32_t* __restrict__ index,
                                                  uint32_t* __restrict__ out, uint32_t* total, uint32_t count,
                                                  uint32_t mode, uint64_t* status, DeviceControl* ctl,
                                                  uint32_t setupCapacity, uint32_t waitSite) {
    __shared__ uint32_t sBlock, sWarp[8], sExclusive;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sBlock = atomicAdd(&ctl->tickets[12], 1u);
    __syncthreads();
    const uint32_t block = sBlock;
    const uint32_t base = block * 256 * kScanItems + tid * kScanItems;
    uint32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint32_t idx = base + j;
        uint32_t x = 0;
        if (idx < count) {
            if (mode == GSR_SCAN_GATHER) x = in[index[idx]];
            else x = in[idx];
            if (mode == GSR_SCAN_NONZERO) x = x != 0;
        }
        v[j] = x;
        sum += x;
    }
    uint32_t blockTotal;
    const uint32_t threadExcl = blockExclusiveScan256(sum, sWarp, &blockTotal);
    const uint32_t epoch = ctl->c.epoch;
    if (warp == 0) {
        if (lane == 0)
            stRelease(&status[block], packStatus(epoch, block == 0 ? kFlagInclusive : kFlagAggregate, blockTotal));
        uint32_t exclusive = 0;
        if (block > 0) exclusive = warpLookback(status, int(block), epoch, ctl, waitSite);
        if (lane == 0) {
            if (block > 0) stRelease(&status[block], packStatus(epoch, kFlagInclusive, exclusive + blockTotal));
            sExclusive = exclusive;
        }
    }
    __syncthreads();
    uint32_t run = sExclusive + threadExcl;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint32_t idx = base + j;
        if (idx < count) out[idx] = run;
        run += v[j];
    }
    if (block == gridDim.x - 1 && tid == 255) {
        if (total) *total = run;
        if (setupCapacity) {  // the frame's list: entries = min(M, capacity) (tile_setup.comp:16-24)
            const uint32_t entries = run < setupCapacity ? run : setupCapacity;
            ctl->c.entries = entries;
            ctl->c.overflow = run - entries;
            ctl->c.ranges_groups[0] = (entries + 255u) / 256u;
            ctl->c.ranges_groups[1] = 1;
            ctl->c.ranges_groups[2] = 1;
        }
    }
}

__global__ void pack64Kernel(const uint32_t* lo, const uint32_t* hi, uint64_t* out, uint32_t n) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = (hi ? (uint64_t(hi[k]) << 32) : 0ull) | lo[k];
}
__global__ void unpack64Kernel(const uint64_t* in, uint32_t* lo, uint32_t* hi, uint32_t n) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint64_t v = in[k];
        lo[k] = uint32_t(v);
        if (hi) hi[k] = uint32_t(v >> 32);
    }
}
__global__ void setEntriesKernel(DeviceControl* ctl, uint32_t count) {
    ctl->c.entries = count;
    ctl->c.duplicates = count;
}

uint32_t gridFor(uint32_t n, uint32_t perBlock, uint32_t cap) {
    uint32_t b = (n + perBlock - 1) / perBlock;
    return b < 1 ? 1 : (b > cap ? cap : b);
}

}  // namespace

cudaError_t launchSort(const SortArgs& a, uint32_t histBlocks, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(sortPassKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kSortSmemBytes);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(sortPassPackedKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kBigSmemBytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    sortHistKernel<<<histBlocks < 1 ? 1 : histBlocks, 256, 0, s>>>(a);
    const uint32_t grid = a.maxTiles < 1 ? 1 : a.maxTiles;
    const uint32_t bigGrid = (grid + (kBigTile / kSortTile) - 1) / (kBigTile / kSortTile);
    for (uint32_t p = 0; p < a.passesLaunched; ++p) {
        // the entry layout is decided on the device: both run, the other one returns at once
        if (a.frameMode) sortPassPackedKernel<<<bigGrid, kBigThreads, kBigSmemBytes, s>>>(a, p);
        sortPassKernel<false><<<grid, kSortThreads, kSortSmemBytes, s>>>(a, p);
    }
    return cudaGetLastError();
}

cudaError_t launchRanges(const RenderArgs& a, uint32_t capacity, cudaStream_t s) {
    rangesKernel<<<gridFor(capacity, 256, 148 * 16), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchScan(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
                       uint32_t mode, uint64_t* status, DeviceControl* ctl, cudaStream_t s, uint32_t setupCapacity,
                       uint32_t waitSite) {
    const uint32_t blocks = (count + 256 * kScanItems - 1) / (256 * kScanItems);
    if (blocks == 0) {
        if (total) return cudaMemsetAsync(total, 0, 4, s);
        return cudaSuccess;
    }
    scanKernel<<<blocks, 256, 0, s>>>(in, index, out, total, count, mode, status, ctl, setupCapacity, waitSite);
    return cudaGetLastError();
}

cudaError_t launchPack64(const uint32_t* lo, const uint32_t* hi, uint64_t* out, uint32_t n, cudaStream_t s) {
    if (!n) return cudaSuccess;
    pack64Kernel<<<gridFor(n, 256, 148 * 16), 256, 0, s>>>(lo, hi, out, n);
    return cudaGetLastError();
}
cudaError_t launchUnpack64(const uint64_t* in, uint32_t* lo, uint32_t* hi, uint32_t n, cudaStream_t s) {
    if (!n) return cudaSuccess;
    unpack64Kernel<<<gridFor(n, 256, 148 * 16), 256, 0, s>>>(in, lo, hi, n);
    return cudaGetLastError();
}
cudaError_t launchSetEntries(DeviceControl* ctl, uint32_t count, cudaStream_t s) {
    setEntriesKernel<<<1, 1, 0, s>>>(ctl, count);
    return cudaGetLastError();
}

}  // namespace gsr
