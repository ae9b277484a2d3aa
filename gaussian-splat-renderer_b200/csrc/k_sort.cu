// Sorting the (tile | depth) list, the tile ranges, and the standalone prefix-sum primitive.
//
// The sort is a stable LSD radix sort over 8-bit digits in the onesweep form (Adinets and
// Merrill, 2022): one histogram kernel computes the digit counts of every pass in a single
// read of the keys, then each pass is ONE kernel whose blocks (ordered by a ticket) count the
// digits of their tile and publish the counts at once, rank the tile locally with a warp-level
// multisplit, get their global digit offsets by a decoupled look-back over the earlier tiles,
// and scatter through shared memory. Ties keep their input order (warp order, then item and
// lane order).
//
// The multisplit finds the lanes of a warp that hold the same digit through per-warp lane
// masks in shared memory (each lane ORs its bit into mask[digit], then reads the word back).
// On sm_100a that costs about 40 cycles per warp-step against ~95 for eight vote.ballot rounds
// and ~235 for match.any.sync over random 8-bit digits (measured on B200 with a synthetic
// throughput loop).
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

// The depth sort's key of a depth word: its depth bits (above the record index) minus the
// frame's smallest visible depth bits, in depthBits = bit_width(max - min) bits. Positive floats
// order like their bits, so the offsets of the visible records order like their depths, and no
// digit pass is spent on the bits every real depth shares. (Offsets span fewer bits than the
// bits where min and max differ: 24 against 25 for depths in [6, 22], one pass less at 8-bit
// digits.) A record without tiles (all-ones depth bits) gets some key in the range: it emits no
// entry, so where it sorts changes no offset and no list. The view is not part of the key: each
// view's run of records is sorted on its own (SortArgs::segments).
__device__ __forceinline__ uint32_t depthVirtualKey(uint64_t word, uint32_t indexBits, uint32_t depthBits,
                                                    uint32_t depthMin) {
    return (uint32_t(word >> indexBits) - depthMin) & uint32_t(maskOf(depthBits));
}

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

// Digits of BITS bits (7, 8 or 9): kBins digit values; in the per-digit phases thread tid owns
// digits tid * kPerThread .. tid * kPerThread + kPerThread - 1 (those below kBins).
template <int BITS>
struct Digits {
    static constexpr int kBins = 1 << BITS;
    static constexpr int kPerThread = kBins > 256 ? kBins / 256 : 1;
    static constexpr uint32_t kMask = uint32_t(kBins - 1);
    static_assert(kBins <= kMaxSortBins, "the plan's digit arrays");
    __device__ static uint32_t of(uint32_t q) { return threadIdx.x * kPerThread + q; }
};

// Exclusive scan over the kBins digits in digit order, v and excl in each thread's own digits.
template <int BITS>
__device__ __forceinline__ void blockScanDigits(const uint32_t (&v)[Digits<BITS>::kPerThread],
                                                uint32_t (&excl)[Digits<BITS>::kPerThread], uint32_t* sWarp) {
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < Digits<BITS>::kPerThread; ++q) {
        excl[q] = sum;
        sum += v[q];
    }
    uint32_t total;
    const uint32_t base = blockExclusiveScan256(sum, sWarp, &total);
#pragma unroll
    for (int q = 0; q < Digits<BITS>::kPerThread; ++q) excl[q] += base;
}

// ---- histogram of every pass's digit + the plan ---------------------------------------------
constexpr int kHistItems = 16;
template <int BITS>
__global__ void __launch_bounds__(256) sortHistKernel(const __grid_constant__ SortArgs a) {
    using D = Digits<BITS>;
    __shared__ uint32_t sHist[kMaxSortPasses][D::kBins];
    __shared__ uint32_t sWarp[8];
    __shared__ uint32_t sLast;
    __shared__ uint32_t sAny;
    DeviceControl* ctl = a.ctl;
    const uint32_t entries = a.frameMode == 2 ? a.count : ctl->c.entries;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t lowBits, keyBits, packed = 0, indexBits = 0, depthBits = 0, depthMin = 0;
    if (a.frameMode == 1) {
        const KeyLayout lay = keyLayout(ctl, a.tileCount, a.count, a.binning != 0);
        lowBits = lay.lowBits;
        packed = lay.packed;
        indexBits = lay.indexBits;
        keyBits = bitWidth(ctl->c.tile_max) + lowBits;
    } else if (a.frameMode == 2) {  // binning mode's depth keys: the depth offsets, each view's run apart
        const uint32_t dmin = ctl->c.depth_min_bits, dmax = ctl->c.depth_max_bits;
        lowBits = 0;
        packed = 1;
        indexBits = a.indexBits;
        depthMin = dmin > dmax ? 0u : dmin;
        depthBits = dmin > dmax ? 0u : bitWidth(dmax - dmin);
        keyBits = depthBits;
    } else {
        lowBits = a.fixedLowBits;
        keyBits = a.fixedKeyBits;
    }
    uint32_t passes = entries ? (keyBits + BITS - 1) / BITS : 0;
    if (passes > a.passesLaunched) {  // planned for fewer bits than the keys carry: report
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_KEY_RANGE));
        passes = a.passesLaunched;
    }
    const uint64_t keyMask = maskOf(keyBits);
    for (uint32_t j = threadIdx.x; j < kMaxSortPasses * D::kBins; j += 256) (&sHist[0][0])[j] = 0;
    __syncthreads();
    const uint64_t* keys = a.keys[0];
    // kHistItems independent loads per thread in flight before the counting
    constexpr uint32_t kChunk = 256 * kHistItems;
    static_assert(kChunk == kDepthSortTile, "a depth histogram chunk is one depth sort tile");
    if (a.frameMode == 2) {
        // the depth words, one view's run at a time: a block takes a contiguous share of the runs'
        // tiles (none straddles two runs) and adds its counts to the run's histogram whenever the
        // run changes, and at the end
        const uint32_t tilesPerRun = (a.segLength + kChunk - 1) / kChunk;
        const uint32_t chunks = tilesPerRun * a.segments;
        const uint32_t per = (chunks + gridDim.x - 1) / gridDim.x;
        const uint32_t c0 = blockIdx.x * per, c1 = c0 + per < chunks ? c0 + per : chunks;
        auto flushRun = [&](uint32_t run) {
            for (uint32_t p = 0; p < passes; ++p)
                for (uint32_t d = threadIdx.x; d < uint32_t(D::kBins); d += 256) {
                    const uint32_t c = sHist[p][d];
                    if (c) {
                        atomicAdd(&a.segHist[(size_t(run) * a.passesLaunched + p) * D::kBins + d], c);
                        sHist[p][d] = 0;
                    }
                }
        };
        uint32_t run = c0 < c1 ? c0 / tilesPerRun : 0u;
        for (uint32_t c = c0; c < c1; ++c) {
            const uint32_t v = c / tilesPerRun;  // the same in every thread
            if (v != run) {
                __syncthreads();
                flushRun(run);
                __syncthreads();
                run = v;
            }
            const uint32_t runEnd = (v + 1) * a.segLength;
            const uint32_t base = v * a.segLength + (c - v * tilesPerRun) * kChunk;
            uint64_t k[kHistItems];
#pragma unroll
            for (int j = 0; j < kHistItems; ++j) {
                const uint32_t idx = base + j * 256 + threadIdx.x;
                k[j] = idx < runEnd ? __ldg(&keys[idx]) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < kHistItems; ++j) {
                if (base + j * 256 + threadIdx.x < runEnd) {
                    const uint32_t v2 = depthVirtualKey(k[j], indexBits, depthBits, depthMin);
                    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sHist[p][(v2 >> (BITS * p)) & D::kMask], 1u);
                }
            }
        }
        __syncthreads();
        if (c0 < c1) flushRun(run);
    } else {
        for (uint32_t base = blockIdx.x * kChunk; base < entries; base += gridDim.x * kChunk) {
            uint64_t k[kHistItems];
#pragma unroll
            for (int j = 0; j < kHistItems; ++j) {
                const uint32_t idx = base + j * 256 + threadIdx.x;
                k[j] = idx < entries ? __ldg(&keys[idx]) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < kHistItems; ++j) {
                if (base + j * 256 + threadIdx.x < entries) {
                    const uint64_t v = packed ? (k[j] >> indexBits) : virtualKey(k[j], lowBits, keyMask);
                    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sHist[p][uint32_t(v >> (BITS * p)) & D::kMask], 1u);
                }
            }
        }
        __syncthreads();
        for (uint32_t p = 0; p < passes; ++p)
            for (uint32_t d = threadIdx.x; d < uint32_t(D::kBins); d += 256) {
                const uint32_t c = sHist[p][d];
                if (c) atomicAdd(&a.plan->hist[p][d], c);
            }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sLast = atomicAdd(&ctl->histDone[a.frameMode == 2 ? 1 : 0], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!sLast) return;
    __threadfence();
    // the last block: per-pass activity, digit bases, buffer parity
    SortPlan* plan = a.plan;
    uint32_t activeCount = 0;
    for (uint32_t p = 0; p < kMaxSortPasses; ++p) {
        bool active;
        if (a.frameMode == 2) {
            // each warp scans the runs warp, warp + 8, ...: the run's digit bases start at its first
            // record; the pass is needed unless, in every run, one digit holds all of its keys
            constexpr int kPerLane = D::kBins / 32;
            if (threadIdx.x == 0) sAny = 0;
            __syncthreads();
            for (uint32_t v = warp; p < passes && v < a.segments; v += 8) {
                const size_t at = (size_t(v) * a.passesLaunched + p) * D::kBins + lane * kPerLane;
                uint32_t c[kPerLane], sum = 0;
                bool whole = false;
#pragma unroll
                for (int q = 0; q < kPerLane; ++q) {
                    c[q] = ldAcquire32(&a.segHist[at + q]);
                    whole |= c[q] == a.segLength;
                    sum += c[q];
                }
                uint32_t incl = sum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= uint32_t(o)) incl += t;
                }
                uint32_t base = v * a.segLength + incl - sum;
#pragma unroll
                for (int q = 0; q < kPerLane; ++q) {
                    a.segBase[at + q] = base;
                    base += c[q];
                }
                if (!__any_sync(0xFFFFFFFFu, whole) && lane == 0) sAny = 1;
            }
            __syncthreads();
            active = p < passes && sAny;
        } else {
            uint32_t c[D::kPerThread];
#pragma unroll
            for (int q = 0; q < D::kPerThread; ++q) {
                const uint32_t d = D::of(q);
                c[q] = p < passes && d < uint32_t(D::kBins) ? ldAcquire32(&plan->hist[p][d]) : 0u;
            }
            if (threadIdx.x == 0) sAny = 0;
            __syncthreads();
#pragma unroll
            for (int q = 0; q < D::kPerThread; ++q)
                if (p < passes && D::of(q) < uint32_t(D::kBins) && c[q] == entries) sAny = 1;  // one digit holds every key
            __syncthreads();
            active = p < passes && !sAny;
            uint32_t excl[D::kPerThread];
            blockScanDigits<BITS>(c, excl, sWarp);
#pragma unroll
            for (int q = 0; q < D::kPerThread; ++q)
                if (D::of(q) < uint32_t(D::kBins)) plan->digitBase[p][D::of(q)] = excl[q];
        }
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
        plan->digitBits = BITS;
        plan->depthBits = depthBits;
        plan->depthMin = depthMin;
        plan->sortedBuffer = activeCount & 1u;
        if (a.frameMode == 2) return;  // the list's own plan fills the control block
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
// Decoupled look-back of digit d for tile t: the sum of the digit's counts over tiles 0..t-1
// (status words [tile][BINS]). Eight predecessors are read per round trip; a word that is not
// yet published (or carries an older frame's epoch) stops the window and is re-read after a
// short sleep. Waits are bounded by kSpinLimit (then the timeout is reported and the partial
// sum returned).
template <int BINS>
__device__ __forceinline__ uint32_t digitLookback(const uint64_t* status, uint32_t t, uint32_t d, uint32_t epoch,
                                                  DeviceControl* ctl) {
    constexpr int kWindow = 8;
    const uint32_t forced = ctl->forceTimeout;
    uint32_t exclusive = 0, spins = 0;
    int q = int(t) - 1;
    while (q >= 0) {
        uint64_t w[kWindow];
#pragma unroll
        for (int j = 0; j < kWindow; ++j)
            w[j] = q - j >= 0 ? ldRelaxed(&status[size_t(q - j) * BINS + d]) : packStatus(epoch, kFlagInclusive, 0);
        int used = 0;
        bool found = false;
#pragma unroll
        for (int j = 0; j < kWindow; ++j) {
            if (found || used != j) continue;
            bool ready = statusReady(w[j], epoch);
            if (forced && spins < forced) ready = false;  // test hook: behave as if nobody published
            if (!ready) continue;
            exclusive += uint32_t(w[j]);
            ++used;
            if (statusFlag(w[j]) == kFlagInclusive) found = true;
        }
        if (found) break;
        q -= used;
        if (used < kWindow) {
            if (++spins >= kSpinLimit || (forced && spins >= forced)) {
                reportTimeout(ctl, kWaitSort);
                break;
            }
            __nanosleep(32);
        }
    }
    return exclusive;
}

// One pass over 256-thread tiles of kItems keys per thread. PAIRS = false: the entries are
// single words (vkey << indexBits | index), 24 per thread; PAIRS = true: (tile << 32 | depth)
// keys with a 32-bit value array, 16 per thread. The frame launches both and the one that does
// not match the plan's layout returns at once. BITS: the digit width.
//   1) load; per-warp digit counts -> the tile's counts, published at once (aggregate, or
//      inclusive for tile 0), and the tile's digit starts;
//   2) ranks: peer masks of each warp step, a warp-private running count per digit; every key
//      goes straight to its place in the tile's stable order in shared memory;
//   3) the look-back of each digit a thread owns gives the global offset of the tile's run of
//      that digit;
//   4) the runs are written out, coalesced.
// Items past the end of the list are loaded as all-ones keys: their digit is the largest one
// the key width allows, they rank after every real key of the tile and are never stored.
template <bool PAIRS, int ITEMS, int BITS>
struct PassShape {
    static constexpr int kItems = ITEMS;
    static constexpr int kTile = kSortThreads * kItems;
    static constexpr int kBins = 1 << BITS;
    // keys, values, per-warp running counts [8][kBins], per-warp peer masks [8][2][kBins]
    static constexpr int kSmemBytes = kTile * 8 + (PAIRS ? kTile * 4 : 0) + 8 * kBins * 4 * 3;
};
static_assert(kSortThreads == 256, "256 threads own the digits");
static_assert(PassShape<true, 16, 8>::kTile == kSortTile, "the status array is sized by the smaller tile");
static_assert(PassShape<true, 16, 9>::kSmemBytes == PassShape<false, 24, 9>::kSmemBytes, "one launch serves both layouts");
static_assert(PassShape<false, kDepthSortItems, 8>::kTile == kDepthSortTile, "the depth status array is sized by this tile");

// The blocks of a pass are persistent: each takes tiles by ticket (the tile order of the
// look-back) until the list is done, so a pass launches a fixed grid of blocks that all stay
// resident (blocks only ever wait on tiles already taken by running blocks).
template <bool PAIRS, int ITEMS, int BITS, bool DEPTH = false>
__device__ __forceinline__ void sortPassTiles(const SortArgs& a, uint32_t p, unsigned char* smem, uint32_t* sOff,
                                              uint32_t* sScan, uint32_t& sTile) {
    using S = PassShape<PAIRS, ITEMS, BITS>;
    using D = Digits<BITS>;
    constexpr int kItems = S::kItems, kTile = S::kTile, kBins = D::kBins, P = D::kPerThread;
    uint64_t* sKeys = reinterpret_cast<uint64_t*>(smem);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(smem + kTile * 8);
    uint32_t* sWarpCnt = reinterpret_cast<uint32_t*>(smem + kTile * (PAIRS ? 12 : 8));  // [8][kBins]
    uint32_t* sMask = sWarpCnt + 8 * kBins;                                             // [8][2][kBins]
    const SortPlan* plan = a.plan;
    DeviceControl* ctl = a.ctl;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t entries = a.frameMode == 2 ? a.count : ctl->c.entries;
    const uint32_t ticket = (a.frameMode == 2 ? kDepthSortTickets : kListSortTickets) + p;
    for (;;) {
    if (tid == 0) sTile = atomicAdd(&ctl->tickets[ticket], 1u);
#pragma unroll
    for (int j = 0; j < 24 * kBins / 256; ++j) sWarpCnt[j * 256 + tid] = 0;
    __syncthreads();
    const uint32_t t = sTile;
    // the tile's keys [tileBase, tileEnd), and whether it starts its look-back chains (the list's
    // first tile; in the depth sort, the first tile of its view's run, whose digits start at the
    // run's first record)
    uint32_t tileBase, tileEnd, seg = 0;
    bool first;
    if constexpr (DEPTH) {
        const uint32_t tilesPerRun = (a.segLength + kTile - 1) / kTile;
        if (t >= tilesPerRun * a.segments || t >= a.maxTiles) return;
        seg = t / tilesPerRun;
        const uint32_t local = t - seg * tilesPerRun;
        tileBase = seg * a.segLength + local * kTile;
        tileEnd = tileBase + kTile < (seg + 1) * a.segLength ? tileBase + kTile : (seg + 1) * a.segLength;
        first = local == 0;
    } else {
        tileBase = t * kTile;
        if (tileBase >= entries || t >= a.maxTiles) return;
        tileEnd = entries;
        first = t == 0;
    }
    const uint32_t in = plan->inBuffer[p];
    const uint64_t* keysIn = a.keys[in];
    const uint32_t* valsIn = a.values[in];
    uint64_t* keysOut = a.keys[in ^ 1u];
    uint32_t* valsOut = a.values[in ^ 1u];
    const uint32_t lowBits = plan->lowBits;
    const uint64_t keyMask = maskOf(plan->keyBits);
    const uint32_t shift = BITS * p + (PAIRS || DEPTH ? 0u : plan->indexBits);
    const uint32_t indexBits = plan->indexBits, depthBits = plan->depthBits, depthMin = plan->depthMin;
    auto digit = [&](uint64_t k) -> uint32_t {
        if constexpr (DEPTH) return (depthVirtualKey(k, indexBits, depthBits, depthMin) >> shift) & D::kMask;
        return PAIRS ? uint32_t(virtualKey(k, lowBits, keyMask) >> shift) & D::kMask : uint32_t(k >> shift) & D::kMask;
    };

    // 1) load, count, publish
    const uint32_t itemBase = tileBase + warp * (32 * kItems) + lane;
    uint64_t key[kItems];
    uint32_t val[PAIRS ? kItems : 1];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t idx = itemBase + j * 32;
        key[j] = idx < tileEnd ? __ldg(&keysIn[idx]) : ~0ull;
        if (PAIRS) val[PAIRS ? j : 0] = idx < tileEnd ? __ldg(&valsIn[idx]) : 0u;
    }
    uint32_t* wc = sWarpCnt + warp * kBins;
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        if (itemBase + j * 32 < tileEnd) atomicAdd(&wc[digit(key[j])], 1u);
    __syncthreads();
    const uint32_t epoch = ctl->c.epoch;
    uint64_t* status = a.status + (size_t(p) * a.maxTiles) * kBins;
    uint32_t blockCount[P];
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const uint32_t d = D::of(q);
        blockCount[q] = 0;
        if (d >= uint32_t(kBins)) continue;
#pragma unroll
        for (int w = 0; w < 8; ++w) {  // warp offsets of digit d, exclusive over the warps
            const uint32_t c = sWarpCnt[w * kBins + d];
            sWarpCnt[w * kBins + d] = blockCount[q];
            blockCount[q] += c;
        }
        stRelaxed(&status[size_t(t) * kBins + d], packStatus(epoch, first ? kFlagInclusive : kFlagAggregate, blockCount[q]));
    }
    uint32_t blockStart[P];
    blockScanDigits<BITS>(blockCount, blockStart, sScan);
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const uint32_t d = D::of(q);
        if (d >= uint32_t(kBins)) continue;
#pragma unroll
        for (int w = 0; w < 8; ++w) sWarpCnt[w * kBins + d] += blockStart[q];
    }
    __syncthreads();

    // 2) ranks and the local stable order
    const uint32_t ltMask = laneMaskLt();
    uint32_t prevDigit = 0, prevLeader = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t dj = digit(key[j]);
        uint32_t* mask = sMask + (warp * 2 + (j & 1)) * kBins;
        atomicOr(&mask[dj], 1u << lane);
        __syncwarp();
        const uint32_t peers = mask[dj];
        const uint32_t run = wc[dj];  // the digit's running position in this warp's order
        // the previous step's masks were read by every lane before the last __syncwarp
        if (j > 0 && prevLeader) sMask[(warp * 2 + ((j & 1) ^ 1)) * kBins + prevDigit] = 0;
        const uint32_t below = peers & ltMask;
        prevDigit = dj;
        prevLeader = below == 0;
        const uint32_t pos = run + __popc(below);
        if (itemBase + j * 32 < tileEnd) {
            sKeys[pos] = key[j];
            if (PAIRS) sVals[pos] = val[PAIRS ? j : 0];
        }
        __syncwarp();  // every lane has read wc[dj] before its digit's leader advances it
        if (below == 0) wc[dj] = run + __popc(peers);
    }

    // 3) global offsets of this thread's digits' runs
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const uint32_t d = D::of(q);
        if (d >= uint32_t(kBins)) continue;
        uint32_t exclusive = 0;
        if (!first) {  // a chain ends at the first inclusive status: the run's (or the list's) first tile
            exclusive = digitLookback<kBins>(status, t, d, epoch, ctl);
            stRelaxed(&status[size_t(t) * kBins + d], packStatus(epoch, kFlagInclusive, exclusive + blockCount[q]));
        }
        const uint32_t digitBase =
            DEPTH ? a.segBase[(size_t(seg) * a.passesLaunched + p) * kBins + d] : plan->digitBase[p][d];
        sOff[d] = digitBase + exclusive - blockStart[q];
    }
    __syncthreads();

    // 4) write-out
    const uint32_t n = tileEnd - tileBase < uint32_t(kTile) ? tileEnd - tileBase : uint32_t(kTile);
#pragma unroll 4
    for (uint32_t k = tid; k < n; k += kSortThreads) {
        const uint64_t kk = sKeys[k];
        const uint32_t g = sOff[digit(kk)] + k;
        if (g < entries) {
            keysOut[g] = kk;
            if (PAIRS) valsOut[g] = sVals[k];
        } else {
            atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
        }
    }
    __syncthreads();  // the next tile reuses the shared buffers and sTile
    }
}

// One pass in the layout the plan chose on the device (a skipped pass returns at once).
template <int BITS>
__global__ void __launch_bounds__(kSortThreads, BITS == 9 ? 2 : 3) sortPassKernel(const __grid_constant__ SortArgs a,
                                                                                 uint32_t p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t sOff[1 << BITS], sScan[8], sTile;
    const SortPlan* plan = a.plan;
    if (!plan->active[p]) return;
    if (plan->packed) sortPassTiles<false, 24, BITS>(a, p, smem, sOff, sScan, sTile);
    else sortPassTiles<true, 16, BITS>(a, p, smem, sOff, sScan, sTile);
}

// One pass of binning mode's depth sort: always single words, 4096-key tiles (N / 4096 tiles, one
// wave at N ~ 1M). Measured on B200 at N = 1.24M, 4 passes of 8 bits: 16 keys per thread 86 us,
// 12: 86, 24 (the list sort's tile): 92, 8: 94, 4: 120.
template <int BITS>
__global__ void __launch_bounds__(kSortThreads, BITS == 9 ? 2 : 4) depthPassKernel(const __grid_constant__ SortArgs a,
                                                                                  uint32_t p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t sOff[1 << BITS], sScan[8], sTile;
    if (!a.plan->active[p]) return;
    sortPassTiles<false, kDepthSortItems, BITS, true>(a, p, smem, sOff, sScan, sTile);
}

// ---- tile ranges (tile_ranges.comp:22-44) -----------------------------------------------------
// Each thread takes 8 consecutive sorted entries (four 16-byte loads) and the entry before them,
// so the loads stream at the copy's width; a range starts where the tile changes and ends where
// the next one starts (or at the list's end).
constexpr uint32_t kRangeItems = 8;
__global__ void __launch_bounds__(256) rangesKernel(const __grid_constant__ RenderArgs a) {
    const DeviceControl* ctl = a.ctl;
    const uint32_t n = ctl->c.entries;
    const uint64_t* keys = a.keys[ctl->c.sorted_buffer & 1u];
    const uint32_t tileCount = a.totalTiles;  // every view's tiles; the sentinel is this id
    uint2* ranges = reinterpret_cast<uint2*>(a.ranges);
    const uint32_t shift = a.plan->packed ? a.plan->indexBits + a.plan->lowBits : 32u;
    const uint32_t stride = gridDim.x * blockDim.x * kRangeItems;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * kRangeItems; base < n; base += stride) {
        uint32_t t[kRangeItems];
        if (base + kRangeItems <= n) {
            const uint4* v = reinterpret_cast<const uint4*>(keys + base);
#pragma unroll
            for (uint32_t j = 0; j < kRangeItems / 2; ++j) {
                const uint4 w = __ldg(&v[j]);
                t[2 * j] = uint32_t(((uint64_t(w.y) << 32) | w.x) >> shift);
                t[2 * j + 1] = uint32_t(((uint64_t(w.w) << 32) | w.z) >> shift);
            }
        } else {
#pragma unroll
            for (uint32_t j = 0; j < kRangeItems; ++j) t[j] = base + j < n ? uint32_t(keys[base + j] >> shift) : 0u;
        }
        uint32_t prev = base > 0 ? uint32_t(keys[base - 1] >> shift) : 0u;
#pragma unroll
        for (uint32_t j = 0; j < kRangeItems; ++j) {
            const uint32_t k = base + j;
            if (k >= n) break;
            const uint32_t tile = t[j];
            if (tile >= tileCount) {
                // the sentinel tile (sorted last) closes the last real tile's range
                if (k > 0 && prev < tileCount) ranges[prev].y = k;
            } else {
                if (k == 0) {
                    ranges[tile].x = 0;
                } else if (prev != tile) {
                    if (prev < tileCount) ranges[prev].y = k;
                    ranges[tile].x = k;
                }
                if (k == n - 1) ranges[tile].y = n;
            }
            prev = tile;
        }
    }
}

// ---- standalone exclusive scan (GpuScan plain / kNonZero / kGather) ---------------------------
constexpr int kScanItems = int(kScanBlockItems / 256);
static_assert(256 * kScanItems == int(kScanBlockItems), "one scan block = 256 threads x kScanItems");
__global__ void __launch_bounds__(256) scanKernel(const uint32_t* __restrict__ in, const uint32_t* __restrict__ index,
                                                  uint32_t* __restrict__ out, uint32_t* total, uint32_t count,
                                                  uint32_t mode, uint64_t* status, DeviceControl* ctl,
                                                  uint32_t setupCapacity, uint32_t waitSite,
                                                  const __grid_constant__ ScanGather gather) {
    __shared__ uint32_t sBlock, sWarp[8], sExclusive;
    const uint64_t* words = mode == kScanGatherSorted ? gather.words[gather.plan->sortedBuffer & 1u] : nullptr;
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
            else if (mode == kScanGatherSorted) x = in[uint32_t(words[idx] & gather.mask)];
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
            stRelaxed(&status[block], packStatus(epoch, block == 0 ? kFlagInclusive : kFlagAggregate, blockTotal));
        uint32_t exclusive = 0;
        if (block > 0) exclusive = warpLookback(status, int(block), epoch, ctl, waitSite);
        if (lane == 0) {
            if (block > 0) stRelaxed(&status[block], packStatus(epoch, kFlagInclusive, exclusive + blockTotal));
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

namespace {
template <int BITS>
cudaError_t launchSortBits(const SortArgs& a, uint32_t histBlocks, cudaStream_t s) {
    static std::atomic<int> passGrids[64] = {}, depthGrids[64] = {};
    std::atomic<int>& passGrid = perDevice(passGrids);
    std::atomic<int>& depthGrid = perDevice(depthGrids);
    constexpr int kListSmem = PassShape<false, 24, BITS>::kSmemBytes;
    constexpr int kDepthSmem = PassShape<false, kDepthSortItems, BITS>::kSmemBytes;
    if (!passGrid) {
        cudaError_t e = cudaFuncSetAttribute(sortPassKernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, kListSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(depthPassKernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepthSmem);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 148, perSm = 3, depthPerSm = 4;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, sortPassKernel<BITS>, kSortThreads, kListSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&depthPerSm, depthPassKernel<BITS>, kSortThreads, kDepthSmem);
        depthGrid = sms * (depthPerSm > 0 ? depthPerSm : 1);
        passGrid = sms * (perSm > 0 ? perSm : 1);
    }
    sortHistKernel<BITS><<<histBlocks < 1 ? 1 : histBlocks, 256, 0, s>>>(a);
    const bool depth = a.frameMode == 2;
    const uint32_t tiles = a.maxTiles < 1 ? 1 : a.maxTiles;
    const uint32_t limit = uint32_t(depth ? depthGrid : passGrid);
    const uint32_t grid = tiles < limit ? tiles : limit;
    for (uint32_t p = 0; p < a.passesLaunched; ++p) {
        if (depth) depthPassKernel<BITS><<<grid, kSortThreads, kDepthSmem, s>>>(a, p);
        else sortPassKernel<BITS><<<grid, kSortThreads, kListSmem, s>>>(a, p);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launchSort(const SortArgs& a, uint32_t histBlocks, cudaStream_t s) {
    if (a.passesLaunched > uint32_t(kMaxSortPasses)) return cudaErrorInvalidValue;
    switch (a.digitBits) {
        case 7: return launchSortBits<7>(a, histBlocks, s);
        case 9: return launchSortBits<9>(a, histBlocks, s);
        case 0:
        case 8: return launchSortBits<8>(a, histBlocks, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchRanges(const RenderArgs& a, uint32_t capacity, cudaStream_t s) {
    rangesKernel<<<gridFor((capacity + kRangeItems - 1) / kRangeItems, 256, 148 * 16), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchScan(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
                       uint32_t mode, uint64_t* status, DeviceControl* ctl, cudaStream_t s, uint32_t setupCapacity,
                       uint32_t waitSite, const ScanGather* gather) {
    const uint32_t blocks = (count + kScanBlockItems - 1) / kScanBlockItems;
    if (blocks == 0) {
        if (total) return cudaMemsetAsync(total, 0, 4, s);
        return cudaSuccess;
    }
    const ScanGather g = gather ? *gather : ScanGather{{nullptr, nullptr}, nullptr, 0};
    scanKernel<<<blocks, 256, 0, s>>>(in, index, out, total, count, mode, status, ctl, setupCapacity, waitSite, g);
    return cudaGetLastError();
}

// The scratch of gsr_scan_static: a fixed array instead of a per-call allocation (control
// block at offset 0, look-back words from kStaticScanCtlBytes). Zero at module load; every
// call clears what it uses. One array per device, shared by all calls on that device.
static __device__ __align__(256) unsigned char gStaticScanScratch[kStaticScanScratchBytes];

cudaError_t staticScanScratch(void** base) { return cudaGetSymbolAddress(base, gStaticScanScratch); }

// Loads the scan kernel's code on the current device now (with lazy module loading a kernel is
// loaded, and may allocate device memory, at its first launch).
cudaError_t loadScanKernel() {
    cudaFuncAttributes attr;
    return cudaFuncGetAttributes(&attr, scanKernel);
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
