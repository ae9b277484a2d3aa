// Device-side building blocks shared by the splat-tiles kernels (sm_100a).
//
// Exactness rules of the bit-exact stages (preprocess, coverage, key emission): those
// translation units are compiled with -fmad=false (no contraction into FMA), keep CUDA's
// IEEE division and square root (-prec-div/-prec-sqrt, the nvcc default), and spell every
// expression in the reference's evaluation order. std::min/std::max/std::clamp and the
// x86-64 int(float) conversion are restated below with their exact semantics.
#pragma once

#include <cstdint>

#include "gsr_types.h"

namespace gsr {

// ---- exact scalar semantics -------------------------------------------------------------
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
__device__ __forceinline__ int imax(int a, int b) { return (a < b) ? b : a; }
__device__ __forceinline__ int imin(int a, int b) { return (b < a) ? b : a; }
// int(float) as x86-64 cvttss2si: truncation, INT_MIN for NaN and out-of-range values.
__device__ __forceinline__ int ftoi(float x) {
    return (x >= -2147483648.0f && x < 2147483648.0f) ? __float2int_rz(x) : int(0x80000000u);
}

// ---- memory ordering for flag-based cross-block communication ------------------------------
// Look-back status words carry their value in the word itself, so they are written and read
// with relaxed (strong, GPU-scope) operations: no acquire/release ordering is needed, and a
// window of relaxed loads is in flight at once (acquire loads would complete one by one).
__device__ __forceinline__ uint64_t ldRelaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void stRelaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ldAcquire32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Look-back status words: [63:34] epoch, [33:32] flag, [31:0] value.
constexpr uint64_t kFlagAggregate = 1, kFlagInclusive = 2;
__device__ __forceinline__ uint64_t packStatus(uint32_t epoch, uint64_t flag, uint32_t value) {
    return (uint64_t(epoch & 0x3FFFFFFFu) << 34) | (flag << 32) | value;
}
__device__ __forceinline__ bool statusReady(uint64_t s, uint32_t epoch) {
    return uint32_t(s >> 34) == (epoch & 0x3FFFFFFFu) && ((s >> 32) & 3u) != 0;
}
__device__ __forceinline__ uint64_t statusFlag(uint64_t s) { return (s >> 32) & 3u; }

__device__ __forceinline__ void reportTimeout(DeviceControl* ctl, uint32_t where) {
    atomicOr(&ctl->c.status, uint32_t(GSR_CONTROL_TIMEOUT));
    atomicExch(&ctl->c.timeout_where, where);
}

// Decoupled look-back (single-pass chained scan, Merrill & Garland 2016) of one tile's
// exclusive prefix, done by one full warp: lane j inspects predecessor (tile - 1 - j) so a
// window of 32 predecessors is read per step. Returns the sum of the values of all tiles
// before `tile`. Waits are bounded by kSpinLimit (then reportTimeout and a partial sum).
__device__ __forceinline__ uint32_t warpLookback(const uint64_t* status, int tile, uint32_t epoch,
                                                 DeviceControl* ctl, uint32_t where) {
    const int lane = threadIdx.x & 31;
    uint32_t exclusive = 0;
    int base = tile - 1;
    uint32_t spins = 0;
    const uint32_t forced = ctl->forceTimeout;
    while (base >= 0) {
        const int idx = base - lane;
        uint64_t s = idx >= 0 ? ldRelaxed(&status[idx]) : packStatus(epoch, kFlagInclusive, 0);
        bool ready = statusReady(s, epoch);
        if (forced && spins < forced) ready = false;  // test hook: behave as if nobody published
        if (!__all_sync(0xFFFFFFFFu, ready)) {
            if (++spins >= kSpinLimit || (forced && spins >= forced)) {
                if (lane == 0) reportTimeout(ctl, where);
                break;
            }
            __nanosleep(32);
            continue;
        }
        const uint32_t incl = __ballot_sync(0xFFFFFFFFu, statusFlag(s) == kFlagInclusive);
        uint32_t v = uint32_t(s);
        if (incl) {
            const int first = __ffs(incl) - 1;
            if (lane > first) v = 0;
        }
        exclusive += __reduce_add_sync(0xFFFFFFFFu, v);
        if (incl) break;
        base -= 32;
    }
    return exclusive;
}

// ---- the layout of the frame's list entries -----------------------------------------------
// The sort key is (tile, depth bits). All depth bits above the highest bit where the frame's
// smallest and largest visible depth differ are equal in every key, so the key is ordered by
// the "virtual key" vkey = tile << W | depth mod 2^W, W = bit_width(depthMin ^ depthMax). When
// tile bits + W + index bits fit in 64, an entry is ONE word, (vkey << indexBits) | index: the
// index breaks ties, so sorting these words orders the list exactly like a stable sort of the
// (tile, depth) keys in index order, and the sort moves 8 bytes per entry instead of 12.
// Otherwise entries are the two arrays (tile << 32 | depth bits, index). Every kernel derives the
// same layout from the control block (written by the preprocess) and the grid.
struct KeyLayout {
    uint32_t packed;     // 1: one 64-bit word per entry
    uint32_t lowBits;    // W
    uint32_t indexBits;  // bits of the gaussian index (packed)
    uint32_t tileBits;   // bits of the largest tile id incl. the sentinel
};
__device__ __forceinline__ uint32_t bitWidth32(uint32_t x) { return x ? 32u - __clz(x) : 0u; }
// binning: the list is emitted in (depth, index) order and sorted stably by tile alone, so its
// entries carry no depth bits (W = 0): (tile << indexBits) | index, always one word.
__device__ __forceinline__ KeyLayout keyLayout(const DeviceControl* ctl, uint32_t tileCount, uint32_t count,
                                               bool binning = false) {
    KeyLayout l;
    const uint32_t dmin = ctl->c.depth_min_bits, dmax = ctl->c.depth_max_bits;
    l.lowBits = binning || dmin > dmax ? 0u : bitWidth32(dmin ^ dmax);
    l.indexBits = count > 1 ? bitWidth32(count - 1) : 1u;
    l.tileBits = bitWidth32(tileCount);  // the sentinel tile id is tileCount
    l.packed = l.tileBits + l.lowBits + l.indexBits <= 64 ? 1u : 0u;
    return l;
}

// ---- the C library's logf, exactly -------------------------------------------------------
// The reference evaluates 2 ln(255 o) with std::log(float) (tile_coverage.cpp:36). Here: the
// correctly rounded log (from the double-precision log), corrected by the build-time table of
// inputs where the C library's logf is one ulp away (gen_logf_fixups.c). Inputs outside
// [1, 255] (opacity above 1) use the correctly rounded value.
__device__ __forceinline__ float libcLogf(float x, const LogfFixups& t) {
    const float r = float(log(double(x)));
    const uint32_t xb = __float_as_uint(x);
    if (xb < t.base || xb > t.last) return r;
    const uint32_t off = xb - t.base;
    const uint32_t b = off >> 10;
    if (!((__ldg(&t.groups[off >> 8]) >> ((off >> 3) & 31u)) & 1u)) return r;  // none among its 8 neighbours
    uint32_t lo = __ldg(&t.bucketStart[b]), hi = __ldg(&t.bucketStart[b + 1]);
    while (lo < hi) {  // lower bound of off in entries[lo, hi)
        const uint32_t mid = (lo + hi) >> 1;
        if ((__ldg(&t.entries[mid]) >> 1) < off) lo = mid + 1;
        else hi = mid;
    }
    if (lo < t.count) {
        const uint32_t e = __ldg(&t.entries[lo]);
        if ((e >> 1) == off) return __uint_as_float((e & 1u) ? __float_as_uint(r) + 1u : __float_as_uint(r) - 1u);
    }
    return r;
}

}  // namespace gsr
