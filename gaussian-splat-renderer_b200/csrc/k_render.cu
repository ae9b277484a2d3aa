// The tile rasterizer (INRIA renderCUDA; the reference's shaders/tile_render.comp:281-400 and
// the CPU reference's per-pixel loop, src/splat/reference_renderer.cpp:120-222).
//
// One 256-thread block per 16x16 tile, one thread per pixel; warp w owns an 8 x 4 pixel block.
// The tile's entries [ranges[tile].x, ranges[tile].y) are walked front to back in batches of
// 256 records, double-buffered: while batch b is blended, the records of batch b+1 are gathered
// into shared memory with cp.async (16-byte LDGSTS, the record of gaussian values[j]). Each
// entry is then prepared once per block: its power, in base 2 and with log2(opacity) added,
// expanded as a quadratic in the pixel's offset from the centre of its 32 x 16 cell (powerAt), so that
//   alpha = min(0.99, 2^p) = min(0.99, o * exp(power))
// costs five FMAs and one MUFU.EX2, and the warp strips its alpha >= 1/255 cutoff ellipse (the
// reference's threshold with a wider margin, tile_coverage.cpp:24-50) meets, so that a warp skips a
// splat that cannot reach any of its 32 pixels (every skipped pair has alpha < 1/255, which the
// loop would skip anyway). Per pair, INRIA's test-before-accept rule:
//   skip power > 0; skip alpha < 1/255; testT = T (1 - alpha); testT < 1e-4 -> done;
//   C += colour alpha T; T = testT
// and a whole-tile vote (__syncthreads_count) ends the tile once every pixel is done.
//
// Tiles are the frame's tiles over all of its views (DevView): tile t belongs to the view whose
// [tileBase, tileBase + tilesX * tilesY) holds it, the records of that view's gaussians are at
// view * N + g, and its pixels at the view's pixelBase. Two schedules of the same per-tile body:
// one block per tile (a single view), or a persistent grid (a few blocks per SM) whose blocks
// take the next tile from a queue counter until every tile of every view is done, which keeps
// the SMs busy across views of uneven size.
//
// The expanded power, FMA contraction and the hardware exp2 and log2 make the float image differ
// from the CPU reference's in the last bits (and, for pairs within rounding of the 1/255 or 1e-4
// thresholds, by one such pair's contribution); tests bound it: float PSNR > 60 dB and the 8-bit
// image within 1/255. The image does not depend on the tile shape, the schedule or the gather.
#include <cuda.h>  // CUtensorMap (the type only; maps are encoded by the host)

#include "gsr_device.cuh"
#include "kernels.cuh"
#include "render_splat.cuh"

namespace gsr {

namespace {

constexpr int kRenderThreads = 256;
constexpr int kPersistentBlocksPerSm = 4;
constexpr uint32_t kRenderQueueTicket = 13;  // DeviceControl::tickets slot of the persistent queue
constexpr float kMaxAlpha = 0.99f;
constexpr float kMinTransmittance = 1e-4f;
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ void cpAsync16(void* smemDst, const void* gsrc) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smemDst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpAsync8(void* smemDst, const void* gsrc) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smemDst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ float fastExp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float approxSqrt(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Render tiles by their code: 16 (16 x 16, INRIA's), 8 (8 x 8) or 32 (32 x 8).
__host__ __device__ constexpr int tileW(int code) { return code; }
__host__ __device__ constexpr int tileH(int code) { return code == 32 ? 8 : code; }
__host__ __device__ constexpr int tilePixels(int code) { return tileW(code) * tileH(code); }

// The warp strips (8 x 4 pixel blocks of a tile; bit w = warp w's) that a record's
// cutoff ellipse q(d) = A dx^2 + 2B dx dy + C dy^2 <= t meets, computed once per record. At
// distance dy = cy - y from the centre the ellipse's run is cx + (B/A) dy -/+ sqrt((t - (D/A) dy^2)
// / A); over a strip row's y-range its right edge (concave in dy) peaks at the ellipse's
// rightmost point dy = B sqrt(t / (C D)) clamped into the range, its left edge at the mirror
// point. The test keeps the margins of the tile-coverage box: t + 0.2 %, the y-range widened by
// 0.05 px, the run by 0.1 % + 0.05 px, over a continuous y-range (a superset of the pixel rows),
// so a strip holding a pixel with alpha >= 1/255 is always set; a NaN sets the strip.
template <int TILE>
__device__ __forceinline__ uint32_t stripMask(float cx, float cy, float A, float B, float C, float D, float t,
                                              float tileX, float tileY) {
    constexpr uint32_t kStripsX = tileW(TILE) / 8, kGroups = tileH(TILE) / 4;
    const float tt = t * 1.002f;
    const float ia = 1.0f / A, bA = B * ia, dA = D * ia;
    const float ey = approxSqrt(tt / dA);
    const float dyR = B * approxSqrt(tt / (C * D));
    uint32_t mask = 0;
#pragma unroll
    for (uint32_t g = 0; g < kGroups; ++g) {
        const float ya = tileY + float(4 * g) - 0.05f, yb = tileY + float(4 * g + 3) + 0.05f;
        const float lo = fmaxf(cy - yb, -ey), hi = fminf(cy - ya, ey);  // dy range inside the ellipse
        if (lo > hi) continue;
        const float dr = fminf(fmaxf(dyR, lo), hi), dl = fminf(fmaxf(-dyR, lo), hi);
        const float hr = fmaf(approxSqrt(fmaxf(fmaf(-dA * dr, dr, tt), 0.0f) * ia), 1.001f, 0.05f);
        const float hl = fmaf(approxSqrt(fmaxf(fmaf(-dA * dl, dl, tt), 0.0f) * ia), 1.001f, 0.05f);
        const float right = fmaf(bA, dr, cx) + hr, left = fmaf(bA, dl, cx) - hl;
#pragma unroll
        for (uint32_t c = 0; c < kStripsX; ++c) {
            const float x0 = tileX + float(8 * c), x1 = x0 + 7.0f;
            if (!(right < x0) && !(left > x1)) mask |= 1u << (g * kStripsX + c);
        }
    }
    return mask;
}

// 32 x 8 tiles: the strips (bit g * 4 + c: columns 8c .. 8c + 7 of the tile, either row group)
// inside the splat's 16-px tile rectangle along x, [16 minX, 16 maxX) with the preprocess's
// tileRect arithmetic (its upper clamp to the grid only removes pixels past the image). The
// rectangle's edges are multiples of 16 and the strips' multiples of 8, so a strip is wholly in
// or out. (Along y the tile's 8 rows always lie inside or outside the rectangle's 16-px rows.)
__device__ __forceinline__ uint32_t rectStrips32(float cx, float radius, uint32_t tileX) {
    const float fr = float(ftoi(radius));
    const int x0 = 16 * imax(0, ftoi((cx - fr) / float(kTileSize)));
    const int x1 = 16 * imax(0, ftoi((cx + fr + float(kTileSize - 1)) / float(kTileSize)));
    uint32_t m = 0;
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
        const int s = int(tileX + 8 * c);
        if (s >= x0 && s < x1) m |= 0x11u << c;
    }
    return m;
}

// How a batch's records reach shared memory.
constexpr int kGatherCpAsync = 0;  // every thread copies its record with 16-byte cp.async
constexpr int kGatherTma = 1;      // one warp gathers four records per cp.async.bulk.tensor tile::gather4

// The staging area of a batch (double-buffered). cp.async: full 3 x 16 B, p32 2 x 16 B, p24
// 3 x 8 B per record (as uint2 rows of N in the first half of the area). TMA: quads of four
// 48-byte records as gather4 writes them, each quad in a 256-byte slot so that every
// destination is 128-byte aligned; one mbarrier per buffer and its completed uses (the phase).
template <int N, int GATHER>
struct StageArea {
    float4 raw[2][3][N];
};
template <int N>
struct StageArea<N, kGatherTma> {
    alignas(128) unsigned char quad[2][N / 4][256];
    uint64_t bar[2];
    uint32_t uses[2];
};

// N = the batch (one entry per thread of the tile's block)
template <int N, int GATHER = kGatherCpAsync>
struct RenderShared {
    StageArea<N, GATHER> st;
    float4 power0[N];     // qa, qb, qc, d of the expanded power (powerAt)
    float4 power1[N];     // e, f, the sign-test bound, -
    uint32_t strips[N];   // the warp strips the cutoff ellipse meets (stripMask)
    float4 color[N];      // r, g, b, -
    uint32_t hits[N / 32][32];  // per warp: the records of its current 32 that meet its strip, in list order
    uint32_t tile;        // persistent schedule: the block's current tile
};

// The exponent of alpha in base 2, log2(o) + log2(e) * power, at pixel offset (X, Y) from the
// centre of the 32 x 16 pixel cell that holds the tile (the same origin for every tile shape,
// so the image does not depend on it). With qa, qb, qc the conic scaled by -log2(e)/2, -log2(e),
// -log2(e)/2 and (cx, cy) the centre relative to the cell,
//   qa (cx-X)^2 + qb (cx-X)(cy-Y) + qc (cy-Y)^2 + log2(o) = X (qa X + qb Y + d) + Y (qc Y + e) + f
// with d = -(2 qa cx + qb cy), e = -(2 qc cy + qb cx), f = the left side at (0, 0): five FMAs a
// pair and o folded in. The power > 0 test reads p > log2(o); for a positive definite conic the
// power is never positive and the bound is +inf (the expanded sum's rounding near the centre
// must not drop the splat there).
__device__ __forceinline__ float powerAt(const float4& u, const float4& w, float X, float Y) {
    return fmaf(X, fmaf(u.x, X, fmaf(u.y, Y, u.w)), fmaf(Y, fmaf(u.z, Y, w.x), w.y));
}

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Four records (rows of the 2-D tensor map over the frame's record array: 12 fp32 columns, one
// row per record) into 192 contiguous bytes at dst, completed on bar. Column 0 is the only
// x coordinate used (16-byte aligned); the box is one row high.
__device__ __forceinline__ void tmaGather4(void* dst, const CUtensorMap* map, const uint32_t (&row)[4], uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        :: "r"(smemAddr(dst)), "l"(map), "r"(0), "r"(row[0]), "r"(row[1]), "r"(row[2]), "r"(row[3]), "r"(smemAddr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbarDone(uint64_t* bar, uint32_t parity) {
    uint32_t done = 0;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(smemAddr(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait for a buffer's gathers; on expiry the frame is marked GSR_CONTROL_TIMEOUT (site
// kWaitGather) and its image is untrusted.
__device__ __forceinline__ void mbarWaitBounded(uint64_t* bar, uint32_t parity, DeviceControl* ctl) {
    for (uint32_t spins = 0; !mbarDone(bar, parity); ++spins) {
        if (spins >= kSpinLimit) {
            if ((threadIdx.x & 31) == 0) reportTimeout(ctl, kWaitGather);
            return;
        }
    }
}

// The view holding frame tile t: the last view whose tileBase <= t (views are in tile order).
__device__ __forceinline__ uint32_t viewOfTile(const RenderArgs& a, uint32_t t) {
    uint32_t lo = 0, hi = a.viewCount;  // invariant: views[lo].tileBase <= t < views[hi].tileBase
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.views[mid].tileBase <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The whole per-tile pass for frame tile `tile`; every thread of the block calls it.
// StopThePop's per-pixel window (tile_render.comp:201-279): the pixel's K = a.sortWindow pending
// splats ordered by their ray depth (nearest first, ties in list order), in CAP >= K register
// slots. While fewer than K wait, a splat is inserted; once K wait, the nearest of the window and
// the new splat is blended (the usual test-before-accept rule) and the other one takes its place.
// The rest is blended nearest first at the end of the list. Every loop runs over the constant CAP
// with K as a predicate, so the slots stay in registers for CAP <= 16.
template <int CAP>
struct SortWindow {
    float d[CAP], al[CAP], r[CAP], g[CAP], b[CAP];
    uint32_t count = 0;
};
__device__ __forceinline__ void blendOver(float alpha, float r, float g, float b, float& T, float& c0, float& c1,
                                          float& c2, bool& done) {
    const float testT = T * (1.0f - alpha);
    if (testT < kMinTransmittance) {
        done = true;
        return;
    }
    const float w = alpha * T;
    c0 += r * w;
    c1 += g * w;
    c2 += b * w;
    T = testT;
}
template <int CAP>
__device__ __forceinline__ void windowPush(SortWindow<CAP>& q, uint32_t K, float depth, float alpha, float4 col,
                                           float& T, float& c0, float& c1, float& c2, bool& done) {
    if (!(depth < 3.0e38f)) depth = 3.0e38f;  // finite (NaN / infinity of a degenerate splat)
    if (q.count < K) {
        // not full: insertion from the back
        bool placed = false;
#pragma unroll
        for (int i = CAP - 1; i > 0; --i) {
            if (uint32_t(i) < K && !placed) {
                if (uint32_t(i - 1) < q.count && q.d[i - 1] > depth) {
                    q.d[i] = q.d[i - 1];
                    q.al[i] = q.al[i - 1];
                    q.r[i] = q.r[i - 1];
                    q.g[i] = q.g[i - 1];
                    q.b[i] = q.b[i - 1];
                } else if (uint32_t(i - 1) < q.count) {
                    q.d[i] = depth;
                    q.al[i] = alpha;
                    q.r[i] = col.x;
                    q.g[i] = col.y;
                    q.b[i] = col.z;
                    placed = true;
                }
            }
        }
        if (!placed) {
            q.d[0] = depth;
            q.al[0] = alpha;
            q.r[0] = col.x;
            q.g[0] = col.y;
            q.b[0] = col.z;
        }
        ++q.count;
        return;
    }
    // full: the nearest of the window and the new splat leaves it and is blended now
    if (depth < q.d[0]) {
        blendOver(alpha, col.x, col.y, col.z, T, c0, c1, c2, done);
        return;
    }
    blendOver(q.al[0], q.r[0], q.g[0], q.b[0], T, c0, c1, c2, done);
    // slots move left while they are not farther than the new splat; it takes the first other
    // slot, or the last one (K - 1). (One loop: a separate "store at K - 1" loop is turned into an
    // indexed store by the compiler, which moves the window to local memory.)
    bool placed = false;
#pragma unroll
    for (int i = 0; i < CAP; ++i) {
        if (!placed && uint32_t(i) < K) {
            if (i + 1 < CAP && uint32_t(i + 1) < K && q.d[i + 1 < CAP ? i + 1 : i] <= depth) {
                const int n = i + 1 < CAP ? i + 1 : i;
                q.d[i] = q.d[n];
                q.al[i] = q.al[n];
                q.r[i] = q.r[n];
                q.g[i] = q.g[n];
                q.b[i] = q.b[n];
            } else {
                q.d[i] = depth;
                q.al[i] = alpha;
                q.r[i] = col.x;
                q.g[i] = col.y;
                q.b[i] = col.z;
                placed = true;
            }
        }
    }
}

// MODE: the record layout (kRenderSplatFull / P32 / P24), a compile-time parameter so that each
// layout's kernel carries only its own gather and decode (a runtime switch measured 8 % slower).
// CAP: 0, or the StopThePop window's register capacity; `ray` is then the shared area of the
// gathered ray-depth parameters (3 x 16 B per entry, double-buffered).
// TILE: the tile's code, 16 (INRIA's 16 x 16 tiles), 8 (8 x 8) or 32 (32 x 8); one thread per pixel, batches of
// a tile's pixel count
// entries, and each warp owns an 8 x 4 pixel block of the tile (its strip: a squarer footprint
// meets fewer ellipses than a 16 x 2 row pair).
// STATS: the instrumented build (TileSettings::stats, tile_render.comp's GSR_TILE_STATS): the
// kTileStatCount words of the tile (list length, fetched, evaluated, blended, terminated, lane
// slots, max depth, pixels) and the frame's count of the pairs this kernel tested. "Evaluated"
// keeps the reference's meaning, the list entries a pixel visits until it terminates (all of
// them when it does not); "tested" are the pairs this kernel computed alpha for (a pixel still
// blending and a record whose cutoff ellipse meets the pixel's warp strip).
// GATHER: how the batch reaches shared memory (kGatherCpAsync or kGatherTma; TMA only with the
// full records, no window and no statistics); map = the tensor map of the record array (TMA).
template <int MODE, int CAP, int TILE, bool STATS, int GATHER>
__device__ __forceinline__ void renderTile(const RenderArgs& a, RenderShared<tilePixels(TILE), GATHER>& sm,
                                           float4 (*ray)[3][tilePixels(TILE)], uint32_t tile, const CUtensorMap* map) {
    static_assert(GATHER == kGatherCpAsync || (MODE == kRenderSplatFull && CAP == 0 && !STATS), "the TMA gather");
    constexpr uint32_t kTW = tileW(TILE), kTH = tileH(TILE);
    constexpr uint32_t kThreads = kTW * kTH, kStripW = 8, kRows = 4, kStripsX = kTW / kStripW;
    static_assert(kThreads <= kRenderThreads && kStripW * kRows == 32 && kTW % kStripW == 0 && kTH % kRows == 0,
                  "tile shape");
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t sx = (warp % kStripsX) * kStripW, sy = (warp / kStripsX) * kRows;
    const uint32_t view = viewOfTile(a, tile);
    const DevView vw = a.views[view];
    const uint32_t local = tile - vw.tileBase;
    const uint32_t tx = local % vw.tilesX, ty = local / vw.tilesX;
    const uint32_t px = tx * kTW + sx + (lane % kStripW), py = ty * kTH + sy + (lane / kStripW);
    const bool inside = px < vw.width && py < vw.height;
    uint2 range = reinterpret_cast<const uint2*>(a.ranges)[tile];
    // a frame whose look-back gave up (GSR_CONTROL_TIMEOUT) has meaningless ranges: every index
    // read below stays inside the list and the scene all the same
    const uint32_t entries = a.ctl->c.entries;
    range.y = range.y < entries ? range.y : entries;
    range.x = range.x < range.y ? range.x : range.y;
    const uint32_t sortedBuffer = a.ctl->c.sorted_buffer & 1u;
    const uint32_t* values = a.values[sortedBuffer];
    const uint64_t* packedKeys = a.keys[sortedBuffer];
    const bool packed = a.plan->packed != 0;
    const uint64_t indexMask = (1ull << a.plan->indexBits) - 1ull;
    const float4* records = reinterpret_cast<const float4*>(a.splats) + size_t(view) * a.count * 3;
    const uint4* records32 = reinterpret_cast<const uint4*>(a.packed) + size_t(view) * a.count * 2;
    const uint2* records24 = reinterpret_cast<const uint2*>(a.packed) + size_t(view) * a.count * 3;
    constexpr int mode = MODE;
    const float fx = float(px), fy = float(py);
    // the pixel relative to the centre of its 32 x 16 cell (exact small integers, -16..15 and
    // -8..7: the expansion's terms stay small against the power it sums to)
    const float X = float(int(px) - int((tx * kTW) & ~31u) - 16), Y = float(int(py) - int((ty * kTH) & ~15u) - 8);
    // this warp's pixel strip
    float T = 1.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    bool done = !inside;

    // TMA: the buffers' mbarrier phases, the same in every thread (each thread counts the uses)
    uint32_t phase0 = 0, phase1 = 0;
    if constexpr (GATHER == kGatherTma) {
        phase0 = sm.st.uses[0];
        phase1 = sm.st.uses[1];
    }
    auto issue = [&](uint32_t start, int buf) {
        if constexpr (GATHER == kGatherTma) {
            // warp 0 reads the batch's gaussian indices and gathers the records four at a time
            if (warp != 0) return;
            const uint32_t n = range.y - start < kThreads ? range.y - start : kThreads;
            const uint32_t quads = (n + 3u) / 4u;
            if (lane == 0)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smemAddr(&sm.st.bar[buf])),
                             "r"(quads * 192u) : "memory");
            __syncwarp();
            for (uint32_t q = lane; q < quads; q += 32u) {
                uint32_t row[4];
#pragma unroll
                for (uint32_t r = 0; r < 4; ++r) {
                    const uint32_t slot = 4u * q + r;
                    const uint32_t j = start + (slot < n ? slot : n - 1u);  // a short last quad repeats its last record
                    uint32_t g = packed ? uint32_t(__ldg(&packedKeys[j]) & indexMask) : __ldg(&values[j]);
                    if (g >= a.count) {
                        atomicOr(&a.ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
                        g = 0;
                    }
                    row[r] = view * a.count + g;  // the host uses TMA only while V N < 2^31
                }
                tmaGather4(&sm.st.quad[buf][q][0], map, row, &sm.st.bar[buf]);
            }
        } else {
            const uint32_t j = start + tid;
            if (j < range.y) {
                uint32_t g = packed ? uint32_t(__ldg(&packedKeys[j]) & indexMask) : __ldg(&values[j]);
                if (g >= a.count) {
                    atomicOr(&a.ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
                    g = 0;
                }
                if constexpr (mode == kRenderSplatFull) {
                    const float4* rec = records + size_t(g) * 3;
                    cpAsync16(&sm.st.raw[buf][0][tid], rec);
                    cpAsync16(&sm.st.raw[buf][1][tid], rec + 1);
                    cpAsync16(&sm.st.raw[buf][2][tid], rec + 2);
                } else if constexpr (mode == kRenderSplatP32) {
                    const uint4* rec = records32 + size_t(g) * 2;
                    cpAsync16(&sm.st.raw[buf][0][tid], rec);
                    cpAsync16(&sm.st.raw[buf][1][tid], rec + 1);
                } else {  // 24-byte records start on 8-byte boundaries
                    const uint2* rec = records24 + size_t(g) * 3;
                    uint2* dst = reinterpret_cast<uint2*>(&sm.st.raw[buf][0][0]);
                    cpAsync8(&dst[tid], rec);
                    cpAsync8(&dst[kThreads + tid], rec + 1);
                    cpAsync8(&dst[2 * kThreads + tid], rec + 2);
                }
                if constexpr (CAP > 0) {
                    const float4* rp = a.rayDepth + (size_t(view) * a.count + g) * 3;
                    cpAsync16(&ray[buf][0][tid], rp);
                    cpAsync16(&ray[buf][1][tid], rp + 1);
                    cpAsync16(&ray[buf][2][tid], rp + 2);
                }
            }
            cpAsyncCommit();
        }
    };
    // TMA: every thread waits for the buffer's gathers (bounded) and counts the use
    auto waitTma = [&](int buf) {
        if constexpr (GATHER == kGatherTma) {
            mbarWaitBounded(&sm.st.bar[buf], buf ? phase1 : phase0, a.ctl);
            if (buf) phase1 ^= 1u;
            else phase0 ^= 1u;
        }
    };
    // StopThePop: the pixel's ray t (vx, vy, 1) in camera space (pixel = f x / z + (size - 1) / 2)
    SortWindow<(CAP > 0 ? CAP : 1)> window;
    const uint32_t K = a.sortWindow;
    float vx = 0.0f, vy = 0.0f;
    if constexpr (CAP > 0) {
        vx = (fx - 0.5f * (float(vw.width) - 1.0f)) / a.cam[view].focalX;
        vy = (fy - 0.5f * (float(vw.height) - 1.0f)) / a.cam[view].focalY;
    }

    // STATS counters (per thread; stIters is uniform over the warp)
    uint32_t stEval = 0, stBlend = 0, stIters = 0, stFetched = 0, stTested = 0;
    bool stTerm = false;

    // Two block barriers a batch: the vote, which also publishes the batch's gathered records (each
    // thread has waited for its own copies) and orders the previous batch's reads of the staging
    // buffer and of the prepared arrays before this batch overwrites them; and the end of the
    // preparation. Every batch issued is waited for at the top of the next iteration, which
    // always runs, so none is in flight after the loop.
    int buf = 0;
    if (range.x < range.y) issue(range.x, 0);
    for (uint32_t start = range.x; start < range.y; start += kThreads, buf ^= 1) {
        if constexpr (GATHER == kGatherTma) waitTma(buf);
        else cpAsyncWait<0>();
        if (__syncthreads_count(done) == int(kThreads)) break;
        if constexpr (STATS) stFetched += range.y - start < kThreads ? range.y - start : kThreads;
        // the next batch is gathered while this one is prepared and blended
        const uint32_t next = start + kThreads;
        if (next < range.y) issue(next, buf ^ 1);
        if (start + tid < range.y) {
            float2 r0;  // cx, cy
            float A, B, C, o;
            float4 r2;  // r, g, b, -
            float radius = 0.0f;  // as the preprocess's 16-px rectangle read it (truncated)
            if constexpr (mode == kRenderSplatFull) {
                float4 w0, w1;
                if constexpr (GATHER == kGatherTma) {
                    const float4* rec = reinterpret_cast<const float4*>(&sm.st.quad[buf][tid >> 2][(tid & 3u) * 48u]);
                    w0 = rec[0];
                    w1 = rec[1];
                    r2 = rec[2];
                } else {
                    w0 = sm.st.raw[buf][0][tid];  // cx, cy, depth, cull
                    w1 = sm.st.raw[buf][1][tid];  // A, B, C, opacity
                    r2 = sm.st.raw[buf][2][tid];  // r, g, b, radius
                }
                r0 = make_float2(w0.x, w0.y);
                A = w1.x;
                B = w1.y;
                C = w1.z;
                o = w1.w;
                radius = r2.w;
            } else if constexpr (mode == kRenderSplatP32) {
                const float4 w0 = sm.st.raw[buf][0][tid];  // cx, cy, A, B
                const float4 w1 = sm.st.raw[buf][1][tid];  // C, opacity, h(r, g), h(b) | radius
                r0 = make_float2(w0.x, w0.y);
                A = w0.z;
                B = w0.w;
                C = w1.x;
                o = w1.y;
                const uint32_t rg = __float_as_uint(w1.z), bw = __float_as_uint(w1.w);
                r2 = make_float4(halfLoF(rg), halfHiF(rg), halfLoF(bw), 0.0f);
                radius = float(bw >> 16);
            } else {
                const uint2* w = reinterpret_cast<const uint2*>(&sm.st.raw[buf][0][0]);
                const uint2 w0 = w[tid], w1 = w[kThreads + tid], w2 = w[2 * kThreads + tid];
                r0 = make_float2(__uint_as_float(w0.x), __uint_as_float(w0.y));
                p24DecodeConic(w1.x, w1.y, A, B, C, o);
                r2 = make_float4(halfLoF(w2.x), halfHiF(w2.x), halfLoF(w2.y), 0.0f);
                radius = float(w2.y >> 16);
            }
            // the strips the cutoff ellipse meets (makeCutoffEllipse's threshold, wider margin):
            // none below opacity 1/255, all for an invalid conic
            uint32_t strips = (1u << (kThreads / 32)) - 1u;
            const float D = A * C - B * B;
            const bool ellipse = A > 0.0f && C > 0.0f && D > 0.0f;
            if (!(o >= 1.0f / 255.0f)) {
                strips = 0u;
            } else if (ellipse) {
                const float qmax = 2.0f * __logf(255.0f * o) + 1e-3f;
                const float rho = fabsf(B) * rsqrtf(A * C);
                const float K = 2.0f / fmaxf(1.0f - rho, 1e-30f);
                const float t = qmax + (2e-3f + 4e-5f * K) * fmaxf(qmax, 1.0f) + 4e-3f;
                if (t < 1e30f) strips = stripMask<TILE>(r0.x, r0.y, A, B, C, D, t, float(tx * kTW), float(ty * kTH));
            }
            // 32 x 8 tiles: a bin's 32 columns can reach 16 px past the splat's 16-px rectangle,
            // which bounds the splat's pixels wherever the coverage used it (rect and tight
            // bounds, and cutoff-only bounds for a splat without an ellipse)
            if constexpr (TILE == 32)
                if (a.bounds != kBoundsCutoff || !ellipse) strips &= rectStrips32(r0.x, radius, tx * kTW);
            sm.strips[tid] = strips;
            // the expanded power about the cell origin (powerAt); only a record with strips is
            // visited, so its opacity is at least 1/255 and log2(o) finite
            const float qa = -0.5f * kLog2e * A, qb = -kLog2e * B, qc = -0.5f * kLog2e * C;
            const float lg = __log2f(o);
            const float cx = r0.x - (float(px) - X), cy = r0.y - (float(py) - Y);  // the cell centre: exact
            const float d = -fmaf(2.0f * qa, cx, qb * cy), e = -fmaf(2.0f * qc, cy, qb * cx);
            const float f = fmaf(cx, fmaf(qa, cx, qb * cy), fmaf(cy, qc * cy, lg));
            sm.power0[tid] = make_float4(qa, qb, qc, d);
            sm.power1[tid] = make_float4(e, f, ellipse ? __int_as_float(0x7f800000) : lg, 0.0f);
            sm.color[tid] = r2;
        }
        __syncthreads();
        const uint32_t n = range.y - start < kThreads ? range.y - start : kThreads;
        // the warp takes 32 records at a time, one per lane, lists those that meet its strip in
        // list order (each such lane writes its record at its rank among them) and visits the
        // list: a load a record instead of finding and clearing the next set bit of the ballot
        uint32_t* hits = sm.hits[warp];
        const uint32_t below = (1u << lane) - 1u;
        for (uint32_t q0 = 0; q0 < n && !__all_sync(0xffffffffu, done); q0 += 32) {
            const uint32_t ql = q0 + lane;
            const bool hit = ql < n && ((sm.strips[ql] >> warp) & 1u) != 0u;
            const uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (hit) hits[__popc(m & below)] = ql;
            __syncwarp();
            const uint32_t listed = uint32_t(__popc(m));
            for (uint32_t h = 0; h < listed; ++h) {
                const uint32_t q = hits[h];
                if constexpr (STATS) {
                    ++stIters;
                    stTested += done ? 0u : 1u;
                }
                const float4 pw0 = sm.power0[q], pw1 = sm.power1[q];
                const float p = powerAt(pw0, pw1, X, Y);
                const float alpha = fminf(kMaxAlpha, fastExp2(p));
                // skipped: a finished pixel, power > 0, alpha below 1/255 (one predicate)
                if (done || p > pw1.z || alpha < (1.0f / 255.0f)) continue;
                if constexpr (CAP > 0) {
                    // the depth of the gaussian's maximum along the pixel ray: (v . b) / (v^T P v)
                    const float4 pa = ray[buf][0][q], pb = ray[buf][1][q];
                    const float pc = ray[buf][2][q].x;
                    const float vPv = pa.x * vx * vx + 2.0f * pa.y * vx * vy + 2.0f * pa.z * vx + pa.w * vy * vy +
                                      2.0f * pb.x * vy + pb.y;
                    const float vb = pb.z * vx + pb.w * vy + pc;
                    windowPush(window, K, vb / vPv, alpha, sm.color[q], T, c0, c1, c2, done);
                    continue;
                }
                const float testT = T * (1.0f - alpha);
                if (testT < kMinTransmittance) {
                    done = true;
                    if constexpr (STATS) {
                        stTerm = true;
                        stEval = start + q - range.x + 1u;  // the entries visited, the terminating one included
                    }
                    continue;
                }
                const float4 col = sm.color[q];
                const float w = alpha * T;
                c0 += col.x * w;
                c1 += col.y * w;
                c2 += col.z * w;
                T = testT;
                if constexpr (STATS) ++stBlend;
            }
            __syncwarp();  // every lane has read the list before the next group writes it
        }
    }
    if constexpr (CAP > 0) {  // the end of the list: what waits is blended, nearest first
#pragma unroll
        for (int i = 0; i < CAP; ++i)
            if (!done && uint32_t(i) < window.count) blendOver(window.al[i], window.r[i], window.g[i], window.b[i], T, c0, c1, c2, done);
    }
    if constexpr (GATHER == kGatherTma) {
        // no batch is in flight here (see the loop); the phases are kept for the next tile
        __syncthreads();
        if (tid == 0) {
            sm.st.uses[0] = phase0;
            sm.st.uses[1] = phase1;
        }
    } else {
        cpAsyncWait<0>();
    }
    if constexpr (STATS) {
        if (!stTerm) stEval = inside ? range.y - range.x : 0u;
        __shared__ uint32_t sStat[kTileStatWords];
        if (tid < kTileStatWords) sStat[tid] = 0u;
        __syncthreads();
        const uint32_t eSum = __reduce_add_sync(0xffffffffu, stEval), bSum = __reduce_add_sync(0xffffffffu, stBlend);
        const uint32_t tSum = __popc(__ballot_sync(0xffffffffu, stTerm)), pSum = __popc(__ballot_sync(0xffffffffu, inside));
        const uint32_t eMax = __reduce_max_sync(0xffffffffu, stEval), tested = __reduce_add_sync(0xffffffffu, stTested);
        if (lane == 0) {
            atomicAdd(&sStat[kTileStatEvaluated], eSum);
            atomicAdd(&sStat[kTileStatBlended], bSum);
            atomicAdd(&sStat[kTileStatTerminated], tSum);
            atomicAdd(&sStat[kTileStatLaneSlots], stIters * 32u);
            atomicMax(&sStat[kTileStatMaxDepth], eMax);
            atomicAdd(&sStat[kTileStatPixels], pSum);
            atomicAdd(a.testedPairs, (unsigned long long)tested);
        }
        __syncthreads();
        if (tid == 0) {
            sStat[kTileStatListLength] = range.y - range.x;
            sStat[kTileStatFetched] = stFetched;
        }
        __syncthreads();
        if (tid < kTileStatWords) a.tileStats[size_t(tile) * kTileStatWords + tid] = sStat[tid];
    }
    if (!inside) return;
    const size_t p = vw.pixelBase + size_t(py) * vw.width + px;
    if (a.imageFormat == 0) {
        reinterpret_cast<float4*>(a.image)[p] = make_float4(c0, c1, c2, 1.0f - T);
    } else if (a.imageFormat == 1) {
        reinterpret_cast<uint2*>(a.image)[p] = make_uint2(packHalf2(c0, c1), packHalf2(c2, 1.0f - T));
    } else {
        const float v[4] = {c0, c1, c2, 1.0f - T};
        uint32_t w = 0;
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) {
            const float cl = v[ch] < 0.0f ? 0.0f : (v[ch] > 1.0f ? 1.0f : v[ch]);
            w |= uint32_t(roundf(cl * 255.0f)) << (8 * ch);
        }
        reinterpret_cast<uint32_t*>(a.image)[p] = w;
    }
    if (a.rgb8) {
        const float v[3] = {c0, c1, c2};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const float cl = v[ch] < 0.0f ? 0.0f : (v[ch] > 1.0f ? 1.0f : v[ch]);
            a.rgb8[p * 3 + ch] = uint8_t(roundf(cl * 255.0f));  // lround(clamp(v, 0, 1) * 255), image_io.cpp:55-56
        }
    }
}

// One block per frame tile.
// the shared area of a block: RenderShared, then for a StopThePop kernel the ray-depth parameters
template <int CAP, int N, int GATHER>
constexpr size_t renderSmemBytes() {
    return sizeof(RenderShared<N, GATHER>) + (CAP > 0 ? sizeof(float4) * 2 * 3 * N : 0);
}
template <int N, int GATHER>
__device__ __forceinline__ float4 (*rayArea(unsigned char* smem))[3][N] {
    return reinterpret_cast<float4(*)[3][N]>(smem + sizeof(RenderShared<N, GATHER>));
}

// TMA: the buffers' mbarriers, initialized once per block (their phases then run across tiles)
template <int N, int GATHER>
__device__ __forceinline__ void initStage(RenderShared<N, GATHER>& sm) {
    if constexpr (GATHER == kGatherTma) {
        if (threadIdx.x == 0) {
            for (int b = 0; b < 2; ++b) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smemAddr(&sm.st.bar[b])) : "memory");
                sm.st.uses[b] = 0;
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
}

// Without the window: five 256-thread blocks (or the same threads in 8-px tiles) per SM, 48
// registers a thread (the strip masks would take 61, four blocks, 5 % slower).
template <int MODE, int CAP, int TILE, bool STATS, int GATHER>
__global__ void __launch_bounds__(tilePixels(TILE), CAP == 0 ? 5 * 256 / (tilePixels(TILE)) : 1)
    renderKernel(const __grid_constant__ RenderArgs a, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(128) unsigned char smemRaw[];
    RenderShared<tilePixels(TILE), GATHER>& sm = *reinterpret_cast<RenderShared<tilePixels(TILE), GATHER>*>(smemRaw);
    initStage(sm);
    renderTile<MODE, CAP, TILE, STATS, GATHER>(a, sm, CAP > 0 ? rayArea<tilePixels(TILE), GATHER>(smemRaw) : nullptr,
                                               blockIdx.x + a.tileOffset, &map);
}

// Persistent schedule: each block takes tiles from the frame's queue counter (reset by frame
// begin) until the counter passes the last tile.
template <int MODE, int CAP, int TILE, bool STATS, int GATHER>
__global__ void __launch_bounds__(tilePixels(TILE), CAP == 0 ? 5 * 256 / (tilePixels(TILE)) : 1)
    renderPersistentKernel(const __grid_constant__ RenderArgs a, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(128) unsigned char smemRaw[];
    RenderShared<tilePixels(TILE), GATHER>& sm = *reinterpret_cast<RenderShared<tilePixels(TILE), GATHER>*>(smemRaw);
    initStage(sm);
    for (;;) {
        if (threadIdx.x == 0) sm.tile = atomicAdd(&a.ctl->tickets[kRenderQueueTicket], 1u);
        __syncthreads();
        const uint32_t tile = sm.tile;
        if (tile >= a.totalTiles) break;
        renderTile<MODE, CAP, TILE, STATS, GATHER>(a, sm, CAP > 0 ? rayArea<tilePixels(TILE), GATHER>(smemRaw) : nullptr,
                                                   tile, &map);
        __syncthreads();  // every thread has read sm.tile and left the tile's shared buffers
    }
}

template <int MODE, int CAP, int TILE, bool STATS = false, int GATHER = kGatherCpAsync>
cudaError_t launchRenderMode(const RenderArgs& a, cudaStream_t s) {
    constexpr size_t smem = renderSmemBytes<CAP, tilePixels(TILE), GATHER>();
    constexpr uint32_t threads = tilePixels(TILE);
    static std::atomic<bool> configuredOn[64] = {};
    std::atomic<bool>& configured = perDevice(configuredOn);
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(renderKernel<MODE, CAP, TILE, STATS, GATHER>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(renderPersistentKernel<MODE, CAP, TILE, STATS, GATHER>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    CUtensorMap map{};  // read by the TMA kernels only
    if constexpr (GATHER == kGatherTma) map = *static_cast<const CUtensorMap*>(a.splatMap);
    if (a.persistent) {
        int sms = 148, dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // as many resident threads per SM for either tile size
        const uint32_t grid = uint32_t(sms) * kPersistentBlocksPerSm * (kRenderThreads / threads);
        renderPersistentKernel<MODE, CAP, TILE, STATS, GATHER>
            <<<grid < a.totalTiles ? grid : a.totalTiles, threads, smem, s>>>(a, map);
    } else {
        renderKernel<MODE, CAP, TILE, STATS, GATHER><<<a.tileLaunch ? a.tileLaunch : a.totalTiles, threads, smem, s>>>(a, map);
    }
    return cudaGetLastError();
}

// the window capacity for K: 4, 16 or 64 register slots
template <int MODE, int TILE>
cudaError_t launchRenderWindow(const RenderArgs& a, cudaStream_t s) {
    if (a.tileStats) return launchRenderMode<MODE, 0, TILE, true>(a, s);  // the stats build has no window
    if constexpr (MODE == kRenderSplatFull) {
        if (a.sortWindow == 0 && a.splatMap) return launchRenderMode<MODE, 0, TILE, false, kGatherTma>(a, s);
    }
    if (a.sortWindow == 0) return launchRenderMode<MODE, 0, TILE>(a, s);
    if (a.sortWindow <= 4) return launchRenderMode<MODE, 4, TILE>(a, s);
    if (a.sortWindow <= 16) return launchRenderMode<MODE, 16, TILE>(a, s);
    return launchRenderMode<MODE, 64, TILE>(a, s);
}
template <int MODE>
cudaError_t launchRenderTile(const RenderArgs& a, cudaStream_t s) {
    if (a.tileSize == 8) return launchRenderWindow<MODE, 8>(a, s);
    if (a.tileSize == 32) return launchRenderWindow<MODE, 32>(a, s);
    return launchRenderWindow<MODE, 16>(a, s);
}

}  // namespace

cudaError_t launchRender(const RenderArgs& a, cudaStream_t s) {
    if (a.totalTiles == 0) return cudaSuccess;
    if (a.renderSplat == kRenderSplatP32) return launchRenderTile<kRenderSplatP32>(a, s);
    if (a.renderSplat == kRenderSplatP24) return launchRenderTile<kRenderSplatP24>(a, s);
    return launchRenderTile<kRenderSplatFull>(a, s);
}

}  // namespace gsr
