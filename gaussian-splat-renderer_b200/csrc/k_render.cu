// The tile rasterizer (INRIA renderCUDA; the reference's shaders/tile_render.comp:281-400 and
// the CPU reference's per-pixel loop, src/splat/reference_renderer.cpp:120-222).
//
// One 256-thread block per 16x16 tile, one thread per pixel. The tile's entries
// [ranges[tile].x, ranges[tile].y) of the sorted list are walked front to back in batches of
// 256: the block gathers the batch's splat records into shared memory (one record per
// thread), then every pixel blends the batch with INRIA's test-before-accept rule:
//   power = -0.5 (A dx^2 + C dy^2) - B dx dy; skip power > 0
//   alpha = min(0.99, o exp(power));          skip alpha < 1/255
//   testT = T (1 - alpha); testT < 1e-4 -> the pixel is done (this splat is not blended)
//   C += colour alpha T; T = testT
// A whole-tile vote (__syncthreads_count) ends the tile once every pixel is done. Expressions
// follow the CPU reference's order (this unit is built without FMA contraction), so the float
// image differs from the CPU's only where CUDA's expf and the C library's expf round apart.
#include "gsr_device.cuh"
#include "kernels.cuh"

namespace gsr {

namespace {

constexpr int kRenderThreads = 256;
constexpr float kMaxAlpha = 0.99f;
constexpr float kMinTransmittance = 1e-4f;

__global__ void __launch_bounds__(kRenderThreads) renderKernel(const __grid_constant__ RenderArgs a) {
    __shared__ float4 sCenter[kRenderThreads];  // cx, cy, depth, cullReason
    __shared__ float4 sConic[kRenderThreads];   // A, B, C, opacity
    __shared__ float4 sColor[kRenderThreads];   // r, g, b, radius
    const uint32_t tile = blockIdx.x;
    const uint32_t tid = threadIdx.x;
    const uint32_t tx = tile % a.tilesX, ty = tile / a.tilesX;
    const uint32_t px = tx * 16 + (tid & 15), py = ty * 16 + (tid >> 4);
    const bool inside = px < a.width && py < a.height;
    uint2 range = reinterpret_cast<const uint2*>(a.ranges)[tile];
    // a frame whose look-back gave up (GSR_CONTROL_TIMEOUT) has meaningless ranges: every index
    // read below stays inside the list and the scene all the same
    const uint32_t entries = a.ctl->c.entries;
    range.y = range.y < entries ? range.y : entries;
    range.x = range.x < range.y ? range.x : range.y;
    const uint32_t* values = a.values[a.ctl->c.sorted_buffer & 1u];
    const float4* records = reinterpret_cast<const float4*>(a.splats);
    const float fx = float(px), fy = float(py);
    float T = 1.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    bool done = !inside;
    for (uint32_t start = range.x; start < range.y; start += kRenderThreads) {
        if (__syncthreads_count(done) == kRenderThreads) break;
        const uint32_t j = start + tid;
        if (j < range.y) {
            uint32_t g = __ldg(&values[j]);
            if (g >= a.count) {
                atomicOr(&a.ctl->c.status, uint32_t(GSR_CONTROL_BOUNDS));
                g = 0;
            }
            sCenter[tid] = __ldg(&records[size_t(g) * 3]);
            sConic[tid] = __ldg(&records[size_t(g) * 3 + 1]);
            sColor[tid] = __ldg(&records[size_t(g) * 3 + 2]);
        }
        __syncthreads();
        const uint32_t n = range.y - start < uint32_t(kRenderThreads) ? range.y - start : uint32_t(kRenderThreads);
        for (uint32_t q = 0; !done && q < n; ++q) {
            const float4 c = sCenter[q];
            const float4 co = sConic[q];
            const float dx = c.x - fx;
            const float dy = c.y - fy;
            const float power = -0.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
            if (power > 0.0f) continue;
            const float alpha = fminf(kMaxAlpha, co.w * expf(power));
            if (alpha < (1.0f / 255.0f)) continue;
            const float testT = T * (1.0f - alpha);
            if (testT < kMinTransmittance) {
                done = true;
                break;
            }
            const float4 col = sColor[q];
            c0 = c0 + col.x * alpha * T;
            c1 = c1 + col.y * alpha * T;
            c2 = c2 + col.z * alpha * T;
            T = testT;
        }
        __syncthreads();
    }
    if (!inside) return;
    const size_t p = size_t(py) * a.width + px;
    a.image[p] = make_float4(c0, c1, c2, 1.0f - T);
    if (a.rgb8) {
        const float v[3] = {c0, c1, c2};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const float cl = v[ch] < 0.0f ? 0.0f : (v[ch] > 1.0f ? 1.0f : v[ch]);
            a.rgb8[p * 3 + ch] = uint8_t(roundf(cl * 255.0f));  // lround(clamp(v, 0, 1) * 255), image_io.cpp:55-56
        }
    }
}

}  // namespace

cudaError_t launchRender(const RenderArgs& a, cudaStream_t s) {
    const uint32_t tiles = a.tilesX * a.tilesY;
    if (tiles == 0) return cudaSuccess;
    renderKernel<<<tiles, kRenderThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace gsr
