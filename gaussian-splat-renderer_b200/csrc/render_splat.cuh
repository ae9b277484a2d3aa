// The packed render records of the emission and the rasterizer (shaders/render_splat.glsl; CPU
// twin src/render/render_splat.h). Integer and exact conversions only, so both the bit-exact
// front (built with -fmad=false) and the rasterizer include it.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

namespace gsr {

// ---- packed render records (shaders/render_splat.glsl; CPU twin src/render/render_splat.h) ----
// p32, 8 words: cx, cy, a, b | c, opacity, h(r, g), h(b) | radius << 16
// p24, 6 words: cx, cy | h(a S, b S), h(c S, opacity) | h(r, g), h(b) | radius << 16, S = 2^12
// h() is the fp16 bit pattern rounded to nearest even; the conic is scaled by S so that the
// entries of large splats stay in fp16's normal range. Decoding is exact (fp16 -> fp32, then a
// multiply by 2^-12).
constexpr int kRenderSplatFull = 0, kRenderSplatP32 = 1, kRenderSplatP24 = 2;
constexpr float kConicScaleP24 = 4096.0f;

__device__ __forceinline__ uint32_t halfBits(float v) { return uint32_t(__half_as_ushort(__float2half_rn(v))); }
__device__ __forceinline__ uint32_t packHalf2(float lo, float hi) { return halfBits(lo) | (halfBits(hi) << 16); }
__device__ __forceinline__ float halfLoF(uint32_t w) { return __half2float(__ushort_as_half(uint16_t(w & 0xFFFFu))); }
__device__ __forceinline__ float halfHiF(uint32_t w) { return __half2float(__ushort_as_half(uint16_t(w >> 16))); }
// h(b) | radius << 16 with radius clamped as std::min(radius, 65535.0f), then truncated
__device__ __forceinline__ uint32_t packColorRadius(float b, float radius) {
    const float r = (65535.0f < radius) ? 65535.0f : radius;
    return halfBits(b) | (uint32_t(__float2uint_rz(r)) << 16);
}
// p24's conic (a, b, c) and opacity as the passes that read the record see them
__device__ __forceinline__ void p24ConicWords(float a, float b, float c, float o, uint32_t& w0, uint32_t& w1) {
    w0 = packHalf2(a * kConicScaleP24, b * kConicScaleP24);
    w1 = packHalf2(c * kConicScaleP24, o);
}
__device__ __forceinline__ void p24DecodeConic(uint32_t w0, uint32_t w1, float& a, float& b, float& c, float& o) {
    const float inv = 1.0f / kConicScaleP24;
    a = halfLoF(w0) * inv;
    b = halfHiF(w0) * inv;
    c = halfLoF(w1) * inv;
    o = halfHiF(w1);
}

}  // namespace gsr
