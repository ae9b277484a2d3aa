// The front of the splat-tiles frame, the reference's passes 0-7 (splat_tile_renderer.cpp:653-739):
//
//   frameBegin   reset of the control block and the tile ranges
//   preprocess   per gaussian: scene decode, near/opacity culls, cov3D, EWA cov2D, conic/radius,
//                pixel centre, 16-px rectangle, SH colour, tight tile count (streaming, no waits)
//   scan         exclusive prefix of the counts in index order (GpuScan, k_sort.cu) = the list
//                offsets, whose last block clamps the list to the capacity (tile_setup)
//   duplicate    per gaussian: one (tile << 32 | depth bits, index) entry per covered tile
//
// The placement comes from the scan in index order (INRIA's scheme), so the unsorted list equals
// the reference's entry for entry; atomics are used only for counters. Built with -fmad=false:
// see splat_math.cuh.
#include <cuda_fp16.h>

#include "kernels.cuh"
#include "mlp.cuh"
#include "splat_math.cuh"
#include "tcgen05.cuh"

namespace gsr {

namespace {

constexpr int kFrontThreads = 256;

__device__ __forceinline__ float halfLo(uint32_t w) { return __half2float(__ushort_as_half(uint16_t(w & 0xFFFFu))); }
__device__ __forceinline__ float halfHi(uint32_t w) { return __half2float(__ushort_as_half(uint16_t(w >> 16))); }
__device__ __forceinline__ uint32_t word(const uint4& v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }

// ---- scene decode (shaders/scene_decode.glsl; CPU twin decodeGaussian,
//      src/scene/scene_compression.cpp:382-460) ------------------------------------------
template <int GEOM>
__device__ __forceinline__ float4 loadPosAlpha(const SceneArgs& s, uint32_t i) {
    if (GEOM == GSR_GEOMETRY_SOA_F32) {
        const uint4 w = __ldg(&s.b0[i]);
        return make_float4(__uint_as_float(w.x), __uint_as_float(w.y), __uint_as_float(w.z), __uint_as_float(w.w));
    }
    const uint4 w = __ldg(&s.b0[size_t(i) * s.geometryStride]);
    if (GEOM == GSR_GEOMETRY_RECORD_F32)
        return make_float4(__uint_as_float(w.x), __uint_as_float(w.y), __uint_as_float(w.z), __uint_as_float(w.w));
    return make_float4(__uint_as_float(w.x), __uint_as_float(w.y), __uint_as_float(w.z), halfLo(w.w));
}

template <int GEOM>
__device__ __forceinline__ void loadShape(const SceneArgs& s, uint32_t i, float sigma[3], float q[4], uint32_t& meta) {
    if (GEOM == GSR_GEOMETRY_SOA_F32) {
        const uint4 sc = __ldg(&s.b1[i]);
        const uint4 ro = __ldg(&s.b2[i]);
        sigma[0] = __uint_as_float(sc.x); sigma[1] = __uint_as_float(sc.y); sigma[2] = __uint_as_float(sc.z);
        meta = sc.w;
        q[0] = __uint_as_float(ro.x); q[1] = __uint_as_float(ro.y); q[2] = __uint_as_float(ro.z); q[3] = __uint_as_float(ro.w);
    } else if (GEOM == GSR_GEOMETRY_RECORD_F32) {
        const size_t base = size_t(i) * s.geometryStride;
        const uint4 g1 = __ldg(&s.b0[base + 1]);
        const uint4 g2 = __ldg(&s.b0[base + 2]);
        sigma[0] = __uint_as_float(g1.x); sigma[1] = __uint_as_float(g1.y); sigma[2] = __uint_as_float(g1.z);
        meta = g1.w;
        q[0] = __uint_as_float(g2.x); q[1] = __uint_as_float(g2.y); q[2] = __uint_as_float(g2.z); q[3] = __uint_as_float(g2.w);
    } else {  // G16: word 3 = h(alpha, sx), 4 = h(sy, sz), 5 = h(qw, qx), 6 = h(qy, qz), 7 = meta
        const size_t base = size_t(i) * s.geometryStride;
        const uint32_t w3 = __ldg(&s.b0[base].w);
        const uint4 b = __ldg(&s.b0[base + 1]);
        sigma[0] = halfHi(w3); sigma[1] = halfLo(b.x); sigma[2] = halfHi(b.x);
        const float r0 = halfLo(b.y), r1 = halfHi(b.y), r2 = halfLo(b.z), r3 = halfHi(b.z);
        // decodeGaussian: q * (1 / sqrt(len2)), identity for a zero quaternion
        const float len2 = r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3;
        if (len2 > 0.0f) {
            const float inv = 1.0f / sqrtf(len2);
            q[0] = r0 * inv; q[1] = r1 * inv; q[2] = r2 * inv; q[3] = r3 * inv;
        } else {
            q[0] = 1.0f; q[1] = 0.0f; q[2] = 0.0f; q[3] = 0.0f;
        }
        meta = b.w;
    }
}

// The first `used` SH triplets of gaussian i into sh[k*3 + c] (loadSH, scene_decode.glsl:107-190).
template <int COLOR>
__device__ __forceinline__ void loadSH(const SceneArgs& s, uint32_t i, uint32_t used, uint32_t meta, float sh[48]) {
    const uint32_t K = s.storedCoeffs;
    if (COLOR == GSR_COLOR_SOA_F32) {
        if (K == 16 && s.variableSh == GSR_VARIABLE_SH_OFF) {
            const float4* p = reinterpret_cast<const float4*>(s.shSoa) + size_t(i) * 12;
#pragma unroll
            for (int v = 0; v < 12; ++v) {
                if (uint32_t(v) * 4 < used * 3) {
                    const float4 f = __ldg(&p[v]);
                    sh[v * 4 + 0] = f.x; sh[v * 4 + 1] = f.y; sh[v * 4 + 2] = f.z; sh[v * 4 + 3] = f.w;
                }
            }
            return;
        }
        const size_t base = s.variableSh == GSR_VARIABLE_SH_COMPACT ? size_t(meta & 0x3FFFFFFFu) : size_t(i) * K * 3;
#pragma unroll
        for (int k = 0; k < 48; ++k)
            if (uint32_t(k) < used * 3) sh[k] = __ldg(&s.shSoa[base + k]);
        return;
    }
    const size_t base = s.variableSh == GSR_VARIABLE_SH_COMPACT ? size_t(meta & 0x3FFFFFFFu)
                                                                : size_t(i) * s.colorStride + s.colorOffset;
    if (COLOR == GSR_COLOR_RECORD_F32) {
#pragma unroll
        for (int v = 0; v < 12; ++v) {
            if (uint32_t(v) * 4 < K * 3 && uint32_t(v) * 4 < used * 3) {
                const uint4 w = __ldg(&s.b1[base + v]);
                sh[v * 4 + 0] = __uint_as_float(w.x); sh[v * 4 + 1] = __uint_as_float(w.y);
                sh[v * 4 + 2] = __uint_as_float(w.z); sh[v * 4 + 3] = __uint_as_float(w.w);
            }
        }
    } else if (COLOR == GSR_COLOR_RECORD_F16) {
#pragma unroll
        for (int v = 0; v < 6; ++v) {
            if (uint32_t(v) * 8 < K * 3 && uint32_t(v) * 8 < used * 3) {
                const uint4 w = __ldg(&s.b1[base + v]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    sh[v * 8 + 2 * j] = halfLo(word(w, j));
                    sh[v * 8 + 2 * j + 1] = halfHi(word(w, j));
                }
            }
        }
    } else if (COLOR == GSR_COLOR_CODEBOOK) {
        // CB record (h(dc.r, dc.g), h(dc.b) | index << 16), two per 16 bytes when the colour stride
        // is 0 (split); the rest from codebook entry `index`, fp32 (scene_decode.glsl:96-103, 177-188)
        uint2 r;
        if (s.colorStride == 0) {
            const uint4 v = __ldg(&s.b1[i >> 1]);
            r = (i & 1u) ? make_uint2(v.z, v.w) : make_uint2(v.x, v.y);
        } else {
            const uint4 v = __ldg(&s.b1[size_t(i) * s.colorStride + s.colorOffset]);
            r = make_uint2(v.x, v.y);
        }
        sh[0] = halfLo(r.x);
        sh[1] = halfHi(r.x);
        sh[2] = halfLo(r.y);
        if (used > 1 && K > 1) {
            const size_t entry = size_t(min(r.y >> 16, s.codebookLast)) * s.codebookStride;
#pragma unroll
            for (int v = 0; v < 12; ++v) {
                if (uint32_t(v) * 4 < (K - 1) * 3 && uint32_t(v) * 4 < (used - 1) * 3) {
                    const uint4 w = __ldg(&s.b2[entry + v]);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int k = 3 + v * 4 + j;  // rest word v*4+j -> sh[3 + v*4 + j]
                        if (k < 48) sh[k] = __uint_as_float(word(w, j));
                    }
                }
            }
        }
    } else {  // Q8: w0 = h(dc.r, dc.g), w1 = h(dc.b, s1), w2 = h(s2, s3), int8 rest from byte 12
        uint4 w[4];
#pragma unroll
        for (int v = 0; v < 4; ++v)
            w[v] = (uint32_t(v) * 16 < 12 + (K - 1) * 3 && uint32_t(v) * 16 < 12 + (used - 1) * 3) ? __ldg(&s.b1[base + v])
                                                                                                    : make_uint4(0, 0, 0, 0);
        sh[0] = halfLo(w[0].x); sh[1] = halfHi(w[0].x); sh[2] = halfLo(w[0].y);
        const float scale1 = halfHi(w[0].y), scale2 = halfLo(w[0].z), scale3 = halfHi(w[0].z);
#pragma unroll
        for (int k = 1; k < 16; ++k) {
            if (uint32_t(k) >= used) continue;
            const float sc = k < 4 ? scale1 : (k < 9 ? scale2 : scale3);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                const int j = (k - 1) * 3 + ch;
                const uint32_t wd = word(w[(3 + j / 4) >> 2], (3 + j / 4) & 3);
                const int q = int(int8_t(uint8_t(wd >> (8 * (j % 4)))));
                sh[k * 3 + ch] = float(q) * sc;
            }
        }
    }
}

__device__ __forceinline__ uint32_t gaussianDegree(const SceneArgs& s, uint32_t meta) {
    return s.variableSh == GSR_VARIABLE_SH_OFF ? 3u : (meta >> 30);
}

// normalize(mean - camera position), glm::normalize's order (the SH colour's direction and the
// learned colour's direction input).
__device__ __forceinline__ void viewDirection(const float4& pa, const float (&camPos)[3], float (&dir)[3]) {
    const float d0 = pa.x - camPos[0], d1 = pa.y - camPos[1], d2 = pa.z - camPos[2];
    const float inv = 1.0f / sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
    dir[0] = d0 * inv;
    dir[1] = d1 * inv;
    dir[2] = d2 * inv;
}

// What the colour of a visible gaussian needs once its geometry is done.
struct ColourJob {
    uint32_t meta, degree;
    float dir[3];  // normalize(mean - camera position), glm::normalize's order
};

// Staged SH (soa scenes with 16 stored coefficients and no per-gaussian degree): at block start
// one thread copies the block's 256 x 192 bytes of SH into shared memory with one bulk copy
// (cp.async.bulk, completed on an mbarrier), so the coefficients arrive while the geometry is
// computed and the colour reads them from shared memory. Every wait is bounded: on expiry the
// frame records GSR_CONTROL_TIMEOUT (kWaitShStage) and the thread reads global memory instead.
__shared__ alignas(8) uint64_t gShBarrier;
extern __shared__ float4 gShStage[];  // [kFrontThreads * 12]

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool shStageReady() {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(smemAddr(&gShBarrier)) : "memory");
    return done != 0;
}

// honorForce: the test hook (DeviceControl::forceTimeout) makes the wait see no completion for
// that many spins and give up; the wait before the block exits ignores it.
__device__ __forceinline__ bool waitShStage(DeviceControl* ctl, bool honorForce) {
    const uint32_t forced = honorForce ? ctl->forceTimeout : 0u;
    for (uint32_t spins = 0; spins < kSpinLimit; ++spins) {
        if (forced) {
            if (spins >= forced) break;
            continue;
        }
        if (shStageReady()) return true;
    }
    reportTimeout(ctl, kWaitShStage);
    return false;
}

// Thread 0, after the barrier's init is visible: the block's SH range [i0, i0 + n).
__device__ __forceinline__ void issueShStage(const SceneArgs& s, uint32_t i0, uint32_t n) {
    const uint32_t bytes = n * 192u;
    const float* src = s.shSoa + size_t(i0) * 48;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smemAddr(&gShBarrier)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smemAddr(gShStage)), "l"(src), "r"(bytes), "r"(smemAddr(&gShBarrier)) : "memory");
}

// The plain colour: the gaussian's SH coefficients, evaluated in the view direction.
template <int COLOR>
__device__ __forceinline__ void shColour(const FrontArgs& a, uint32_t i, const ColourJob& job, DevSplat& s) {
    float color[3];
    if (COLOR == GSR_COLOR_SOA_F32 && a.shStaged && waitShStage(a.ctl, true)) {
        // straight from the staged copy: the coefficients are read as the bands need them, with
        // no 48-register array (evalSH reads the first (degree + 1)^2 triplets)
        evalSH(int(job.degree), reinterpret_cast<const float*>(gShStage + threadIdx.x * 12), job.dir[0], job.dir[1],
               job.dir[2], color);
    } else {
        float sh[48];
        loadSH<COLOR>(a.scene, i, (job.degree + 1) * (job.degree + 1), job.meta, sh);
        evalSH(int(job.degree), sh, job.dir[0], job.dir[1], job.dir[2], color);
    }
    s.r = color[0];
    s.g = color[1];
    s.b = color[2];
}

// preprocessGaussian (splat_math.cpp:153-193) with the GPU culls of splat_preprocess.comp.
// LEARNED: the colour of a visible gaussian is left to the caller (job), which decodes it with
// the colour model or falls back to shColour.
template <int GEOM, int COLOR, bool LEARNED>
__device__ __forceinline__ uint32_t preprocessOne(const FrontArgs& a, const DevCamera& cam, uint32_t i, DevSplat& s,
                                                  TileRect& rect, ColourJob& job, float4* ray) {
    const float4 pa = loadPosAlpha<GEOM>(a.scene, i);
    const float* v = cam.v;
    const float t[3] = {v[0] * pa.x + v[4] * pa.y + v[8] * pa.z + v[12], v[1] * pa.x + v[5] * pa.y + v[9] * pa.z + v[13],
                        v[2] * pa.x + v[6] * pa.y + v[10] * pa.z + v[14]};
    s.depth = t[2];
    if (!(t[2] > kNearCullDepth)) return kCullNear;
    if (pa.w < GSR_MIN_ALPHA) return kCullLowOpacity;
    float sigma[3], q[4];
    uint32_t meta = 0;
    loadShape<GEOM>(a.scene, i, sigma, q, meta);
    float S[9], cov[3], conic[3], radius = 0.0f;
    cov3d(sigma[0], sigma[1], sigma[2], q[0], q[1], q[2], q[3], S);
    cov2d(t, S, cam, cov);
    if (!conicAndRadius(cov, conic, radius)) return kCullSingular;
    const float ndcX = t[0] / (t[2] * cam.tanHalfFovX);
    const float ndcY = t[1] / (t[2] * cam.tanHalfFovY);
    const float cx = ((ndcX + 1.0f) * float(cam.width) - 1.0f) * 0.5f;
    const float cy = ((ndcY + 1.0f) * float(cam.height) - 1.0f) * 0.5f;
    rect = tileRect(cx, cy, radius, cam.tilesX, cam.tilesY);
    s.cx = cx;
    s.cy = cy;
    if (rect.maxX <= rect.minX || rect.maxY <= rect.minY) return kCullOffScreen;
    const uint32_t gdeg = gaussianDegree(a.scene, meta);
    job.meta = meta;
    job.degree = uint32_t(a.evalDegree) < gdeg ? uint32_t(a.evalDegree) : gdeg;
    viewDirection(pa, cam.pos, job.dir);
    if (!LEARNED) shColour<COLOR>(a, i, job, s);
    s.conicA = conic[0];
    s.conicB = conic[1];
    s.conicC = conic[2];
    s.opacity = pa.w;
    s.radius = radius;
    if (ray) {  // StopThePop: the ray-depth parameters of the visible gaussian
        float4 rp[3];
        rayDepthParams(sigma, q, t, cam, rp);
        ray[0] = rp[0];
        ray[1] = rp[1];
        ray[2] = rp[2];
    }
    return kCullVisible;
}

// The learned colour of the warp's visible gaussians (every lane calls it): the MLP decode on
// the tensor cores for gaussians with a kept latent, the SH colour for the others.
struct LearnedShared {
    DecoderWeights w;
    __nv_bfloat16 stage[kFrontThreads / 32][32][16];
    float out4[kFrontThreads / 32][32][4];
};
template <int COLOR>
__device__ __forceinline__ void learnedColour(const FrontArgs& a, LearnedShared& sl, uint32_t i, size_t rec,
                                              bool visible, const ColourJob& job, DevSplat& s) {
    if (a.decoded) {  // decoded by the tensor-core pre-pass
        if (visible) {
            if (!latentIsFallback(__ldg(&a.latents[i]))) {
                const float4 c = __ldg(&a.decoded[rec]);
                s.r = c.x;
                s.g = c.y;
                s.b = c.z;
            } else {
                shColour<COLOR>(a, i, job, s);
            }
        }
        return;
    }
    bool mlp = false;
    float feat[kMlpIn];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) feat[k] = 0.0f;
    if (visible) {
        const uint4 q = __ldg(&a.latents[i]);
        mlp = !latentIsFallback(q);
        const uint32_t qw[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < kMlpLatent; ++k) feat[k] = __half2float(__ushort_as_half(uint16_t(qw[k >> 1] >> (16 * (k & 1)))));
#pragma unroll
        for (int c = 0; c < 3; ++c) feat[kMlpLatent + c] = job.dir[c];
    }
    if (__any_sync(0xFFFFFFFFu, mlp)) {
        const uint32_t warp = threadIdx.x >> 5;
        float rgb[3];
        mlpDecodeWarp(sl.w, feat, sl.stage[warp], sl.out4[warp], rgb);
        if (mlp) {
            s.r = rgb[0];
            s.g = rgb[1];
            s.b = rgb[2];
        }
    }
    if (visible && !mlp) shColour<COLOR>(a, i, job, s);
}

// Decoded SH coefficients [N][48] (zeros past each gaussian's evaluated degree) and degrees,
// for training the colour model from any scene format.
template <int GEOM, int COLOR>
__global__ void __launch_bounds__(kFrontThreads) shDecodeKernel(const __grid_constant__ SceneArgs scene, uint32_t count,
                                                                int evalDegree, float* __restrict__ out,
                                                                uint8_t* __restrict__ degrees) {
    const uint32_t i = blockIdx.x * kFrontThreads + threadIdx.x;
    if (i >= count) return;
    float sigma[3], q[4];
    uint32_t meta = 0;
    loadShape<GEOM>(scene, i, sigma, q, meta);
    const uint32_t gdeg = gaussianDegree(scene, meta);
    const uint32_t degree = uint32_t(evalDegree) < gdeg ? uint32_t(evalDegree) : gdeg;
    float sh[48];
#pragma unroll
    for (int k = 0; k < 48; ++k) sh[k] = 0.0f;
    loadSH<COLOR>(scene, i, (degree + 1) * (degree + 1), meta, sh);
#pragma unroll
    for (int k = 0; k < 48; ++k) out[size_t(i) * 48 + k] = uint32_t(k) < (degree + 1) * (degree + 1) * 3 ? sh[k] : 0.0f;
    degrees[i] = uint8_t(degree);
}

// 1) Preprocess + tight count, one thread per (view, gaussian) (splat_preprocess.comp:283-318,
//    GSR_TILES); grid.y = view. Writes the splat record of visible gaussians and every gaussian's
//    tile count; cull counters with one ballot per warp and one atomic per block and reason. No
//    waits: a streaming kernel.
// writeRenderSplat (splat_preprocess.comp:74-91), packed forms: the record, the packed tile
// rectangle and the depth bits, each in its own array.
__device__ __forceinline__ void writePackedSplat(const FrontArgs& a, size_t rec, const DevSplat& s, const TileRect& rect,
                                                 uint32_t p24w0, uint32_t p24w1) {
    const uint32_t cr = packColorRadius(s.b, s.radius);
    if (a.renderSplat == kRenderSplatP32) {
        uint4* p = reinterpret_cast<uint4*>(a.packed) + rec * 2;
        p[0] = make_uint4(__float_as_uint(s.cx), __float_as_uint(s.cy), __float_as_uint(s.conicA), __float_as_uint(s.conicB));
        p[1] = make_uint4(__float_as_uint(s.conicC), __float_as_uint(s.opacity), packHalf2(s.r, s.g), cr);
    } else {
        uint2* p = reinterpret_cast<uint2*>(a.packed) + rec * 3;
        p[0] = make_uint2(__float_as_uint(s.cx), __float_as_uint(s.cy));
        p[1] = make_uint2(p24w0, p24w1);
        p[2] = make_uint2(packHalf2(s.r, s.g), cr);
    }
    a.rects[rec] = packRect(rect);
    a.depths[rec] = __float_as_uint(s.depth);
}

// EXTRAS: the optional outputs, told apart at run time: packed render records (p32 / p24) instead
// of the 48-byte record, and the StopThePop ray-depth parameters. A compile-time switch, so that
// the default kernel carries none of their code.
template <int GEOM, int COLOR, bool LEARNED, bool EXTRAS>
__global__ void __launch_bounds__(kFrontThreads, 4) preprocessKernel(const __grid_constant__ FrontArgs a) {
    __shared__ DevCamera sCam;  // the view's camera, read once per block from its device copy
    __shared__ uint32_t sCull[kCullReasonCount];
    __shared__ uint32_t sDepthMin, sDepthMax;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    // the views vary fastest along the grid: the blocks of one gaussian range for every view run
    // side by side, so one of them reads the range's scene data from DRAM and the others from L2
    const uint32_t view = blockIdx.x % a.viewCount, i0 = blockIdx.x / a.viewCount * kFrontThreads;
    if (tid < kCullReasonCount) sCull[tid] = 0;
    if (tid == 0) {
        sDepthMin = 0xFFFFFFFFu;
        sDepthMax = 0;
    }
    static_assert(sizeof(DevCamera) == sizeof(DevCameraArgs) && sizeof(DevCamera) % 4 == 0, "camera layout");
    if (tid < sizeof(DevCamera) / 4)
        reinterpret_cast<uint32_t*>(&sCam)[tid] = reinterpret_cast<const uint32_t*>(a.cam + view)[tid];
    const bool staged = COLOR == GSR_COLOR_SOA_F32 && a.shStaged;
    if (staged && tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smemAddr(&gShBarrier)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issueShStage(a.scene, i0, a.count - i0 < kFrontThreads ? a.count - i0 : kFrontThreads);
    }
    LearnedShared* sl = nullptr;
    if constexpr (LEARNED) {
        __shared__ LearnedShared sLearned;
        static_assert(sizeof(DecoderWeights) % 4 == 0, "decoder layout");
        if (!a.decoded)
            for (uint32_t e = tid; e < sizeof(DecoderWeights) / 4; e += kFrontThreads)
                reinterpret_cast<uint32_t*>(&sLearned.w)[e] = reinterpret_cast<const uint32_t*>(a.decoder)[e];
        sl = &sLearned;
    }
    __syncthreads();
    const uint32_t i = i0 + tid;
    const size_t rec = size_t(view) * a.count + i;
    // the binning grid: ceil(size / bin) bins (INRIA's rectangles stay on the 16-px tiles)
    const BinShape bs = binShapeOf(a.binSize);
    const int gx = (int(sCam.width) + bs.sx - 1) >> bs.lx, gy = (int(sCam.height) + bs.sy - 1) >> bs.ly;
    uint32_t reason = kCullReasonCount;  // threads past the end
    uint32_t dmin = 0xFFFFFFFFu, dmax = 0;
    DevSplat s;
    TileRect rect{0, 0, 0, 0};
    ColourJob job{};
    if (i < a.count)
        reason = preprocessOne<GEOM, COLOR, LEARNED>(a, sCam, i, s, rect, job,
                                                     EXTRAS && a.rayDepth ? a.rayDepth + rec * 3 : nullptr);
    if constexpr (LEARNED) learnedColour<COLOR>(a, *sl, i, rec, reason == kCullVisible, job, s);  // warp-collective
    if (i < a.count) {
        uint32_t count = 0;
        if (reason == kCullVisible) {
            // the conic and opacity as the emission and the rasterizer will read them: p24 keeps
            // them in fp16, so its tiles are counted with the decoded values
            float cA = s.conicA, cB = s.conicB, cC = s.conicC, cO = s.opacity;
            uint32_t p24w0 = 0, p24w1 = 0;
            if (EXTRAS && a.renderSplat == kRenderSplatP24) {
                p24ConicWords(cA, cB, cC, cO, p24w0, p24w1);
                p24DecodeConic(p24w0, p24w1, cA, cB, cC, cO);
            }
            const Coverage cv = makeCoverage(a.bounds, rect, bs, gx, gy, s.cx, s.cy, cA, cB, cC, cO, a.logf);
            const RowGeom g = rowGeom(cv);
            if (a.bounds != kBoundsRect) {
                uint32_t* hintWords = reinterpret_cast<uint32_t*>(a.hints + rec);
                int r0, rows;
                bool spanForm;
                count = coverageCountSpans(cv, g, bs, gx, hintWords, reinterpret_cast<uint32_t*>(a.spanRows + rec),
                                           r0, rows, spanForm);
                if (spanForm) {
                    hintWords[0] = kSpanMarker | uint32_t(r0) | (uint32_t(rows) << 16);
                } else {
                    a.hints[rec] = coverageHint(cv, g);
                }
            } else {
                count = coverageCount(cv, g, bs);
            }
            s.cullReason = kCullVisible;
            if (!EXTRAS || a.renderSplat == kRenderSplatFull) reinterpret_cast<DevSplat*>(a.splats)[rec] = s;
            else writePackedSplat(a, rec, s, rect, p24w0, p24w1);
            dmin = dmax = __float_as_uint(s.depth);  // positive: the bits order like the values
        }
        a.tileCounts[rec] = count;
        // binning mode: the record's depth word, depth bits above the record index (positive
        // floats: the bits order like the depths); records that emit no tile get all-ones depth
        // bits (the sort places them anywhere: they add no entry).
        // Frames of several views put the view above the depth bits: the depth sort then orders
        // by (view, depth, record), so the emission walks one view's records at a time (each
        // tile's entries come from one view, so the list is the same)
        if (a.binning)
            a.depthKeys[0][rec] = (a.depthViewShift ? uint64_t(view) << a.depthViewShift : 0ull) |
                                  (uint64_t(count ? __float_as_uint(s.depth) : 0xFFFFFFFFu) << a.recordBits) | rec;
    }
#pragma unroll
    for (uint32_t r = 0; r < kCullReasonCount; ++r) {
        const uint32_t n = __popc(__ballot_sync(0xFFFFFFFFu, reason == r));
        if (lane == 0 && n) atomicAdd(&sCull[r], n);
    }
    // the visible depth range (the list keys' depths lie in it): one atomic pair per block
    dmin = __reduce_min_sync(0xFFFFFFFFu, dmin);
    dmax = __reduce_max_sync(0xFFFFFFFFu, dmax);
    if (lane == 0 && dmin <= dmax) {
        atomicMin(&sDepthMin, dmin);
        atomicMax(&sDepthMax, dmax);
    }
    __syncthreads();
    // the bulk copy must have landed before the block's shared memory is released; if this
    // bounded wait expires the copy may still be writing after the block ends, so the frame is
    // marked GSR_CONTROL_TIMEOUT (its records untrusted; the host reports a failed frame)
    if (staged && tid == 0 && !shStageReady()) waitShStage(a.ctl, false);
    if (tid < kCullReasonCount && sCull[tid]) atomicAdd(&a.ctl->c.cull_counts[tid], sCull[tid]);
    if (tid == 0 && sDepthMin <= sDepthMax) {
        atomicMin(&a.ctl->c.depth_min_bits, sDepthMin);
        atomicMax(&a.ctl->c.depth_max_bits, sDepthMax);
    }
}

// 3) Key emission, one thread per (view, gaussian) in index order (tile_duplicate.comp:177-221,
//    global mode): the splat's tiles row by row at offsets [offset, offset + count), dropped at or
//    past the capacity. The coverage is rebuilt from the splat's record with the same functions
//    and the same inputs as the count, so it enumerates exactly `count` tiles; a disagreement
//    would be counted (coverageMismatch) and padded with the sentinel tile, as the reference
//    does. The key's tile is the view's tile base + the tile in the view, so the list orders by
//    view first and each view's entries form the single-view list.
// BINNING (the reference's default construction, tile_duplicate.comp's binning build): one thread
// per slot j of the records sorted by (depth, record index), emitting the record's tiles at the
// offsets of the scan in that order; the entry carries the tile and the gaussian only, and the
// stable sort by tile that follows leaves each tile's entries in (depth, index) order.
template <bool BINNING>
__global__ void __launch_bounds__(kFrontThreads) duplicateKernel(const __grid_constant__ FrontArgs a) {
    __shared__ uint32_t sTileMax, sMismatch, sAny;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        sTileMax = 0;
        sMismatch = 0;
        sAny = 0;
    }
    __syncthreads();
    uint32_t view, i, count = 0;
    size_t rec, slot;
    if (BINNING) {
        const uint32_t records = a.count * a.viewCount;
        slot = size_t(blockIdx.x) * kFrontThreads + tid;
        const uint64_t* sorted = a.depthKeys[a.depthPlan->sortedBuffer & 1u];
        const uint64_t word = slot < records ? sorted[slot] : 0ull;
        rec = uint32_t(word & ((1ull << a.recordBits) - 1ull));
        view = a.depthViewShift ? uint32_t(word >> a.depthViewShift) : uint32_t(rec) / a.count;
        i = uint32_t(rec - size_t(view) * a.count);
        count = slot < records && view < a.viewCount ? a.tileCounts[rec] : 0u;
    } else {
        view = blockIdx.y;
        i = blockIdx.x * kFrontThreads + tid;
        rec = size_t(view) * a.count + i;
        slot = rec;
        count = i < a.count ? a.tileCounts[rec] : 0u;
    }
    // (staging a warp's entries in shared memory for one coalesced write-out of its range
    // measured slower: 0.494 against 0.424 ms for scan + emission of an 8-view 1080p frame)
    auto putKey = [&](uint32_t k, uint64_t key) {
        if (k < a.capacity) a.keys[k] = key;
    };
    if (count > 0) {
        const uint32_t sentinel = a.totalTiles;
        const KeyLayout lay = keyLayout(a.ctl, sentinel, a.count, BINNING);
        const uint32_t offset = a.offsets[slot];
        const DevView vw = a.views[view];
        const int gx = int(vw.tilesX), gy = int(vw.tilesY);  // the view's binning grid
        const float4 hint = a.bounds != kBoundsRect ? a.hints[rec] : make_float4(-2.0f, 0.0f, 0.0f, 0.0f);
        if (isSpanHint(hint)) {
            // the runs the count was made of: no record, no ellipse (binning keys need no depth)
            const uint32_t head = __float_as_uint(hint.x);
            const int r0 = int(head & 0xFFFFu), rows = int((head >> 16) & 0x7u);
            uint32_t span[kSpanRows] = {__float_as_uint(hint.y), __float_as_uint(hint.z), __float_as_uint(hint.w),
                                        0u, 0u, 0u, 0u};
            if (rows > 3) {
                const uint4 more = a.spanRows[rec];
                span[3] = more.x;
                span[4] = more.y;
                span[5] = more.z;
                span[6] = more.w;
            }
            uint64_t depthBits = 0;
            if (!BINNING || !lay.packed)
                depthBits = a.renderSplat == kRenderSplatFull ? __float_as_uint(reinterpret_cast<const DevSplat*>(a.splats)[rec].depth)
                                                              : a.depths[rec];
            const uint64_t packedBase =
                ((lay.lowBits >= 32 ? depthBits : (depthBits & ((1ull << lay.lowBits) - 1ull))) << lay.indexBits) | i;
            const uint32_t tileShift = lay.lowBits + lay.indexBits;
            uint32_t k = offset, written = 0, tileMax = 0;
#pragma unroll
            for (int r = 0; r < kSpanRows; ++r) {
                if (r < rows) {
                    const uint32_t x0 = span[r] & 0xFFFFu, x1 = span[r] >> 16;
                    const uint32_t rowBase = vw.tileBase + uint32_t(r0 + r) * uint32_t(gx);
                    for (uint32_t x = x0; x < x1 && written < count; ++x, ++written, ++k) {
                        const uint32_t tile = rowBase + x;
                        tileMax = tile > tileMax ? tile : tileMax;
                        if (lay.packed) {
                            putKey(k, (uint64_t(tile) << tileShift) | packedBase);
                        } else if (k < a.capacity) {
                            a.keys[k] = (uint64_t(tile) << 32) | depthBits;
                            a.values[k] = i;
                        }
                    }
                }
            }
            if (written != count) {  // the runs hold the count's tiles: never, but treated as below
                atomicAdd(&sMismatch, 1u);
                tileMax = sentinel;
                for (; written < count; ++written, ++k) {
                    if (lay.packed) {
                        putKey(k, (uint64_t(sentinel) << tileShift) | packedBase);
                    } else if (k < a.capacity) {
                        a.keys[k] = (uint64_t(sentinel) << 32) | depthBits;
                        a.values[k] = i;
                    }
                }
            }
            atomicMax(&sTileMax, tileMax);
            sAny = 1;
        } else {
        // centre, conic, rectangle and depth from the record (full) or the packed arrays
        float cx, cy, cA, cB, cC;
        TileRect rect;
        uint64_t depthBits;
        if (a.renderSplat == kRenderSplatFull) {
            const DevSplat s = reinterpret_cast<const DevSplat*>(a.splats)[rec];
            cx = s.cx;
            cy = s.cy;
            cA = s.conicA;
            cB = s.conicB;
            cC = s.conicC;
            rect = tileRect(s.cx, s.cy, s.radius, (vw.width + 15) / 16, (vw.height + 15) / 16);
            depthBits = __float_as_uint(s.depth);
        } else {
            rect = unpackRect(a.rects[rec]);
            depthBits = a.depths[rec];
            if (a.renderSplat == kRenderSplatP32) {
                const uint4 w = reinterpret_cast<const uint4*>(a.packed)[rec * 2];
                cx = __uint_as_float(w.x);
                cy = __uint_as_float(w.y);
                cA = __uint_as_float(w.z);
                cB = __uint_as_float(w.w);
                cC = __uint_as_float(reinterpret_cast<const uint32_t*>(a.packed)[rec * 8 + 4]);
            } else {
                const uint2 w0 = reinterpret_cast<const uint2*>(a.packed)[rec * 3];
                const uint2 w1 = reinterpret_cast<const uint2*>(a.packed)[rec * 3 + 1];
                cx = __uint_as_float(w0.x);
                cy = __uint_as_float(w0.y);
                float o;
                p24DecodeConic(w1.x, w1.y, cA, cB, cC, o);
            }
        }
        RowGeom g;
        const BinShape S = binShapeOf(a.binSize);
        const Coverage cv = coverageFromHint(a.bounds, rect, S, gx, gy, cx, cy, cA, cB, cC, hint, g);
        // packed: (((tile << W) | depth mod 2^W) << indexBits) | index; the tile part added per entry
        const uint64_t packedBase =
            ((lay.lowBits >= 32 ? depthBits : (depthBits & ((1ull << lay.lowBits) - 1ull))) << lay.indexBits) | i;
        const uint32_t tileShift = lay.lowBits + lay.indexBits;
        auto emit = [&](uint32_t k, uint32_t tile) {
            if (lay.packed) {
                putKey(k, (uint64_t(tile) << tileShift) | packedBase);
            } else if (k < a.capacity) {
                a.keys[k] = (uint64_t(tile) << 32) | depthBits;
                a.values[k] = i;
            }
        };
        int r0, r1;
        coverageRows(cv, S, r0, r1);
        uint32_t written = 0;
        uint32_t k = offset;
        uint32_t tileMax = 0;
        for (int row = r0; row < r1 && written < count; ++row) {
            int x0, x1;
            coverageRowSpan(cv, g, row, S, x0, x1);
            for (int x = x0; x < x1 && written < count; ++x, ++written, ++k) {
                const uint32_t tile = vw.tileBase + uint32_t(row) * uint32_t(gx) + uint32_t(x);
                tileMax = tile > tileMax ? tile : tileMax;
                emit(k, tile);
            }
        }
        if (written != count) {
            atomicAdd(&sMismatch, 1u);
            tileMax = sentinel;
            for (; written < count; ++written, ++k) emit(k, sentinel);
        }
        atomicMax(&sTileMax, tileMax);
        sAny = 1;
        }
    }
    __syncthreads();
    if (tid == 0 && sAny) {
        DeviceControl* ctl = a.ctl;
        atomicMax(&ctl->c.tile_max, sTileMax);
        if (sMismatch) atomicAdd(&ctl->c.coverage_mismatch, sMismatch);
    }
}

// Per-frame reset of the control block (vkCmdUpdateBuffer of TileControl{N, 0, ...}) and of the
// tile ranges (vkCmdFillBuffer 0), splat_tile_renderer.cpp:653-661. Block 0 resets the control
// block and the sort histograms; every block zeroes a part of the ranges and of `clear` (the
// depth sort's per-view digit counts).
__global__ void frameBeginKernel(DeviceControl* ctl, uint32_t count, uint32_t capacity, uint4* ranges,
                                 uint32_t rangeVec4s, SortPlan* plan, uint32_t forceTimeout, SortPlan* plan2,
                                 uint32_t* clear, uint32_t clearCount) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t j = g; j < rangeVec4s; j += gridDim.x * blockDim.x) ranges[j] = make_uint4(0, 0, 0, 0);
    for (uint32_t j = g; j < clearCount; j += gridDim.x * blockDim.x) clear[j] = 0;
    if (blockIdx.x != 0) return;
    SortPlan* plans[2] = {plan, plan2};
    for (int k = 0; k < 2; ++k) {
        if (!plans[k]) continue;
        uint32_t* h = &plans[k]->hist[0][0];
        for (uint32_t j = threadIdx.x; j < kMaxSortPasses * kMaxSortBins; j += blockDim.x) h[j] = 0;
    }
    if (threadIdx.x == 0) {
        GsrControl& c = ctl->c;
        const uint32_t epoch = ((c.epoch + 1u) & 0x3FFFFFFFu) ? ((c.epoch + 1u) & 0x3FFFFFFFu) : 1u;
        c.gaussian_count = count;
        c.visible = 0;
        c.duplicates = 0;
        c.entries = 0;
        for (int r = 0; r < 8; ++r) c.cull_counts[r] = 0;
        c.overflow = 0;
        c.ranges_groups[0] = 0;
        c.ranges_groups[1] = 1;
        c.ranges_groups[2] = 1;
        c.coverage_mismatch = 0;
        c.status = 0;
        c.timeout_where = 0;
        c.epoch = epoch;
        c.sort_passes = 0;
        c.key_bits = 0;
        c.depth_low_bits = 0;
        c.depth_min_bits = 0xFFFFFFFFu;
        c.depth_max_bits = 0;
        c.tile_max = 0;
        c.sorted_buffer = 0;
        c.capacity = capacity;
        for (int t = 0; t < kControlTickets; ++t) ctl->tickets[t] = 0;
        ctl->histDone[0] = 0;
        ctl->histDone[1] = 0;
        ctl->forceTimeout = forceTimeout;
    }
}

__global__ void logfTableKernel(float* out, LogfFixups t) {
    const uint32_t n = t.last - t.base + 1;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        out[j] = libcLogf(__uint_as_float(t.base + j), t);
}

}  // namespace

cudaError_t loadFrameBeginKernel() {
    cudaFuncAttributes attr;
    return cudaFuncGetAttributes(&attr, frameBeginKernel);
}

cudaError_t launchFrameBegin(DeviceControl* ctl, uint32_t count, uint32_t capacity, uint32_t* ranges,
                             uint32_t rangeWords, SortPlan* plan, uint32_t forceTimeout, cudaStream_t s,
                             SortPlan* plan2, uint32_t* clearWords, uint32_t clearCount) {
    const uint32_t vec4s = (rangeWords + 3) / 4;
    const uint32_t work = vec4s > clearCount ? vec4s : clearCount;
    uint32_t blocks = (work + 255) / 256;
    blocks = blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks);
    frameBeginKernel<<<blocks, 256, 0, s>>>(ctl, count, capacity, reinterpret_cast<uint4*>(ranges), vec4s, plan,
                                             forceTimeout, plan2, clearWords, clearWords ? clearCount : 0u);
    return cudaGetLastError();
}

// ---- the learned colour's decode on the tcgen05 tensor cores (GSR_DECODE_TCGEN05) ----------------
// A pre-pass before the preprocess. Persistent 128-thread blocks take 128-gaussian tiles of one
// view at a time (the views of one gaussian range side by side, so the latents and positions are
// read from DRAM once). Thread t builds row t of the decoder input (the fp16 latent and the view
// direction as BF16, zero-padded to K = 16) in shared memory; one thread issues each layer as
// tcgen05.mma products of M = 128 rows (the tile's gaussians) with FP32 accumulators in tensor
// memory: 16 -> 32 (1 MMA), 32 -> 32 (2 MMAs of K = 16), 32 -> 16 (2 MMAs; 3 outputs used),
// each completion signalled through tcgen05.commit on an mbarrier. After each layer every warp
// reads its 32 rows back (tcgen05.ld, thread t = row t = TMEM lane t), adds the bias and applies
// ReLU (sigmoid at the output), and writes the next layer's BF16 operand. The colours of the
// kept gaussians go to decoded[view][g]. The rounding points are the in-preprocess decode's
// (BF16 inputs, weights and hidden units, FP32 accumulation); the bias is added after the
// products instead of seeding the accumulator, so colours can differ in the last bits of FP32.
constexpr uint32_t kDecodeTcThreads = 128, kDecodeTcCols = 64;  // layer 1 and 3 at column 0, layer 2 at 32
struct alignas(128) DecodeTcSmem {
    alignas(128) unsigned char a1[128 * 16 * 2];  // layer inputs, M = 128 rows, K-major no swizzle
    alignas(128) unsigned char a2[128 * 32 * 2];
    alignas(128) unsigned char a3[128 * 32 * 2];
    alignas(128) unsigned char b1[32 * 16 * 2];   // weights [n][k]: N = 32, 32, 16 (rows 3..15 zero)
    alignas(128) unsigned char b2[32 * 32 * 2];
    alignas(128) unsigned char b3[16 * 32 * 2];
    float bias1[32], bias2[32], bias3[4];
    uint64_t mbar;
    uint32_t tmem;
};
// 28 KB a block: at most 8 blocks per SM, so the blocks' TMEM (64 columns each) always fits the
// SM's 512 columns and no allocation waits.
constexpr uint32_t kDecodeTcSmem = 28 * 1024;
static_assert(sizeof(DecodeTcSmem) + 128 <= kDecodeTcSmem, "the decode's shared memory");

// Eight floats as BF16 into one 16-byte row chunk of an operand.
__device__ __forceinline__ void storeRowChunk(unsigned char* base, uint32_t off, const float* v) {
    *reinterpret_cast<uint4*>(base + off) =
        make_uint4(packBf16(v[0], v[1]), packBf16(v[2], v[3]), packBf16(v[4], v[5]), packBf16(v[6], v[7]));
}

template <int GEOM>
__global__ void __launch_bounds__(kDecodeTcThreads) decodeColoursTcKernel(const __grid_constant__ FrontArgs a) {
    extern __shared__ __align__(128) unsigned char decodeRaw[];
    DecodeTcSmem& S = *reinterpret_cast<DecodeTcSmem*>(decodeRaw + ((128u - (tc::smem32(decodeRaw) & 127u)) & 127u));
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const DecoderWeights& W = *a.decoder;
    // the weights in the operand layout, the biases, the barrier and the tensor memory
    if (tid < 64) {
        const uint32_t n = tid >> 1, c = tid & 1;
        *reinterpret_cast<uint4*>(S.b1 + tc::operandOffset(n, 8 * c, 16)) = *reinterpret_cast<const uint4*>(&W.w1[n][8 * c]);
    }
    {
        const uint32_t n = tid >> 2, c = tid & 3;
        *reinterpret_cast<uint4*>(S.b2 + tc::operandOffset(n, 8 * c, 32)) = *reinterpret_cast<const uint4*>(&W.w2[n][8 * c]);
    }
    if (tid < 64) {
        const uint32_t n = tid >> 2, c = tid & 3;
        *reinterpret_cast<uint4*>(S.b3 + tc::operandOffset(n, 8 * c, 32)) =
            n < 8 ? *reinterpret_cast<const uint4*>(&W.w3[n][8 * c]) : make_uint4(0, 0, 0, 0);
    }
    if (tid < 32) {
        S.bias1[tid] = W.b1[tid];
        S.bias2[tid] = W.b2[tid];
    }
    if (tid < 4) S.bias3[tid] = W.b3[tid];
    if (tid == 0) tc::mbarInit(&S.mbar, 1);
    if (warp == 0) tc::tmemAlloc(&S.tmem, kDecodeTcCols);
    tc::fenceProxyAsync();
    tc::fenceBeforeSync();
    __syncthreads();
    tc::fenceAfterSync();
    const uint32_t tmem = S.tmem, lane0 = (warp * 32u) << 16;
    const uint32_t a1 = tc::smem32(S.a1), a2 = tc::smem32(S.a2), a3 = tc::smem32(S.a3);
    const uint32_t b1 = tc::smem32(S.b1), b2 = tc::smem32(S.b2), b3 = tc::smem32(S.b3);
    const uint32_t tiles = (a.count + 127u) / 128u * a.viewCount;
    uint32_t phase = 0;
    bool failed = false;
    // every thread waits for the layer's commit; a wait that runs out stops the whole block
    auto layerDone = [&]() -> bool {
        const bool ok = tc::mbarWait(&S.mbar, phase, kSpinLimit);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = true;
            return false;
        }
        tc::fenceAfterSync();
        return true;
    };
    // the inputs of a tile: its latent and position, loaded one tile ahead (while the current
    // tile's products run)
    auto fetch = [&](uint32_t tile, uint4& q, float4& pa) {
        const uint32_t g = tile / a.viewCount * 128u + tid;
        q = make_uint4(0, 0, 0, 0xFFFFFFFFu);  // a fallback marker: no colour
        pa = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (tile < tiles && g < a.count) {
            q = __ldg(&a.latents[g]);
            if (!latentIsFallback(q)) pa = loadPosAlpha<GEOM>(a.scene, g);
        }
    };
    uint4 qNext;
    float4 paNext;
    fetch(blockIdx.x, qNext, paNext);
    for (uint32_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const uint32_t view = tile % a.viewCount, g = tile / a.viewCount * 128u + tid;
        const uint4 q = qNext;
        const float4 pa = paNext;
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) f[k] = 0.0f;
        const bool kept = g < a.count && !latentIsFallback(q);
        if (kept) {
            const uint32_t qw[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int k = 0; k < kMlpLatent; ++k) f[k] = __half2float(__ushort_as_half(uint16_t(qw[k >> 1] >> (16 * (k & 1)))));
            const float camPos[3] = {a.cam[view].pos[0], a.cam[view].pos[1], a.cam[view].pos[2]};
            float dir[3];
            viewDirection(pa, camPos, dir);
            f[8] = dir[0];
            f[9] = dir[1];
            f[10] = dir[2];
        }
        storeRowChunk(S.a1, tc::operandOffset(tid, 0, 16), f);
        storeRowChunk(S.a1, tc::operandOffset(tid, 8, 16), f + 8);
        tc::fenceProxyAsync();
        tc::fenceBeforeSync();
        __syncthreads();
        if (tid == 0) {
            tc::fenceAfterSync();
            tc::mma(tmem, tc::operandDescriptor(a1, 0, 16), tc::operandDescriptor(b1, 0, 16), tc::instrDescriptorBf16(128, 32),
                    false);
            tc::commit(&S.mbar);
        }
        fetch(tile + gridDim.x, qNext, paNext);
        if (!layerDone()) break;
        uint32_t acc[32];
        tc::ld32(tmem + lane0, acc);
        tc::waitLd();
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) h[e] = fmaxf(__uint_as_float(acc[8 * c + e]) + S.bias1[8 * c + e], 0.0f);
            storeRowChunk(S.a2, tc::operandOffset(tid, 8 * c, 32), h);
        }
        tc::fenceProxyAsync();
        tc::fenceBeforeSync();
        __syncthreads();
        if (tid == 0) {
            tc::fenceAfterSync();
            for (uint32_t ks = 0; ks < 2; ++ks)
                tc::mma(tmem + 32, tc::operandDescriptor(a2, ks, 32), tc::operandDescriptor(b2, ks, 32),
                        tc::instrDescriptorBf16(128, 32), ks > 0);
            tc::commit(&S.mbar);
        }
        if (!layerDone()) break;
        tc::ld32(tmem + lane0 + 32, acc);
        tc::waitLd();
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) h[e] = fmaxf(__uint_as_float(acc[8 * c + e]) + S.bias2[8 * c + e], 0.0f);
            storeRowChunk(S.a3, tc::operandOffset(tid, 8 * c, 32), h);
        }
        tc::fenceProxyAsync();
        tc::fenceBeforeSync();
        __syncthreads();
        if (tid == 0) {
            tc::fenceAfterSync();
            for (uint32_t ks = 0; ks < 2; ++ks)
                tc::mma(tmem, tc::operandDescriptor(a3, ks, 32), tc::operandDescriptor(b3, ks, 32),  // layer 1 read back
                        tc::instrDescriptorBf16(128, 16), ks > 0);
            tc::commit(&S.mbar);
        }
        if (!layerDone()) break;
        uint32_t out[16];
        tc::ld16(tmem + lane0, out);
        tc::waitLd();
        if (kept)
            a.decoded[size_t(view) * a.count + g] =
                make_float4(sigmoidF(__uint_as_float(out[0]) + S.bias3[0]), sigmoidF(__uint_as_float(out[1]) + S.bias3[1]),
                            sigmoidF(__uint_as_float(out[2]) + S.bias3[2]), 0.0f);
        tc::fenceBeforeSync();  // this tile's TMEM reads before the next tile's products
    }
    if (failed && tid == 0) {
        reportTimeout(a.ctl, kWaitDecode);
        tc::mbarWait(&S.mbar, phase ^ 1u, kSpinLimit);  // the products in flight, once more (bounded)
    }
    tc::fenceBeforeSync();
    __syncthreads();
    if (warp == 0) {
        tc::fenceAfterSync();
        tc::tmemFree(tmem, kDecodeTcCols);
    }
}

namespace {
constexpr int kShStageBytes = kFrontThreads * 192;
template <int GEOM, int COLOR, bool LEARNED, bool EXTRAS>
void launchPreprocessT(const FrontArgs& a, dim3 blocks, cudaStream_t s) {
    static std::atomic<bool> configuredOn[64] = {};
    std::atomic<bool>& configured = perDevice(configuredOn);
    if (COLOR == GSR_COLOR_SOA_F32 && !configured) {  // (a failure here fails the staged launch below)
        configured = cudaFuncSetAttribute(preprocessKernel<GEOM, COLOR, LEARNED, EXTRAS>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, kShStageBytes) == cudaSuccess;
    }
    preprocessKernel<GEOM, COLOR, LEARNED, EXTRAS><<<blocks, kFrontThreads, a.shStaged ? kShStageBytes : 0, s>>>(a);
}
template <int GEOM, int COLOR>
void launchPreprocess(const FrontArgs& a, dim3 blocks, cudaStream_t s) {
    const bool extras = a.renderSplat != kRenderSplatFull || a.rayDepth != nullptr;
    FrontArgs b = a;
    // staging: soa with 16 stored coefficients and no per-gaussian degree (192 bytes a gaussian,
    // so every block's range starts on a 16-byte boundary); not with the learned colour, which
    // reads SH only for its fallback gaussians
    b.shStaged = COLOR == GSR_COLOR_SOA_F32 && !a.latents && a.scene.storedCoeffs == 16 &&
                 a.scene.variableSh == GSR_VARIABLE_SH_OFF && (reinterpret_cast<uintptr_t>(a.scene.shSoa) & 15u) == 0;
    if (a.latents) {
        if (extras) launchPreprocessT<GEOM, COLOR, true, true>(b, blocks, s);
        else launchPreprocessT<GEOM, COLOR, true, false>(b, blocks, s);
    } else {
        if (extras) launchPreprocessT<GEOM, COLOR, false, true>(b, blocks, s);
        else launchPreprocessT<GEOM, COLOR, false, false>(b, blocks, s);
    }
}
template <int GEOM, int COLOR>
void launchShDecodeT(const SceneArgs& scene, uint32_t count, int evalDegree, float* out, uint8_t* degrees, cudaStream_t s) {
    shDecodeKernel<GEOM, COLOR><<<(count + kFrontThreads - 1) / kFrontThreads, kFrontThreads, 0, s>>>(scene, count, evalDegree,
                                                                                                    out, degrees);
}
}  // namespace

cudaError_t launchShDecode(const SceneArgs& scene, uint32_t geometry, uint32_t color, uint32_t count, int evalDegree,
                           float* out, uint8_t* degrees, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    if (geometry == GSR_GEOMETRY_SOA_F32 && color == GSR_COLOR_SOA_F32)
        launchShDecodeT<GSR_GEOMETRY_SOA_F32, GSR_COLOR_SOA_F32>(scene, count, evalDegree, out, degrees, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F32 && color == GSR_COLOR_RECORD_F32)
        launchShDecodeT<GSR_GEOMETRY_RECORD_F32, GSR_COLOR_RECORD_F32>(scene, count, evalDegree, out, degrees, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_RECORD_F16)
        launchShDecodeT<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_RECORD_F16>(scene, count, evalDegree, out, degrees, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_Q8)
        launchShDecodeT<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_Q8>(scene, count, evalDegree, out, degrees, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_CODEBOOK)
        launchShDecodeT<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_CODEBOOK>(scene, count, evalDegree, out, degrees, s);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// The preprocess grid: one block per (gaussian block, view), the view fastest (records = count x
// views fit 32 bits, so the block count stays below 2^24).
static dim3 preprocessGrid(const FrontArgs& a) { return dim3((a.count + kFrontThreads - 1) / kFrontThreads * a.viewCount); }

cudaError_t launchFrontBinningKeys(const FrontArgs& a, uint32_t geometry, uint32_t color, cudaStream_t s) {
    const dim3 blocks = preprocessGrid(a);
    if (blocks.x == 0) return cudaSuccess;
    if (geometry == GSR_GEOMETRY_SOA_F32 && color == GSR_COLOR_SOA_F32)
        launchPreprocess<GSR_GEOMETRY_SOA_F32, GSR_COLOR_SOA_F32>(a, blocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F32 && color == GSR_COLOR_RECORD_F32)
        launchPreprocess<GSR_GEOMETRY_RECORD_F32, GSR_COLOR_RECORD_F32>(a, blocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_RECORD_F16)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_RECORD_F16>(a, blocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_Q8)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_Q8>(a, blocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_CODEBOOK)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_CODEBOOK>(a, blocks, s);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launchFrontBinningEmit(const FrontArgs& a, cudaStream_t s) {
    const uint32_t records = a.count * a.viewCount;
    if (records == 0) return cudaSuccess;
    // the counts in (depth, record) order: the scan gathers them through the sorted depth words;
    // its last block clamps the list to the capacity (tile_setup), in depth order
    const ScanGather gather{{a.depthKeys[0], a.depthKeys[1]}, a.depthPlan, (1ull << a.recordBits) - 1ull};
    cudaError_t e = launchScan(a.tileCounts, nullptr, a.offsets, &a.ctl->c.duplicates, records, kScanGatherSorted,
                               a.scanStatus, a.ctl, s, a.capacity, kWaitScan, &gather);
    if (e != cudaSuccess) return e;
    duplicateKernel<true><<<(records + kFrontThreads - 1) / kFrontThreads, kFrontThreads, 0, s>>>(a);
    return cudaGetLastError();
}

namespace {
template <int GEOM>
cudaError_t launchDecodeTcT(const FrontArgs& a, cudaStream_t s) {
    static std::atomic<int> grids[64] = {};
    std::atomic<int>& grid = perDevice(grids);
    if (!grid) {
        cudaError_t e = cudaFuncSetAttribute(decodeColoursTcKernel<GEOM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(kDecodeTcSmem));
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 148, perSm = 4;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, decodeColoursTcKernel<GEOM>, kDecodeTcThreads, kDecodeTcSmem);
        grid = sms * (perSm > 0 ? (perSm < 8 ? perSm : 8) : 1);
    }
    const uint32_t tiles = (a.count + 127u) / 128u * a.viewCount;
    const uint32_t blocks = tiles < uint32_t(grid) ? tiles : uint32_t(grid);
    decodeColoursTcKernel<GEOM><<<blocks, kDecodeTcThreads, kDecodeTcSmem, s>>>(a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launchDecodeColoursTc(const FrontArgs& a, uint32_t geometry, cudaStream_t s) {
    if (a.count == 0 || a.viewCount == 0 || !a.latents || !a.decoder || !a.decoded) return cudaSuccess;
    if (geometry == GSR_GEOMETRY_SOA_F32) return launchDecodeTcT<GSR_GEOMETRY_SOA_F32>(a, s);
    if (geometry == GSR_GEOMETRY_RECORD_F32) return launchDecodeTcT<GSR_GEOMETRY_RECORD_F32>(a, s);
    if (geometry == GSR_GEOMETRY_RECORD_F16) return launchDecodeTcT<GSR_GEOMETRY_RECORD_F16>(a, s);
    return cudaErrorInvalidValue;
}

cudaError_t launchFront(const FrontArgs& a, uint32_t geometry, uint32_t color, cudaStream_t s) {
    const dim3 blocks((a.count + kFrontThreads - 1) / kFrontThreads, a.viewCount), pblocks = preprocessGrid(a);
    if (blocks.x == 0 || blocks.y == 0) return cudaSuccess;
    // 1) preprocess + count, one block per (gaussian block, view)
    if (geometry == GSR_GEOMETRY_SOA_F32 && color == GSR_COLOR_SOA_F32)
        launchPreprocess<GSR_GEOMETRY_SOA_F32, GSR_COLOR_SOA_F32>(a, pblocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F32 && color == GSR_COLOR_RECORD_F32)
        launchPreprocess<GSR_GEOMETRY_RECORD_F32, GSR_COLOR_RECORD_F32>(a, pblocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_RECORD_F16)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_RECORD_F16>(a, pblocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_Q8)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_Q8>(a, pblocks, s);
    else if (geometry == GSR_GEOMETRY_RECORD_F16 && color == GSR_COLOR_CODEBOOK)
        launchPreprocess<GSR_GEOMETRY_RECORD_F16, GSR_COLOR_CODEBOOK>(a, pblocks, s);
    else
        return cudaErrorInvalidValue;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // 2) exclusive scan of the counts (GpuScan over V * N, view-major), the list size and its
    //    clamp (tile_setup.comp:16-24) by the scan's last block
    e = launchScan(a.tileCounts, nullptr, a.offsets, &a.ctl->c.duplicates, a.count * a.viewCount, GSR_SCAN_PLAIN,
                   a.scanStatus, a.ctl, s, a.capacity, kWaitScan);
    if (e != cudaSuccess) return e;
    // 3) key emission
    duplicateKernel<false><<<blocks, kFrontThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchLogfTable(float* out, LogfFixups t, cudaStream_t s) {
    logfTableKernel<<<148 * 8, 256, 0, s>>>(out, t);
    return cudaGetLastError();
}

}  // namespace gsr
