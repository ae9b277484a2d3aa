// GPU scene encoder: the reference's encodeScene (src/scene/scene_compression.cpp:150-380) for
// the f32, f16 and q8 formats in the soa, split and aos layouts, with the per-gaussian SH degree
// (selectShDegree, :53-68) and the compacted colour data of the variable-degree layouts. The
// reference runs it on the CPU at load time (GpuScene::upload); here it runs on the device
// over the uploaded f32 arrays. Built with -fmad=false: the degree selection and the q8 scale
// search must round exactly like the reference.
#include "gsr_device.cuh"
#include "encode.cuh"

namespace gsr {

namespace {

__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }

// floatToHalf (src/scene/half.h:32-58): round to nearest even, subnormals, inf/NaN.
__device__ __forceinline__ uint16_t floatToHalf(float value) {
    const uint32_t f = __float_as_uint(value);
    const uint32_t sign = (f >> 16) & 0x8000u;
    const uint32_t absBits = f & 0x7FFFFFFFu;
    if (absBits >= 0x7F800000u) return uint16_t(sign | 0x7C00u | (absBits > 0x7F800000u ? 0x200u : 0u));
    if (absBits >= 0x477FF000u) return uint16_t(sign | 0x7C00u);
    if (absBits < 0x38800000u) {
        if (absBits < 0x33000000u) return uint16_t(sign);
        const uint32_t exponent = absBits >> 23;
        const uint32_t mantissa = (absBits & 0x7FFFFFu) | 0x800000u;
        const uint32_t shift = 126u - exponent;
        uint32_t half = mantissa >> shift;
        const uint32_t rest = mantissa & ((1u << shift) - 1u);
        const uint32_t halfway = 1u << (shift - 1u);
        if (rest > halfway || (rest == halfway && (half & 1u))) ++half;
        return uint16_t(sign | half);
    }
    uint32_t half = (absBits - 0x38000000u) >> 13;
    const uint32_t rest = absBits & 0x1FFFu;
    if (rest > 0x1000u || (rest == 0x1000u && (half & 1u))) ++half;
    return uint16_t(sign | half);
}

// halfToFloat (half.h:60-71): exact.
__device__ __forceinline__ float halfToFloat(uint16_t h) {
    const uint32_t sign = uint32_t(h & 0x8000u) << 16;
    const uint32_t exponent = (h >> 10) & 0x1Fu;
    const uint32_t mantissa = h & 0x3FFu;
    if (exponent == 0) {
        const float v = float(mantissa) * (1.0f / 16777216.0f);
        return sign ? -v : v;
    }
    if (exponent == 31) return __uint_as_float(sign | 0x7F800000u | (mantissa << 13));
    return __uint_as_float(sign | ((exponent + 112u) << 23) | (mantissa << 13));
}

__device__ __forceinline__ uint32_t packHalf2(float lo, float hi) {
    return uint32_t(floatToHalf(lo)) | (uint32_t(floatToHalf(hi)) << 16);
}

__device__ __forceinline__ float smaxf(float a, float b) { return (a < b) ? b : a; }

__device__ __forceinline__ float shValue(const EncodeArgs& a, uint32_t i, uint32_t kept, uint32_t k, uint32_t c) {
    return k < kept ? a.sh[(size_t(i) * a.srcK + k) * 3 + c] : 0.0f;
}

// shBandMaxContribution + selectShDegree (scene_compression.cpp:53-68).
__device__ int selectDegree(const EncodeArgs& a, uint32_t i, float opacity) {
    const float threshold = a.threshold255 / 255.0f;
    for (int band = a.degree; band >= 1; --band) {
        const int k0 = band * band, k1 = (band + 1) * (band + 1);
        float sq0 = 0.0f, sq1 = 0.0f, sq2 = 0.0f;
        for (int k = k0; k < k1; ++k) {
            const float* s = &a.sh[(size_t(i) * a.srcK + k) * 3];
            sq0 = sq0 + s[0] * s[0];
            sq1 = sq1 + s[1] * s[1];
            sq2 = sq2 + s[2] * s[2];
        }
        const float norm = sqrtf(smaxf(sq0, smaxf(sq1, sq2)));
        const float kInv4Pi = 0.07957747154594767f;
        const float contribution = sqrtf(float(2 * band + 1) * kInv4Pi) * norm;
        if (opacity * contribution > threshold) return band;
    }
    return 0;
}

__device__ __forceinline__ uint32_t vec4sFor(uint32_t bytes) { return (bytes + 15u) / 16u; }
__device__ __forceinline__ uint32_t colorWordsFor(uint32_t color, uint32_t k) {
    switch (color) {
        case GSR_COLOR_RECORD_F32: return vec4sFor(k * 3 * 4) * 4;
        case GSR_COLOR_RECORD_F16: return vec4sFor(k * 3 * 2) * 4;
        default: return vec4sFor(12 + (k - 1) * 3) * 4;  // q8
    }
}

// Pass 1: per-gaussian kept degree and the size of its (compacted) colour data.
__global__ void degreeKernel(const __grid_constant__ EncodeArgs a, uint8_t* degrees, uint32_t* sizes) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int d = a.variable ? selectDegree(a, i, a.pa[i].w) : a.degree;
        degrees[i] = uint8_t(d);
        const uint32_t kept = uint32_t((d + 1) * (d + 1));
        if (sizes) sizes[i] = a.layout == GSR_LAYOUT_SOA ? kept * 3 : colorWordsFor(a.color, kept) / 4;
    }
}

// quantizeBandQ8 (scene_compression.cpp:130-148).
__device__ uint16_t quantizeBand(const float* v, uint32_t n, int8_t* q) {
    float m = 0.0f;
    for (uint32_t j = 0; j < n; ++j)
        if (isfinite(v[j])) m = smaxf(m, fabsf(v[j]));
    if (m == 0.0f) {
        for (uint32_t j = 0; j < n; ++j) q[j] = 0;
        return 0;
    }
    uint16_t h = floatToHalf(m / 127.0f);
    if (h == 0) h = 1;
    while (halfToFloat(h) * 127.0f < m) ++h;
    const float s = halfToFloat(h);
    for (uint32_t j = 0; j < n; ++j) {
        const float x = isfinite(v[j]) ? v[j] / s : 0.0f;
        long r = lroundf(x);
        r = r < -127L ? -127L : (r > 127L ? 127L : r);
        q[j] = int8_t(r);
    }
    return h;
}

// Pass 2: the records.
__global__ void encodeKernel(const __grid_constant__ EncodeArgs a, const uint8_t* degrees, const uint32_t* offsets) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const float4 pa = a.pa[i], sc = a.sc[i], ro = a.ro[i];
        const uint32_t d = degrees[i];
        const uint32_t kept = a.variable ? (d + 1) * (d + 1) : a.K;
        if (a.layout == GSR_LAYOUT_SOA) {
            uint32_t* b0 = reinterpret_cast<uint32_t*>(a.out[0]);
            uint32_t* b1 = reinterpret_cast<uint32_t*>(a.out[1]);
            uint32_t* b2 = reinterpret_cast<uint32_t*>(a.out[2]);
            uint32_t* b3 = reinterpret_cast<uint32_t*>(a.out[3]);
            b0[size_t(i) * 4 + 0] = fbits(pa.x); b0[size_t(i) * 4 + 1] = fbits(pa.y);
            b0[size_t(i) * 4 + 2] = fbits(pa.z); b0[size_t(i) * 4 + 3] = fbits(pa.w);
            b1[size_t(i) * 4 + 0] = fbits(sc.x); b1[size_t(i) * 4 + 1] = fbits(sc.y);
            b1[size_t(i) * 4 + 2] = fbits(sc.z); b1[size_t(i) * 4 + 3] = fbits(sc.w);
            b2[size_t(i) * 4 + 0] = fbits(ro.x); b2[size_t(i) * 4 + 1] = fbits(ro.y);
            b2[size_t(i) * 4 + 2] = fbits(ro.z); b2[size_t(i) * 4 + 3] = fbits(ro.w);
            size_t base = size_t(i) * a.K * 3;
            if (a.variable) {
                base = offsets[i];
                b1[size_t(i) * 4 + 3] = (d << 30) | offsets[i];
                for (uint32_t k = 0; k < kept; ++k)
                    for (uint32_t c = 0; c < 3; ++c) b3[base + k * 3 + c] = fbits(shValue(a, i, kept, k, c));
                continue;
            }
            for (uint32_t k = 0; k < a.K; ++k)
                for (uint32_t c = 0; c < 3; ++c) b3[base + k * 3 + c] = fbits(shValue(a, i, kept, k, c));
            continue;
        }
        // geometry record (encodeGeometry, scene_compression.cpp:34-49)
        uint32_t g[12];
        for (int j = 0; j < 12; ++j) g[j] = 0;
        if (a.geometry == GSR_GEOMETRY_RECORD_F32) {
            g[0] = fbits(pa.x); g[1] = fbits(pa.y); g[2] = fbits(pa.z); g[3] = fbits(pa.w);
            g[4] = fbits(sc.x); g[5] = fbits(sc.y); g[6] = fbits(sc.z); g[7] = 0;
            g[8] = fbits(ro.x); g[9] = fbits(ro.y); g[10] = fbits(ro.z); g[11] = fbits(ro.w);
        } else {
            g[0] = fbits(pa.x); g[1] = fbits(pa.y); g[2] = fbits(pa.z);
            g[3] = packHalf2(pa.w, sc.x);
            g[4] = packHalf2(sc.y, sc.z);
            g[5] = packHalf2(ro.x, ro.y);
            g[6] = packHalf2(ro.z, ro.w);
            g[7] = 0;
        }
        // colour record, the full-size one (truncated when compacted)
        uint32_t c[48];
        for (int j = 0; j < 48; ++j) c[j] = 0;
        if (a.color == GSR_COLOR_RECORD_F32) {
            for (uint32_t k = 0; k < a.K; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch) c[k * 3 + ch] = fbits(shValue(a, i, kept, k, ch));
        } else if (a.color == GSR_COLOR_RECORD_F16) {
            for (uint32_t k = 0; k < a.K; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch) {
                    const uint32_t hi = k * 3 + ch;
                    const uint32_t h = floatToHalf(shValue(a, i, kept, k, ch));
                    c[hi / 2] = (hi & 1u) ? ((c[hi / 2] & 0x0000FFFFu) | (h << 16)) : ((c[hi / 2] & 0xFFFF0000u) | h);
                }
        } else if (a.color == GSR_COLOR_CODEBOOK) {  // DC + the codebook entry (scene_compression.cpp:309-314)
            c[0] = packHalf2(shValue(a, i, kept, 0, 0), shValue(a, i, kept, 0, 1));
            c[1] = uint32_t(floatToHalf(shValue(a, i, kept, 0, 2))) | ((a.cbIndex ? a.cbIndex[i] : 0u) << 16);
        } else {  // q8
            c[0] = packHalf2(shValue(a, i, kept, 0, 0), shValue(a, i, kept, 0, 1));
            uint16_t bandScale[4] = {0, 0, 0, 0};
            int8_t q[45];
            for (int j = 0; j < 45; ++j) q[j] = 0;
            for (uint32_t band = 1; band * band < kept; ++band) {
                const uint32_t k0 = band * band, k1 = (band + 1) * (band + 1);
                float values[21];
                uint32_t m = 0;
                for (uint32_t k = k0; k < k1; ++k)
                    for (uint32_t ch = 0; ch < 3; ++ch) values[m++] = shValue(a, i, kept, k, ch);
                bandScale[band] = quantizeBand(values, m, &q[(k0 - 1) * 3]);
            }
            c[1] = uint32_t(floatToHalf(shValue(a, i, kept, 0, 2))) | (uint32_t(bandScale[1]) << 16);
            c[2] = uint32_t(bandScale[2]) | (uint32_t(bandScale[3]) << 16);
            const uint32_t restDims = (a.K - 1) * 3;
            for (uint32_t j = 0; j < restDims; ++j) c[3 + j / 4] |= uint32_t(uint8_t(q[j])) << (8 * (j % 4));
        }
        // variable degree: the degree in word 7, plus the compacted colour offset in the split
        // layout (scene_compression.cpp:320-337); cb records stay fixed-size (degree only)
        const bool compact = a.variable && a.layout == GSR_LAYOUT_SPLIT && a.color != GSR_COLOR_CODEBOOK;
        uint32_t colorWords = a.colorWords;
        if (compact) {
            g[7] = (d << 30) | offsets[i];
            colorWords = colorWordsFor(a.color, kept);
        } else if (a.variable) {
            g[7] = d << 30;
        }
        uint32_t* gdst;
        uint32_t* cdst;
        if (a.layout == GSR_LAYOUT_SPLIT) {
            gdst = reinterpret_cast<uint32_t*>(a.out[0]) + size_t(i) * a.geomWords;
            cdst = reinterpret_cast<uint32_t*>(a.out[1]) + (compact ? size_t(offsets[i]) * 4 : size_t(i) * a.colorWords);
        } else {
            uint32_t* rec = reinterpret_cast<uint32_t*>(a.out[0]) + size_t(i) * (a.geomWords + a.colorWords);
            gdst = rec;
            cdst = rec + a.geomWords;
        }
        for (uint32_t j = 0; j < a.geomWords; ++j) gdst[j] = g[j];
        for (uint32_t j = 0; j < colorWords; ++j) cdst[j] = c[j];
    }
}

uint32_t gridFor(uint32_t n) {
    uint32_t b = (n + 255) / 256;
    return b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b);
}

// ---- the cb codebook's k-means (kmeans.cpp) --------------------------------------------------
__global__ void codebookPointsKernel(const __grid_constant__ EncodeArgs a, const uint8_t* degrees, float* points) {
    const uint32_t dims = (a.K - 1) * 3;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const uint32_t d = degrees[i];
        const uint32_t kept = a.variable ? (d + 1) * (d + 1) : a.K;
        for (uint32_t k = 1; k < a.K; ++k)
            for (uint32_t c = 0; c < 3; ++c) {
                const float v = shValue(a, i, kept, k, c);
                points[size_t(i) * dims + (k - 1) * 3 + c] = isfinite(v) ? v : 0.0f;
            }
    }
}

__global__ void codebookGatherKernel(const float* points, uint32_t dims, const uint32_t* index, uint32_t count,
                                     float* out) {
    const size_t total = size_t(count) * dims;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x)
        out[e] = points[size_t(index[e / dims]) * dims + e % dims];
}

// nearestAvx2 (kmeans.cpp:153-190) per point: x.c_j accumulated over the dimensions in order with
// one fused multiply-add per dimension, the distance |c_j|^2 - 2 x.c_j fused as well, the first
// smallest distance wins; then max(0, |x|^2 + best) with |x|^2 summed in double (assignAll,
// :196-223). A block's 256 threads take 256 points; the centroids pass through shared memory in
// tiles of 64, transposed so that one 16-byte load feeds four centroids' chains.
constexpr int kCentroidTile = 64;
template <int DIMS>
__global__ void __launch_bounds__(256) nearestCentroidKernel(const float* __restrict__ points, uint32_t count,
                                                             const float* __restrict__ centroids,
                                                             const float* __restrict__ norm2, uint32_t k,
                                                             uint32_t* assignment, float* sqDist) {
    __shared__ __align__(16) float sC[DIMS][kCentroidTile];
    __shared__ float sN[kCentroidTile];
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    const bool valid = i < count;
    float x[DIMS];
    double x2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) x[d] = valid ? points[size_t(i) * DIMS + d] : 0.0f;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) x2 += double(x[d]) * double(x[d]);
    float best = __uint_as_float(0x7F800000u);
    uint32_t bestIndex = 0;
    for (uint32_t t0 = 0; t0 < k; t0 += kCentroidTile) {
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < uint32_t(DIMS * kCentroidTile); e += 256) {
            const uint32_t j = e / DIMS, d = e % DIMS;
            sC[d][j] = t0 + j < k ? centroids[size_t(t0 + j) * DIMS + d] : 0.0f;
        }
        if (threadIdx.x < uint32_t(kCentroidTile))
            sN[threadIdx.x] = t0 + threadIdx.x < k ? norm2[t0 + threadIdx.x] : __uint_as_float(0x7F800000u);
        __syncthreads();
        const uint32_t m = k - t0 < uint32_t(kCentroidTile) ? k - t0 : uint32_t(kCentroidTile);
        for (uint32_t j = 0; j < m; j += 4) {  // slots past m: c = 0, |c|^2 = +inf, never chosen
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
            for (int d = 0; d < DIMS; ++d) {
                const float4 c = *reinterpret_cast<const float4*>(&sC[d][j]);
                a0 = fmaf(x[d], c.x, a0);
                a1 = fmaf(x[d], c.y, a1);
                a2 = fmaf(x[d], c.z, a2);
                a3 = fmaf(x[d], c.w, a3);
            }
            const float acc[4] = {a0, a1, a2, a3};
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const float dist = fmaf(-2.0f, acc[l], sN[j + l]);
                if (dist < best) {
                    best = dist;
                    bestIndex = t0 + j + uint32_t(l);
                }
            }
        }
    }
    if (valid) {
        assignment[i] = bestIndex;
        const float v = float(x2) + best;
        sqDist[i] = (0.0f < v) ? v : 0.0f;  // std::max(0.0f, v)
    }
}

}  // namespace

cudaError_t launchEncodeDegrees(const EncodeArgs& a, uint8_t* degrees, uint32_t* sizes, cudaStream_t s) {
    degreeKernel<<<gridFor(a.n), 256, 0, s>>>(a, degrees, sizes);
    return cudaGetLastError();
}

cudaError_t launchEncodeRecords(const EncodeArgs& a, const uint8_t* degrees, const uint32_t* offsets, cudaStream_t s) {
    encodeKernel<<<gridFor(a.n), 256, 0, s>>>(a, degrees, offsets);
    return cudaGetLastError();
}

cudaError_t launchCodebookPoints(const EncodeArgs& a, const uint8_t* degrees, float* points, cudaStream_t s) {
    codebookPointsKernel<<<gridFor(a.n), 256, 0, s>>>(a, degrees, points);
    return cudaGetLastError();
}

cudaError_t launchCodebookGather(const float* points, uint32_t dims, const uint32_t* index, uint32_t count, float* out,
                                 cudaStream_t s) {
    const uint64_t total = uint64_t(count) * dims;
    const uint32_t blocks = uint32_t(total / 256 + 1 < 148 * 32 ? total / 256 + 1 : 148 * 32);
    codebookGatherKernel<<<blocks, 256, 0, s>>>(points, dims, index, count, out);
    return cudaGetLastError();
}

cudaError_t launchNearestCentroid(const float* points, uint32_t count, uint32_t dims, const float* centroids,
                                  const float* norm2, uint32_t k, uint32_t* assignment, float* sqDist, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const uint32_t blocks = (count + 255) / 256;
    switch (dims) {
        case 9: nearestCentroidKernel<9><<<blocks, 256, 0, s>>>(points, count, centroids, norm2, k, assignment, sqDist); break;
        case 24: nearestCentroidKernel<24><<<blocks, 256, 0, s>>>(points, count, centroids, norm2, k, assignment, sqDist); break;
        case 45: nearestCentroidKernel<45><<<blocks, 256, 0, s>>>(points, count, centroids, norm2, k, assignment, sqDist); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace gsr
