// The per-gaussian math of the splat-tiles preprocess and the tight tile coverage, on the
// device. Include only from translation units built with -fmad=false: every expression below
// is spelled in the reference's evaluation order so that depths, conics, radii, rectangles
// and tile runs are bit-identical to the reference's CPU code.
//
// Sources followed (evaluation order of the GLM products: k ascending, left to right):
//   src/splat/splat_math.cpp  quaternionToMatrix, computeCov3D, computeCov2D, projectToPixel,
//                             conicAndRadius, computeTileRect, evalSH, preprocessGaussian
//   src/splat/tile_coverage.cpp  makeCutoffEllipse, ellipseRows, ellipseRowBounds,
//                             ellipseRowSpan, rectToBins, makeCoverage, coverageCount
//   shaders/splat_preprocess.comp:147-223  the GPU culls (NaN-safe near test, o < 1/255)
#pragma once

#include "gsr_device.cuh"
#include "render_splat.cuh"

namespace gsr {

// INRIA constants (src/splat/splat_math.h:26-40).
constexpr float kNearCullDepth = 0.2f;
constexpr float kLowPassFilter = 0.3f;
constexpr float kFrustumClampFactor = 1.3f;
#define GSR_MIN_ALPHA (1.0f / 255.0f)
constexpr float kShC0 = 0.28209479177387814f;
constexpr float kShC1 = 0.4886025119029199f;
constexpr float kShC2_0 = 1.0925484305920792f, kShC2_1 = -1.0925484305920792f, kShC2_2 = 0.31539156525252005f,
                kShC2_3 = -1.0925484305920792f, kShC2_4 = 0.5462742152960396f;
constexpr float kShC3_0 = -0.5900435899266435f, kShC3_1 = 2.890611442640554f, kShC3_2 = -0.4570457994644658f,
                kShC3_3 = 0.3731763325901154f, kShC3_4 = -0.4570457994644658f, kShC3_5 = 1.445305721320277f,
                kShC3_6 = -0.5900435899266435f;

// gsr::SplatCamera (splat_math.h:43-50); viewInria column-major v[c*4 + r].
struct DevCamera {
    float v[16];
    float pos[3];
    uint32_t width, height;
    float tanHalfFovX, tanHalfFovY, focalX, focalY;
    uint32_t tilesX, tilesY;
};

// The 48-byte ProjectedSplat / GLSL Splat (splat_math.h:115-122, splat_common.glsl:25-32).
struct __align__(16) DevSplat {
    float cx, cy, depth;
    uint32_t cullReason;
    float conicA, conicB, conicC, opacity;
    float r, g, b, radius;
};
static_assert(sizeof(DevSplat) == 48, "ProjectedSplat layout");

struct TileRect { int minX, minY, maxX, maxY; };

// the packed render records' tile rectangle: minX | minY << 16, maxX | maxY << 16 (packRect,
// render_splat.glsl)
__device__ __forceinline__ uint2 packRect(const TileRect& r) {
    return make_uint2(uint32_t(r.minX) | (uint32_t(r.minY) << 16), uint32_t(r.maxX) | (uint32_t(r.maxY) << 16));
}
__device__ __forceinline__ TileRect unpackRect(uint2 w) {
    return TileRect{int(w.x & 0xFFFFu), int(w.x >> 16), int(w.y & 0xFFFFu), int(w.y >> 16)};
}

// computeCov3D (splat_math.cpp:44-63): S[c*3 + r] = sum_k M[k][r] M[k][c], M = R diag(sigma).
__device__ __forceinline__ void cov3d(float sx, float sy, float sz, float qr, float qx, float qy, float qz, float S[9]) {
    const float r = qr, x = qx, y = qy, z = qz;
    float R[9];
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + r * z); R[2] = 2.0f * (x * z - r * y);
    R[3] = 2.0f * (x * y - r * z); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + r * x);
    R[6] = 2.0f * (x * z + r * y); R[7] = 2.0f * (y * z - r * x); R[8] = 1.0f - 2.0f * (x * x + y * y);
    float M[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        M[0 + k] = R[0 + k] * sx;
        M[3 + k] = R[3 + k] * sy;
        M[6 + k] = R[6 + k] * sz;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int row = 0; row < 3; ++row)
            S[c * 3 + row] = M[0 * 3 + row] * M[0 * 3 + c] + M[1 * 3 + row] * M[1 * 3 + c] + M[2 * 3 + row] * M[2 * 3 + c];
}

// computeCov2D (splat_math.cpp:65-91). out = (a, b, c) of [[a b][b c]].
__device__ __forceinline__ void cov2d(const float t[3], const float S[9], const DevCamera& cam, float out[3]) {
    const float limX = kFrustumClampFactor * cam.tanHalfFovX;
    const float limY = kFrustumClampFactor * cam.tanHalfFovY;
    const float txtz = t[0] / t[2];
    const float tytz = t[1] / t[2];
    const float tx = smin(limX, smax(-limX, txtz)) * t[2];
    const float ty = smin(limY, smax(-limY, tytz)) * t[2];
    const float tz = t[2];
    float J[6];  // J[c*2 + r]: 3 columns, 2 rows; the zero entries take part in the products
    J[0] = cam.focalX / tz; J[1] = 0.0f;
    J[2] = 0.0f;            J[3] = cam.focalY / tz;
    J[4] = -(cam.focalX * tx) / (tz * tz);
    J[5] = -(cam.focalY * ty) / (tz * tz);
    float T[6], A[6];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 2; ++r)
            T[c * 2 + r] = J[0 * 2 + r] * cam.v[c * 4 + 0] + J[1 * 2 + r] * cam.v[c * 4 + 1] + J[2 * 2 + r] * cam.v[c * 4 + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 2; ++r)
            A[c * 2 + r] = T[0 * 2 + r] * S[c * 3 + 0] + T[1 * 2 + r] * S[c * 3 + 1] + T[2 * 2 + r] * S[c * 3 + 2];
    const float c00 = A[0] * T[0] + A[2] * T[2] + A[4] * T[4];
    const float c01 = A[1] * T[0] + A[3] * T[2] + A[5] * T[4];
    const float c11 = A[1] * T[1] + A[3] * T[3] + A[5] * T[5];
    out[0] = c00 + kLowPassFilter;
    out[1] = c01;
    out[2] = c11 + kLowPassFilter;
}

// conicAndRadius (splat_math.cpp:102-114).
__device__ __forceinline__ bool conicAndRadius(const float cov[3], float conic[3], float& radius) {
    const float det = cov[0] * cov[2] - cov[1] * cov[1];
    if (det == 0.0f) return false;
    const float detInv = 1.0f / det;
    conic[0] = cov[2] * detInv;
    conic[1] = -cov[1] * detInv;
    conic[2] = cov[0] * detInv;
    const float mid = 0.5f * (cov[0] + cov[2]);
    const float lambda1 = mid + sqrtf(smax(0.1f, mid * mid - det));
    const float lambda2 = mid - sqrtf(smax(0.1f, mid * mid - det));
    radius = ceilf(3.0f * sqrtf(smax(lambda1, lambda2)));
    return true;
}

// computeTileRect (splat_math.cpp:116-127): INRIA getRect with int truncation.
__device__ __forceinline__ TileRect tileRect(float px, float py, float radius, uint32_t tilesX, uint32_t tilesY) {
    const int gx = int(tilesX), gy = int(tilesY);
    const int r = ftoi(radius);
    const float fr = float(r);
    TileRect t;
    t.minX = imin(gx, imax(0, ftoi((px - fr) / float(kTileSize))));
    t.minY = imin(gy, imax(0, ftoi((py - fr) / float(kTileSize))));
    t.maxX = imin(gx, imax(0, ftoi((px + fr + float(kTileSize - 1)) / float(kTileSize))));
    t.maxY = imin(gy, imax(0, ftoi((py + fr + float(kTileSize - 1)) / float(kTileSize))));
    return t;
}

// computeRayDepthParams (splat_math.cpp:195-205) for the StopThePop window: with M = the upper-left
// 3x3 of viewInria times quaternionToMatrix(q) (the gaussian's axes in camera space), s = sigma
// clamped below at max(1e-4 max(sigma), 1e-12) and w = 1 / s^2, P = sum_k w_k M_k M_k^T (k = 0, 1,
// 2 added to a zero matrix) and b = P tCam. The depth of the gaussian's maximum along the pixel
// ray t (vx, vy, 1) is then (v . b) / (v^T P v). out: (P00, P01, P02, P11), (P12, P22, b0, b1),
// (b2, 0, 0, 0).
__device__ __forceinline__ void rayDepthParams(const float sigma[3], const float q[4], const float t[3],
                                               const DevCamera& cam, float4 out[3]) {
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    float R[9];  // R[c*3 + row], quaternionToMatrix
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + r * z); R[2] = 2.0f * (x * z - r * y);
    R[3] = 2.0f * (x * y - r * z); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + r * x);
    R[6] = 2.0f * (x * z + r * y); R[7] = 2.0f * (y * z - r * x); R[8] = 1.0f - 2.0f * (x * x + y * y);
    float M[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int row = 0; row < 3; ++row)
            M[c * 3 + row] = cam.v[0 * 4 + row] * R[c * 3 + 0] + cam.v[1 * 4 + row] * R[c * 3 + 1] + cam.v[2 * 4 + row] * R[c * 3 + 2];
    const float sMax = smax(sigma[0], smax(sigma[1], sigma[2]));
    const float floorS = smax(1e-4f * sMax, 1e-12f);
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sk = smax(sigma[k], floorS);
        w[k] = 1.0f / (sk * sk);
    }
    float P[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) P[i * 3 + j] = P[i * 3 + j] + w[k] * (M[k * 3 + j] * M[k * 3 + i]);
    float b[3];
#pragma unroll
    for (int row = 0; row < 3; ++row) b[row] = P[0 * 3 + row] * t[0] + P[1 * 3 + row] * t[1] + P[2 * 3 + row] * t[2];
    out[0] = make_float4(P[0], P[1], P[2], P[4]);
    out[1] = make_float4(P[5], P[8], b[0], b[1]);
    out[2] = make_float4(b[2], 0.0f, 0.0f, 0.0f);
}

// evalSH (splat_math.cpp:129-151) over 16 coefficient triplets sh[k*3 + c] (only the first
// (degree+1)^2 are read).
__device__ __forceinline__ void evalSH(int degree, const float* sh, float dx, float dy, float dz, float out[3]) {
    float res0 = kShC0 * sh[0], res1 = kShC0 * sh[1], res2 = kShC0 * sh[2];
    if (degree > 0) {
        const float x = dx, y = dy, z = dz;
        const float a = kShC1 * y, b = kShC1 * z, d = kShC1 * x;
        res0 = res0 - a * sh[3] + b * sh[6] - d * sh[9];
        res1 = res1 - a * sh[4] + b * sh[7] - d * sh[10];
        res2 = res2 - a * sh[5] + b * sh[8] - d * sh[11];
        if (degree > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float t4 = kShC2_0 * xy, t5 = kShC2_1 * yz, t6 = kShC2_2 * (2.0f * zz - xx - yy);
            const float t7 = kShC2_3 * xz, t8 = kShC2_4 * (xx - yy);
            res0 = res0 + t4 * sh[12] + t5 * sh[15] + t6 * sh[18] + t7 * sh[21] + t8 * sh[24];
            res1 = res1 + t4 * sh[13] + t5 * sh[16] + t6 * sh[19] + t7 * sh[22] + t8 * sh[25];
            res2 = res2 + t4 * sh[14] + t5 * sh[17] + t6 * sh[20] + t7 * sh[23] + t8 * sh[26];
            if (degree > 2) {
                const float t9 = kShC3_0 * y * (3.0f * xx - yy), t10 = kShC3_1 * xy * z;
                const float t11 = kShC3_2 * y * (4.0f * zz - xx - yy);
                const float t12 = kShC3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
                const float t13 = kShC3_4 * x * (4.0f * zz - xx - yy), t14 = kShC3_5 * z * (xx - yy);
                const float t15 = kShC3_6 * x * (xx - 3.0f * yy);
                res0 = res0 + t9 * sh[27] + t10 * sh[30] + t11 * sh[33] + t12 * sh[36] + t13 * sh[39] + t14 * sh[42] + t15 * sh[45];
                res1 = res1 + t9 * sh[28] + t10 * sh[31] + t11 * sh[34] + t12 * sh[37] + t13 * sh[40] + t14 * sh[43] + t15 * sh[46];
                res2 = res2 + t9 * sh[29] + t10 * sh[32] + t11 * sh[35] + t12 * sh[38] + t13 * sh[41] + t14 * sh[44] + t15 * sh[47];
            }
        }
    }
    res0 = res0 + 0.5f;
    res1 = res1 + 0.5f;
    res2 = res2 + 0.5f;
    out[0] = smax(res0, 0.0f);
    out[1] = smax(res1, 0.0f);
    out[2] = smax(res2, 0.0f);
}

// ---- tight coverage (tile_coverage.cpp) ---------------------------------------------------
struct Ellipse {
    float cx, cy, A, B, C, D, t, exPad, eyPad;
    bool valid;
};
struct BinRect { int x0, y0, x1, y1; };
struct Coverage {
    BinRect bins;
    Ellipse e;
    bool useEllipse;
};

// makeCutoffEllipse (tile_coverage.cpp:24-50).
__device__ __forceinline__ Ellipse makeEllipse(float cx, float cy, float A, float B, float C, float opacity,
                                               const LogfFixups& logf) {
    Ellipse e;
    e.cx = cx;
    e.cy = cy;
    const float D = A * C - B * B;
    e.A = A; e.B = B; e.C = C; e.D = D;
    e.t = -1.0f;
    e.exPad = 0.0f;
    e.eyPad = 0.0f;
    e.valid = A > 0.0f && C > 0.0f && D > 0.0f;
    if (!e.valid) return e;
    if (!(opacity >= GSR_MIN_ALPHA)) return e;
    const float qmax = 2.0f * libcLogf(255.0f * opacity, logf);
    const float rho = fabsf(B) / sqrtf(A * C);
    const float K = 2.0f / smax(1.0f - rho, 1e-30f);
    const float t = qmax + (1e-3f + 2e-5f * K) * smax(qmax, 1.0f) + 2e-3f;
    if (!(t < 1e30f)) {
        e.valid = false;
        return e;
    }
    e.t = t;
    const float ex = sqrtf(t * C / D);
    const float ey = sqrtf(t * A / D);
    e.exPad = ex + (0.02f + 2e-3f * ex);
    e.eyPad = ey + (0.02f + 2e-3f * ey);
    return e;
}

// The bins of the binning grid, sx x sy pixels (lx, ly their base-2 logarithms). The reference's
// bins are square, S x S with S = 16 or 8 (tile_coverage.cpp); code 32 names 32 x 8 bins, as many
// pixels as a 16 x 16 tile. With sx = sy = S every expression below is the reference's.
struct BinShape {
    int sx, sy, lx, ly;
};
__device__ __forceinline__ BinShape binShapeOf(int code) {
    const int sy = code == 32 ? 8 : code;
    return BinShape{code, sy, code == 32 ? 5 : (code == 16 ? 4 : 3), sy == 16 ? 4 : 3};
}

// floorDivClamped (tile_coverage.cpp:54). S is 32, 16 or 8: dividing by a power of two is exactly
// multiplying by its reciprocal (both give the exact quotient, or round the same exact value),
// so the quotient is the reference's without a division sequence.
__device__ __forceinline__ int floorDivClamped(float v, int S) {
    const float inv = S == 16 ? 0.0625f : (S == 8 ? 0.125f : (S == 32 ? 0.03125f : 0.0f));
    const float c = sclamp(v, -65536.0f, 1048576.0f);
    return ftoi(floorf(inv != 0.0f ? c * inv : c / float(S)));
}

// rectToBins (tile_coverage.cpp:102-105): the bins holding the 16-px rectangle's pixels (its
// first bin rounds down, its end up; for bins that divide 16 this is the reference's r * 16 / S).
__device__ __forceinline__ BinRect rectToBins(const TileRect& r, const BinShape& bs, int gx, int gy) {
    return {(r.minX << 4) >> bs.lx, (r.minY << 4) >> bs.ly, imin(((r.maxX << 4) + bs.sx - 1) >> bs.lx, gx),
            imin(((r.maxY << 4) + bs.sy - 1) >> bs.ly, gy)};
}

// makeCoverage (tile_coverage.cpp:107-117).
__device__ __forceinline__ Coverage makeCoverage(uint32_t mode, const TileRect& rect16, const BinShape& S, int gx, int gy,
                                                 float cx, float cy, float A, float B, float C, float opacity,
                                                 const LogfFixups& logf) {
    Coverage cv;
    cv.bins = mode == kBoundsCutoff ? BinRect{0, 0, gx, gy} : rectToBins(rect16, S, gx, gy);
    cv.useEllipse = false;
    cv.e.valid = false;
    cv.e.t = -1.0f;
    if (mode != kBoundsRect) {
        cv.e = makeEllipse(cx, cy, A, B, C, opacity, logf);
        cv.useEllipse = cv.e.valid;
        if (!cv.e.valid && mode == kBoundsCutoff) cv.bins = rectToBins(rect16, S, gx, gy);
    }
    return cv;
}

// coverageRows (tile_coverage.cpp:119-122) with ellipseRows (56-63).
__device__ __forceinline__ void coverageRows(const Coverage& cv, const BinShape& S, int& r0, int& r1) {
    if (!cv.useEllipse) {
        r0 = cv.bins.y0;
        r1 = imax(cv.bins.y0, cv.bins.y1);
        return;
    }
    const Ellipse& e = cv.e;
    if (e.t < 0.0f) {
        r0 = 0;
        r1 = 0;
        return;
    }
    const float y0 = ceilf(e.cy - e.eyPad);
    const float y1 = floorf(e.cy + e.eyPad);
    const int lo = imax(cv.bins.y0, floorDivClamped(y0, S.sy));
    const int hi = imin(cv.bins.y1, floorDivClamped(y1, S.sy) + 1);
    r0 = lo;
    r1 = imax(lo, hi);
}

// The row-independent terms of ellipseRowSpan (tile_coverage.cpp:81-90), computed once per
// ellipse with the reference's expressions: exTrue = sqrt(t C / D), eyRight0 = -B exTrue / C
// (eyLeft0 = B exTrue / C is exactly -eyRight0: IEEE products and quotients are sign-symmetric),
// At = A t, pad = 0.02 + 2e-3 exTrue. Only used when the ellipse is valid with t >= 0.
struct RowGeom {
    float exTrue, eyRight0, At, pad;
};
__device__ __forceinline__ RowGeom rowGeom(const Coverage& cv) {
    RowGeom g{0.0f, 0.0f, 0.0f, 0.0f};
    const Ellipse& e = cv.e;
    if (!cv.useEllipse || e.t < 0.0f) return g;
    g.exTrue = sqrtf(e.t * e.C / e.D);
    g.eyRight0 = -e.B * g.exTrue / e.C;
    g.At = e.A * e.t;
    g.pad = 0.02f + 2e-3f * g.exTrue;
    return g;
}

// coverageRowSpan (tile_coverage.cpp:124-127) with ellipseRowBounds/ellipseRowSpan (70-96).
__device__ __forceinline__ void coverageRowSpan(const Coverage& cv, const RowGeom& g, int row, const BinShape& S, int& x0,
                                                int& x1) {
    if (!cv.useEllipse) {
        x0 = cv.bins.x0;
        x1 = imax(cv.bins.x0, cv.bins.x1);
        return;
    }
    const Ellipse& e = cv.e;
    const float ey0 = float(row * S.sy) - e.cy;
    const float ey1 = float(row * S.sy + S.sy - 1) - e.cy;
    const float lo = smax(ey0, -e.eyPad);
    const float hi = smin(ey1, e.eyPad);
    if (!(lo <= hi)) {
        x0 = cv.bins.x0;
        x1 = cv.bins.x0;
        return;
    }
    const float eyRight = sclamp(g.eyRight0, lo, hi);
    const float eyLeft = sclamp(-g.eyRight0, lo, hi);
    const float xRight = (-e.B * eyRight + sqrtf(smax(0.0f, g.At - e.D * eyRight * eyRight))) / e.A;
    const float xLeft = (-e.B * eyLeft - sqrtf(smax(0.0f, g.At - e.D * eyLeft * eyLeft))) / e.A;
    const float fx0 = e.cx + xLeft - g.pad;
    const float fx1 = e.cx + xRight + g.pad;
    const int a = imax(cv.bins.x0, floorDivClamped(ceilf(fx0), S.sx));
    const int c = imin(cv.bins.x1, floorDivClamped(floorf(fx1), S.sx) + 1);
    x0 = a;
    x1 = imax(a, c);
}

// coverageCount (tile_coverage.cpp:129-138).
__device__ __forceinline__ uint32_t coverageCount(const Coverage& cv, const RowGeom& g, const BinShape& S) {
    int r0, r1;
    coverageRows(cv, S, r0, r1);
    if (!cv.useEllipse) return uint32_t(imax(0, cv.bins.x1 - cv.bins.x0) * (r1 - r0));
    uint32_t n = 0;
    for (int r = r0; r < r1; ++r) {
        int x0, x1;
        coverageRowSpan(cv, g, r, S, x0, x1);
        n += uint32_t(x1 - x0);
    }
    return n;
}

// Span hints: the coverage of a visible gaussian as its rows' runs, kept by the preprocess (which
// computes them for the count anyway) when it has at most kSpanRows rows and fewer than 65536
// bins a row, so that the emission needs neither the record nor the ellipse's square roots and
// quotients. Word x of the hint is a quiet NaN carrying r0 (16 bits) and the row count (3 bits),
// which no float hint has (their x is t: finite, or -2); words y, z, w hold rows 0-2 as
// x0 | x1 << 16, the second array's four words rows 3-6.
constexpr int kSpanRows = 7;
constexpr uint32_t kSpanMarker = 0x7FC00000u;
__device__ __forceinline__ bool isSpanHint(const float4& h) {
    return (__float_as_uint(h.x) & 0xFFC00000u) == kSpanMarker;
}

// coverageCount that also stores the rows' runs of a span hint (spanForm: rows <= kSpanRows and
// the grid's width below 65536) into `hint` (rows 0-2, words 1-3) and `more` (rows 3-6).
__device__ __forceinline__ uint32_t coverageCountSpans(const Coverage& cv, const RowGeom& g, const BinShape& S, int gx,
                                                       uint32_t* hint, uint32_t* more, int& r0, int& rows,
                                                       bool& spanForm) {
    int r1;
    coverageRows(cv, S, r0, r1);
    rows = r1 - r0;
    spanForm = r1 - r0 <= kSpanRows && gx < 65536 && r0 >= 0 && r0 < 65536;
    uint32_t n = 0;
    for (int r = r0; r < r1; ++r) {
        int x0, x1;
        coverageRowSpan(cv, g, r, S, x0, x1);
        n += uint32_t(x1 - x0);
        if (spanForm) {
            const int k = r - r0;
            const uint32_t w = uint32_t(x0) | (uint32_t(x1) << 16);
            if (k < 3) hint[1 + k] = w;
            else more[k - 3] = w;
        }
    }
    return n;
}

// What the key emission needs of a visible gaussian's coverage beyond its record, kept by the
// preprocess so that the emission does not evaluate the logarithm, the square roots and the
// quotients of the cutoff ellipse again: (t, ex, ey, eyRight0), t = -2 for an invalid ellipse.
// coverageFromHint rebuilds the same Coverage and RowGeom from the record and the hint.
__device__ __forceinline__ float4 coverageHint(const Coverage& cv, const RowGeom& g) {
    const Ellipse& e = cv.e;
    if (!e.valid) return make_float4(-2.0f, 0.0f, 0.0f, 0.0f);
    if (e.t < 0.0f) return make_float4(e.t, 0.0f, 0.0f, 0.0f);
    // makeEllipse's ey = sqrt(t A / D); ex = sqrt(t C / D) = exTrue
    return make_float4(e.t, g.exTrue, sqrtf(e.t * e.A / e.D), g.eyRight0);
}

__device__ __forceinline__ Coverage coverageFromHint(uint32_t mode, const TileRect& rect16, const BinShape& S, int gx, int gy,
                                                     float cx, float cy, float A, float B, float C, const float4& h,
                                                     RowGeom& g) {
    Coverage cv;
    cv.bins = mode == kBoundsCutoff ? BinRect{0, 0, gx, gy} : rectToBins(rect16, S, gx, gy);
    cv.useEllipse = false;
    cv.e.valid = false;
    cv.e.t = -1.0f;
    g = RowGeom{0.0f, 0.0f, 0.0f, 0.0f};
    if (mode == kBoundsRect) return cv;
    Ellipse& e = cv.e;
    e.cx = cx;
    e.cy = cy;
    e.A = A; e.B = B; e.C = C; e.D = A * C - B * B;
    e.valid = h.x != -2.0f;
    e.t = e.valid ? h.x : -1.0f;
    e.exPad = 0.0f;
    e.eyPad = 0.0f;
    if (e.valid && e.t >= 0.0f) {
        e.exPad = h.y + (0.02f + 2e-3f * h.y);  // makeEllipse's pads
        e.eyPad = h.z + (0.02f + 2e-3f * h.z);
        g.exTrue = h.y;
        g.eyRight0 = h.w;
        g.At = e.A * e.t;
        g.pad = 0.02f + 2e-3f * h.y;
    }
    cv.useEllipse = e.valid;
    if (!e.valid && mode == kBoundsCutoff) cv.bins = rectToBins(rect16, S, gx, gy);
    return cv;
}

}  // namespace gsr
