/* Test infrastructure: the CPU oracle of the splat-tiles frame path (see gsr_oracle.h).
 * Only tests/, tests/golden/make_golden.py and bench.py's CPU-baseline legs use it.
 *
 * Written against the reference's CPU code; every function cites the reference file:line
 * it restates. Evaluation order is the GLM-subset order documented in
 * oracle/glm_shim/glm/glm.hpp; std::min/std::max/std::clamp are restated with their exact
 * comparison semantics (NaN included), and int(float) with the x86-64 cvttss2si result
 * (INT_MIN for NaN and out-of-range values), which is what the reference compiles to. */
#define _GNU_SOURCE
#include "gsr_oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

/* ---- scalar helpers ------------------------------------------------------------------ */
static inline float smax(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline float smin(float a, float b) { return (b < a) ? b : a; } /* std::min */
static inline int imax(int a, int b) { return (a < b) ? b : a; }
static inline int imin(int a, int b) { return (b < a) ? b : a; }
static inline float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : (hi < v) ? hi : v; } /* std::clamp */
static inline int ftoi(float x) { return (x >= -2147483648.0f && x < 2147483648.0f) ? (int)x : INT_MIN; }
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* INRIA constants, src/splat/splat_math.h:26-40 and src/scene/gaussian_scene.h (kShC0). */
static const float kNearCullDepth = 0.2f;
static const float kLowPassFilter = 0.3f;
static const float kFrustumClampFactor = 1.3f;
static const float kMaxAlpha = 0.99f;
#define kMinAlpha (1.0f / 255.0f)
static const float kMinTransmittance = 1e-4f;
static const int kTileSize = 16;
static const float kShC0 = 0.28209479177387814f;
static const float kShC1 = 0.4886025119029199f;
static const float kShC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                               -1.0925484305920792f, 0.5462742152960396f};
static const float kShC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                               0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                               -0.5900435899266435f};

#define M4(m, c, r) (m)[(c)*4 + (r)]

static double nowMs(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
}

/* ---- threads: parallelFor (reference_renderer.cpp:23-37) ------------------------------- */
typedef void (*ForFn)(uint32_t index, void* ctx);
typedef struct { atomic_uint next; uint32_t count, chunk; ForFn fn; void* ctx; } ForJob;
static void* forWorker(void* p) {
    ForJob* j = (ForJob*)p;
    for (;;) {
        const uint32_t begin = atomic_fetch_add(&j->next, j->chunk);
        if (begin >= j->count) return NULL;
        const uint32_t end = j->count - begin < j->chunk ? j->count : begin + j->chunk;
        for (uint32_t i = begin; i < end; ++i) j->fn(i, j->ctx);
    }
}
static void parallelFor(uint32_t count, unsigned threads, uint32_t chunk, ForFn fn, void* ctx) {
    ForJob job;
    atomic_init(&job.next, 0u);
    job.count = count;
    job.chunk = chunk;
    job.fn = fn;
    job.ctx = ctx;
    pthread_t pool[512];
    unsigned started = 0;
    for (unsigned t = 1; t < threads && t < 512; ++t)
        if (pthread_create(&pool[started], NULL, forWorker, &job) == 0) ++started;
    forWorker(&job);
    for (unsigned t = 0; t < started; ++t) pthread_join(pool[t], NULL);
}
static unsigned hardwareThreads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (unsigned)n : 1u;
}

/* ---- camera ------------------------------------------------------------------------- */
static void normalize3(const float v[3], float out[3]) {
    const float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    out[0] = v[0] * inv;
    out[1] = v[1] * inv;
    out[2] = v[2] * inv;
}
static void cross3(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - b[1] * a[2];
    out[1] = a[2] * b[0] - b[2] * a[0];
    out[2] = a[0] * b[1] - b[0] * a[1];
}
static float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* glm::lookAtRH, the view matrix the reference's tests and camera build (test_tile_raster.cpp:407). */
void gsr_oracle_look_at(const float eye[3], const float center[3], const float up[3], float view[16]) {
    float d[3] = {center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]}, f[3], sraw[3], s[3], u[3];
    normalize3(d, f);
    cross3(f, up, sraw);
    normalize3(sraw, s);
    cross3(s, f, u);
    for (int i = 0; i < 16; ++i) view[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    M4(view, 0, 0) = s[0]; M4(view, 1, 0) = s[1]; M4(view, 2, 0) = s[2];
    M4(view, 0, 1) = u[0]; M4(view, 1, 1) = u[1]; M4(view, 2, 1) = u[2];
    M4(view, 0, 2) = -f[0]; M4(view, 1, 2) = -f[1]; M4(view, 2, 2) = -f[2];
    M4(view, 3, 0) = -dot3(s, eye);
    M4(view, 3, 1) = -dot3(u, eye);
    M4(view, 3, 2) = dot3(f, eye);
}

/* glm::perspectiveRH_ZO (GLM_FORCE_DEPTH_ZERO_TO_ONE); callers flip proj[1][1] for Vulkan. */
void gsr_oracle_perspective(float fovy, float aspect, float zNear, float zFar, float proj[16]) {
    const float tanHalfFovy = tanf(fovy / 2.0f);
    for (int i = 0; i < 16; ++i) proj[i] = 0.0f;
    M4(proj, 0, 0) = 1.0f / (aspect * tanHalfFovy);
    M4(proj, 1, 1) = 1.0f / tanHalfFovy;
    M4(proj, 2, 2) = zFar / (zNear - zFar);
    M4(proj, 2, 3) = -1.0f;
    M4(proj, 3, 2) = -(zFar * zNear) / (zFar - zNear);
}

static void mul4(const float* a, const float* b, float* r) {
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            M4(r, c, row) = M4(a, 0, row) * M4(b, c, 0) + M4(a, 1, row) * M4(b, c, 1) + M4(a, 2, row) * M4(b, c, 2) +
                            M4(a, 3, row) * M4(b, c, 3);
}

/* makeSplatCamera (splat_math.cpp:9-27) and splatCameraFromViewer (splat_math.cpp:29-42). */
void gsr_oracle_camera_from_viewer(const float* view, const float* proj, const float* model, uint32_t width,
                                   uint32_t height, GsrOracleCamera* cam) {
    float flip[16], fv[16];
    for (int i = 0; i < 16; ++i) flip[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    M4(flip, 1, 1) = -1.0f;
    M4(flip, 2, 2) = -1.0f;
    mul4(flip, view, fv);
    mul4(fv, model, cam->viewInria);
    const float tanHalfFovX = 1.0f / M4(proj, 0, 0);
    const float tanHalfFovY = 1.0f / fabsf(M4(proj, 1, 1));
    const float* V = cam->viewInria;
    /* position = -(transpose(R) * t), t = column 3 */
    for (int r = 0; r < 3; ++r)
        cam->position[r] = -(M4(V, r, 0) * M4(V, 3, 0) + M4(V, r, 1) * M4(V, 3, 1) + M4(V, r, 2) * M4(V, 3, 2));
    cam->width = width;
    cam->height = height;
    cam->tanHalfFovX = tanHalfFovX;
    cam->tanHalfFovY = tanHalfFovY;
    cam->focalX = (float)width / (2.0f * tanHalfFovX);
    cam->focalY = (float)height / (2.0f * tanHalfFovY);
    cam->tilesX = (width + kTileSize - 1) / kTileSize;
    cam->tilesY = (height + kTileSize - 1) / kTileSize;
}

/* ---- per-gaussian math (splat_math.cpp) ---------------------------------------------- */
/* quaternionToMatrix (splat_math.cpp:44-53) + computeCov3D (55-63); S[c*3 + r]. */
static void cov3d(const float sigma[3], const float q[4], float S[9]) {
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    float R[9];
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + r * z); R[2] = 2.0f * (x * z - r * y);
    R[3] = 2.0f * (x * y - r * z); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + r * x);
    R[6] = 2.0f * (x * z + r * y); R[7] = 2.0f * (y * z - r * x); R[8] = 1.0f - 2.0f * (x * x + y * y);
    float M[9];
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) M[c * 3 + k] = R[c * 3 + k] * sigma[c];
    for (int c = 0; c < 3; ++c)
        for (int row = 0; row < 3; ++row)
            S[c * 3 + row] = M[0 * 3 + row] * M[0 * 3 + c] + M[1 * 3 + row] * M[1 * 3 + c] + M[2 * 3 + row] * M[2 * 3 + c];
}

/* computeCov2D (splat_math.cpp:65-91). */
static void cov2d(const float t[3], const float S[9], const GsrOracleCamera* cam, float out[3]) {
    const float limX = kFrustumClampFactor * cam->tanHalfFovX;
    const float limY = kFrustumClampFactor * cam->tanHalfFovY;
    const float txtz = t[0] / t[2];
    const float tytz = t[1] / t[2];
    const float tx = smin(limX, smax(-limX, txtz)) * t[2];
    const float ty = smin(limY, smax(-limY, tytz)) * t[2];
    const float tz = t[2];
    float J[6] = {0, 0, 0, 0, 0, 0}; /* J[c*2 + r], 3 columns x 2 rows */
    J[0 * 2 + 0] = cam->focalX / tz;
    J[2 * 2 + 0] = -(cam->focalX * tx) / (tz * tz);
    J[1 * 2 + 1] = cam->focalY / tz;
    J[2 * 2 + 1] = -(cam->focalY * ty) / (tz * tz);
    const float* V = cam->viewInria;
    float T[6], A[6];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 2; ++r)
            T[c * 2 + r] = J[0 * 2 + r] * M4(V, c, 0) + J[1 * 2 + r] * M4(V, c, 1) + J[2 * 2 + r] * M4(V, c, 2);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 2; ++r)
            A[c * 2 + r] = T[0 * 2 + r] * S[c * 3 + 0] + T[1 * 2 + r] * S[c * 3 + 1] + T[2 * 2 + r] * S[c * 3 + 2];
    float cov[4];
    for (int c = 0; c < 2; ++c)
        for (int r = 0; r < 2; ++r)
            cov[c * 2 + r] = A[0 * 2 + r] * T[0 * 2 + c] + A[1 * 2 + r] * T[1 * 2 + c] + A[2 * 2 + r] * T[2 * 2 + c];
    out[0] = cov[0] + kLowPassFilter;
    out[1] = cov[1];
    out[2] = cov[3] + kLowPassFilter;
}

/* conicAndRadius (splat_math.cpp:102-114). */
static int conicAndRadius(const float cov[3], float conic[3], float* radius) {
    const float det = cov[0] * cov[2] - cov[1] * cov[1];
    if (det == 0.0f) return 0;
    const float detInv = 1.0f / det;
    conic[0] = cov[2] * detInv;
    conic[1] = -cov[1] * detInv;
    conic[2] = cov[0] * detInv;
    const float mid = 0.5f * (cov[0] + cov[2]);
    const float lambda1 = mid + sqrtf(smax(0.1f, mid * mid - det));
    const float lambda2 = mid - sqrtf(smax(0.1f, mid * mid - det));
    *radius = ceilf(3.0f * sqrtf(smax(lambda1, lambda2)));
    return 1;
}

typedef struct { int minX, minY, maxX, maxY; } TileRect;
/* computeTileRect (splat_math.cpp:116-127). */
static TileRect tileRect(const float p[2], float radius, uint32_t tilesX, uint32_t tilesY) {
    const int gx = (int)tilesX, gy = (int)tilesY;
    const int r = ftoi(radius);
    TileRect t;
    t.minX = imin(gx, imax(0, ftoi((p[0] - (float)r) / (float)kTileSize)));
    t.minY = imin(gy, imax(0, ftoi((p[1] - (float)r) / (float)kTileSize)));
    t.maxX = imin(gx, imax(0, ftoi((p[0] + (float)r + (float)(kTileSize - 1)) / (float)kTileSize)));
    t.maxY = imin(gy, imax(0, ftoi((p[1] + (float)r + (float)(kTileSize - 1)) / (float)kTileSize)));
    return t;
}
static int rectEmpty(TileRect t) { return t.maxX <= t.minX || t.maxY <= t.minY; }

/* evalSH (splat_math.cpp:129-151); sh = RGB triplets. */
static void evalSH(int degree, const float* sh, const float dir[3], float out[3]) {
    float res[3];
    for (int c = 0; c < 3; ++c) res[c] = kShC0 * sh[c];
    if (degree > 0) {
        const float x = dir[0], y = dir[1], z = dir[2];
        const float a = kShC1 * y, b = kShC1 * z, d = kShC1 * x;
        for (int c = 0; c < 3; ++c) res[c] = res[c] - a * sh[3 + c] + b * sh[6 + c] - d * sh[9 + c];
        if (degree > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float t4 = kShC2[0] * xy, t5 = kShC2[1] * yz, t6 = kShC2[2] * (2.0f * zz - xx - yy);
            const float t7 = kShC2[3] * xz, t8 = kShC2[4] * (xx - yy);
            for (int c = 0; c < 3; ++c)
                res[c] = res[c] + t4 * sh[12 + c] + t5 * sh[15 + c] + t6 * sh[18 + c] + t7 * sh[21 + c] + t8 * sh[24 + c];
            if (degree > 2) {
                const float t9 = kShC3[0] * y * (3.0f * xx - yy), t10 = kShC3[1] * xy * z;
                const float t11 = kShC3[2] * y * (4.0f * zz - xx - yy);
                const float t12 = kShC3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
                const float t13 = kShC3[4] * x * (4.0f * zz - xx - yy), t14 = kShC3[5] * z * (xx - yy);
                const float t15 = kShC3[6] * x * (xx - 3.0f * yy);
                for (int c = 0; c < 3; ++c)
                    res[c] = res[c] + t9 * sh[27 + c] + t10 * sh[30 + c] + t11 * sh[33 + c] + t12 * sh[36 + c] +
                             t13 * sh[39 + c] + t14 * sh[42 + c] + t15 * sh[45 + c];
            }
        }
    }
    for (int c = 0; c < 3; ++c) {
        res[c] = res[c] + 0.5f;
        out[c] = smax(res[c], 0.0f); /* glm::max(v, 0): (v < 0) ? 0 : v */
    }
}

/* preprocessGaussian (splat_math.cpp:153-193); gpuRules adds splat_preprocess.comp:159-177. */
static void preprocessOne(const float* pa, const float* sc, const float* q, const float* sh, int degree,
                          const GsrOracleCamera* cam, int gpuRules, GsrOracleSplat* s) {
    memset(s, 0, sizeof(*s));
    const float* V = cam->viewInria;
    const float t[3] = {M4(V, 0, 0) * pa[0] + M4(V, 1, 0) * pa[1] + M4(V, 2, 0) * pa[2] + M4(V, 3, 0),
                        M4(V, 0, 1) * pa[0] + M4(V, 1, 1) * pa[1] + M4(V, 2, 1) * pa[2] + M4(V, 3, 1),
                        M4(V, 0, 2) * pa[0] + M4(V, 1, 2) * pa[1] + M4(V, 2, 2) * pa[2] + M4(V, 3, 2)};
    s->depth = t[2];
    if (gpuRules ? !(t[2] > kNearCullDepth) : (t[2] <= kNearCullDepth)) {
        s->cullReason = GSR_ORACLE_CULL_NEAR;
        return;
    }
    if (gpuRules && pa[3] < kMinAlpha) {
        s->cullReason = GSR_ORACLE_CULL_LOW_OPACITY;
        return;
    }
    float S[9], cov[3], conic[3], radius = 0.0f;
    cov3d(sc, q, S);
    cov2d(t, S, cam, cov);
    if (!conicAndRadius(cov, conic, &radius)) {
        s->cullReason = GSR_ORACLE_CULL_SINGULAR;
        return;
    }
    /* projectToPixel (splat_math.cpp:93-100) */
    const float ndcX = t[0] / (t[2] * cam->tanHalfFovX);
    const float ndcY = t[1] / (t[2] * cam->tanHalfFovY);
    const float center[2] = {((ndcX + 1.0f) * (float)cam->width - 1.0f) * 0.5f,
                             ((ndcY + 1.0f) * (float)cam->height - 1.0f) * 0.5f};
    if (rectEmpty(tileRect(center, radius, cam->tilesX, cam->tilesY))) {
        s->center[0] = center[0];
        s->center[1] = center[1];
        s->cullReason = GSR_ORACLE_CULL_OFFSCREEN;
        return;
    }
    const float dv[3] = {pa[0] - cam->position[0], pa[1] - cam->position[1], pa[2] - cam->position[2]};
    float dir[3];
    normalize3(dv, dir);
    evalSH(degree, sh, dir, s->color);
    s->center[0] = center[0];
    s->center[1] = center[1];
    s->conicOpacity[0] = conic[0];
    s->conicOpacity[1] = conic[1];
    s->conicOpacity[2] = conic[2];
    s->conicOpacity[3] = pa[3];
    s->radius = radius;
    s->cullReason = GSR_ORACLE_CULL_VISIBLE;
}

void gsr_oracle_preprocess_degrees(uint32_t n, const float* posAlpha, const float* scales, const float* rotations,
                                   const float* sh, uint32_t K, int degree, const uint8_t* degrees,
                                   const GsrOracleCamera* cam, int gpuRules, GsrOracleSplat* out) {
    for (uint32_t i = 0; i < n; ++i) {
        int d = degree;
        if (degrees && (int)degrees[i] < d) d = degrees[i];
        preprocessOne(posAlpha + 4 * (size_t)i, scales + 4 * (size_t)i, rotations + 4 * (size_t)i,
                      sh + (size_t)i * K * 3, d, cam, gpuRules, &out[i]);
    }
}

void gsr_oracle_preprocess(uint32_t n, const float* posAlpha, const float* scales, const float* rotations,
                           const float* sh, uint32_t K, int degree, const GsrOracleCamera* cam, int gpuRules,
                           GsrOracleSplat* out) {
    gsr_oracle_preprocess_degrees(n, posAlpha, scales, rotations, sh, K, degree, NULL, cam, gpuRules, out);
}

/* ---- tight coverage (tile_coverage.cpp) ---------------------------------------------- */
typedef struct { float cx, cy, A, B, C, D, t, exPad, eyPad; int valid; } Ellipse;
typedef struct { int x0, y0, x1, y1; } BinRect;
typedef struct { BinRect bins; Ellipse e; int useEllipse; } Coverage;

/* makeCutoffEllipse (tile_coverage.cpp:24-50). */
static Ellipse makeEllipse(const float c[2], const float conic[3], float opacity) {
    Ellipse e;
    memset(&e, 0, sizeof(e));
    e.cx = c[0];
    e.cy = c[1];
    const float A = conic[0], B = conic[1], C = conic[2];
    const float D = A * C - B * B;
    e.A = A; e.B = B; e.C = C; e.D = D;
    e.t = -1.0f;
    e.valid = A > 0.0f && C > 0.0f && D > 0.0f;
    if (!e.valid) return e;
    if (!(opacity >= kMinAlpha)) return e;
    const float qmax = 2.0f * logf(255.0f * opacity);
    const float rho = fabsf(B) / sqrtf(A * C);
    const float K = 2.0f / smax(1.0f - rho, 1e-30f);
    const float t = qmax + (1e-3f + 2e-5f * K) * smax(qmax, 1.0f) + 2e-3f;
    if (!(t < 1e30f)) {
        e.valid = 0;
        return e;
    }
    e.t = t;
    const float ex = sqrtf(t * C / D);
    const float ey = sqrtf(t * A / D);
    e.exPad = ex + (0.02f + 2e-3f * ex);
    e.eyPad = ey + (0.02f + 2e-3f * ey);
    return e;
}

/* floorDivClamped (tile_coverage.cpp:54). */
static int floorDivClamped(float v, int S) { return ftoi(floorf(sclamp(v, -65536.0f, 1048576.0f) / (float)S)); }

/* The bins of the binning grid: sx x sy pixels. The reference's bins are square, S x S with
 * S = 16 or 8 (tile_coverage.cpp); S = 32 here names 32 x 8 bins (wide bins of 256 pixels, as
 * many as a 16 x 16 tile), for which every S below is the bin's width along x and its height
 * along y. With sx = sy = S every expression is the reference's. */
typedef struct { int sx, sy; } BinShape;
static BinShape binShape(int S) {
    BinShape b = {S, S == 32 ? 8 : S};
    return b;
}

/* ellipseRows (tile_coverage.cpp:56-63). */
static void ellipseRows(const Ellipse* e, BinShape bs, const BinRect* b, int* lo, int* hi) {
    if (e->t < 0.0f) {
        *lo = 0;
        *hi = 0;
        return;
    }
    const float y0 = ceilf(e->cy - e->eyPad);
    const float y1 = floorf(e->cy + e->eyPad);
    const int l = imax(b->y0, floorDivClamped(y0, bs.sy));
    const int h = imin(b->y1, floorDivClamped(y1, bs.sy) + 1);
    *lo = l;
    *hi = imax(l, h);
}

/* ellipseRowBounds (tile_coverage.cpp:70-88). Returns 0 if the strip is empty. */
static int rowBounds(const Ellipse* e, int row, BinShape bs, float* x0, float* x1) {
    const float ey0 = (float)(row * bs.sy) - e->cy;
    const float ey1 = (float)(row * bs.sy + bs.sy - 1) - e->cy;
    const float lo = smax(ey0, -e->eyPad);
    const float hi = smin(ey1, e->eyPad);
    if (!(lo <= hi)) return 0;
    const float exTrue = sqrtf(e->t * e->C / e->D);
    const float eyRight = sclamp(-e->B * exTrue / e->C, lo, hi);
    const float eyLeft = sclamp(e->B * exTrue / e->C, lo, hi);
    const float At = e->A * e->t;
    const float xRight = (-e->B * eyRight + sqrtf(smax(0.0f, At - e->D * eyRight * eyRight))) / e->A;
    const float xLeft = (-e->B * eyLeft - sqrtf(smax(0.0f, At - e->D * eyLeft * eyLeft))) / e->A;
    const float pad = 0.02f + 2e-3f * exTrue;
    *x0 = e->cx + xLeft - pad;
    *x1 = e->cx + xRight + pad;
    return 1;
}

/* ellipseRowSpan (tile_coverage.cpp:90-96). */
static void ellipseRowSpan(const Ellipse* e, int row, BinShape bs, const BinRect* b, int* x0, int* x1) {
    float fx0, fx1;
    if (!rowBounds(e, row, bs, &fx0, &fx1)) {
        *x0 = b->x0;
        *x1 = b->x0;
        return;
    }
    const int a = imax(b->x0, floorDivClamped(ceilf(fx0), bs.sx));
    const int c = imin(b->x1, floorDivClamped(floorf(fx1), bs.sx) + 1);
    *x0 = a;
    *x1 = imax(a, c);
}

/* rectToBins (tile_coverage.cpp:102-105): the bins holding the 16-px rectangle's pixels (its
 * first bin rounds down, its end up; for bins that divide 16 this is the reference's r * 16 / S). */
static BinRect rectToBins(TileRect r, BinShape bs, int gx, int gy) {
    BinRect b = {r.minX * 16 / bs.sx, r.minY * 16 / bs.sy, imin((r.maxX * 16 + bs.sx - 1) / bs.sx, gx),
                 imin((r.maxY * 16 + bs.sy - 1) / bs.sy, gy)};
    return b;
}

/* makeCoverage (tile_coverage.cpp:107-117). */
static Coverage makeCoverage(uint32_t mode, TileRect rect16, BinShape bs, int gx, int gy, const float center[2],
                             const float conic[3], float opacity) {
    Coverage cv;
    memset(&cv, 0, sizeof(cv));
    if (mode == GSR_ORACLE_BOUNDS_CUTOFF) {
        BinRect all = {0, 0, gx, gy};
        cv.bins = all;
    } else {
        cv.bins = rectToBins(rect16, bs, gx, gy);
    }
    cv.e.t = -1.0f;
    if (mode != GSR_ORACLE_BOUNDS_RECT) {
        cv.e = makeEllipse(center, conic, opacity);
        cv.useEllipse = cv.e.valid;
        if (!cv.e.valid && mode == GSR_ORACLE_BOUNDS_CUTOFF) cv.bins = rectToBins(rect16, bs, gx, gy);
    }
    return cv;
}

/* coverageRows / coverageRowSpan (tile_coverage.cpp:119-127). */
static void coverageRows(const Coverage* cv, BinShape bs, int* r0, int* r1) {
    if (!cv->useEllipse) {
        *r0 = cv->bins.y0;
        *r1 = imax(cv->bins.y0, cv->bins.y1);
        return;
    }
    ellipseRows(&cv->e, bs, &cv->bins, r0, r1);
}
static void coverageRowSpan(const Coverage* cv, int row, BinShape bs, int* x0, int* x1) {
    if (!cv->useEllipse) {
        *x0 = cv->bins.x0;
        *x1 = imax(cv->bins.x0, cv->bins.x1);
        return;
    }
    ellipseRowSpan(&cv->e, row, bs, &cv->bins, x0, x1);
}

/* coverageCount (tile_coverage.cpp:129-138). */
static uint32_t coverageCount(const Coverage* cv, BinShape bs) {
    int r0, r1;
    coverageRows(cv, bs, &r0, &r1);
    if (!cv->useEllipse) return (uint32_t)(imax(0, cv->bins.x1 - cv->bins.x0) * (r1 - r0));
    uint32_t n = 0;
    for (int r = r0; r < r1; ++r) {
        int x0, x1;
        ellipseRowSpan(&cv->e, r, bs, &cv->bins, &x0, &x1);
        n += (uint32_t)(x1 - x0);
    }
    return n;
}

/* splatCoverage (tile_coverage.cpp:140-144). */
static Coverage splatCoverage(uint32_t mode, const GsrOracleSplat* s, const GsrOracleCamera* cam, BinShape bs) {
    const int gx = (int)((cam->width + bs.sx - 1) / bs.sx), gy = (int)((cam->height + bs.sy - 1) / bs.sy);
    const TileRect rect = tileRect(s->center, s->radius, cam->tilesX, cam->tilesY);
    return makeCoverage(mode, rect, bs, gx, gy, s->center, s->conicOpacity, s->conicOpacity[3]);
}

void gsr_oracle_coverage_counts(uint32_t n, const GsrOracleSplat* splats, const GsrOracleCamera* cam, uint32_t bounds,
                                int S, uint32_t* counts) {
    for (uint32_t i = 0; i < n; ++i) {
        if (splats[i].cullReason != GSR_ORACLE_CULL_VISIBLE) {
            counts[i] = 0;
            continue;
        }
        const Coverage cv = splatCoverage(bounds, &splats[i], cam, binShape(S));
        counts[i] = coverageCount(&cv, binShape(S));
    }
}

uint32_t gsr_oracle_coverage_tiles(const GsrOracleSplat* s, const GsrOracleCamera* cam, uint32_t bounds, int S,
                                   uint32_t* tiles, uint32_t cap) {
    const BinShape bs = binShape(S);
    const int gx = (int)((cam->width + bs.sx - 1) / bs.sx);
    const Coverage cv = splatCoverage(bounds, s, cam, bs);
    int r0, r1;
    coverageRows(&cv, bs, &r0, &r1);
    uint32_t k = 0;
    for (int r = r0; r < r1; ++r) {
        int x0, x1;
        coverageRowSpan(&cv, r, bs, &x0, &x1);
        for (int x = x0; x < x1; ++x) {
            if (k < cap) tiles[k] = (uint32_t)(r * gx + x);
            ++k;
        }
    }
    return k;
}

static int nearInteger(float v, float eps) { return fabsf(v - roundf(v)) < eps; }

/* coverageIsBorderline (tile_coverage.cpp:146-164). */
int gsr_oracle_coverage_borderline(const GsrOracleSplat* s, const GsrOracleCamera* cam, uint32_t bounds, int S,
                                   float eps) {
    const BinShape bs = binShape(S);
    const Coverage cv = splatCoverage(bounds, s, cam, bs);
    if (!cv.useEllipse || cv.e.t < 0.0f) return 0;
    const float rho = fabsf(cv.e.B) / sqrtf(cv.e.A * cv.e.C);
    const float K = 2.0f / smax(1.0f - rho, 1e-30f);
    eps += (1e-7f * K + 1e-12f * K * K) * (cv.e.exPad + cv.e.eyPad);
    if (nearInteger(cv.e.cy - cv.e.eyPad, eps) || nearInteger(cv.e.cy + cv.e.eyPad, eps)) return 1;
    int r0, r1;
    coverageRows(&cv, bs, &r0, &r1);
    for (int r = r0; r < r1; ++r) {
        float x0, x1;
        if (!rowBounds(&cv.e, r, bs, &x0, &x1)) continue;
        if (nearInteger(x0, eps) || nearInteger(x1, eps)) return 1;
        const float ey0 = (float)(r * bs.sy) - cv.e.cy, ey1 = (float)(r * bs.sy + bs.sy - 1) - cv.e.cy;
        if (fabsf(ey1 + cv.e.eyPad) < eps || fabsf(ey0 - cv.e.eyPad) < eps) return 1;
    }
    return 0;
}

/* ---- the global-mode tile list (tile_duplicate.comp:177-221, radix sort, tile_ranges.comp) */
typedef struct { uint32_t tile, depth, value, pos; } Entry;
static int entryCmp(const void* a, const void* b) {
    const Entry* x = (const Entry*)a;
    const Entry* y = (const Entry*)b;
    if (x->tile != y->tile) return x->tile < y->tile ? -1 : 1;
    if (x->depth != y->depth) return x->depth < y->depth ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

uint64_t gsr_oracle_tile_list(uint32_t n, const GsrOracleSplat* splats, const uint32_t* counts,
                              const GsrOracleCamera* cam, uint32_t bounds, int S, uint32_t capacity, uint32_t* keysLo,
                              uint32_t* keysHi, uint32_t* values, uint32_t* ranges) {
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) total += counts[i];
    const uint64_t kept = total < capacity ? total : capacity;
    Entry* e = (Entry*)malloc(sizeof(Entry) * (kept ? kept : 1));
    uint32_t* tiles = NULL;
    uint32_t tilesCap = 0;
    uint64_t k = 0;
    for (uint32_t i = 0; i < n && k < kept; ++i) {
        if (counts[i] == 0) continue;
        if (counts[i] > tilesCap) {
            tilesCap = counts[i];
            tiles = (uint32_t*)realloc(tiles, sizeof(uint32_t) * tilesCap);
        }
        const uint32_t m = gsr_oracle_coverage_tiles(&splats[i], cam, bounds, S, tiles, tilesCap);
        for (uint32_t j = 0; j < counts[i] && k < kept; ++j, ++k) {
            e[k].tile = j < m ? tiles[j] : ((cam->width + binShape(S).sx - 1) / binShape(S).sx) *
                                               ((cam->height + binShape(S).sy - 1) / binShape(S).sy);
            e[k].depth = fbits(splats[i].depth);
            e[k].value = i;
            e[k].pos = (uint32_t)k;
        }
    }
    free(tiles);
    qsort(e, (size_t)kept, sizeof(Entry), entryCmp);
    const uint32_t T = ((cam->width + binShape(S).sx - 1) / binShape(S).sx) * ((cam->height + binShape(S).sy - 1) / binShape(S).sy);
    if (ranges) memset(ranges, 0, sizeof(uint32_t) * 2 * T);
    for (uint64_t j = 0; j < kept; ++j) {
        if (keysLo) keysLo[j] = e[j].depth;
        if (keysHi) keysHi[j] = e[j].tile;
        if (values) values[j] = e[j].value;
        const uint32_t t = e[j].tile;
        if (ranges && t < T) {
            if (j == 0 || e[j - 1].tile != t) ranges[2 * t] = (uint32_t)j;
            ranges[2 * t + 1] = (uint32_t)(j + 1);
        }
    }
    free(e);
    return total;
}

/* ---- depth sort (depth_sort.cpp) --------------------------------------------------------- */
/* radixSortPairs (depth_sort.cpp:46-75). */
uint32_t gsr_oracle_radix_sort_pairs(uint32_t n, uint32_t* keys, uint32_t* values) {
    uint32_t* kt = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* vt = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* k = keys;
    uint32_t* v = values;
    uint32_t passes = 0;
    for (uint32_t shift = 0; shift < 32; shift += 8) {
        uint32_t hist[256];
        memset(hist, 0, sizeof(hist));
        for (uint32_t i = 0; i < n; ++i) hist[(k[i] >> shift) & 0xFFu]++;
        if (n == 0 || hist[(k[0] >> shift) & 0xFFu] == n) continue;
        uint32_t sum = 0;
        for (int d = 0; d < 256; ++d) {
            const uint32_t c = hist[d];
            hist[d] = sum;
            sum += c;
        }
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t dst = hist[(k[i] >> shift) & 0xFFu]++;
            kt[dst] = k[i];
            vt[dst] = v[i];
        }
        uint32_t* tk = k; k = kt; kt = tk;
        uint32_t* tv = v; v = vt; vt = tv;
        ++passes;
    }
    if (k != keys) {
        memcpy(keys, k, sizeof(uint32_t) * n);
        memcpy(values, v, sizeof(uint32_t) * n);
        kt = k;
        vt = v;
    }
    free(kt);
    free(vt);
    return passes;
}

/* DepthSorter::sort (depth_sort.cpp:17-44) with viewDepth (splat_math.h:70-72). */
uint32_t gsr_oracle_depth_sort(uint32_t n, const float* posAlpha, const float* V, uint32_t* order, uint32_t* keys) {
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float* p = posAlpha + 4 * (size_t)i;
        const float z = M4(V, 0, 2) * p[0] + M4(V, 1, 2) * p[1] + M4(V, 2, 2) * p[2] + M4(V, 3, 2);
        if (!(z > kNearCullDepth)) continue;
        keys[m] = fbits(z);
        order[m] = i;
        ++m;
    }
    gsr_oracle_radix_sort_pairs(m, keys, order);
    return m;
}

/* ---- computeRayDepthParams (splat_math.cpp:195-205) and RayDepthParams::depthAt
 *      (splat_math.h:134-141), the StopThePop window's per-gaussian ray depth ------------- */
static void rayDepthParams(const float* sigma, const float* q, const float t[3], const float* V, float out[9]) {
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    float R[9]; /* quaternionToMatrix, R[c*3 + row] */
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + r * z); R[2] = 2.0f * (x * z - r * y);
    R[3] = 2.0f * (x * y - r * z); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + r * x);
    R[6] = 2.0f * (x * z + r * y); R[7] = 2.0f * (y * z - r * x); R[8] = 1.0f - 2.0f * (x * x + y * y);
    float M[9]; /* mat3(viewInria) * R */
    for (int c = 0; c < 3; ++c)
        for (int row = 0; row < 3; ++row)
            M[c * 3 + row] = M4(V, 0, row) * R[c * 3 + 0] + M4(V, 1, row) * R[c * 3 + 1] + M4(V, 2, row) * R[c * 3 + 2];
    const float sMax = smax(sigma[0], smax(sigma[1], sigma[2]));
    const float floorS = smax(1e-4f * sMax, 1e-12f);
    float w[3];
    for (int k = 0; k < 3; ++k) {
        const float sk = smax(sigma[k], floorS);
        w[k] = 1.0f / (sk * sk);
    }
    float P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) P[i * 3 + j] = P[i * 3 + j] + w[k] * (M[k * 3 + j] * M[k * 3 + i]);
    float b[3];
    for (int row = 0; row < 3; ++row) b[row] = P[0 * 3 + row] * t[0] + P[1 * 3 + row] * t[1] + P[2 * 3 + row] * t[2];
    const float o[9] = {P[0], P[1], P[2], P[4], P[5], P[8], b[0], b[1], b[2]};
    memcpy(out, o, sizeof(o));
}
static float rayDepthAt(const float* p, float vx, float vy) {
    const float vPv = p[0] * vx * vx + 2.0f * p[1] * vx * vy + 2.0f * p[2] * vx + p[3] * vy * vy + 2.0f * p[4] * vy + p[5];
    const float vb = p[6] * vx + p[7] * vy + p[8];
    return vb / vPv;
}

/* ---- renderReference (reference_renderer.cpp:41-234), with the StopThePop window -------- */
typedef struct {
    uint32_t n, K;
    int degree;
    const float *posAlpha, *scales, *rotations, *sh;
    const GsrOracleCamera* cam;
    GsrOracleSplat* splats;
} PreCtx;
static void preTask(uint32_t i, void* p) {
    PreCtx* c = (PreCtx*)p;
    preprocessOne(c->posAlpha + 4 * (size_t)i, c->scales + 4 * (size_t)i, c->rotations + 4 * (size_t)i,
                  c->sh + (size_t)i * c->K * 3, c->degree, c->cam, 0, &c->splats[i]);
}

typedef struct {
    const GsrOracleCamera* cam;
    const GsrOracleSplat* splats;
    const uint32_t *tileStart, *tileLists;
    float* rgb;
    int earlyTermination;
    uint32_t sortWindow;    /* 0: off; GSR_ORACLE_EXACT_PIXEL_SORT: every pixel sorts all its splats */
    const float* rayDepth;  /* 9 floats per gaussian (rayDepthParams) */
    _Atomic uint64_t evaluated, blended, terminated;
} RasterCtx;

typedef struct {
    float depth, alpha, color[3];
} Pending;

/* the reference's blend lambda (reference_renderer.cpp:150-159) */
static void blendPending(const Pending* e, float* T, float* C, int* done, uint64_t* bl, uint64_t* te) {
    const float testT = *T * (1.0f - e->alpha);
    if (testT < kMinTransmittance) {
        *done = 1;
        ++*te;
        return;
    }
    for (int ch = 0; ch < 3; ++ch) C[ch] = C[ch] + e->color[ch] * e->alpha * *T;
    *T = testT;
    ++*bl;
}

/* std::stable_sort by depth (a.depth < b.depth): a bottom-up merge sort */
static void stableSortByDepth(Pending* a, size_t n) {
    if (n < 2) return;
    Pending* tmp = (Pending*)malloc(sizeof(Pending) * n);
    for (size_t w = 1; w < n; w *= 2) {
        for (size_t lo = 0; lo < n; lo += 2 * w) {
            const size_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            size_t i = lo, j = mid, k = lo;
            while (i < mid && j < hi) tmp[k++] = (a[j].depth < a[i].depth) ? a[j++] : a[i++];
            while (i < mid) tmp[k++] = a[i++];
            while (j < hi) tmp[k++] = a[j++];
        }
        memcpy(a, tmp, sizeof(Pending) * n);
    }
    free(tmp);
}

/* One pixel with the window (reference_renderer.cpp:143-196). */
static void windowPixel(const RasterCtx* c, uint32_t s0, uint32_t s1, float px, float py, Pending* win, float* T,
                        float* C, uint64_t* ev, uint64_t* bl, uint64_t* te) {
    const GsrOracleCamera* cam = c->cam;
    const float vx = (px - 0.5f * ((float)cam->width - 1.0f)) / cam->focalX;
    const float vy = (py - 0.5f * ((float)cam->height - 1.0f)) / cam->focalY;
    const int exact = c->sortWindow == GSR_ORACLE_EXACT_PIXEL_SORT;
    const size_t K = c->sortWindow;
    size_t wn = 0;
    int done = 0;
    for (uint32_t j = s0; j < s1 && !done; ++j) {
        const uint32_t g = c->tileLists[j];
        const GsrOracleSplat* s = &c->splats[g];
        ++*ev;
        const float dx = s->center[0] - px;
        const float dy = s->center[1] - py;
        const float* co = s->conicOpacity;
        const float power = -0.5f * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
        if (power > 0.0f) continue;
        const float alpha = fminf(kMaxAlpha, co[3] * expf(power));
        if (alpha < kMinAlpha) continue;
        Pending e;
        e.depth = rayDepthAt(c->rayDepth + (size_t)g * 9, vx, vy);
        e.alpha = alpha;
        memcpy(e.color, s->color, sizeof(e.color));
        if (exact) {
            win[wn++] = e;
        } else if (wn == K) {
            if (e.depth < win[0].depth) {
                blendPending(&e, T, C, &done, bl, te);
                continue;
            }
            blendPending(&win[0], T, C, &done, bl, te);
            size_t i = 0;
            for (; i + 1 < K && win[i + 1].depth <= e.depth; ++i) win[i] = win[i + 1];
            win[i] = e;
        } else {
            size_t i = wn++;
            for (; i > 0 && win[i - 1].depth > e.depth; --i) win[i] = win[i - 1];
            win[i] = e;
        }
    }
    if (exact) stableSortByDepth(win, wn);
    for (size_t i = 0; i < wn && !done; ++i) blendPending(&win[i], T, C, &done, bl, te);
}
static void rasterTask(uint32_t tile, void* p) {
    RasterCtx* c = (RasterCtx*)p;
    const GsrOracleCamera* cam = c->cam;
    const uint32_t tx = tile % cam->tilesX, ty = tile / cam->tilesX;
    const uint32_t s0 = c->tileStart[tile], s1 = c->tileStart[tile + 1];
    uint64_t ev = 0, bl = 0, te = 0;
    const uint32_t x0 = tx * kTileSize, y0 = ty * kTileSize;
    const uint32_t x1 = cam->width < x0 + kTileSize ? cam->width : x0 + kTileSize;
    const uint32_t y1 = cam->height < y0 + kTileSize ? cam->height : y0 + kTileSize;
    Pending* win = NULL;
    if (c->sortWindow > 0) {
        const size_t cap = c->sortWindow == GSR_ORACLE_EXACT_PIXEL_SORT ? (size_t)(s1 - s0) : c->sortWindow;
        win = (Pending*)malloc(sizeof(Pending) * (cap ? cap : 1));
    }
    for (uint32_t y = y0; y < y1; ++y) {
        for (uint32_t x = x0; x < x1; ++x) {
            const float px = (float)x, py = (float)y;
            float T = 1.0f, C[3] = {0.0f, 0.0f, 0.0f};
            if (win) {
                windowPixel(c, s0, s1, px, py, win, &T, C, &ev, &bl, &te);
                float* dst = &c->rgb[((size_t)y * cam->width + x) * 3];
                for (int ch = 0; ch < 3; ++ch) dst[ch] = C[ch] + T * 0.0f;
                continue;
            }
            for (uint32_t j = s0; j < s1; ++j) {
                const GsrOracleSplat* s = &c->splats[c->tileLists[j]];
                ++ev;
                /* splatAlphaAt (splat_math.h:147-156) */
                const float dx = s->center[0] - px;
                const float dy = s->center[1] - py;
                const float* co = s->conicOpacity;
                const float power = -0.5f * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
                if (power > 0.0f) continue;
                const float alpha = fminf(kMaxAlpha, co[3] * expf(power));
                if (alpha < kMinAlpha) continue;
                const float testT = T * (1.0f - alpha);
                if (c->earlyTermination && testT < kMinTransmittance) {
                    ++te;
                    break;
                }
                for (int ch = 0; ch < 3; ++ch) C[ch] = C[ch] + s->color[ch] * alpha * T;
                T = testT;
                ++bl;
            }
            float* dst = &c->rgb[((size_t)y * cam->width + x) * 3];
            /* C + T * background (black) */
            for (int ch = 0; ch < 3; ++ch) dst[ch] = C[ch] + T * 0.0f;
        }
    }
    free(win);
    atomic_fetch_add(&c->evaluated, ev);
    atomic_fetch_add(&c->blended, bl);
    atomic_fetch_add(&c->terminated, te);
}

int gsr_oracle_render(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                      const float* sh, const GsrOracleCamera* cam, int maxShDegree, uint32_t bounds, uint32_t threads,
                      int earlyTermination, uint32_t sortWindow, float* rgb, GsrOracleRenderStats* stats) {
    const double tStart = nowMs();
    const unsigned nt = threads ? threads : hardwareThreads();
    const uint32_t K = (uint32_t)((shDegree + 1) * (shDegree + 1));
    memset(rgb, 0, sizeof(float) * 3 * (size_t)cam->width * cam->height);
    GsrOracleSplat* splats = (GsrOracleSplat*)malloc(sizeof(GsrOracleSplat) * (n ? n : 1));
    PreCtx pc = {n, K, shDegree < maxShDegree ? shDegree : maxShDegree, posAlpha, scales, rotations, sh, cam, splats};
    parallelFor(n, nt, 4096, preTask, &pc);
    GsrOracleRenderStats st;
    memset(&st, 0, sizeof(st));
    st.gaussians = n;
    st.threads = nt;
    for (uint32_t i = 0; i < n; ++i) {
        switch (splats[i].cullReason) {
            case GSR_ORACLE_CULL_VISIBLE: st.visible++; break;
            case GSR_ORACLE_CULL_NEAR: st.culledNear++; break;
            case GSR_ORACLE_CULL_SINGULAR: st.culledSingular++; break;
            case GSR_ORACLE_CULL_OFFSCREEN: st.culledOffScreen++; break;
            default: break;
        }
    }
    /* StopThePop: the ray-depth parameters of every visible gaussian (reference_renderer.cpp:60-70) */
    float* rayDepth = NULL;
    if (sortWindow > 0) {
        rayDepth = (float*)calloc((size_t)(n ? n : 1) * 9, sizeof(float));
        const float* V = cam->viewInria;
        for (uint32_t i = 0; i < n; ++i) {
            if (splats[i].cullReason != GSR_ORACLE_CULL_VISIBLE) continue;
            const float* pa = posAlpha + 4 * (size_t)i;
            const float t[3] = {M4(V, 0, 0) * pa[0] + M4(V, 1, 0) * pa[1] + M4(V, 2, 0) * pa[2] + M4(V, 3, 0),
                                M4(V, 0, 1) * pa[0] + M4(V, 1, 1) * pa[1] + M4(V, 2, 1) * pa[2] + M4(V, 3, 1),
                                M4(V, 0, 2) * pa[0] + M4(V, 1, 2) * pa[1] + M4(V, 2, 2) * pa[2] + M4(V, 3, 2)};
            rayDepthParams(scales + 4 * (size_t)i, rotations + 4 * (size_t)i, t, V, rayDepth + (size_t)i * 9);
        }
    }
    const double tPre = nowMs();
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    const uint32_t m = gsr_oracle_depth_sort(n, posAlpha, cam->viewInria, order, keys);
    const double tSort = nowMs();

    const uint32_t tileCount = cam->tilesX * cam->tilesY;
    uint32_t* tileStart = (uint32_t*)calloc((size_t)tileCount + 1, sizeof(uint32_t));
    uint32_t* tiles = NULL;
    uint32_t tilesCap = 0;
    for (int phase = 0; phase < 2; ++phase) {
        uint32_t* cursor = NULL;
        uint32_t* lists = NULL;
        if (phase == 1) {
            for (uint32_t t = 0; t < tileCount; ++t) tileStart[t + 1] += tileStart[t];
            st.tileInstances = tileStart[tileCount];
            cursor = (uint32_t*)malloc(sizeof(uint32_t) * (tileCount ? tileCount : 1));
            memcpy(cursor, tileStart, sizeof(uint32_t) * tileCount);
            lists = (uint32_t*)malloc(sizeof(uint32_t) * (tileStart[tileCount] ? tileStart[tileCount] : 1));
        }
        for (uint32_t j = 0; j < m; ++j) {
            const uint32_t idx = order[j];
            const GsrOracleSplat* s = &splats[idx];
            if (s->cullReason != GSR_ORACLE_CULL_VISIBLE) continue;
            const Coverage cv = splatCoverage(bounds, s, cam, binShape(kTileSize));
            const uint32_t cnt = coverageCount(&cv, binShape(kTileSize));
            if (cnt > tilesCap) {
                tilesCap = cnt;
                tiles = (uint32_t*)realloc(tiles, sizeof(uint32_t) * tilesCap);
            }
            const uint32_t got = gsr_oracle_coverage_tiles(s, cam, bounds, kTileSize, tiles, tilesCap);
            for (uint32_t q = 0; q < got && q < tilesCap; ++q) {
                if (phase == 0) tileStart[tiles[q] + 1]++;
                else lists[cursor[tiles[q]]++] = idx;
            }
        }
        if (phase == 1) {
            const double tBin = nowMs();
            RasterCtx rc;
            rc.cam = cam;
            rc.splats = splats;
            rc.tileStart = tileStart;
            rc.tileLists = lists;
            rc.rgb = rgb;
            rc.earlyTermination = earlyTermination;
            rc.sortWindow = sortWindow;
            rc.rayDepth = rayDepth;
            atomic_init(&rc.evaluated, 0);
            atomic_init(&rc.blended, 0);
            atomic_init(&rc.terminated, 0);
            parallelFor(tileCount, nt, 1, rasterTask, &rc);
            const double tEnd = nowMs();
            st.evaluatedFragments = atomic_load(&rc.evaluated);
            st.blendedFragments = atomic_load(&rc.blended);
            st.terminatedPixels = atomic_load(&rc.terminated);
            st.preprocessMs = tPre - tStart;
            st.sortMs = tSort - tPre;
            st.binMs = tBin - tSort;
            st.rasterMs = tEnd - tBin;
            st.totalMs = tEnd - tStart;
            free(cursor);
            free(lists);
        }
    }
    free(rayDepth);
    free(tiles);
    free(tileStart);
    free(order);
    free(keys);
    free(splats);
    if (stats) *stats = st;
    return 0;
}

/* ---- half (src/scene/half.h) --------------------------------------------------------- */
uint16_t gsr_oracle_float_to_half(float value) {
    const uint32_t f = fbits(value);
    const uint32_t sign = (f >> 16) & 0x8000u;
    const uint32_t absBits = f & 0x7FFFFFFFu;
    if (absBits >= 0x7F800000u) return (uint16_t)(sign | 0x7C00u | (absBits > 0x7F800000u ? 0x200u : 0u));
    if (absBits >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);
    if (absBits < 0x38800000u) {
        if (absBits < 0x33000000u) return (uint16_t)sign;
        const uint32_t exponent = absBits >> 23;
        const uint32_t mantissa = (absBits & 0x7FFFFFu) | 0x800000u;
        const uint32_t shift = 126u - exponent;
        uint32_t half = mantissa >> shift;
        const uint32_t rest = mantissa & ((1u << shift) - 1u);
        const uint32_t halfway = 1u << (shift - 1u);
        if (rest > halfway || (rest == halfway && (half & 1u))) ++half;
        return (uint16_t)(sign | half);
    }
    uint32_t half = (absBits - 0x38000000u) >> 13;
    const uint32_t rest = absBits & 0x1FFFu;
    if (rest > 0x1000u || (rest == 0x1000u && (half & 1u))) ++half;
    return (uint16_t)(sign | half);
}

float gsr_oracle_half_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t exponent = (h >> 10) & 0x1Fu;
    const uint32_t mantissa = h & 0x3FFu;
    if (exponent == 0) {
        const float v = (float)mantissa * (1.0f / 16777216.0f);
        return sign ? -v : v;
    }
    if (exponent == 31) return bitsf(sign | 0x7F800000u | (mantissa << 13));
    return bitsf(sign | ((exponent + 112u) << 23) | (mantissa << 13));
}

static uint32_t packHalf2(float lo, float hi) {
    return (uint32_t)gsr_oracle_float_to_half(lo) | ((uint32_t)gsr_oracle_float_to_half(hi) << 16);
}
static float unpackLo(uint32_t w) { return gsr_oracle_half_to_float((uint16_t)(w & 0xFFFFu)); }
static float unpackHi(uint32_t w) { return gsr_oracle_half_to_float((uint16_t)(w >> 16)); }

/* ---- scene formats (scene_compression.cpp) ------------------------------------------- */
enum { FMT_F32 = 0, FMT_F16 = 1, FMT_Q8 = 2, FMT_CB = 3 };
enum { LAYOUT_SOA = 0, LAYOUT_SPLIT = 1, LAYOUT_AOS = 2 };
enum { GEOM_SOA = 0, GEOM_F32 = 1, GEOM_F16 = 2 };
enum { COL_SOA = 0, COL_F32 = 1, COL_F16 = 2, COL_Q8 = 3, COL_CB = 4 };
enum { VSH_OFF = 0, VSH_DEGREE = 1, VSH_COMPACT = 2 };

static uint32_t vec4sFor(uint32_t bytes) { return (bytes + 15u) / 16u; }
static uint32_t bandOf(uint32_t k) { return k < 4 ? 1u : k < 9 ? 2u : 3u; }
static uint32_t geometryRecordBytes(uint32_t g) { return g == GEOM_F16 ? 32u : 48u; }
static uint32_t colorRecordBytes(uint32_t c, uint32_t k) {
    switch (c) {
        case COL_SOA: return k * 3 * 4;
        case COL_F32: return vec4sFor(k * 3 * 4) * 16;
        case COL_F16: return vec4sFor(k * 3 * 2) * 16;
        case COL_Q8: return vec4sFor(12 + (k - 1) * 3) * 16;
        default: return 8;
    }
}

/* shBandMaxContribution / selectShDegree (scene_compression.cpp:53-68). */
static float shBandMax(const float* sh, int band) {
    if (band <= 0) return 0.0f;
    const int k0 = band * band, k1 = (band + 1) * (band + 1);
    float sq[3] = {0.0f, 0.0f, 0.0f};
    for (int k = k0; k < k1; ++k)
        for (int c = 0; c < 3; ++c) sq[c] = sq[c] + sh[k * 3 + c] * sh[k * 3 + c];
    const float norm = sqrtf(smax(sq[0], smax(sq[1], sq[2])));
    const float kInv4Pi = 0.07957747154594767f;
    return sqrtf((float)(2 * band + 1) * kInv4Pi) * norm;
}
int gsr_oracle_select_sh_degree(const float* sh, int storedDegree, float opacity, float threshold255) {
    const float threshold = threshold255 / 255.0f;
    for (int band = storedDegree; band >= 1; --band)
        if (opacity * shBandMax(sh, band) > threshold) return band;
    return 0;
}

/* quantizeBandQ8 (scene_compression.cpp:130-148). */
static uint16_t quantizeBandQ8(const float* v, uint32_t n, int8_t* q) {
    float m = 0.0f;
    for (uint32_t i = 0; i < n; ++i)
        if (isfinite(v[i])) m = smax(m, fabsf(v[i]));
    if (m == 0.0f) {
        memset(q, 0, n);
        return 0;
    }
    uint16_t h = gsr_oracle_float_to_half(m / 127.0f);
    if (h == 0) h = 1;
    while (gsr_oracle_half_to_float(h) * 127.0f < m) ++h;
    const float s = gsr_oracle_half_to_float(h);
    for (uint32_t i = 0; i < n; ++i) {
        const float x = isfinite(v[i]) ? v[i] / s : 0.0f;
        long r = lroundf(x);
        if (r < -127L) r = -127L;
        if (r > 127L) r = 127L;
        q[i] = (int8_t)r;
    }
    return h;
}

/* encodeScene (scene_compression.cpp:150-380) for f32/f16/q8 (the cb format is out of scope). */
int gsr_oracle_encode(uint32_t n, int shDegreeIn, const float* posAlpha, const float* scales, const float* rotations,
                      const float* sh, uint32_t format, uint32_t layout, int maxShDegree, float shThreshold,
                      uint32_t* desc, uint64_t* sizes, void** buffers) {
    if (format == FMT_CB || format > FMT_CB || layout > LAYOUT_AOS) return -1;
    if (format != FMT_F32 && layout == LAYOUT_SOA) return -1;
    int deg = shDegreeIn < maxShDegree ? shDegreeIn : maxShDegree;
    deg = deg < 0 ? 0 : deg > 3 ? 3 : deg;
    const uint32_t K = (uint32_t)((deg + 1) * (deg + 1));
    const uint32_t srcK = (uint32_t)((shDegreeIn + 1) * (shDegreeIn + 1));
    const int variable = shThreshold >= 0.0f && deg > 0;
    uint8_t* degrees = NULL;
    if (variable) {
        degrees = (uint8_t*)malloc(n ? n : 1);
        float c[48];
        for (uint32_t i = 0; i < n; ++i) {
            for (uint32_t k = 0; k < K * 3; ++k) c[k] = sh[(size_t)i * srcK * 3 + k];
            degrees[i] = (uint8_t)gsr_oracle_select_sh_degree(c, deg, posAlpha[4 * (size_t)i + 3], shThreshold);
        }
    }
#define KEPT(i) (variable ? (uint32_t)((degrees[i] + 1) * (degrees[i] + 1)) : K)
#define SHV(i, k, c) ((k) < KEPT(i) ? sh[((size_t)(i) * srcK + (k)) * 3 + (c)] : 0.0f)
    uint32_t geometry, color;
    uint32_t gStride = 0, cStride = 0, cOffset = 0, vsh = VSH_OFF;
    uint64_t sz[4] = {0, 0, 0, 0};
    uint32_t* out[4] = {NULL, NULL, NULL, NULL};
    const int fill = buffers != NULL;
    if (layout == LAYOUT_SOA) {
        geometry = GEOM_SOA;
        color = COL_SOA;
        size_t shFloats = (size_t)n * K * 3;
        uint32_t* shOffset = NULL;
        if (variable) {
            vsh = VSH_COMPACT;
            shOffset = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
            size_t o = 0;
            for (uint32_t i = 0; i < n; ++i) {
                shOffset[i] = (uint32_t)o;
                o += (size_t)KEPT(i) * 3;
            }
            shFloats = o;
        }
        sz[0] = sz[1] = sz[2] = (uint64_t)n * 16;
        sz[3] = (uint64_t)shFloats * 4;
        if (fill) {
            for (int b = 0; b < 4; ++b) out[b] = (uint32_t*)buffers[b];
            for (uint32_t i = 0; i < n; ++i) {
                for (int c = 0; c < 4; ++c) {
                    out[0][(size_t)i * 4 + c] = fbits(posAlpha[4 * (size_t)i + c]);
                    out[1][(size_t)i * 4 + c] = fbits(scales[4 * (size_t)i + c]);
                    out[2][(size_t)i * 4 + c] = fbits(rotations[4 * (size_t)i + c]);
                }
                if (variable) {
                    out[1][(size_t)i * 4 + 3] = ((uint32_t)degrees[i] << 30) | shOffset[i];
                    for (uint32_t k = 0; k < KEPT(i); ++k)
                        for (uint32_t c = 0; c < 3; ++c) out[3][shOffset[i] + k * 3 + c] = fbits(SHV(i, k, c));
                    continue;
                }
                for (uint32_t k = 0; k < K; ++k)
                    for (uint32_t c = 0; c < 3; ++c) out[3][((size_t)i * K + k) * 3 + c] = fbits(SHV(i, k, c));
            }
        }
        free(shOffset);
    } else {
        geometry = format == FMT_F32 ? GEOM_F32 : GEOM_F16;
        color = format == FMT_F32 ? COL_F32 : format == FMT_F16 ? COL_F16 : COL_Q8;
        const uint32_t geomWords = vec4sFor(geometryRecordBytes(geometry)) * 4;
        const uint32_t colorWords = vec4sFor(colorRecordBytes(color, K)) * 4;
        uint32_t* geom = (uint32_t*)calloc((size_t)n * geomWords + 1, 4);
        uint32_t* col = (uint32_t*)calloc((size_t)n * colorWords + 1, 4);
        const uint32_t restDims = (K - 1) * 3;
        for (uint32_t i = 0; i < n; ++i) {
            const float* pa = posAlpha + 4 * (size_t)i;
            const float* sc = scales + 4 * (size_t)i;
            const float* q = rotations + 4 * (size_t)i;
            uint32_t* w = &geom[(size_t)i * geomWords];
            if (geometry == GEOM_F32) {
                const float v[12] = {pa[0], pa[1], pa[2], pa[3], sc[0], sc[1], sc[2], 0.0f, q[0], q[1], q[2], q[3]};
                for (int j = 0; j < 12; ++j) w[j] = fbits(v[j]);
            } else {
                w[0] = fbits(pa[0]);
                w[1] = fbits(pa[1]);
                w[2] = fbits(pa[2]);
                w[3] = packHalf2(pa[3], sc[0]);
                w[4] = packHalf2(sc[1], sc[2]);
                w[5] = packHalf2(q[0], q[1]);
                w[6] = packHalf2(q[2], q[3]);
                w[7] = 0;
            }
            uint32_t* cw = &col[(size_t)i * colorWords];
            if (color == COL_F32) {
                for (uint32_t k = 0; k < K; ++k)
                    for (uint32_t c = 0; c < 3; ++c) cw[k * 3 + c] = fbits(SHV(i, k, c));
            } else if (color == COL_F16) {
                for (uint32_t k = 0; k < K; ++k)
                    for (uint32_t c = 0; c < 3; ++c) {
                        const uint32_t hi = k * 3 + c;
                        const uint32_t h = gsr_oracle_float_to_half(SHV(i, k, c));
                        uint32_t* word = &cw[hi / 2];
                        *word = (hi & 1u) ? ((*word & 0x0000FFFFu) | (h << 16)) : ((*word & 0xFFFF0000u) | h);
                    }
            } else {
                cw[0] = packHalf2(SHV(i, 0, 0), SHV(i, 0, 1));
                uint16_t bandScale[4] = {0, 0, 0, 0};
                int8_t qv[45];
                memset(qv, 0, sizeof(qv));
                for (uint32_t band = 1; band * band < KEPT(i); ++band) {
                    const uint32_t k0 = band * band, k1 = (band + 1) * (band + 1);
                    float values[21];
                    uint32_t m = 0;
                    for (uint32_t k = k0; k < k1; ++k)
                        for (uint32_t c = 0; c < 3; ++c) values[m++] = SHV(i, k, c);
                    bandScale[band] = quantizeBandQ8(values, m, &qv[(k0 - 1) * 3]);
                }
                cw[1] = (uint32_t)gsr_oracle_float_to_half(SHV(i, 0, 2)) | ((uint32_t)bandScale[1] << 16);
                cw[2] = (uint32_t)bandScale[2] | ((uint32_t)bandScale[3] << 16);
                for (uint32_t j = 0; j < restDims; ++j) cw[3 + j / 4] |= (uint32_t)(uint8_t)qv[j] << (8 * (j % 4));
            }
        }
        uint32_t* colFinal = col;
        size_t colFinalWords = (size_t)n * colorWords;
        if (variable) {
            const int compact = layout == LAYOUT_SPLIT;
            vsh = compact ? VSH_COMPACT : VSH_DEGREE;
            if (compact) {
                size_t total = 0;
                for (uint32_t i = 0; i < n; ++i) total += vec4sFor(colorRecordBytes(color, KEPT(i))) * 4;
                uint32_t* packed = (uint32_t*)calloc(total + 1, 4);
                size_t p = 0;
                for (uint32_t i = 0; i < n; ++i) {
                    const uint32_t words = vec4sFor(colorRecordBytes(color, KEPT(i))) * 4;
                    geom[(size_t)i * geomWords + 7] = ((uint32_t)degrees[i] << 30) | (uint32_t)(p / 4);
                    memcpy(&packed[p], &col[(size_t)i * colorWords], (size_t)words * 4);
                    p += words;
                }
                colFinal = packed;
                colFinalWords = total;
            } else {
                for (uint32_t i = 0; i < n; ++i) geom[(size_t)i * geomWords + 7] = (uint32_t)degrees[i] << 30;
            }
        }
        if (layout == LAYOUT_SPLIT) {
            gStride = geomWords / 4;
            cStride = colorWords / 4;
            cOffset = 0;
            sz[0] = (uint64_t)n * geomWords * 4;
            sz[1] = (uint64_t)colFinalWords * 4;
            if (fill) {
                memcpy(buffers[0], geom, (size_t)sz[0]);
                memcpy(buffers[1], colFinal, (size_t)sz[1]);
            }
        } else {
            const uint32_t recordWords = geomWords + colorWords;
            gStride = recordWords / 4;
            cStride = recordWords / 4;
            cOffset = geomWords / 4;
            sz[0] = (uint64_t)n * recordWords * 4;
            if (fill) {
                uint32_t* rec = (uint32_t*)buffers[0];
                for (uint32_t i = 0; i < n; ++i) {
                    memcpy(&rec[(size_t)i * recordWords], &geom[(size_t)i * geomWords], (size_t)geomWords * 4);
                    memcpy(&rec[(size_t)i * recordWords + geomWords], &col[(size_t)i * colorWords],
                           (size_t)colorWords * 4);
                }
            }
        }
        if (colFinal != col) free(colFinal);
        free(geom);
        free(col);
    }
#undef KEPT
#undef SHV
    free(degrees);
    desc[0] = geometry;
    desc[1] = color;
    desc[2] = gStride;
    desc[3] = cStride;
    desc[4] = cOffset;
    desc[5] = 0;
    desc[6] = vsh;
    desc[7] = (uint32_t)deg;
    desc[8] = K;
    desc[9] = format;
    desc[10] = layout;
    for (int b = 0; b < 4; ++b) sizes[b] = sz[b];
    return 0;
}

/* decodeGaussian (scene_compression.cpp:382-460), f32/f16/q8/cb. */
void gsr_oracle_decode(uint32_t n, const uint32_t* desc, const uint64_t* sizes, void* const* buffers, float* posAlpha,
                       float* scales, float* rotations, float* shOut) {
    (void)sizes;
    const uint32_t geometry = desc[0], color = desc[1], gStride = desc[2], cStride = desc[3], cOffset = desc[4];
    const uint32_t vsh = desc[6], Kstored = desc[8], layout = desc[10];
    const uint32_t* b0 = (const uint32_t*)buffers[0];
    const uint32_t* b1 = (const uint32_t*)buffers[1];
    const uint32_t* b2 = (const uint32_t*)buffers[2];
    const uint32_t* b3 = (const uint32_t*)buffers[3];
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t K = Kstored;
        float* pa = posAlpha + 4 * (size_t)i;
        float* sg = scales + 4 * (size_t)i;
        float* ro = rotations + 4 * (size_t)i;
        float* sh = shOut + (size_t)i * Kstored * 3;
        for (uint32_t k = 0; k < Kstored * 3; ++k) sh[k] = 0.0f;
        sg[3] = 0.0f;
        if (geometry == GEOM_SOA) {
            for (int c = 0; c < 4; ++c) pa[c] = bitsf(b0[(size_t)i * 4 + c]);
            for (int c = 0; c < 3; ++c) sg[c] = bitsf(b1[(size_t)i * 4 + c]);
            for (int c = 0; c < 4; ++c) ro[c] = bitsf(b2[(size_t)i * 4 + c]);
            size_t base = (size_t)i * K * 3;
            if (vsh != VSH_OFF) {
                const uint32_t d = b1[(size_t)i * 4 + 3] >> 30;
                if ((d + 1) * (d + 1) < K) K = (d + 1) * (d + 1);
                base = b1[(size_t)i * 4 + 3] & 0x3FFFFFFFu;
            }
            for (uint32_t k = 0; k < K * 3; ++k) sh[k] = bitsf(b3[base + k]);
            continue;
        }
        const uint32_t* g = &b0[(size_t)i * gStride * 4];
        if (geometry == GEOM_F32) {
            for (int c = 0; c < 4; ++c) pa[c] = bitsf(g[c]);
            for (int c = 0; c < 3; ++c) sg[c] = bitsf(g[4 + c]);
            for (int c = 0; c < 4; ++c) ro[c] = bitsf(g[8 + c]);
        } else {
            pa[0] = bitsf(g[0]);
            pa[1] = bitsf(g[1]);
            pa[2] = bitsf(g[2]);
            pa[3] = unpackLo(g[3]);
            sg[0] = unpackHi(g[3]);
            sg[1] = unpackLo(g[4]);
            sg[2] = unpackHi(g[4]);
            const float q[4] = {unpackLo(g[5]), unpackHi(g[5]), unpackLo(g[6]), unpackHi(g[6])};
            const float len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
            if (len2 > 0.0f) {
                const float inv = 1.0f / sqrtf(len2);
                for (int c = 0; c < 4; ++c) ro[c] = q[c] * inv;
            } else {
                ro[0] = 1.0f;
                ro[1] = ro[2] = ro[3] = 0.0f;
            }
        }
        const uint32_t* cb = layout == LAYOUT_AOS ? b0 : b1;
        size_t colorWord = cStride == 0 ? (size_t)i * 2 : ((size_t)i * cStride + cOffset) * 4;
        if (vsh != VSH_OFF) {
            const uint32_t meta = g[7];
            const uint32_t d = meta >> 30;
            if ((d + 1) * (d + 1) < K) K = (d + 1) * (d + 1);
            if (vsh == VSH_COMPACT) colorWord = (size_t)(meta & 0x3FFFFFFFu) * 4;
        }
        const uint32_t* c = cb + colorWord;
        if (color == COL_F32) {
            for (uint32_t k = 0; k < K * 3; ++k) sh[k] = bitsf(c[k]);
        } else if (color == COL_F16) {
            for (uint32_t h = 0; h < K * 3; ++h) sh[h] = (h & 1u) ? unpackHi(c[h / 2]) : unpackLo(c[h / 2]);
        } else if (color == COL_Q8) {
            sh[0] = unpackLo(c[0]);
            sh[1] = unpackHi(c[0]);
            sh[2] = unpackLo(c[1]);
            const float scale[4] = {0.0f, unpackHi(c[1]), unpackLo(c[2]), unpackHi(c[2])};
            for (uint32_t k = 1; k < K; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch) {
                    const uint32_t j = (k - 1) * 3 + ch;
                    const int8_t q = (int8_t)(uint8_t)(c[3 + j / 4] >> (8 * (j % 4)));
                    sh[k * 3 + ch] = (float)q * scale[bandOf(k)];
                }
        } else if (color == COL_CB) {  /* DC in the record, the rest from entry c[1] >> 16 of the codebook */
            sh[0] = unpackLo(c[0]);
            sh[1] = unpackHi(c[0]);
            sh[2] = unpackLo(c[1]);
            const uint32_t* entry = b2 + (size_t)(c[1] >> 16) * desc[5] * 4;
            for (uint32_t k = 1; k < K; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch) sh[k * 3 + ch] = bitsf(entry[(k - 1) * 3 + ch]);
        }
    }
}

void gsr_oracle_quantize_rgb8(uint32_t pixels, const float* rgb, uint32_t srcStride, uint8_t* out) {
    for (uint32_t p = 0; p < pixels; ++p)
        for (int c = 0; c < 3; ++c) {
            const float v = rgb[(size_t)p * srcStride + c];
            const float cl = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
            out[(size_t)p * 3 + c] = (uint8_t)lroundf(cl * 255.0f);
        }
}

void gsr_oracle_logf_range(uint32_t first_bits, uint32_t count, float* out) {
    for (uint32_t j = 0; j < count; ++j) out[j] = logf(bitsf(first_bits + j));
}

/* ---- renderReference over a scalar type (frame_generic.h): the float instance restates the
 *      functions above once more and must equal them bit for bit; the double instance is the
 *      FP64 build the float images are measured against. <tgmath.h> picks each math
 *      function's precision from its argument. ------------------------------------------ */
#include <tgmath.h>
#define REAL float
#define FN(x) x##_f32
#include "frame_generic.h"
#undef REAL
#undef FN
#define REAL double
#define FN(x) x##_f64
#include "frame_generic.h"
#undef REAL
#undef FN
