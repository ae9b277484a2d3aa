/* Test infrastructure: the reference's CPU frame (renderReference) written once over a scalar
 * type, for the FP64 build the float image is measured against. Included twice by
 * gsr_oracle_fp64.c:
 *
 *   REAL = float,  FN(x) = x##_f32   must equal the float restatement (gsr_oracle.c) bit for bit,
 *                                    which pins this body to the reference's own build;
 *   REAL = double, FN(x) = x##_f64   the same operations in IEEE double precision.
 *
 * Every step restates the reference file:line it follows (the same sources gsr_oracle.c cites):
 * splatCameraFromViewer (splat_math.cpp:9-42), preprocessGaussian (splat_math.cpp:44-193), the
 * tight coverage (tile_coverage.cpp:24-144), DepthSorter (depth_sort.cpp:17-75) and the
 * per-pixel loop of renderReference (reference_renderer.cpp:41-234). Evaluation order is the
 * GLM-subset order of oracle/glm_shim. Math functions come from <tgmath.h>, so the float body
 * calls sqrtf / expf / logf / floorf / ceilf as the reference's float code does and the double
 * body calls their double versions. Constants are written as double literals and converted
 * with R(); the float pin test checks that each converts to the reference's float constant. */

#define RR(x) ((REAL)(x))

static inline REAL FN(smax)(REAL a, REAL b) { return (a < b) ? b : a; } /* std::max */
static inline REAL FN(smin)(REAL a, REAL b) { return (b < a) ? b : a; } /* std::min */
static inline REAL FN(sclamp)(REAL v, REAL lo, REAL hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
static inline int FN(toInt)(REAL x) { /* int(x) as x86-64 converts it (INT_MIN out of range / NaN) */
    return (x >= RR(-2147483648.0) && x < RR(2147483648.0)) ? (int)x : INT_MIN;
}

typedef struct {
    REAL V[16]; /* viewInria, column-major */
    REAL position[3];
    uint32_t width, height, tilesX, tilesY;
    REAL tanX, tanY, focalX, focalY;
} FN(Camera);

typedef struct {
    REAL center[2], depth, conic[3], opacity, color[3], radius;
    uint32_t cull;
} FN(Splat);

#define GM4(m, c, r) (m)[(c)*4 + (r)]

static void FN(mul4)(const REAL* a, const REAL* b, REAL* r) {
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            GM4(r, c, row) = GM4(a, 0, row) * GM4(b, c, 0) + GM4(a, 1, row) * GM4(b, c, 1) +
                             GM4(a, 2, row) * GM4(b, c, 2) + GM4(a, 3, row) * GM4(b, c, 3);
}

/* makeSplatCamera / splatCameraFromViewer (splat_math.cpp:9-42) */
static void FN(camera)(const float* view, const float* proj, const float* model, uint32_t width, uint32_t height,
                       FN(Camera) * cam) {
    REAL flip[16], v[16], m[16], fv[16];
    for (int i = 0; i < 16; ++i) {
        flip[i] = (i % 5 == 0) ? RR(1.0) : RR(0.0);
        v[i] = (REAL)view[i];
        m[i] = (REAL)model[i];
    }
    GM4(flip, 1, 1) = RR(-1.0);
    GM4(flip, 2, 2) = RR(-1.0);
    FN(mul4)(flip, v, fv);
    FN(mul4)(fv, m, cam->V);
    cam->tanX = RR(1.0) / (REAL)GM4(proj, 0, 0);
    cam->tanY = RR(1.0) / fabs((REAL)GM4(proj, 1, 1));
    const REAL* V = cam->V;
    for (int r = 0; r < 3; ++r)
        cam->position[r] = -(GM4(V, r, 0) * GM4(V, 3, 0) + GM4(V, r, 1) * GM4(V, 3, 1) + GM4(V, r, 2) * GM4(V, 3, 2));
    cam->width = width;
    cam->height = height;
    cam->focalX = (REAL)width / (RR(2.0) * cam->tanX);
    cam->focalY = (REAL)height / (RR(2.0) * cam->tanY);
    cam->tilesX = (width + 15) / 16;
    cam->tilesY = (height + 15) / 16;
}

/* quaternionToMatrix + computeCov3D (splat_math.cpp:44-63) */
static void FN(cov3d)(const REAL sigma[3], const REAL q[4], REAL S[9]) {
    const REAL r = q[0], x = q[1], y = q[2], z = q[3];
    REAL R_[9];
    R_[0] = RR(1.0) - RR(2.0) * (y * y + z * z); R_[1] = RR(2.0) * (x * y + r * z); R_[2] = RR(2.0) * (x * z - r * y);
    R_[3] = RR(2.0) * (x * y - r * z); R_[4] = RR(1.0) - RR(2.0) * (x * x + z * z); R_[5] = RR(2.0) * (y * z + r * x);
    R_[6] = RR(2.0) * (x * z + r * y); R_[7] = RR(2.0) * (y * z - r * x); R_[8] = RR(1.0) - RR(2.0) * (x * x + y * y);
    REAL M[9];
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) M[c * 3 + k] = R_[c * 3 + k] * sigma[c];
    for (int c = 0; c < 3; ++c)
        for (int row = 0; row < 3; ++row)
            S[c * 3 + row] = M[0 * 3 + row] * M[0 * 3 + c] + M[1 * 3 + row] * M[1 * 3 + c] + M[2 * 3 + row] * M[2 * 3 + c];
}

/* computeCov2D (splat_math.cpp:65-91) */
static void FN(cov2d)(const REAL t[3], const REAL S[9], const FN(Camera) * cam, REAL out[3]) {
    const REAL limX = RR(1.3) * cam->tanX, limY = RR(1.3) * cam->tanY;
    const REAL txtz = t[0] / t[2], tytz = t[1] / t[2];
    const REAL tx = FN(smin)(limX, FN(smax)(-limX, txtz)) * t[2];
    const REAL ty = FN(smin)(limY, FN(smax)(-limY, tytz)) * t[2];
    const REAL tz = t[2];
    REAL J[6] = {0, 0, 0, 0, 0, 0};
    J[0] = cam->focalX / tz;
    J[4] = -(cam->focalX * tx) / (tz * tz);
    J[3] = cam->focalY / tz;
    J[5] = -(cam->focalY * ty) / (tz * tz);
    const REAL* V = cam->V;
    REAL T[6], A[6], cov[4];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 2; ++r)
            T[c * 2 + r] = J[0 * 2 + r] * GM4(V, c, 0) + J[1 * 2 + r] * GM4(V, c, 1) + J[2 * 2 + r] * GM4(V, c, 2);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 2; ++r)
            A[c * 2 + r] = T[0 * 2 + r] * S[c * 3 + 0] + T[1 * 2 + r] * S[c * 3 + 1] + T[2 * 2 + r] * S[c * 3 + 2];
    for (int c = 0; c < 2; ++c)
        for (int r = 0; r < 2; ++r)
            cov[c * 2 + r] = A[0 * 2 + r] * T[0 * 2 + c] + A[1 * 2 + r] * T[1 * 2 + c] + A[2 * 2 + r] * T[2 * 2 + c];
    out[0] = cov[0] + RR(0.3);
    out[1] = cov[1];
    out[2] = cov[3] + RR(0.3);
}

typedef struct { int minX, minY, maxX, maxY; } FN(Rect);

/* computeTileRect (splat_math.cpp:116-127) */
static FN(Rect) FN(tileRect)(const REAL p[2], REAL radius, uint32_t tilesX, uint32_t tilesY) {
    const int gx = (int)tilesX, gy = (int)tilesY, r = FN(toInt)(radius);
    FN(Rect) t;
    t.minX = imin(gx, imax(0, FN(toInt)((p[0] - (REAL)r) / RR(16.0))));
    t.minY = imin(gy, imax(0, FN(toInt)((p[1] - (REAL)r) / RR(16.0))));
    t.maxX = imin(gx, imax(0, FN(toInt)((p[0] + (REAL)r + RR(15.0)) / RR(16.0))));
    t.maxY = imin(gy, imax(0, FN(toInt)((p[1] + (REAL)r + RR(15.0)) / RR(16.0))));
    return t;
}

/* evalSH (splat_math.cpp:129-151) */
static void FN(evalSH)(int degree, const REAL* sh, const REAL dir[3], REAL out[3]) {
    const REAL C0 = RR(0.28209479177387814), C1 = RR(0.4886025119029199);
    const REAL C2[5] = {RR(1.0925484305920792), RR(-1.0925484305920792), RR(0.31539156525252005),
                        RR(-1.0925484305920792), RR(0.5462742152960396)};
    const REAL C3[7] = {RR(-0.5900435899266435), RR(2.890611442640554), RR(-0.4570457994644658),
                        RR(0.3731763325901154), RR(-0.4570457994644658), RR(1.445305721320277),
                        RR(-0.5900435899266435)};
    REAL res[3];
    for (int c = 0; c < 3; ++c) res[c] = C0 * sh[c];
    if (degree > 0) {
        const REAL x = dir[0], y = dir[1], z = dir[2];
        const REAL a = C1 * y, b = C1 * z, d = C1 * x;
        for (int c = 0; c < 3; ++c) res[c] = res[c] - a * sh[3 + c] + b * sh[6 + c] - d * sh[9 + c];
        if (degree > 1) {
            const REAL xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            const REAL t4 = C2[0] * xy, t5 = C2[1] * yz, t6 = C2[2] * (RR(2.0) * zz - xx - yy);
            const REAL t7 = C2[3] * xz, t8 = C2[4] * (xx - yy);
            for (int c = 0; c < 3; ++c)
                res[c] = res[c] + t4 * sh[12 + c] + t5 * sh[15 + c] + t6 * sh[18 + c] + t7 * sh[21 + c] + t8 * sh[24 + c];
            if (degree > 2) {
                const REAL t9 = C3[0] * y * (RR(3.0) * xx - yy), t10 = C3[1] * xy * z;
                const REAL t11 = C3[2] * y * (RR(4.0) * zz - xx - yy);
                const REAL t12 = C3[3] * z * (RR(2.0) * zz - RR(3.0) * xx - RR(3.0) * yy);
                const REAL t13 = C3[4] * x * (RR(4.0) * zz - xx - yy), t14 = C3[5] * z * (xx - yy);
                const REAL t15 = C3[6] * x * (xx - RR(3.0) * yy);
                for (int c = 0; c < 3; ++c)
                    res[c] = res[c] + t9 * sh[27 + c] + t10 * sh[30 + c] + t11 * sh[33 + c] + t12 * sh[36 + c] +
                             t13 * sh[39 + c] + t14 * sh[42 + c] + t15 * sh[45 + c];
            }
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = FN(smax)(res[c] + RR(0.5), RR(0.0));
}

/* preprocessGaussian (splat_math.cpp:153-193), the CPU reference's rules (no opacity cull) */
static void FN(preprocess)(const float* paIn, const float* scIn, const float* qIn, const float* shIn, int degree,
                           const FN(Camera) * cam, FN(Splat) * s) {
    memset(s, 0, sizeof(*s));
    REAL pa[4], sc[3], q[4], sh[48];
    for (int k = 0; k < 4; ++k) pa[k] = (REAL)paIn[k], q[k] = (REAL)qIn[k];
    for (int k = 0; k < 3; ++k) sc[k] = (REAL)scIn[k];
    const int K = (degree + 1) * (degree + 1);
    for (int k = 0; k < K * 3; ++k) sh[k] = (REAL)shIn[k];
    const REAL* V = cam->V;
    const REAL t[3] = {GM4(V, 0, 0) * pa[0] + GM4(V, 1, 0) * pa[1] + GM4(V, 2, 0) * pa[2] + GM4(V, 3, 0),
                       GM4(V, 0, 1) * pa[0] + GM4(V, 1, 1) * pa[1] + GM4(V, 2, 1) * pa[2] + GM4(V, 3, 1),
                       GM4(V, 0, 2) * pa[0] + GM4(V, 1, 2) * pa[1] + GM4(V, 2, 2) * pa[2] + GM4(V, 3, 2)};
    s->depth = t[2];
    if (t[2] <= RR(0.2)) {
        s->cull = 1;
        return;
    }
    REAL S[9], cov[3];
    FN(cov3d)(sc, q, S);
    FN(cov2d)(t, S, cam, cov);
    /* conicAndRadius (splat_math.cpp:102-114) */
    const REAL det = cov[0] * cov[2] - cov[1] * cov[1];
    if (det == RR(0.0)) {
        s->cull = 2;
        return;
    }
    const REAL detInv = RR(1.0) / det;
    s->conic[0] = cov[2] * detInv;
    s->conic[1] = -cov[1] * detInv;
    s->conic[2] = cov[0] * detInv;
    const REAL mid = RR(0.5) * (cov[0] + cov[2]);
    const REAL l1 = mid + sqrt(FN(smax)(RR(0.1), mid * mid - det));
    const REAL l2 = mid - sqrt(FN(smax)(RR(0.1), mid * mid - det));
    s->radius = ceil(RR(3.0) * sqrt(FN(smax)(l1, l2)));
    /* projectToPixel (splat_math.cpp:93-100) */
    const REAL ndcX = t[0] / (t[2] * cam->tanX), ndcY = t[1] / (t[2] * cam->tanY);
    s->center[0] = ((ndcX + RR(1.0)) * (REAL)cam->width - RR(1.0)) * RR(0.5);
    s->center[1] = ((ndcY + RR(1.0)) * (REAL)cam->height - RR(1.0)) * RR(0.5);
    const FN(Rect) rc = FN(tileRect)(s->center, s->radius, cam->tilesX, cam->tilesY);
    if (rc.maxX <= rc.minX || rc.maxY <= rc.minY) {
        s->cull = 3;
        return;
    }
    const REAL dv[3] = {pa[0] - cam->position[0], pa[1] - cam->position[1], pa[2] - cam->position[2]};
    const REAL inv = RR(1.0) / sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    const REAL dir[3] = {dv[0] * inv, dv[1] * inv, dv[2] * inv};
    FN(evalSH)(degree, sh, dir, s->color);
    s->opacity = pa[3];
    s->cull = 0;
}

/* ---- tight coverage (tile_coverage.cpp:24-144), 16-px bins ---------------------------- */
typedef struct { REAL cx, cy, A, B, C, D, t, exPad, eyPad; int valid; } FN(Ellipse);
typedef struct { int x0, y0, x1, y1; } FN(Bins);

/* makeCutoffEllipse (tile_coverage.cpp:24-50) */
static FN(Ellipse) FN(ellipse)(const FN(Splat) * s) {
    FN(Ellipse) e;
    memset(&e, 0, sizeof(e));
    e.cx = s->center[0];
    e.cy = s->center[1];
    e.A = s->conic[0], e.B = s->conic[1], e.C = s->conic[2];
    e.D = e.A * e.C - e.B * e.B;
    e.t = RR(-1.0);
    e.valid = e.A > RR(0.0) && e.C > RR(0.0) && e.D > RR(0.0);
    if (!e.valid || !(s->opacity >= RR(1.0) / RR(255.0))) return e;
    const REAL qmax = RR(2.0) * log(RR(255.0) * s->opacity);
    const REAL rho = fabs(e.B) / sqrt(e.A * e.C);
    const REAL K = RR(2.0) / FN(smax)(RR(1.0) - rho, RR(1e-30));
    const REAL t = qmax + (RR(1e-3) + RR(2e-5) * K) * FN(smax)(qmax, RR(1.0)) + RR(2e-3);
    if (!(t < RR(1e30))) {
        e.valid = 0;
        return e;
    }
    e.t = t;
    const REAL ex = sqrt(t * e.C / e.D), ey = sqrt(t * e.A / e.D);
    e.exPad = ex + (RR(0.02) + RR(2e-3) * ex);
    e.eyPad = ey + (RR(0.02) + RR(2e-3) * ey);
    return e;
}

/* floorDivClamped (tile_coverage.cpp:54) */
static int FN(floorDiv)(REAL v) { return FN(toInt)(floor(FN(sclamp)(v, RR(-65536.0), RR(1048576.0)) / RR(16.0))); }

/* ellipseRowSpan via ellipseRowBounds (tile_coverage.cpp:70-96) */
static void FN(rowSpan)(const FN(Ellipse) * e, int row, const FN(Bins) * b, int* x0, int* x1) {
    const REAL ey0 = (REAL)(row * 16) - e->cy, ey1 = (REAL)(row * 16 + 15) - e->cy;
    const REAL lo = FN(smax)(ey0, -e->eyPad), hi = FN(smin)(ey1, e->eyPad);
    if (!(lo <= hi)) {
        *x0 = *x1 = b->x0;
        return;
    }
    const REAL exTrue = sqrt(e->t * e->C / e->D);
    const REAL eyR = FN(sclamp)(-e->B * exTrue / e->C, lo, hi), eyL = FN(sclamp)(e->B * exTrue / e->C, lo, hi);
    const REAL At = e->A * e->t;
    const REAL xR = (-e->B * eyR + sqrt(FN(smax)(RR(0.0), At - e->D * eyR * eyR))) / e->A;
    const REAL xL = (-e->B * eyL - sqrt(FN(smax)(RR(0.0), At - e->D * eyL * eyL))) / e->A;
    const REAL pad = RR(0.02) + RR(2e-3) * exTrue;
    const REAL fx0 = e->cx + xL - pad, fx1 = e->cx + xR + pad;
    const int a = imax(b->x0, FN(floorDiv)(ceil(fx0)));
    const int c = imin(b->x1, FN(floorDiv)(floor(fx1)) + 1);
    *x0 = a;
    *x1 = imax(a, c);
}

/* makeCoverage + coverageRows / coverageRowSpan (tile_coverage.cpp:102-127); tiles in
 * enumeration order, returns the count (writes at most cap) */
static uint32_t FN(tiles)(const FN(Splat) * s, const FN(Camera) * cam, uint32_t bounds, uint32_t* out, uint32_t cap) {
    const int gx = (int)cam->tilesX, gy = (int)cam->tilesY;
    const FN(Rect) r = FN(tileRect)(s->center, s->radius, cam->tilesX, cam->tilesY);
    FN(Bins) b = {r.minX, r.minY, imin(r.maxX, gx), imin(r.maxY, gy)};
    FN(Ellipse) e;
    int useEllipse = 0;
    if (bounds == 2) b.x0 = 0, b.y0 = 0, b.x1 = gx, b.y1 = gy;
    if (bounds != 0) {
        e = FN(ellipse)(s);
        useEllipse = e.valid;
        if (!e.valid && bounds == 2) b.x0 = r.minX, b.y0 = r.minY, b.x1 = imin(r.maxX, gx), b.y1 = imin(r.maxY, gy);
    }
    int r0, r1;
    if (!useEllipse) {
        r0 = b.y0;
        r1 = imax(b.y0, b.y1);
    } else if (e.t < RR(0.0)) {
        r0 = r1 = 0;
    } else {
        const REAL y0 = ceil(e.cy - e.eyPad), y1 = floor(e.cy + e.eyPad);
        r0 = imax(b.y0, FN(floorDiv)(y0));
        r1 = imax(r0, imin(b.y1, FN(floorDiv)(y1) + 1));
    }
    uint32_t k = 0;
    for (int row = r0; row < r1; ++row) {
        int x0 = b.x0, x1 = imax(b.x0, b.x1);
        if (useEllipse) FN(rowSpan)(&e, row, &b, &x0, &x1);
        for (int x = x0; x < x1; ++x) {
            if (k < cap) out[k] = (uint32_t)(row * gx + x);
            ++k;
        }
    }
    return k;
}

/* ---- renderReference (reference_renderer.cpp:41-234): preprocess, depth order, binning in
 *      depth order, per-pixel front-to-back blending with early termination ------------------- */
typedef struct {
    const float *pa, *sc, *ro, *sh;
    uint32_t K;
    int degree;
    const FN(Camera) * cam;
    FN(Splat) * splats;
    const uint32_t *tileStart, *lists;
    REAL* rgb;
    _Atomic uint64_t evaluated, blended, terminated;
} FN(Ctx);

static void FN(preTask)(uint32_t i, void* p) {
    FN(Ctx)* c = (FN(Ctx)*)p;
    FN(preprocess)(c->pa + 4 * (size_t)i, c->sc + 4 * (size_t)i, c->ro + 4 * (size_t)i, c->sh + (size_t)i * c->K * 3,
                   c->degree, c->cam, &c->splats[i]);
}

static void FN(rasterTask)(uint32_t tile, void* p) {
    FN(Ctx)* c = (FN(Ctx)*)p;
    const FN(Camera)* cam = c->cam;
    const uint32_t tx = tile % cam->tilesX, ty = tile / cam->tilesX;
    const uint32_t s0 = c->tileStart[tile], s1 = c->tileStart[tile + 1];
    const uint32_t x0 = tx * 16, y0 = ty * 16;
    const uint32_t x1 = cam->width < x0 + 16 ? cam->width : x0 + 16;
    const uint32_t y1 = cam->height < y0 + 16 ? cam->height : y0 + 16;
    uint64_t ev = 0, bl = 0, te = 0;
    for (uint32_t y = y0; y < y1; ++y)
        for (uint32_t x = x0; x < x1; ++x) {
            const REAL px = (REAL)x, py = (REAL)y;
            REAL T = RR(1.0), C[3] = {RR(0.0), RR(0.0), RR(0.0)};
            for (uint32_t j = s0; j < s1; ++j) {
                const FN(Splat)* s = &c->splats[c->lists[j]];
                ++ev;
                /* splatAlphaAt (splat_math.h:147-156) */
                const REAL dx = s->center[0] - px, dy = s->center[1] - py;
                const REAL power = RR(-0.5) * (s->conic[0] * dx * dx + s->conic[2] * dy * dy) - s->conic[1] * dx * dy;
                if (power > RR(0.0)) continue;
                const REAL alpha = FN(smin)(RR(0.99), s->opacity * exp(power));
                if (alpha < RR(1.0) / RR(255.0)) continue;
                const REAL testT = T * (RR(1.0) - alpha);
                if (testT < RR(1e-4)) {
                    ++te;
                    break;
                }
                for (int ch = 0; ch < 3; ++ch) C[ch] = C[ch] + s->color[ch] * alpha * T;
                T = testT;
                ++bl;
            }
            REAL* dst = &c->rgb[((size_t)y * cam->width + x) * 3];
            for (int ch = 0; ch < 3; ++ch) dst[ch] = C[ch] + T * RR(0.0);
        }
    atomic_fetch_add(&c->evaluated, ev);
    atomic_fetch_add(&c->blended, bl);
    atomic_fetch_add(&c->terminated, te);
}

typedef struct { REAL depth; uint32_t index; } FN(DepthKey);
static int FN(depthCmp)(const void* a, const void* b) {
    const FN(DepthKey)* x = (const FN(DepthKey)*)a;
    const FN(DepthKey)* y = (const FN(DepthKey)*)b;
    if (x->depth != y->depth) return x->depth < y->depth ? -1 : 1;
    return x->index < y->index ? -1 : (x->index > y->index);
}

int FN(gsr_oracle_render)(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                          const float* sh, const float* view, const float* proj, const float* model, uint32_t width,
                          uint32_t height, int maxShDegree, uint32_t bounds, uint32_t threads, REAL* rgb,
                          GsrOracleRenderStats* stats) {
    FN(Camera) cam;
    FN(camera)(view, proj, model, width, height, &cam);
    const unsigned nt = threads ? threads : hardwareThreads();
    memset(rgb, 0, sizeof(REAL) * 3 * (size_t)width * height);
    FN(Ctx) c;
    memset(&c, 0, sizeof(c));
    c.pa = posAlpha, c.sc = scales, c.ro = rotations, c.sh = sh;
    c.K = (uint32_t)((shDegree + 1) * (shDegree + 1));
    c.degree = shDegree < maxShDegree ? shDegree : maxShDegree;
    c.cam = &cam;
    c.splats = (FN(Splat)*)malloc(sizeof(FN(Splat)) * (n ? n : 1));
    parallelFor(n, nt, 4096, FN(preTask), &c);
    GsrOracleRenderStats st;
    memset(&st, 0, sizeof(st));
    st.gaussians = n;
    st.threads = nt;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t r = c.splats[i].cull;
        st.visible += r == 0, st.culledNear += r == 1, st.culledSingular += r == 2, st.culledOffScreen += r == 3;
    }
    /* DepthSorter::sort (depth_sort.cpp:17-44): depth > 0.2 by (depth, index) */
    FN(DepthKey)* keys = (FN(DepthKey)*)malloc(sizeof(FN(DepthKey)) * (n ? n : 1));
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (c.splats[i].depth > RR(0.2)) keys[m].depth = c.splats[i].depth, keys[m].index = i, ++m;
    qsort(keys, m, sizeof(FN(DepthKey)), FN(depthCmp));
    /* binning in depth order (reference_renderer.cpp:84-118) */
    const uint32_t T = cam.tilesX * cam.tilesY;
    uint32_t* tileStart = (uint32_t*)calloc((size_t)T + 1, sizeof(uint32_t));
    uint32_t *tiles = NULL, cap = 0, *lists = NULL, *cursor = NULL;
    for (int phase = 0; phase < 2; ++phase) {
        if (phase == 1) {
            for (uint32_t t = 0; t < T; ++t) tileStart[t + 1] += tileStart[t];
            st.tileInstances = tileStart[T];
            lists = (uint32_t*)malloc(sizeof(uint32_t) * (tileStart[T] ? tileStart[T] : 1));
            cursor = (uint32_t*)malloc(sizeof(uint32_t) * (T ? T : 1));
            memcpy(cursor, tileStart, sizeof(uint32_t) * T);
        }
        for (uint32_t j = 0; j < m; ++j) {
            const uint32_t g = keys[j].index;
            if (c.splats[g].cull != 0) continue;
            const uint32_t cnt = FN(tiles)(&c.splats[g], &cam, bounds, NULL, 0);
            if (cnt > cap) {
                cap = cnt;
                tiles = (uint32_t*)realloc(tiles, sizeof(uint32_t) * cap);
            }
            FN(tiles)(&c.splats[g], &cam, bounds, tiles, cap);
            for (uint32_t q = 0; q < cnt; ++q) {
                if (phase == 0) tileStart[tiles[q] + 1]++;
                else lists[cursor[tiles[q]]++] = g;
            }
        }
    }
    c.tileStart = tileStart;
    c.lists = lists;
    c.rgb = rgb;
    atomic_init(&c.evaluated, 0);
    atomic_init(&c.blended, 0);
    atomic_init(&c.terminated, 0);
    parallelFor(T, nt, 1, FN(rasterTask), &c);
    st.evaluatedFragments = atomic_load(&c.evaluated);
    st.blendedFragments = atomic_load(&c.blended);
    st.terminatedPixels = atomic_load(&c.terminated);
    if (stats) *stats = st;
    free(tiles);
    free(lists);
    free(cursor);
    free(tileStart);
    free(keys);
    free(c.splats);
    return 0;
}

#undef RR
#undef GM4
