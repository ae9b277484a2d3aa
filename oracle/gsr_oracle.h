/* Test infrastructure: the CPU oracle of the splat-tiles frame path.
 *
 * A plain-C restatement of the reference renderer's CPU code for this path (splat math,
 * tight tile coverage, depth sort, the INRIA forward renderer, scene formats), used ONLY as
 * the checker: by tests/, by tests/golden/make_golden.py and by the CPU-baseline legs of
 * bench.py. The product (the CUDA library) never links or loads it.
 *
 * Parity: every function follows the reference source it cites operation for operation, in
 * IEEE single precision without FMA contraction (built with -ffp-contract=off). It is
 * pinned bit for bit against the reference's own sources compiled in place
 * (oracle/_ref/libgsr_ref.so, see ref_driver.cpp) by tests/test_oracle_pin.py and against
 * committed golden vectors made from that build (tests/golden/).
 *
 * Matrices are column-major float[16] (m[c*4 + r] = column c, row r), as in GLM. */
#ifndef GSR_ORACLE_H
#define GSR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* gsr::SplatCamera (src/splat/splat_math.h:43-50). */
typedef struct GsrOracleCamera {
    float viewInria[16];
    float position[3];
    uint32_t width, height;
    float tanHalfFovX, tanHalfFovY, focalX, focalY;
    uint32_t tilesX, tilesY;
} GsrOracleCamera;

/* gsr::ProjectedSplat (src/splat/splat_math.h:115-122), 48 bytes. */
typedef struct GsrOracleSplat {
    float center[2];
    float depth;
    uint32_t cullReason;
    float conicOpacity[4];
    float color[3];
    float radius;
} GsrOracleSplat;

/* gsr::ReferenceStats (src/splat/reference_renderer.h:51-62), flattened. */
typedef struct GsrOracleRenderStats {
    uint32_t gaussians, visible, culledNear, culledSingular, culledOffScreen, threads;
    uint64_t tileInstances, evaluatedFragments, blendedFragments, terminatedPixels;
    double preprocessMs, sortMs, binMs, rasterMs, totalMs;
} GsrOracleRenderStats;

enum { GSR_ORACLE_CULL_VISIBLE = 0, GSR_ORACLE_CULL_NEAR = 1, GSR_ORACLE_CULL_SINGULAR = 2,
       GSR_ORACLE_CULL_OFFSCREEN = 3, GSR_ORACLE_CULL_LOW_OPACITY = 4 };
enum { GSR_ORACLE_BOUNDS_RECT = 0, GSR_ORACLE_BOUNDS_TIGHT = 1, GSR_ORACLE_BOUNDS_CUTOFF = 2 };

/* Camera construction (glm::lookAt RH, glm::perspective RH with depth 0..1, as the
 * reference builds them with GLM_FORCE_DEPTH_ZERO_TO_ONE, CMakeLists.txt:186-189). */
void gsr_oracle_look_at(const float eye[3], const float center[3], const float up[3], float view[16]);
void gsr_oracle_perspective(float fovyRadians, float aspect, float zNear, float zFar, float proj[16]);
void gsr_oracle_camera_from_viewer(const float* view, const float* proj, const float* model, uint32_t width,
                                   uint32_t height, GsrOracleCamera* out);

/* preprocessGaussian for gaussians [0, n). gpuRules = 0: the CPU function
 * (splat_math.cpp:153-193); gpuRules = 1: the GPU preprocess's culls on top of it
 * (splat_preprocess.comp:159-177: NaN-safe near test and the o < 1/255 LowOpacity cull). */
void gsr_oracle_preprocess(uint32_t n, const float* posAlpha, const float* scales, const float* rotations,
                           const float* sh, uint32_t K, int degree, const GsrOracleCamera* cam, int gpuRules,
                           GsrOracleSplat* out);
/* Per-gaussian SH degree variant: degrees[i] caps the evaluated bands of gaussian i. */
void gsr_oracle_preprocess_degrees(uint32_t n, const float* posAlpha, const float* scales, const float* rotations,
                                   const float* sh, uint32_t K, int degree, const uint8_t* degrees,
                                   const GsrOracleCamera* cam, int gpuRules, GsrOracleSplat* out);

/* Tight coverage (tile_coverage.cpp): counts of visible splats (0 otherwise), and the tiles
 * of one splat in enumeration order (returns the count; writes at most cap). S names the bins:
 * 16 or 8 (the reference's S x S bins) or 32 (32 x 8 bins). */
void gsr_oracle_coverage_counts(uint32_t n, const GsrOracleSplat* splats, const GsrOracleCamera* cam, uint32_t bounds,
                                int S, uint32_t* counts);
uint32_t gsr_oracle_coverage_tiles(const GsrOracleSplat* splat, const GsrOracleCamera* cam, uint32_t bounds, int S,
                                   uint32_t* tiles, uint32_t cap);
int gsr_oracle_coverage_borderline(const GsrOracleSplat* splat, const GsrOracleCamera* cam, uint32_t bounds, int S,
                                   float eps);

/* The sorted (tile, splat) list of the global (64-bit key) mode, built on the CPU from the
 * splats: visible splats in index order, their tiles row by row, truncated to `capacity`,
 * stable-sorted by (tile, depth bits). keysLo = depth bits, keysHi = tile, values = gaussian.
 * ranges: [start, end) per tile, 2 words per tile, (0, 0) for empty tiles. Arrays must hold
 * min(duplicates, capacity) entries; returns the unclamped duplicate count M. */
uint64_t gsr_oracle_tile_list(uint32_t n, const GsrOracleSplat* splats, const uint32_t* counts,
                              const GsrOracleCamera* cam, uint32_t bounds, int S, uint32_t capacity,
                              uint32_t* keysLo, uint32_t* keysHi, uint32_t* values, uint32_t* ranges);

/* renderReference (reference_renderer.cpp:41-234), image = W*H*3 floats, row 0 = top. */
/* sortWindow: 0 = the list's order, K = StopThePop's per-pixel window of K splats, or
 * GSR_ORACLE_EXACT_PIXEL_SORT = every pixel sorts all its splats by ray depth
 * (ReferenceOptions::sortWindow, reference_renderer.h:41-46). */
#define GSR_ORACLE_EXACT_PIXEL_SORT 0xFFFFFFFFu
int gsr_oracle_render(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                      const float* sh, const GsrOracleCamera* cam, int maxShDegree, uint32_t bounds, uint32_t threads,
                      int earlyTermination, uint32_t sortWindow, float* rgb, GsrOracleRenderStats* stats);

/* DepthSorter (depth_sort.cpp). */
uint32_t gsr_oracle_depth_sort(uint32_t n, const float* posAlpha, const float* viewInria, uint32_t* order,
                               uint32_t* keys);
uint32_t gsr_oracle_radix_sort_pairs(uint32_t n, uint32_t* keys, uint32_t* values);

/* half.h */
uint16_t gsr_oracle_float_to_half(float v);
float gsr_oracle_half_to_float(uint16_t h);

/* Scene formats (scene_compression.cpp), f32/f16/q8 in soa/split/aos, variable SH degree.
 * desc: geometry, color, geometryStride, colorStride, colorOffset, codebookStride, variableSh,
 * shDegree, shCoeffs, format, layout. Two calls: sizes (buffers = NULL), then contents. */
int gsr_oracle_encode(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                      const float* sh, uint32_t format, uint32_t layout, int maxShDegree, float shThreshold,
                      uint32_t* desc, uint64_t* sizes, void** buffers);
void gsr_oracle_decode(uint32_t n, const uint32_t* desc, const uint64_t* sizes, void* const* buffers, float* posAlpha,
                       float* scales, float* rotations, float* sh);
int gsr_oracle_select_sh_degree(const float* sh, int storedDegree, float opacity, float threshold255);

/* logf (the C library's) of `count` consecutive float bit patterns starting at first_bits. */
void gsr_oracle_logf_range(uint32_t first_bits, uint32_t count, float* out);

/* Image helpers: quantize like the reference's PNG writer (image_io.cpp:55-56,
 * lround(clamp(v, 0, 1) * 255)), and PSNR with peak 1.0 (tools/imgdiff.cpp:127). */
void gsr_oracle_quantize_rgb8(uint32_t pixels, const float* rgb, uint32_t srcStride, uint8_t* out);

/* renderReference (reference_renderer.cpp:41-234, list order, no window) written once over a
 * scalar type (frame_generic.h), from the viewer matrices: _f32 in float (equal to
 * gsr_oracle_render bit for bit), _f64 the same operations in double (the FP64 build). rgb:
 * width x height x 3 of the instance's type. */
int gsr_oracle_render_f32(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                          const float* sh, const float* view, const float* proj, const float* model, uint32_t width,
                          uint32_t height, int maxShDegree, uint32_t bounds, uint32_t threads, float* rgb,
                          GsrOracleRenderStats* stats);
int gsr_oracle_render_f64(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                          const float* sh, const float* view, const float* proj, const float* model, uint32_t width,
                          uint32_t height, int maxShDegree, uint32_t bounds, uint32_t threads, double* rgb,
                          GsrOracleRenderStats* stats);

#ifdef __cplusplus
}
#endif

#endif
