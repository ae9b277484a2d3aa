// Test infrastructure (the oracle): a C-ABI driver over the reference renderer's OWN CPU
// sources, compiled in place from the reference tree by oracle/Makefile into
// oracle/_ref/libgsr_ref.so. It is used only by tests/, the golden-fixture script and the
// CPU-baseline legs of bench.py, to pin the C restatement (gsr_oracle.c) and to time the
// reference's CPU renderer. Nothing in the product links or loads it.
//
// Every entry point is a thin adapter: it copies flat arrays into the reference's types and
// calls the reference function named in its comment. The struct layouts below are shared
// with gsr_oracle.h (same field order and sizes).
#include "scene/gaussian_scene.h"
#include "scene/half.h"
#include "scene/ply_loader.h"
#include "scene/scene_compression.h"
#include "splat/depth_sort.h"
#include "splat/reference_renderer.h"
#include "splat/splat_math.h"
#include "splat/tile_coverage.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <functional>
#include <span>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace {

struct RefCamera {  // = GsrOracleCamera (gsr_oracle.h)
    float viewInria[16];
    float position[3];
    uint32_t width, height;
    float tanHalfFovX, tanHalfFovY, focalX, focalY;
    uint32_t tilesX, tilesY;
};

struct RefRenderStats {  // = GsrOracleRenderStats (gsr_oracle.h)
    uint32_t gaussians, visible, culledNear, culledSingular, culledOffScreen, threads;
    uint64_t tileInstances, evaluatedFragments, blendedFragments, terminatedPixels;
    double preprocessMs, sortMs, binMs, rasterMs, totalMs;
};

glm::mat4 loadMat4(const float* m) {
    glm::mat4 r;
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 4; ++k) r[c][k] = m[c * 4 + k];
    return r;
}

gsr::SplatCamera toCamera(const RefCamera& c) {
    gsr::SplatCamera cam;
    cam.viewInria = loadMat4(c.viewInria);
    cam.position = {c.position[0], c.position[1], c.position[2]};
    cam.width = c.width;
    cam.height = c.height;
    cam.tanHalfFovX = c.tanHalfFovX;
    cam.tanHalfFovY = c.tanHalfFovY;
    cam.focalX = c.focalX;
    cam.focalY = c.focalY;
    cam.tilesX = c.tilesX;
    cam.tilesY = c.tilesY;
    return cam;
}

RefCamera fromCamera(const gsr::SplatCamera& cam) {
    RefCamera c{};
    for (int col = 0; col < 4; ++col)
        for (int k = 0; k < 4; ++k) c.viewInria[col * 4 + k] = cam.viewInria[col][k];
    c.position[0] = cam.position.x;
    c.position[1] = cam.position.y;
    c.position[2] = cam.position.z;
    c.width = cam.width;
    c.height = cam.height;
    c.tanHalfFovX = cam.tanHalfFovX;
    c.tanHalfFovY = cam.tanHalfFovY;
    c.focalX = cam.focalX;
    c.focalY = cam.focalY;
    c.tilesX = cam.tilesX;
    c.tilesY = cam.tilesY;
    return c;
}

gsr::GaussianScene makeScene(uint32_t n, int shDegree, const float* posAlpha, const float* scales,
                             const float* rotations, const float* sh) {
    gsr::GaussianScene s;
    s.count = n;
    s.shDegree = shDegree;
    s.posAlpha.resize(n);
    s.scales.resize(n);
    s.rotations.resize(n);
    std::memcpy(s.posAlpha.data(), posAlpha, size_t(n) * 16);
    std::memcpy(s.scales.data(), scales, size_t(n) * 16);
    std::memcpy(s.rotations.data(), rotations, size_t(n) * 16);
    const size_t shFloats = size_t(n) * s.shCoeffsPerChannel() * 3;
    s.sh.assign(sh, sh + shFloats);
    return s;
}

}  // namespace

extern "C" {

// splatCameraFromViewer (src/splat/splat_math.cpp:29-42 [file lines of splat_math.cpp]).
void gsr_ref_camera_from_viewer(const float* view, const float* proj, const float* model, uint32_t width,
                                uint32_t height, RefCamera* out) {
    *out = fromCamera(gsr::splatCameraFromViewer(loadMat4(view), loadMat4(proj), loadMat4(model), width, height));
}

// preprocessGaussian (src/splat/splat_math.cpp:153-193) for gaussians [0, n); writes
// ProjectedSplat (48 B each). `degree` = evaluated SH bands; K = stored coefficients.
void gsr_ref_preprocess(uint32_t n, const float* posAlpha, const float* scales, const float* rotations,
                        const float* sh, uint32_t K, int degree, const RefCamera* camera, void* outSplats) {
    const gsr::SplatCamera cam = toCamera(*camera);
    auto* out = static_cast<gsr::ProjectedSplat*>(outSplats);
    for (uint32_t i = 0; i < n; ++i) {
        const glm::vec4 pa(posAlpha[4 * i], posAlpha[4 * i + 1], posAlpha[4 * i + 2], posAlpha[4 * i + 3]);
        const glm::vec3 sigma(scales[4 * i], scales[4 * i + 1], scales[4 * i + 2]);
        const glm::vec4 q(rotations[4 * i], rotations[4 * i + 1], rotations[4 * i + 2], rotations[4 * i + 3]);
        const auto* coeffs = reinterpret_cast<const glm::vec3*>(sh + size_t(i) * K * 3);
        out[i] = gsr::preprocessGaussian(pa, sigma, q, coeffs, degree, cam);
    }
}

// makeCoverage + coverageCount (src/splat/tile_coverage.cpp) of every splat whose cullReason
// is Visible (others: 0), with the 16-px rectangle of computeTileRect and bin tiles of size S.
void gsr_ref_coverage_counts(uint32_t n, const void* splats, const RefCamera* camera, uint32_t bounds, int S,
                             uint32_t* counts) {
    const auto* sp = static_cast<const gsr::ProjectedSplat*>(splats);
    const int gx = int((camera->width + S - 1) / S), gy = int((camera->height + S - 1) / S);
    for (uint32_t i = 0; i < n; ++i) {
        if (sp[i].cullReason != uint32_t(gsr::CullReason::Visible)) {
            counts[i] = 0;
            continue;
        }
        const gsr::Coverage cv =
            gsr::splatCoverage(gsr::TileBounds(bounds), sp[i], camera->tilesX, camera->tilesY, S, gx, gy);
        counts[i] = gsr::coverageCount(cv, S);
    }
}

// The bin tiles of splat i, in the order the duplicate pass enumerates them (coverageRows,
// then coverageRowSpan per row). Returns the number written (<= cap).
uint32_t gsr_ref_coverage_tiles(const void* splat, const RefCamera* camera, uint32_t bounds, int S, uint32_t* tiles,
                                uint32_t cap) {
    const auto& s = *static_cast<const gsr::ProjectedSplat*>(splat);
    const int gx = int((camera->width + S - 1) / S), gy = int((camera->height + S - 1) / S);
    const gsr::Coverage cv = gsr::splatCoverage(gsr::TileBounds(bounds), s, camera->tilesX, camera->tilesY, S, gx, gy);
    const auto [r0, r1] = gsr::coverageRows(cv, S);
    uint32_t k = 0;
    for (int r = r0; r < r1; ++r) {
        const auto [x0, x1] = gsr::coverageRowSpan(cv, r, S);
        for (int x = x0; x < x1; ++x) {
            if (k < cap) tiles[k] = uint32_t(r * gx + x);
            ++k;
        }
    }
    return k;
}

// coverageIsBorderline (src/splat/tile_coverage.cpp:146-164) of one splat.
int gsr_ref_coverage_borderline(const void* splat, const RefCamera* camera, uint32_t bounds, int S, float eps) {
    const auto& s = *static_cast<const gsr::ProjectedSplat*>(splat);
    const int gx = int((camera->width + S - 1) / S), gy = int((camera->height + S - 1) / S);
    const gsr::Coverage cv = gsr::splatCoverage(gsr::TileBounds(bounds), s, camera->tilesX, camera->tilesY, S, gx, gy);
    return gsr::coverageIsBorderline(cv, S, eps) ? 1 : 0;
}

// renderReference (src/splat/reference_renderer.cpp:41-234): rgb = W*H*3 floats.
int gsr_ref_render(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                   const float* sh, const RefCamera* camera, int maxShDegree, uint32_t bounds, uint32_t threads,
                   int earlyTermination, uint32_t sortWindow, float* rgb, RefRenderStats* stats) {
    try {
        const gsr::GaussianScene scene = makeScene(n, shDegree, posAlpha, scales, rotations, sh);
        gsr::ReferenceOptions o;
        o.maxShDegree = maxShDegree;
        o.bounds = gsr::TileBounds(bounds);
        o.threads = threads;
        o.earlyTermination = earlyTermination != 0;
        o.sortWindow = sortWindow;
        const gsr::ReferenceImage img = gsr::renderReference(scene, toCamera(*camera), o);
        std::memcpy(rgb, img.rgb.data(), img.rgb.size() * sizeof(float));
        if (stats) {
            const gsr::ReferenceStats& s = img.stats;
            *stats = RefRenderStats{s.gaussians,     s.visible,          s.culledNear,          s.culledSingular,
                                    s.culledOffScreen, s.threads,        s.tileInstances,       s.evaluatedFragments,
                                    s.blendedFragments, s.terminatedPixels, s.preprocessMs,    s.sortMs,
                                    s.binMs,         s.rasterMs,         s.totalMs};
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// DepthSorter::sort (src/splat/depth_sort.cpp:17-44): indices of gaussians with view z > 0.2,
// nearest first, ties by index. Returns the count written to order/keys.
uint32_t gsr_ref_depth_sort(uint32_t n, const float* posAlpha, const float* viewInria, uint32_t* order,
                            uint32_t* keys) {
    gsr::DepthSorter sorter;
    sorter.sort(reinterpret_cast<const glm::vec4*>(posAlpha), n, loadMat4(viewInria));
    std::copy(sorter.order().begin(), sorter.order().end(), order);
    std::copy(sorter.keys().begin(), sorter.keys().end(), keys);
    return uint32_t(sorter.order().size());
}

// DepthSorter::radixSortPairs (src/splat/depth_sort.cpp:46-75), in place. Returns passes run.
uint32_t gsr_ref_radix_sort_pairs(uint32_t n, uint32_t* keys, uint32_t* values) {
    std::vector<uint32_t> k(keys, keys + n), v(values, values + n), kt, vt;
    const uint32_t passes = gsr::DepthSorter::radixSortPairs(k, v, kt, vt);
    std::copy(k.begin(), k.end(), keys);
    std::copy(v.begin(), v.end(), values);
    return passes;
}

// floatToHalf / halfToFloat (src/scene/half.h).
uint16_t gsr_ref_float_to_half(float v) { return gsr::floatToHalf(v); }
float gsr_ref_half_to_float(uint16_t h) { return gsr::halfToFloat(h); }

// encodeScene (src/scene/scene_compression.cpp:150-380). Fills `desc` (11 words: geometry,
// color, geometryStride, colorStride, colorOffset, codebookStride, variableSh, shDegree,
// shCoeffs, format, layout) and the byte size of each of the 4 buffers; if `buffers` is
// non-null, also copies the buffer contents (each buffers[b] must hold sizes[b] bytes).
// Call twice: sizes first, then contents. Returns 0, or -1 on an invalid combination.
int gsr_ref_encode(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                   const float* sh, uint32_t format, uint32_t layout, int maxShDegree, float shThreshold,
                   uint32_t* desc, uint64_t* sizes, void** buffers) {
    try {
        const gsr::GaussianScene scene = makeScene(n, shDegree, posAlpha, scales, rotations, sh);
        gsr::CompressionOptions o;
        o.format = gsr::SceneFormat(format);
        o.layout = gsr::SceneLayout(layout);
        o.maxShDegree = maxShDegree;
        o.shThreshold = shThreshold;
        o.threads = 1;
        const gsr::EncodedScene e = gsr::encodeScene(scene, o);
        desc[0] = uint32_t(e.geometry);
        desc[1] = uint32_t(e.color);
        desc[2] = e.geometryStride;
        desc[3] = e.colorStride;
        desc[4] = e.colorOffset;
        desc[5] = e.codebookStride;
        desc[6] = uint32_t(e.variableSh);
        desc[7] = uint32_t(e.shDegree);
        desc[8] = e.shCoeffs;
        desc[9] = uint32_t(e.format);
        desc[10] = uint32_t(e.layout);
        for (int b = 0; b < 4; ++b) {
            const size_t bytes = b < int(e.buffers.size()) ? e.buffers[b].size() * 4 : 0;
            sizes[b] = bytes;
            if (buffers && buffers[b] && bytes) std::memcpy(buffers[b], e.buffers[b].data(), bytes);
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// encodeScene with the codebook options (the cb format's k-means): codebookSize, iterations,
// samples as CompressionOptions; otherwise as gsr_ref_encode. stats: entries, samples, iterations,
// emptyReseeded, simd (the AVX2 kernel was used).
int gsr_ref_encode_codebook(uint32_t n, int shDegree, const float* posAlpha, const float* scales, const float* rotations,
                            const float* sh, uint32_t layout, int maxShDegree, float shThreshold, uint32_t codebookSize,
                            uint32_t iterations, uint32_t samples, uint32_t* desc, uint64_t* sizes, void** buffers,
                            uint32_t* stats) {
    try {
        const gsr::GaussianScene scene = makeScene(n, shDegree, posAlpha, scales, rotations, sh);
        gsr::CompressionOptions o;
        o.format = gsr::SceneFormat::Codebook;
        o.layout = gsr::SceneLayout(layout);
        o.maxShDegree = maxShDegree;
        o.shThreshold = shThreshold;
        o.codebookSize = codebookSize;
        o.codebookIterations = iterations;
        o.codebookSamples = samples;
        o.threads = 0;
        const gsr::EncodedScene e = gsr::encodeScene(scene, o);
        desc[0] = uint32_t(e.geometry);
        desc[1] = uint32_t(e.color);
        desc[2] = e.geometryStride;
        desc[3] = e.colorStride;
        desc[4] = e.colorOffset;
        desc[5] = e.codebookStride;
        desc[6] = uint32_t(e.variableSh);
        desc[7] = uint32_t(e.shDegree);
        desc[8] = e.shCoeffs;
        desc[9] = uint32_t(e.format);
        desc[10] = uint32_t(e.layout);
        for (int b = 0; b < 4; ++b) {
            const size_t bytes = b < int(e.buffers.size()) ? e.buffers[b].size() * 4 : 0;
            sizes[b] = bytes;
            if (buffers && buffers[b] && bytes) std::memcpy(buffers[b], e.buffers[b].data(), bytes);
        }
        if (stats) {
            stats[0] = e.codebook.entries;
            stats[1] = e.codebook.samples;
            stats[2] = e.codebook.iterations;
            stats[3] = e.codebook.emptyReseeded;
            stats[4] = e.codebook.simd ? 1u : 0u;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// decodeGaussian (src/scene/scene_compression.cpp:382-460) for gaussians [0, n) of an encoded
// scene given as (desc, buffers) like gsr_ref_encode; writes posAlpha, sigma (vec4, w = 0),
// rotation and K = desc[8] SH triplets per gaussian.
void gsr_ref_decode(uint32_t n, const uint32_t* desc, const uint64_t* sizes, void* const* buffers, float* posAlpha,
                    float* scales, float* rotations, float* sh) {
    gsr::EncodedScene e;
    e.geometry = gsr::GeometryEncoding(desc[0]);
    e.color = gsr::ColorEncoding(desc[1]);
    e.geometryStride = desc[2];
    e.colorStride = desc[3];
    e.colorOffset = desc[4];
    e.codebookStride = desc[5];
    e.variableSh = gsr::VariableSh(desc[6]);
    e.shDegree = int(desc[7]);
    e.shCoeffs = desc[8];
    e.format = gsr::SceneFormat(desc[9]);
    e.layout = gsr::SceneLayout(desc[10]);
    e.count = n;
    e.buffers.resize(4);
    for (int b = 0; b < 4; ++b) {
        const auto* w = static_cast<const uint32_t*>(buffers[b]);
        if (w && sizes[b]) e.buffers[b].assign(w, w + sizes[b] / 4);
    }
    gsr::DecodedGaussian g;
    const uint32_t K = e.shCoeffs;
    for (uint32_t i = 0; i < n; ++i) {
        gsr::decodeGaussian(e, i, g);
        for (int c = 0; c < 4; ++c) posAlpha[4 * i + c] = g.posAlpha[c];
        for (int c = 0; c < 3; ++c) scales[4 * i + c] = g.sigma[c];
        scales[4 * i + 3] = 0.0f;
        for (int c = 0; c < 4; ++c) rotations[4 * i + c] = g.rotation[c];
        for (uint32_t k = 0; k < K; ++k)
            for (int c = 0; c < 3; ++c) sh[(size_t(i) * K + k) * 3 + c] = g.sh[k][c];
    }
}

// selectShDegree (src/scene/scene_compression.cpp:63-68).
int gsr_ref_select_sh_degree(const float* sh, int storedDegree, float opacity, float threshold255) {
    return gsr::selectShDegree(reinterpret_cast<const glm::vec3*>(sh), storedDegree, opacity, threshold255);
}

// ---- the PLY loader (src/scene/ply_loader.cpp) ---------------------------------------------
// gsr_ref_ply_load / _memory return a GaussianScene handle, or NULL with the exception's text
// in err and *kind = 1 (PlyError) or 2 (any other exception).
struct RefSceneStats {  // = GsrSceneStats (include/gsr_b200.h)
    float bboxMin[3], bboxMax[3], robustMin[3], robustMax[3];
    float alphaMin, alphaMax, alphaMean;
    uint32_t alphaBelowVisible;
    float sigmaMin, sigmaMax, sigmaMaxMedian, quatNormMin, quatNormMax;
    uint32_t zeroQuaternions;
    uint64_t nonFiniteValues;
};

static void* plyResult(const std::function<gsr::GaussianScene()>& load, char* err, size_t cap, int* kind) {
    *kind = 0;
    try {
        return new gsr::GaussianScene(load());
    } catch (const gsr::PlyError& e) {
        *kind = 1;
        std::snprintf(err, cap, "%s", e.what());
    } catch (const std::exception& e) {
        *kind = 2;
        std::snprintf(err, cap, "%s", e.what());
    }
    return nullptr;
}

void* gsr_ref_ply_load(const char* path, char* err, size_t cap, int* kind) {
    return plyResult([&] { return gsr::loadGaussianPly(std::filesystem::path(path)); }, err, cap, kind);
}

void* gsr_ref_ply_load_memory(const uint8_t* bytes, size_t size, const char* name, char* err, size_t cap, int* kind) {
    return plyResult([&] { return gsr::loadGaussianPly(std::span<const uint8_t>(bytes, size), std::string(name)); }, err,
                     cap, kind);
}

void gsr_ref_ply_info(const void* h, uint32_t* count, int* degree, uint32_t* comments, uint32_t* warnings,
                      RefSceneStats* stats) {
    const auto& s = *static_cast<const gsr::GaussianScene*>(h);
    *count = s.count;
    *degree = s.shDegree;
    *comments = uint32_t(s.comments.size());
    *warnings = uint32_t(s.warnings.size());
    const gsr::SceneStats& t = s.stats;
    for (int c = 0; c < 3; ++c) {
        stats->bboxMin[c] = t.bboxMin[c];
        stats->bboxMax[c] = t.bboxMax[c];
        stats->robustMin[c] = t.robustMin[c];
        stats->robustMax[c] = t.robustMax[c];
    }
    stats->alphaMin = t.alphaMin;
    stats->alphaMax = t.alphaMax;
    stats->alphaMean = t.alphaMean;
    stats->alphaBelowVisible = t.alphaBelowVisible;
    stats->sigmaMin = t.sigmaMin;
    stats->sigmaMax = t.sigmaMax;
    stats->sigmaMaxMedian = t.sigmaMaxMedian;
    stats->quatNormMin = t.quatNormMin;
    stats->quatNormMax = t.quatNormMax;
    stats->zeroQuaternions = t.zeroQuaternions;
    stats->nonFiniteValues = t.nonFiniteValues;
}

// posAlpha/scales/rotations/rawRotation float4[N], sh float[N K 3], rawOpacity [N], rawLogScale float3[N]
void gsr_ref_ply_arrays(const void* h, float* posAlpha, float* scales, float* rotations, float* sh, float* rawOpacity,
                        float* rawLogScale, float* rawRotation) {
    const auto& s = *static_cast<const gsr::GaussianScene*>(h);
    for (uint32_t i = 0; i < s.count; ++i) {
        for (int c = 0; c < 4; ++c) {
            posAlpha[i * 4 + c] = s.posAlpha[i][c];
            scales[i * 4 + c] = s.scales[i][c];
            rotations[i * 4 + c] = s.rotations[i][c];
            rawRotation[i * 4 + c] = s.rawRotation[i][c];
        }
        for (int c = 0; c < 3; ++c) rawLogScale[i * 3 + c] = s.rawLogScale[i][c];
        rawOpacity[i] = s.rawOpacity[i];
    }
    std::copy(s.sh.begin(), s.sh.end(), sh);
}

const char* gsr_ref_ply_comment(const void* h, uint32_t i) {
    return static_cast<const gsr::GaussianScene*>(h)->comments.at(i).c_str();
}

const char* gsr_ref_ply_warning(const void* h, uint32_t i) {
    return static_cast<const gsr::GaussianScene*>(h)->warnings.at(i).c_str();
}

void gsr_ref_ply_free(void* h) { delete static_cast<gsr::GaussianScene*>(h); }

}  // extern "C"
