// Host side of the B200 splat-tiles path: the C ABI of include/gsr_b200.h over a C++ renderer
// that mirrors gsr::SplatTileRenderer (src/render/splat_tile_renderer.h:143-290) and
// gsr::GpuScene (src/render/gpu_scene.h:42-78), launching the kernels of k_front.cu,
// k_sort.cu, k_render.cu and k_encode.cu on the caller's stream.
//
// Per frame (render):
//   frameBegin   reset of the control block + tile ranges      (splat_tile_renderer.cpp:653-661)
//   front        preprocess + count + scan + setup + duplicate (passes 1, 2, 6, 7)
//   sort         histogram/plan + onesweep passes               (pass 8, global 64-bit keys)
//   ranges       per-tile [start, end)                          (pass 9)
//   render       the tile rasterizer                            (pass 10)
//   readback     control block -> the frame slot's pinned buffer, read frames_in_flight later
//
// Counts (V, M, entries) exist only on the device; grids over the list are sized for the
// capacity and read the entry count from the control block, as the reference's indirect
// dispatches do. The adaptive list (splat_tile_renderer.cpp:444-486) follows the measured M.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <random>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "encode.cuh"
#include "gsr_b200.h"
#include "kernels.cuh"

extern "C" {
extern const uint32_t gsr_logf_fixup_base, gsr_logf_fixup_last, gsr_logf_fixup_count, gsr_logf_bucket_count;
extern const uint32_t gsr_logf_fixups[];
extern const uint32_t gsr_logf_bucket_start[];
}

namespace {

using namespace gsr;

thread_local std::string g_lastError;

int fail(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return status;
}

}  // namespace

namespace gsr {
// the calling thread's failure message (the scene input units report through it)
void setLastError(const std::string& message) { g_lastError = message; }
}  // namespace gsr

namespace {

// IEEE binary16 bits -> float, exactly (normal, subnormal, infinity, NaN)
float halfToFloat(uint16_t h) {
    const uint32_t sign = uint32_t(h & 0x8000u) << 16, e = (h >> 10) & 0x1Fu, m = h & 0x3FFu;
    if (e == 0) {
        const float v = float(m) * (1.0f / 16777216.0f);  // m 2^-24
        return sign ? -v : v;
    }
    const uint32_t bits = e == 31 ? (sign | 0x7F800000u | (m << 13)) : (sign | ((e + 112u) << 23) | (m << 13));
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

int cudaFail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(GSR_ERROR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(GSR_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define GSR_CUDA(call)                                           \
    do {                                                         \
        const cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cudaFail(e_, #call);       \
    } while (0)

constexpr uint32_t kBlockSize = 2048;                    // list capacity granularity (GpuRadixSort::kBlockSize)
constexpr uint32_t kMinAdaptiveCapacity = 256u * 1024u;  // entries (splat_tile_renderer.cpp:104)

uint32_t bitWidth(uint32_t x) { return x ? 32u - uint32_t(__builtin_clz(x)) : 0u; }

uint32_t roundUpToBlock(uint64_t n) {
    const uint64_t b = kBlockSize;
    return uint32_t(std::min<uint64_t>((n + b - 1) / b * b, 0xFFFFF800ull));
}

// ---- device-wide constant tables (the logf fixups), once per device ---------------------------
struct DeviceTables {
    uint32_t* entries = nullptr;
    uint32_t* buckets = nullptr;
    uint32_t* groups = nullptr;
};
std::mutex g_tablesMutex;
DeviceTables g_tables[64];

int deviceTables(LogfFixups* out) {
    int dev = 0;
    GSR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(GSR_ERROR_UNSUPPORTED, "device index %d", dev);
    std::lock_guard<std::mutex> lock(g_tablesMutex);
    DeviceTables& t = g_tables[dev];
    if (!t.entries) {
        const size_t eb = size_t(std::max(gsr_logf_fixup_count, 1u)) * 4, bb = size_t(gsr_logf_bucket_count) * 4;
        GSR_CUDA(cudaMalloc(&t.entries, eb));
        GSR_CUDA(cudaMalloc(&t.buckets, bb));
        GSR_CUDA(cudaMemcpy(t.entries, gsr_logf_fixups, eb, cudaMemcpyHostToDevice));
        GSR_CUDA(cudaMemcpy(t.buckets, gsr_logf_bucket_start, bb, cudaMemcpyHostToDevice));
        // one bit per 8 consecutive inputs, set when one of them holds a fixup (1 MB)
        std::vector<uint32_t> groups(size_t(gsr_logf_bucket_count) * 4, 0u);
        for (uint32_t k = 0; k < gsr_logf_fixup_count; ++k) {
            const uint32_t off = gsr_logf_fixups[k] >> 1;
            groups[off >> 8] |= 1u << ((off >> 3) & 31u);
        }
        GSR_CUDA(cudaMalloc(&t.groups, groups.size() * 4));
        GSR_CUDA(cudaMemcpy(t.groups, groups.data(), groups.size() * 4, cudaMemcpyHostToDevice));
    }
    out->entries = t.entries;
    out->bucketStart = t.buckets;
    out->groups = t.groups;
    out->base = gsr_logf_fixup_base;
    out->last = gsr_logf_fixup_last;
    out->count = gsr_logf_fixup_count;
    return GSR_OK;
}

// ---- TMA tensor maps (the rasterizer's gather) -------------------------------------------------
// cuTensorMapEncodeTiled through the runtime's driver entry point (the library links no libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensorMapEncoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The full records as a 2-D tensor for tile::gather4: rows = records (48 bytes apart), 12 fp32
// columns, a box of one row of 12 columns (48 bytes, a multiple of 16), no swizzle, zero fill.
bool encodeRecordMap(CUtensorMap* map, void* records, uint64_t rows) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensorMapEncoder();
    if (!encode || !records || rows == 0 || rows >= (1ull << 31) || reinterpret_cast<uintptr_t>(records) % 16) return false;
    const cuuint64_t dims[2] = {12, rows};
    const cuuint64_t strides[1] = {48};
    const cuuint32_t box[2] = {12, 1};
    const cuuint32_t elemStrides[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, records, dims, strides, box, elemStrides,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---- the static scratch of gsr_scan_static, made ready once per device -----------------------
// gsr_scan_static is for callers that must not allocate device memory: recovery code running
// after an allocation failed (the device's memory is held by a resident scene), hooks of a
// caching allocator that must not re-enter it, and streams that must not stall behind cudaFree
// (it synchronizes the whole device). Under CUDA's lazy module loading a module's device arrays
// and a kernel's code are loaded on first use, and loading can allocate. So the array's address
// is looked up and the two kernels the call launches are loaded here, once per device, by every
// set-up call of this library on a device (scene and renderer creation, gsr_scan,
// gsr_sort_pairs) and by gsr_scan_static itself (count 0 does nothing else).
std::mutex g_staticScanMutex;
void* g_staticScanBase[64] = {};

int staticScanReady(void** base) {
    int dev = 0;
    GSR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(GSR_ERROR_UNSUPPORTED, "device index %d", dev);
    std::lock_guard<std::mutex> lock(g_staticScanMutex);
    if (!g_staticScanBase[dev]) {
        void* p = nullptr;
        GSR_CUDA(staticScanScratch(&p));
        GSR_CUDA(loadScanKernel());
        GSR_CUDA(loadFrameBeginKernel());
        g_staticScanBase[dev] = p;
    }
    if (base) *base = g_staticScanBase[dev];
    return GSR_OK;
}

// ---- camera (splat_math.cpp:9-42), host, same evaluation order as the device and the oracle --
void mul4(const float* a, const float* b, float* r) {
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r[c * 4 + row] = a[0 * 4 + row] * b[c * 4 + 0] + a[1 * 4 + row] * b[c * 4 + 1] + a[2 * 4 + row] * b[c * 4 + 2] +
                             a[3 * 4 + row] * b[c * 4 + 3];
}

void splatCamera(const GsrCamera& in, GsrSplatCamera& cam) {
    float flip[16], fv[16];
    for (int i = 0; i < 16; ++i) flip[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    flip[1 * 4 + 1] = -1.0f;
    flip[2 * 4 + 2] = -1.0f;
    mul4(flip, in.view, fv);
    mul4(fv, in.model, cam.view_inria);
    const float tanX = 1.0f / in.proj[0];
    const float tanY = 1.0f / std::fabs(in.proj[1 * 4 + 1]);
    const float* V = cam.view_inria;
    for (int r = 0; r < 3; ++r)
        cam.position[r] = -(V[r * 4 + 0] * V[12] + V[r * 4 + 1] * V[13] + V[r * 4 + 2] * V[14]);
    cam.width = in.width;
    cam.height = in.height;
    cam.tan_half_fov_x = tanX;
    cam.tan_half_fov_y = tanY;
    cam.focal_x = float(in.width) / (2.0f * tanX);
    cam.focal_y = float(in.height) / (2.0f * tanY);
    cam.tiles_x = (in.width + 15) / 16;
    cam.tiles_y = (in.height + 15) / 16;
}

// ---- device buffer RAII -------------------------------------------------------------------
// A 48-byte ProjectedSplat record as the host reads it back (only the depth is used here).
struct DevSplat48 {
    float cx, cy;
    uint32_t depthBits, cullReason;
    float rest[8];
};
static_assert(sizeof(DevSplat48) == 48, "ProjectedSplat layout");

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        bytes = n;
        return cudaMalloc(&p, std::max<size_t>(n, 16));
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// The kernels' view of a scene's buffers and format.
SceneArgs sceneArgs(const GsrSceneDesc& scene) {
    SceneArgs s{};
    s.b0 = static_cast<const uint4*>(scene.buffers[0]);
    s.b1 = static_cast<const uint4*>(scene.layout == GSR_LAYOUT_AOS ? scene.buffers[0] : scene.buffers[1]);
    s.b2 = static_cast<const uint4*>(scene.buffers[2]);
    s.shSoa = static_cast<const float*>(scene.buffers[3]);
    s.geometryStride = scene.geometry_stride;
    s.colorStride = scene.color_stride;
    s.colorOffset = scene.color_offset;
    s.storedCoeffs = scene.sh_coeffs;
    s.codebookStride = scene.codebook_stride;
    const uint64_t entryBytes = uint64_t(scene.codebook_stride) * 16;
    s.codebookLast = entryBytes && scene.buffer_bytes[2] >= entryBytes ? uint32_t(scene.buffer_bytes[2] / entryBytes - 1) : 0u;
    s.variableSh = scene.variable_sh;
    return s;
}

}  // namespace

// ====================================================================================== colour model
struct GsrColorModel {
    uint32_t count = 0;
    int degree = 3;
    GsrColorModelStats stats{};
    GsrColorModelOptions options{};
    uint32_t step = 0;        // Adam steps taken
    std::vector<float> loss;  // of every step taken
    // fp32 parameters, latents, packed decoder; Adam's moments and the device step counter
    // ({step, scratch}) stay with the model so that training can resume from it
    DevBuf params, latents, decoder, mom, vel, stepDev;
};

// ====================================================================================== scene
struct GsrScene {
    GsrSceneDesc desc{};
    DevBuf buffers[4];
    GsrCodebookStats codebook{};
};

namespace {

double msSince(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// The k-means of the cb codebook (kmeans.cpp:193-300, KMeansOptions seed 0x5EED5EED): the host
// draws the training sample and the initial centroids with the same generator and bound, runs the
// Lloyd updates (sequential double sums in sample order) and the re-seeding of empty clusters;
// the nearest-centroid searches (the sample's each iteration and every point's at the end) run on
// the GPU in the AVX2 kernel's arithmetic. `points` (device, n x dims) are the SH-rest vectors;
// `assignment` (device, n) receives every gaussian's entry; `centroids` the codebook (k x dims).
int trainCodebook(const float* points, uint32_t n, uint32_t dims, uint32_t kRequested, uint32_t iterations,
                  uint32_t samples, uint32_t* assignment, std::vector<float>& centroids, GsrCodebookStats& st) {
    const auto start = std::chrono::steady_clock::now();
    st = GsrCodebookStats{};
    st.dimensions = dims;
    if (n == 0 || dims == 0) return GSR_OK;
    const uint32_t k = std::max(1u, std::min(kRequested, n));
    st.entries = k;
    // 1. training sample (sorted indices)
    const uint32_t S = std::min(n, samples ? std::max(samples, k) : uint32_t(std::min<uint64_t>(n, 32ull * k)));
    std::mt19937_64 rng(0x5EED5EEDull);
    auto uniformBelow = [&](uint32_t bound) { return uint32_t((rng() >> 32) * bound >> 32); };
    std::vector<uint32_t> sample;
    if (S == n) {
        sample.resize(n);
        std::iota(sample.begin(), sample.end(), 0u);
    } else {
        std::vector<uint32_t> perm(n);
        std::iota(perm.begin(), perm.end(), 0u);
        for (uint32_t i = 0; i < S; ++i) std::swap(perm[i], perm[i + uniformBelow(n - i)]);  // partial Fisher-Yates
        sample.assign(perm.begin(), perm.begin() + S);
        std::sort(sample.begin(), sample.end());
    }
    st.samples = S;
    DevBuf dSample, dSamplePts, dCent, dNorm, dAssign, dDist, dFullDist;
    GSR_CUDA(dSample.alloc(size_t(S) * 4));
    GSR_CUDA(cudaMemcpy(dSample.p, sample.data(), size_t(S) * 4, cudaMemcpyHostToDevice));
    GSR_CUDA(dSamplePts.alloc(size_t(S) * dims * 4));
    GSR_CUDA(launchCodebookGather(points, dims, dSample.as<uint32_t>(), S, dSamplePts.as<float>(), nullptr));
    std::vector<float> x(size_t(S) * dims);  // the sample's points, in sample order
    GSR_CUDA(cudaMemcpy(x.data(), dSamplePts.p, x.size() * 4, cudaMemcpyDeviceToHost));
    // 2. initial centroids: k distinct sample points
    std::vector<uint32_t> pick(S);
    std::iota(pick.begin(), pick.end(), 0u);
    for (uint32_t i = 0; i < k; ++i) std::swap(pick[i], pick[i + uniformBelow(S - i)]);
    centroids.assign(size_t(k) * dims, 0.0f);
    for (uint32_t j = 0; j < k; ++j) std::copy_n(&x[size_t(pick[j]) * dims], dims, &centroids[size_t(j) * dims]);
    GSR_CUDA(dCent.alloc(size_t(k) * dims * 4));
    GSR_CUDA(dNorm.alloc(size_t(k) * 4));
    GSR_CUDA(dAssign.alloc(size_t(S) * 4));
    GSR_CUDA(dDist.alloc(size_t(S) * 4));
    std::vector<float> norm2(k);
    auto upload = [&]() -> int {  // CentroidTable::build: |c|^2 summed in double
        for (uint32_t j = 0; j < k; ++j) {
            double s = 0.0;
            for (uint32_t d = 0; d < dims; ++d) {
                const float v = centroids[size_t(j) * dims + d];
                s += double(v) * v;
            }
            norm2[j] = float(s);
        }
        GSR_CUDA(cudaMemcpy(dCent.p, centroids.data(), centroids.size() * 4, cudaMemcpyHostToDevice));
        GSR_CUDA(cudaMemcpy(dNorm.p, norm2.data(), size_t(k) * 4, cudaMemcpyHostToDevice));
        return GSR_OK;
    };
    // 3. Lloyd iterations on the sample
    std::vector<uint32_t> assign(S, 0u), previous(S, ~0u);
    std::vector<float> dist(S, 0.0f);
    std::vector<double> sums(size_t(k) * dims);
    std::vector<uint32_t> counts(k);
    for (uint32_t it = 0; it < iterations; ++it) {
        int rc = upload();
        if (rc) return rc;
        GSR_CUDA(launchNearestCentroid(dSamplePts.as<float>(), S, dims, dCent.as<float>(), dNorm.as<float>(), k,
                                       dAssign.as<uint32_t>(), dDist.as<float>(), nullptr));
        GSR_CUDA(cudaMemcpy(assign.data(), dAssign.p, size_t(S) * 4, cudaMemcpyDeviceToHost));
        GSR_CUDA(cudaMemcpy(dist.data(), dDist.p, size_t(S) * 4, cudaMemcpyDeviceToHost));
        st.iterations = it + 1;
        const bool converged = assign == previous;
        previous = assign;
        // update, sequential in sample order
        std::fill(sums.begin(), sums.end(), 0.0);
        std::fill(counts.begin(), counts.end(), 0u);
        for (uint32_t s = 0; s < S; ++s) {
            const float* xs = &x[size_t(s) * dims];
            double* sum = &sums[size_t(assign[s]) * dims];
            for (uint32_t d = 0; d < dims; ++d) sum[d] += xs[d];
            ++counts[assign[s]];
        }
        // empty clusters take the sample points farthest from their centroid
        std::vector<uint32_t> empty;
        for (uint32_t j = 0; j < k; ++j)
            if (counts[j] == 0) empty.push_back(j);
        if (!empty.empty()) {
            std::vector<uint32_t> far(S);
            std::iota(far.begin(), far.end(), 0u);
            const size_t m = std::min(empty.size(), far.size());
            std::partial_sort(far.begin(), far.begin() + std::ptrdiff_t(m), far.end(), [&](uint32_t a, uint32_t b) {
                return dist[a] != dist[b] ? dist[a] > dist[b] : a < b;
            });
            for (size_t e = 0; e < m; ++e) std::copy_n(&x[size_t(far[e]) * dims], dims, &centroids[size_t(empty[e]) * dims]);
            st.empty_reseeded += uint32_t(m);
        }
        for (uint32_t j = 0; j < k; ++j) {
            if (counts[j] == 0) continue;
            for (uint32_t d = 0; d < dims; ++d)
                centroids[size_t(j) * dims + d] = float(sums[size_t(j) * dims + d] / double(counts[j]));
        }
        if (converged) break;
    }
    st.train_ms = msSince(start);
    // 4. every point's entry under the trained centroids, and the errors
    int rc = upload();
    if (rc) return rc;
    const auto tf = std::chrono::steady_clock::now();
    GSR_CUDA(dFullDist.alloc(size_t(n) * 4));
    GSR_CUDA(launchNearestCentroid(points, n, dims, dCent.as<float>(), dNorm.as<float>(), k, assignment,
                                   dFullDist.as<float>(), nullptr));
    std::vector<float> fullDist(n);
    GSR_CUDA(cudaMemcpy(fullDist.data(), dFullDist.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    st.assign_ms = msSince(tf);
    double sampleErr = 0.0, fullErr = 0.0;
    for (uint32_t s = 0; s < S; ++s) sampleErr += fullDist[sample[s]];
    for (uint32_t i = 0; i < n; ++i) fullErr += fullDist[i];
    st.sample_mse = sampleErr / (double(S) * dims);
    st.full_mse = fullErr / (double(n) * dims);
    st.total_ms = msSince(start);
    return GSR_OK;
}

}  // namespace

// ====================================================================================== renderer
struct GsrRenderer {
    GsrSceneDesc scene{};
    GsrSettings settings{};
    int evalDegree = 3;
    LogfFixups logf{};
    // learned colour (gsr_renderer_set_color_model): null = SH colour
    const uint4* colorLatents = nullptr;
    const DecoderWeights* colorDecoder = nullptr;

    // per gaussian
    DevBuf splats, hints, spanRows, tileCounts, offsets, scanStatus;
    DevBuf decodedColours;  // GSR_DECODE_TCGEN05: the pre-pass's colours, 16 B per (view, gaussian)
    DevBuf packedSplats, rects, depths;  // packed render records (P32 / P24) and their side arrays
    DevBuf rayDepth;                     // StopThePop ray-depth parameters (3 x float4 per record)
    // control + plan
    DevBuf control, plan;
    // binning mode: the records' depth words (ping-pong), their sort's look-back words and plan
    DevBuf depthKeys[2], depthStatus, depthPlan;
    // the depth sort's per-view digit counts and bases, [views][depthPasses()][1 << digitBits] each
    DevBuf depthRuns;
    bool binning() const { return settings.list_mode == GSR_LIST_BINNING; }
    // the radix digit width of both sorts, and the depth sort's passes: its keys are the varying
    // depth bits and the no-tile bit, at most 32 bits (depths are positive floats)
    uint32_t digitBits() const { return settings.sort_digit_bits ? settings.sort_digit_bits : 8u; }
    // the binning / render tiles: tile_size 16 or 8 (square), 32 (32 x 8)
    uint32_t tileW() const { return settings.tile_size; }
    uint32_t tileH() const { return settings.tile_size == 32 ? 8u : settings.tile_size; }
    // The depth words of a frame of v views carry the view above the depth bits when the word
    // has room (record bits + 32 depth bits + view bits <= 64): the depth sort then orders by
    // (view, depth), one view's records after another's. 0: no view field (one view, or no room).
    uint32_t depthViewBits(size_t v) const {
        if (v <= 1) return 0u;
        const uint64_t n = uint64_t(scene.count) * v;
        const uint32_t rb = n > 1 ? bitWidth(uint32_t(n - 1)) : 1u, vb = bitWidth(uint32_t(v - 1));
        return rb + 32u + vb <= 64u ? vb : 0u;
    }
    // Passes launched for the depth sort: the depth word's 32 bits (the plan skips the ones the
    // frame's depth range does not need); each view's records are sorted as a run of their own,
    // so the view costs no pass
    uint32_t depthPasses() const { return (32u + digitBits() - 1u) / digitBits(); }
    // its tiles: each view's run of N records in ceil(N / tile) tiles (none straddles two views)
    uint32_t depthTiles(size_t v) const {
        return uint32_t(v * ((size_t(scene.count) + kDepthSortTile - 1) / kDepthSortTile));
    }
    uint32_t depthRunWords(size_t v) const { return uint32_t(v * depthPasses() * statusWordsPerTile()); }
    size_t statusWordsPerTile() const { return size_t(1) << digitBits(); }
    // the output image: bytes per pixel, the kernel's format code, and the RGB8 companion
    uint32_t imageBytes() const {
        const uint32_t f = settings.output_format;
        return f == GSR_OUTPUT_RGBA8 ? 4u : (f == GSR_OUTPUT_RGBA16F || f == GSR_OUTPUT_RGBA16F_AND_RGB8) ? 8u : 16u;
    }
    uint32_t imageFormatCode() const { return imageBytes() == 16 ? 0u : imageBytes() == 8 ? 1u : 2u; }
    bool withRgb8() const {
        return settings.output_format == GSR_OUTPUT_RGBA32F_AND_RGB8 || settings.output_format == GSR_OUTPUT_RGBA16F_AND_RGB8;
    }
    // words of one packed render record (P32: 8, P24: 6)
    uint32_t packedWords() const { return settings.render_splat == GSR_RENDER_SPLAT_P32 ? 8u : 6u; }
    uint32_t recordBits() const {
        const uint64_t n = uint64_t(scene.count) * std::max<size_t>(views.size(), 1);
        return n > 1 ? bitWidth(uint32_t(n - 1)) : 1u;
    }
    // list
    struct List {
        uint32_t capacity = 0;
        uint32_t maxTiles = 0;
        uint32_t passes = 0;
        DevBuf keys[2], values[2], status;
        cudaEvent_t lastUse = nullptr;
        ~List() {
            if (lastUse) cudaEventDestroy(lastUse);
        }
    };
    std::unique_ptr<List> list;
    std::vector<std::unique_ptr<List>> retired;
    uint32_t maxCapacity = 0;
    uint32_t listResizes = 0;
    uint32_t shrinkFrames = 0, shrinkWindowMax = 0;
    uint64_t lastAdaptedFrame = ~0ull;
    // views of the current frame layout (one for gsr_render); width..tilesY are view 0's
    std::vector<GsrViewLayout> views;
    uint32_t totalTiles = 0;
    uint64_t totalPixels = 0;
    uint32_t allocViews = 0;     // per-gaussian arrays and camera slots are sized for this many views
    uint64_t layoutVersion = 0;  // changes whenever the buffers of the layout are re-created
    DevBuf viewsDevice;          // DevView[views]
    // per tile / image
    uint32_t width = 0, height = 0, tilesX = 0, tilesY = 0;
    uint32_t passesUpper = 0;
    DevBuf ranges, image, rgb8;
    DevBuf tileStats, testedPairs;  // the stats build: kTileStatWords per frame tile, one 64-bit total
    // the TMA gather: the tensor map over `splats` (valid while splatMapOk)
    alignas(64) CUtensorMap splatMap{};
    bool splatMapOk = false;
    bool tcDecode() const { return settings.color_decode == GSR_DECODE_TCGEN05; }
    bool tmaGather() const {
        return settings.raster_gather == GSR_GATHER_TMA && settings.render_splat == GSR_RENDER_SPLAT_FULL &&
               settings.sort_window == 0 && !settings.tile_stats;
    }
    // readback slots (2 frames late)
    // Per frame slot: the control readback, the camera (pinned, copied to the slot's device
    // copy by the frame itself), and the frame captured as a CUDA graph.
    struct Slot {
        GsrControl* host = nullptr;
        DevCameraArgs* camHost = nullptr;
        DevBuf camDevice;
        cudaEvent_t done = nullptr;
        bool used = false;
        uint64_t frameIndex = 0;
        cudaGraphExec_t graph = nullptr;
        const void* graphList = nullptr;   // the list / layout the graph was captured with
        uint64_t graphLayout = ~0ull;
        bool graphSplit = false;           // ... and whether it rasterizes view by view
        std::vector<cudaEvent_t> viewDone;  // view-by-view frames: each view's image is complete
        ~Slot() {
            if (graph) cudaGraphExecDestroy(graph);
            for (cudaEvent_t e : viewDone) cudaEventDestroy(e);
        }
    };
    std::vector<std::unique_ptr<Slot>> slots;
    GsrControl lastStats{};
    bool lastStatsValid = false;
    uint64_t lastStatsFrame = 0;
    uint64_t frameIndex = 0;
    uint64_t kernelLaunches = 0;  // kernels of this library launched by render()
    uint32_t forceTimeout = 0;
    // timing
    bool timing = false;
    // events between the passes: global mode times 5 passes, binning mode 7 (its front in three)
    static constexpr int kPasses = 7;
    cudaEvent_t ev[kPasses + 1] = {};
    int evCount = 0;       // events recorded by the last frame (passes + 1)
    bool timed = false;
    void mark(cudaStream_t stream) {
        if (timing && evCount <= kPasses) cudaEventRecord(ev[evCount++], stream);
    }

    cudaStream_t captureStream = nullptr;  // graphs are captured here (never the legacy stream)
    // gsr_render_views_to_host: the frame's views are rasterized one launch each, and each view's
    // image goes to the host on copyStream as soon as it is complete (hostCopies asks for it,
    // lastSplit / lastSlot tell how the last frame ran; row bands of a single view measured no
    // faster, so one-view frames stay whole)
    bool hostCopies = false, lastSplit = false, splitViews = false;
    Slot* lastSlot = nullptr;
    // the parts of such a frame: one per view (its tiles and its pixels)
    struct RenderPart {
        uint32_t tileOffset, tiles;
        uint64_t pixelOffset, pixels;
    };
    std::vector<RenderPart> parts;
    // gsr_render_views_to_host_async: after the frame's copies the copy stream records
    // imageCopied; the next frame's rasterization (of any kind) waits for it, so only the next
    // frame's front overlaps this frame's copies (about 1 ms of copies against 2 ms of front
    // for 8 views at 1080p). hostDone[t mod kHostTickets] marks the end of ticket t's copies
    // (tickets complete in order).
    bool hostAsync = false;
    cudaEvent_t imageCopied = nullptr;
    static constexpr uint32_t kHostTickets = 8;
    cudaEvent_t hostDone[kHostTickets] = {};
    uint64_t hostTickets = 0;
    // the wait before a rasterization launch: an external event node when captured
    int waitCopied(cudaEvent_t e, cudaStream_t stream) {
        if (!e) return GSR_OK;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        GSR_CUDA(cudaStreamIsCapturing(stream, &cs));
        GSR_CUDA(cudaStreamWaitEvent(stream, e, cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0));
        return GSR_OK;
    }
    void planParts() {
        parts.clear();
        for (const GsrViewLayout& L : views)
            parts.push_back(RenderPart{L.tile_base, L.tiles_x * L.tiles_y, L.pixel_base, uint64_t(L.width) * L.height});
    }
    cudaStream_t copyStream = nullptr;

    ~GsrRenderer() {
        for (auto& s : slots) {
            if (s->host) cudaFreeHost(s->host);
            if (s->camHost) cudaFreeHost(s->camHost);
            if (s->done) cudaEventDestroy(s->done);
        }
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (captureStream) cudaStreamDestroy(captureStream);
        if (copyStream) cudaStreamDestroy(copyStream);
        if (imageCopied) cudaEventDestroy(imageCopied);
        for (cudaEvent_t e : hostDone)
            if (e) cudaEventDestroy(e);
    }

    // the (view, tile) queue rasterizer: asked for, or chosen by the auto schedule for batches
    bool persistentRaster(uint32_t viewCount) const {
        return settings.raster_schedule == GSR_RASTER_PERSISTENT ||
               (settings.raster_schedule == GSR_RASTER_AUTO && viewCount > 1);
    }

    uint32_t passesFor(uint32_t tileCount) const {
        // the largest key: tile ids < tileCount + 1 (sentinel) above up to 32 depth bits (global)
        // or alone (binning)
        const uint32_t keyBits = bitWidth(tileCount) + (binning() ? 0u : 32u);
        return (keyBits + digitBits() - 1) / digitBits();
    }

    double bytesPerEntry() const {
        // keys (8 B) + values (4 B), each ping-ponged (binning: the one-word entries alone), + the
        // look-back words of the passes
        const double statusPerPass = double(statusWordsPerTile()) * 8.0 / double(kSortTile);
        return (binning() ? 16.0 : 24.0) + statusPerPass * double(std::max<uint32_t>(passesUpper, 6));
    }

    uint32_t capacityForBytes(double bytes) const {
        uint32_t c = uint32_t(std::clamp(bytes / bytesPerEntry(), double(kBlockSize), double(0xFFFFF800u)));
        return c - c % kBlockSize;
    }

    int createList(uint32_t capacity, std::unique_ptr<List>& out) {
        auto l = std::make_unique<List>();
        l->capacity = capacity;
        l->maxTiles = (capacity + kSortTile - 1) / kSortTile;
        l->passes = passesUpper;
        for (int b = 0; b < 2; ++b) {
            GSR_CUDA(l->keys[b].alloc(size_t(capacity) * 8));
            if (!binning()) GSR_CUDA(l->values[b].alloc(size_t(capacity) * 4));  // binning entries are one word
        }
        GSR_CUDA(l->status.alloc(size_t(l->passes) * l->maxTiles * statusWordsPerTile() * 8));
        GSR_CUDA(cudaMemset(l->status.p, 0, l->status.bytes));
        GSR_CUDA(cudaEventCreateWithFlags(&l->lastUse, cudaEventDisableTiming));
        out = std::move(l);
        return GSR_OK;
    }

    // Per-gaussian arrays and the frame slots' camera copies for `v` views (grown, never shrunk).
    int ensureViews(uint32_t v) {
        if (v <= allocViews) return GSR_OK;
        const size_t n = size_t(scene.count) * v;
        if (settings.render_splat == GSR_RENDER_SPLAT_FULL) {
            GSR_CUDA(splats.alloc(n * 48));
            GSR_CUDA(cudaMemset(splats.p, 0, splats.bytes));
            splatMapOk = tmaGather() && encodeRecordMap(&splatMap, splats.p, n);
        } else {
            GSR_CUDA(packedSplats.alloc(n * packedWords() * 4));
            GSR_CUDA(cudaMemset(packedSplats.p, 0, packedSplats.bytes));
            GSR_CUDA(rects.alloc(n * 8));
            GSR_CUDA(cudaMemset(rects.p, 0, rects.bytes));
            GSR_CUDA(depths.alloc(n * 4));
            GSR_CUDA(cudaMemset(depths.p, 0, depths.bytes));
        }
        GSR_CUDA(hints.alloc(n * 16));
        GSR_CUDA(spanRows.alloc(n * 16));
        if (settings.sort_window > 0) GSR_CUDA(rayDepth.alloc(n * 48));
        if (tcDecode()) GSR_CUDA(decodedColours.alloc(n * 16));
        if (binning()) {
            for (auto& k : depthKeys) GSR_CUDA(k.alloc(n * 8));
            GSR_CUDA(depthStatus.alloc(size_t(depthPasses()) * depthTiles(v) * statusWordsPerTile() * 8));
            GSR_CUDA(cudaMemset(depthStatus.p, 0, depthStatus.bytes));
            GSR_CUDA(depthRuns.alloc(size_t(depthRunWords(v)) * 2 * 4));
            GSR_CUDA(cudaMemset(depthRuns.p, 0, depthRuns.bytes));
        }
        GSR_CUDA(tileCounts.alloc(n * 4));
        GSR_CUDA(offsets.alloc(n * 4));
        GSR_CUDA(scanStatus.alloc((n + 255) / 256 * 8));
        GSR_CUDA(cudaMemset(scanStatus.p, 0, scanStatus.bytes));
        for (auto& s : slots) {
            if (s->camHost) cudaFreeHost(s->camHost);
            s->camHost = nullptr;
            GSR_CUDA(cudaMallocHost(&s->camHost, sizeof(DevCameraArgs) * v));
            GSR_CUDA(s->camDevice.alloc(sizeof(DevCameraArgs) * v));
        }
        allocViews = v;
        return GSR_OK;
    }

    // onRenderTargetsChanged for the views' sizes: the per-tile and image buffers of the frame's
    // tiles and pixels over all views, and the list when the key width changes.
    int setLayout(const uint32_t* w, const uint32_t* h, uint32_t v) {
        if (v == 0 || v > GSR_MAX_VIEWS) return fail(GSR_ERROR_INVALID_ARGUMENT, "views %u (1..%u)", v, GSR_MAX_VIEWS);
        if (copyStream) GSR_CUDA(cudaStreamSynchronize(copyStream));  // copies still reading the old images
        if (uint64_t(scene.count) * v > 0xFFFFF800ull)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "views x gaussians = %llu exceeds 2^32",
                        (unsigned long long)(uint64_t(scene.count) * v));
        bool same = list && views.size() == v;
        uint64_t tiles = 0, pixels = 0;
        for (uint32_t i = 0; i < v; ++i) {
            if (w[i] == 0 || h[i] == 0 || w[i] > 32768 || h[i] > 32768)
                return fail(GSR_ERROR_INVALID_ARGUMENT, "render size %ux%u", w[i], h[i]);
            if (same && (views[i].width != w[i] || views[i].height != h[i])) same = false;
            tiles += uint64_t((w[i] + tileW() - 1) / tileW()) * ((h[i] + tileH() - 1) / tileH());
            pixels += uint64_t(w[i]) * h[i];
        }
        if (same) return GSR_OK;
        if (tiles >= (1ull << 31)) return fail(GSR_ERROR_INVALID_ARGUMENT, "%llu tiles in one frame", (unsigned long long)tiles);
        GSR_CUDA(cudaDeviceSynchronize());  // the reference calls onRenderTargetsChanged with the GPU idle
        int rc = ensureViews(v);
        if (rc) return rc;
        views.assign(v, GsrViewLayout{});
        std::vector<DevView> dv(v);
        uint32_t tileBase = 0;
        uint64_t pixelBase = 0;
        for (uint32_t i = 0; i < v; ++i) {
            GsrViewLayout& L = views[i];
            L.width = w[i];
            L.height = h[i];
            L.tiles_x = (w[i] + tileW() - 1) / tileW();
            L.tiles_y = (h[i] + tileH() - 1) / tileH();
            L.tile_base = tileBase;
            L.pixel_base = pixelBase;
            dv[i] = DevView{L.tile_base, L.tiles_x, L.tiles_y, L.width, L.height, 0, L.pixel_base};
            tileBase += L.tiles_x * L.tiles_y;
            pixelBase += uint64_t(w[i]) * h[i];
        }
        totalTiles = uint32_t(tiles);
        totalPixels = pixels;
        width = views[0].width;
        height = views[0].height;
        tilesX = views[0].tiles_x;
        tilesY = views[0].tiles_y;
        GSR_CUDA(viewsDevice.alloc(sizeof(DevView) * v));
        GSR_CUDA(cudaMemcpy(viewsDevice.p, dv.data(), sizeof(DevView) * v, cudaMemcpyHostToDevice));
        const uint32_t tileCount = totalTiles;
        GSR_CUDA(ranges.alloc(size_t(tileCount) * 8));
        GSR_CUDA(cudaMemset(ranges.p, 0, ranges.bytes));
        if (settings.tile_stats) {
            GSR_CUDA(tileStats.alloc(size_t(tileCount) * kTileStatWords * 4));
            GSR_CUDA(cudaMemset(tileStats.p, 0, tileStats.bytes));
            GSR_CUDA(testedPairs.alloc(8));
        }
        GSR_CUDA(image.alloc(size_t(pixels) * imageBytes()));
        if (withRgb8()) GSR_CUDA(rgb8.alloc(size_t(pixels) * 3));
        else rgb8.release();
        ++layoutVersion;
        const uint32_t passes = passesFor(tileCount);
        if (passes != passesUpper || !list) {
            passesUpper = passes;
            retired.clear();
            maxCapacity = capacityForBytes(double(std::max(settings.budget_mb, 1u)) * 1024.0 * 1024.0);
            uint32_t initial = maxCapacity;
            if (settings.adaptive_list) {
                const uint64_t guess = settings.adaptive_initial_entries
                                           ? settings.adaptive_initial_entries
                                           : std::max<uint64_t>(4ull * scene.count * v, 1u << 20);
                initial = std::min(maxCapacity, roundUpToBlock(guess));
            }
            rc = createList(initial, list);
            if (rc) return rc;
        }
        return GSR_OK;
    }

    int resize(uint32_t w, uint32_t h) { return setLayout(&w, &h, 1); }

    // readSlot (splat_tile_renderer.cpp:572-613): consume a completed readback.
    void readSlot(Slot& s) {
        if (!s.used) return;
        if (cudaEventQuery(s.done) != cudaSuccess) return;  // not finished: try again later
        s.used = false;
        if (lastStatsValid && s.frameIndex < lastStatsFrame) return;
        lastStats = *s.host;
        lastStatsValid = true;
        lastStatsFrame = s.frameIndex;
    }

    // adaptCapacity (splat_tile_renderer.cpp:444-486).
    int adaptCapacity(cudaStream_t stream) {
        for (size_t i = 0; i < retired.size();) {
            if (cudaEventQuery(retired[i]->lastUse) == cudaSuccess) retired.erase(retired.begin() + std::ptrdiff_t(i));
            else ++i;
        }
        (void)stream;
        if (!settings.adaptive_list || !lastStatsValid || lastStatsFrame == lastAdaptedFrame) return GSR_OK;
        lastAdaptedFrame = lastStatsFrame;
        const uint32_t m = lastStats.duplicates;
        const uint32_t cap = list->capacity;
        uint64_t target = 0;
        if (double(m) > 0.9 * cap) {
            target = uint64_t(1.5 * m);
            shrinkFrames = 0;
            shrinkWindowMax = 0;
        } else if (double(m) < 0.4 * cap) {
            shrinkWindowMax = std::max(shrinkWindowMax, m);
            if (++shrinkFrames >= 120) {
                target = uint64_t(1.5 * shrinkWindowMax);
                shrinkFrames = 0;
                shrinkWindowMax = 0;
            }
        } else {
            shrinkFrames = 0;
            shrinkWindowMax = 0;
        }
        if (target == 0) return GSR_OK;
        const uint32_t newCap = std::clamp(roundUpToBlock(target), std::min(kMinAdaptiveCapacity, maxCapacity), maxCapacity);
        if (newCap == cap || (newCap < cap && double(newCap) > 0.75 * cap)) return GSR_OK;
        std::unique_ptr<List> fresh;
        const int rc = createList(newCap, fresh);
        if (rc) return rc;
        retired.push_back(std::move(list));  // freed once its last frame has completed
        list = std::move(fresh);
        ++listResizes;
        return GSR_OK;
    }

    int render(const GsrSplatCamera& cam, cudaStream_t stream) { return renderViews(&cam, 1, stream); }

    // One frame over cameras[0..v): the layout follows the cameras' sizes.
    int renderViews(const GsrSplatCamera* cams, uint32_t v, cudaStream_t stream) {
        if (v == 0 || v > GSR_MAX_VIEWS) return fail(GSR_ERROR_INVALID_ARGUMENT, "views %u (1..%u)", v, GSR_MAX_VIEWS);
        bool same = views.size() == v;
        for (uint32_t i = 0; same && i < v; ++i) same = cams[i].width == views[i].width && cams[i].height == views[i].height;
        if (!same) {
            std::vector<uint32_t> w(v), h(v);
            for (uint32_t i = 0; i < v; ++i) w[i] = cams[i].width, h[i] = cams[i].height;
            const int rc = setLayout(w.data(), h.data(), v);
            if (rc) return rc;
        }
        for (uint32_t i = 0; i < v; ++i)
            if (cams[i].tiles_x != (views[i].width + 15) / 16 || cams[i].tiles_y != (views[i].height + 15) / 16)
                return fail(GSR_ERROR_INVALID_ARGUMENT, "camera %u: tiles %ux%u for a %ux%u image", i, cams[i].tiles_x,
                            cams[i].tiles_y, cams[i].width, cams[i].height);
        if (slots.empty()) return fail(GSR_ERROR_INVALID_ARGUMENT, "renderer not initialised");
        Slot& slot = *slots[frameIndex % slots.size()];
        readSlot(slot);
        if (slot.used) {  // still in flight: wait for it (the reference's frame fence)
            GSR_CUDA(cudaEventSynchronize(slot.done));
            readSlot(slot);
        }
        int rc = adaptCapacity(stream);
        if (rc) return rc;
        // the slot's previous frame has completed: its pinned cameras may be overwritten
        static_assert(sizeof(DevCameraArgs) == sizeof(GsrSplatCamera), "camera layout");
        std::memcpy(slot.camHost, cams, sizeof(GsrSplatCamera) * v);
        // view by view: several per-tile views with their images wanted on the host
        // (the streaming call rasterizes the frame whole: its copies overlap the next frame's
        // front, so they need not start view by view)
        const bool split = hostCopies && v > 1 && !hostAsync && !persistentRaster(v);
        if (split) planParts();
        while (split && slot.viewDone.size() < parts.size()) {
            cudaEvent_t e = nullptr;
            GSR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            slot.viewDone.push_back(e);
        }

        splitViews = split;
        lastSplit = split;
        lastSlot = &slot;
        const bool graphed = settings.use_graph && !timing && forceTimeout == 0;
        if (graphed) {
            if (!slot.graph || slot.graphList != list.get() || slot.graphLayout != layoutVersion ||
                slot.graphSplit != split) {
                if (slot.graph) cudaGraphExecDestroy(slot.graph);
                slot.graph = nullptr;
                if (!captureStream) GSR_CUDA(cudaStreamCreateWithFlags(&captureStream, cudaStreamNonBlocking));
                GSR_CUDA(cudaStreamBeginCapture(captureStream, cudaStreamCaptureModeThreadLocal));
                const int erc = enqueue(slot, captureStream);
                cudaGraph_t g = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(captureStream, &g);
                if (erc) {
                    if (g) cudaGraphDestroy(g);
                    return erc;
                }
                if (ce != cudaSuccess) return cudaFail(ce, "cudaStreamEndCapture");
                const cudaError_t ie = cudaGraphInstantiate(&slot.graph, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return cudaFail(ie, "cudaGraphInstantiate");
                slot.graphList = list.get();
                slot.graphLayout = layoutVersion;
                slot.graphSplit = split;
            }
            GSR_CUDA(cudaGraphLaunch(slot.graph, stream));
        } else {
            rc = enqueue(slot, stream);
            if (rc) return rc;
        }
        // completion of this frame (outside any capture: an event recorded while capturing only
        // orders the captured work and is not a usable event afterwards)
        GSR_CUDA(cudaEventRecord(slot.done, stream));
        GSR_CUDA(cudaEventRecord(list->lastUse, stream));
        mark(stream);
        forceTimeout = 0;
        slot.used = true;
        slot.frameIndex = frameIndex;
        // frameBegin, preprocess, scan, duplicate, histogram, one per pass, ranges, render
        // binning: frameBegin, preprocess, depth histogram + passes, scan, duplicate, list
        // histogram + passes, ranges, render
        kernelLaunches += (binning() ? 8 + depthPasses() + list->passes : 7 + list->passes) + (split ? uint32_t(parts.size()) - 1 : 0) +
                          (colorLatents && tcDecode() ? 1u : 0u);
        timed = timing;
        ++frameIndex;
        return GSR_OK;
    }

    // The frame's work on `stream`: the camera copy, the kernels, the control readback and the
    // completion events (captured once per slot when graphs are on).
    int enqueue(Slot& slot, cudaStream_t stream) {
        List& l = *list;
        DeviceControl* ctl = control.as<DeviceControl>();
        SortPlan* sortPlan = plan.as<SortPlan>();
        const uint32_t tileCount = totalTiles;
        const uint32_t viewCount = uint32_t(views.size());
        evCount = 0;
        mark(stream);
        GSR_CUDA(cudaMemcpyAsync(slot.camDevice.p, slot.camHost, sizeof(DevCameraArgs) * viewCount,
                                 cudaMemcpyHostToDevice, stream));
        GSR_CUDA(launchFrameBegin(ctl, scene.count * viewCount, l.capacity, ranges.as<uint32_t>(), tileCount * 2,
                                  sortPlan, forceTimeout, stream, binning() ? depthPlan.as<SortPlan>() : nullptr,
                                  binning() ? depthRuns.as<uint32_t>() : nullptr,
                                  binning() ? depthRunWords(viewCount) : 0u));
        FrontArgs fa{};
        fa.cam = slot.camDevice.as<DevCameraArgs>();
        fa.views = viewsDevice.as<DevView>();
        fa.viewCount = viewCount;
        fa.totalTiles = tileCount;
        fa.scene = sceneArgs(scene);
        fa.latents = colorLatents;
        fa.decoder = colorDecoder;
        fa.decoded = colorLatents && tcDecode() ? decodedColours.as<float4>() : nullptr;
        fa.count = scene.count;
        fa.evalDegree = evalDegree;
        fa.bounds = settings.bounds;
        fa.binSize = int(settings.tile_size);
        fa.capacity = l.capacity;
        fa.splats = splats.p;
        fa.renderSplat = settings.render_splat;
        fa.packed = packedSplats.p;
        fa.rects = rects.as<uint2>();
        fa.depths = depths.as<uint32_t>();
        fa.rayDepth = settings.sort_window > 0 ? rayDepth.as<float4>() : nullptr;
        fa.hints = hints.as<float4>();
        fa.spanRows = spanRows.as<uint4>();
        fa.tileCounts = tileCounts.as<uint32_t>();
        fa.offsets = offsets.as<uint32_t>();
        fa.keys = l.keys[0].as<uint64_t>();
        fa.values = l.values[0].as<uint32_t>();
        fa.scanStatus = scanStatus.as<uint64_t>();
        fa.ctl = ctl;
        fa.logf = logf;
        if (fa.decoded) GSR_CUDA(launchDecodeColoursTc(fa, scene.geometry, stream));  // timed with the preprocess
        if (binning()) {
            fa.binning = 1;
            fa.depthKeys[0] = depthKeys[0].as<uint64_t>();
            fa.depthKeys[1] = depthKeys[1].as<uint64_t>();
            fa.depthPlan = depthPlan.as<SortPlan>();
            fa.recordBits = recordBits();
            const uint32_t viewBits = depthViewBits(viewCount);
            fa.depthViewShift = viewBits ? fa.recordBits + 32u : 0u;
            GSR_CUDA(launchFrontBinningKeys(fa, scene.geometry, scene.color, stream));
            mark(stream);
            // each view's records by (depth, record index): 32 depth bits above the record index,
            // the views' runs sorted side by side in one launch per pass
            SortArgs sd{};
            sd.keys[0] = fa.depthKeys[0];
            sd.keys[1] = fa.depthKeys[1];
            sd.status = depthStatus.as<uint64_t>();
            sd.maxTiles = depthTiles(viewCount);
            sd.plan = depthPlan.as<SortPlan>();
            sd.ctl = ctl;
            sd.passesLaunched = depthPasses();
            sd.digitBits = digitBits();
            sd.frameMode = 2;
            sd.count = scene.count * viewCount;
            sd.indexBits = fa.recordBits;
            sd.segments = viewCount;
            sd.segLength = scene.count;
            sd.segHist = depthRuns.as<uint32_t>();
            sd.segBase = depthRuns.as<uint32_t>() + depthRunWords(allocViews);
            GSR_CUDA(launchSort(sd, 148 * 2, stream));
            mark(stream);
            GSR_CUDA(launchFrontBinningEmit(fa, stream));
        } else {
            GSR_CUDA(launchFront(fa, scene.geometry, scene.color, stream));
        }
        mark(stream);

        SortArgs sa{};
        for (int b = 0; b < 2; ++b) {
            sa.keys[b] = l.keys[b].as<uint64_t>();
            sa.values[b] = l.values[b].as<uint32_t>();
        }
        sa.status = l.status.as<uint64_t>();
        sa.maxTiles = l.maxTiles;
        sa.plan = sortPlan;
        sa.ctl = ctl;
        sa.passesLaunched = l.passes;
        sa.digitBits = digitBits();
        sa.frameMode = 1;
        sa.binning = binning() ? 1u : 0u;
        sa.tileCount = tileCount;
        sa.count = scene.count;
        GSR_CUDA(launchSort(sa, 148 * 4, stream));
        mark(stream);

        RenderArgs ra{};
        ra.splats = splats.p;
        ra.renderSplat = settings.render_splat;
        ra.packed = packedSplats.p;
        ra.rayDepth = rayDepth.as<float4>();
        ra.cam = slot.camDevice.as<DevCameraArgs>();
        ra.sortWindow = settings.sort_window;
        ra.tileSize = settings.tile_size;
        ra.bounds = settings.bounds;
        for (int b = 0; b < 2; ++b) {
            ra.values[b] = l.values[b].as<uint32_t>();
            ra.keys[b] = l.keys[b].as<uint64_t>();
        }
        ra.ranges = ranges.as<uint32_t>();
        ra.image = image.p;
        ra.imageFormat = imageFormatCode();
        ra.rgb8 = rgb8.as<uint8_t>();
        ra.views = viewsDevice.as<DevView>();
        ra.viewCount = viewCount;
        ra.totalTiles = tileCount;
        ra.persistent = persistentRaster(viewCount);
        ra.count = scene.count;
        ra.ctl = ctl;
        ra.plan = sortPlan;
        ra.splatMap = splatMapOk && tmaGather() ? &splatMap : nullptr;
        if (settings.tile_stats) {
            ra.tileStats = tileStats.as<uint32_t>();
            ra.testedPairs = testedPairs.as<unsigned long long>();
            GSR_CUDA(cudaMemsetAsync(testedPairs.p, 0, 8, stream));
        }
        GSR_CUDA(launchRanges(ra, l.capacity, stream));
        mark(stream);
        // the images may still be on their way to the host (the streaming call): wait for it
        if (int rc = waitCopied(imageCopied, stream)) return rc;
        if (splitViews) {
            // inside a capture the view events become external event nodes (recorded by each
            // launch of the graph); outside one they are plain records
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            GSR_CUDA(cudaStreamIsCapturing(stream, &cs));
            const unsigned recordFlags = cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
            for (size_t j = 0; j < parts.size(); ++j) {
                ra.tileOffset = parts[j].tileOffset;
                ra.tileLaunch = parts[j].tiles;
                GSR_CUDA(launchRender(ra, stream));
                GSR_CUDA(cudaEventRecordWithFlags(slot.viewDone[j], stream, recordFlags));
            }
        } else {
            GSR_CUDA(launchRender(ra, stream));
        }
        mark(stream);

        GSR_CUDA(cudaMemcpyAsync(slot.host, &ctl->c, sizeof(GsrControl), cudaMemcpyDeviceToHost, stream));
        return GSR_OK;
    }
};

namespace {

int validateScene(const GsrSceneDesc& s) {
    if (s.count == 0) return fail(GSR_ERROR_INVALID_ARGUMENT, "empty scene");
    if (s.sh_degree < 0 || s.sh_degree > 3) return fail(GSR_ERROR_INVALID_ARGUMENT, "sh_degree %d", s.sh_degree);
    if (s.sh_coeffs != uint32_t((s.sh_degree + 1) * (s.sh_degree + 1)))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "sh_coeffs %u for degree %d", s.sh_coeffs, s.sh_degree);
    const bool soa = s.geometry == GSR_GEOMETRY_SOA_F32 && s.color == GSR_COLOR_SOA_F32;
    const bool f32 = s.geometry == GSR_GEOMETRY_RECORD_F32 && s.color == GSR_COLOR_RECORD_F32;
    const bool f16 = s.geometry == GSR_GEOMETRY_RECORD_F16 && s.color == GSR_COLOR_RECORD_F16;
    const bool q8 = s.geometry == GSR_GEOMETRY_RECORD_F16 && s.color == GSR_COLOR_Q8;
    const bool cb = s.geometry == GSR_GEOMETRY_RECORD_F16 && s.color == GSR_COLOR_CODEBOOK;
    if (cb && (!s.buffers[2] || s.codebook_stride == 0 || s.buffer_bytes[2] < uint64_t(s.codebook_stride) * 16))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "a codebook scene needs the codebook buffer and its stride");
    if (cb && s.variable_sh == GSR_VARIABLE_SH_COMPACT)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "cb colour records are fixed-size (no compacted variable SH)");
    if (!(soa || f32 || f16 || q8 || cb))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "geometry encoding %u with colour encoding %u", s.geometry, s.color);
    if (s.variable_sh > GSR_VARIABLE_SH_COMPACT) return fail(GSR_ERROR_INVALID_ARGUMENT, "variable_sh %u", s.variable_sh);
    if (soa && (!s.buffers[0] || !s.buffers[1] || !s.buffers[2] || !s.buffers[3]))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "soa scene needs 4 buffers");
    if (!soa && (!s.buffers[0] || (s.layout != GSR_LAYOUT_AOS && !s.buffers[1])))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "record scene needs its buffers");
    if (!soa && s.geometry_stride == 0) return fail(GSR_ERROR_INVALID_ARGUMENT, "geometry_stride 0");
    for (int b = 0; b < 4; ++b)
        if (reinterpret_cast<uintptr_t>(s.buffers[b]) % 16 != 0)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "scene buffer %d is not 16-byte aligned", b);
    return GSR_OK;
}

}  // namespace

// ====================================================================================== C ABI
extern "C" {

int gsr_abi_version(void) { return GSR_ABI_VERSION; }

const char* gsr_error_string(int status) {
    switch (status) {
        case GSR_OK: return "ok";
        case GSR_ERROR_INVALID_ARGUMENT: return "invalid argument";
        case GSR_ERROR_UNSUPPORTED: return "unsupported";
        case GSR_ERROR_CUDA: return "CUDA error";
        case GSR_ERROR_OUT_OF_MEMORY: return "out of device memory";
        case GSR_ERROR_DEVICE_TIMEOUT: return "a device-side wait timed out";
        case GSR_ERROR_NOT_READY: return "not ready";
        case GSR_ERROR_FORMAT: return "malformed input file";
        case GSR_ERROR_IO: return "file I/O error";
        default: return "unknown status";
    }
}

const char* gsr_last_error_message(void) { return g_lastError.c_str(); }

void gsr_settings_default(GsrSettings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->bounds = GSR_BOUNDS_TIGHT;
    s->tile_size = 16;
    s->budget_mb = 256;
    s->adaptive_list = 1;
    s->adaptive_initial_entries = 0;
    s->max_sh_degree = 3;
    s->output_format = GSR_OUTPUT_RGBA32F;
    s->frames_in_flight = 2;
    s->use_graph = 0;
}

int gsr_splat_camera_from_viewer(const GsrCamera* camera, GsrSplatCamera* out) {
    if (!camera || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    splatCamera(*camera, *out);
    return GSR_OK;
}

void gsr_look_at(const float eye[3], const float center[3], const float up[3], float view[16]) {
    auto normalize = [](const float v[3], float o[3]) {
        const float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        o[0] = v[0] * inv;
        o[1] = v[1] * inv;
        o[2] = v[2] * inv;
    };
    auto cross = [](const float a[3], const float b[3], float o[3]) {
        o[0] = a[1] * b[2] - b[1] * a[2];
        o[1] = a[2] * b[0] - b[2] * a[0];
        o[2] = a[0] * b[1] - b[0] * a[1];
    };
    auto dot = [](const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const float d[3] = {center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]};
    float f[3], sr[3], s[3], u[3];
    normalize(d, f);
    cross(f, up, sr);
    normalize(sr, s);
    cross(s, f, u);
    for (int i = 0; i < 16; ++i) view[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    view[0] = s[0]; view[4] = s[1]; view[8] = s[2];
    view[1] = u[0]; view[5] = u[1]; view[9] = u[2];
    view[2] = -f[0]; view[6] = -f[1]; view[10] = -f[2];
    view[12] = -dot(s, eye);
    view[13] = -dot(u, eye);
    view[14] = dot(f, eye);
}

void gsr_perspective_vk(float fovy, float aspect, float zNear, float zFar, float proj[16]) {
    const float t = std::tan(fovy / 2.0f);
    for (int i = 0; i < 16; ++i) proj[i] = 0.0f;
    proj[0] = 1.0f / (aspect * t);
    proj[5] = -(1.0f / t);
    proj[10] = zFar / (zNear - zFar);
    proj[11] = -1.0f;
    proj[14] = -(zFar * zNear) / (zFar - zNear);
}

// ---- scene ------------------------------------------------------------------------------------
int gsr_scene_create(const GsrHostScene* host, const GsrCompression* options, GsrScene** out) {
    if (!host || !options || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (host->count == 0 || host->sh_degree < 0 || host->sh_degree > 3 || !host->pos_alpha || !host->scales ||
        !host->rotations || !host->sh)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "host scene (count %u, degree %d)", host->count, host->sh_degree);
    const uint32_t fmt = options->format, layout = options->layout;
    if (fmt > GSR_FORMAT_CB || layout > GSR_LAYOUT_AOS) return fail(GSR_ERROR_INVALID_ARGUMENT, "format %u layout %u", fmt, layout);
    if (fmt != GSR_FORMAT_F32 && layout == GSR_LAYOUT_SOA)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "scene layout 'soa' exists only for the f32 format (use split or aos)");
    const int ready = staticScanReady(nullptr);  // gsr_scan_static's scratch and kernels on this device
    if (ready) return ready;
    const uint32_t n = host->count;
    const uint32_t srcK = uint32_t((host->sh_degree + 1) * (host->sh_degree + 1));
    const int degree = std::clamp(std::min(host->sh_degree, options->max_sh_degree), 0, 3);
    const uint32_t K = uint32_t((degree + 1) * (degree + 1));
    const bool variable = options->sh_threshold >= 0.0f && degree > 0;

    auto scene = std::make_unique<GsrScene>();
    GsrSceneDesc& d = scene->desc;
    d.count = n;
    d.sh_degree = degree;
    d.sh_coeffs = K;
    d.format = fmt;
    d.layout = layout;
    // staging: the activated f32 arrays on the device
    DevBuf pa, sc, ro, sh, degrees, sizes, offs;
    GSR_CUDA(pa.alloc(size_t(n) * 16));
    GSR_CUDA(sc.alloc(size_t(n) * 16));
    GSR_CUDA(ro.alloc(size_t(n) * 16));
    GSR_CUDA(sh.alloc(size_t(n) * srcK * 12));
    GSR_CUDA(cudaMemcpy(pa.p, host->pos_alpha, pa.bytes, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(sc.p, host->scales, sc.bytes, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(ro.p, host->rotations, ro.bytes, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(sh.p, host->sh, sh.bytes, cudaMemcpyHostToDevice));

    EncodeArgs ea{};
    ea.pa = pa.as<float4>();
    ea.sc = sc.as<float4>();
    ea.ro = ro.as<float4>();
    ea.sh = sh.as<float>();
    ea.n = n;
    ea.srcK = srcK;
    ea.K = K;
    ea.degree = degree;
    ea.variable = variable ? 1 : 0;
    ea.threshold255 = options->sh_threshold;
    ea.layout = layout;
    if (layout == GSR_LAYOUT_SOA) {
        ea.geometry = GSR_GEOMETRY_SOA_F32;
        ea.color = GSR_COLOR_SOA_F32;
    } else {
        ea.geometry = fmt == GSR_FORMAT_F32 ? GSR_GEOMETRY_RECORD_F32 : GSR_GEOMETRY_RECORD_F16;
        ea.color = fmt == GSR_FORMAT_F32   ? GSR_COLOR_RECORD_F32
                   : fmt == GSR_FORMAT_F16 ? GSR_COLOR_RECORD_F16
                   : fmt == GSR_FORMAT_Q8  ? GSR_COLOR_Q8
                                           : GSR_COLOR_CODEBOOK;
    }
    const bool cb = ea.color == GSR_COLOR_CODEBOOK;
    auto vec4sFor = [](uint32_t bytes) { return (bytes + 15u) / 16u; };
    ea.geomWords = ea.geometry == GSR_GEOMETRY_RECORD_F16 ? 8u : 12u;
    ea.colorWords = ea.color == GSR_COLOR_RECORD_F32   ? vec4sFor(K * 12) * 4
                    : ea.color == GSR_COLOR_RECORD_F16 ? vec4sFor(K * 6) * 4
                    : ea.color == GSR_COLOR_Q8         ? vec4sFor(12 + (K - 1) * 3) * 4
                    : cb                               ? (layout == GSR_LAYOUT_SPLIT ? 2u : 4u)  // two 8-byte records per uvec4 (split)
                                                       : 0;
    GSR_CUDA(degrees.alloc(n));
    const bool compact = variable && !cb && (layout == GSR_LAYOUT_SOA || layout == GSR_LAYOUT_SPLIT);
    uint64_t compactTotal = 0;
    if (compact) {
        GSR_CUDA(sizes.alloc(size_t(n) * 4));
        GSR_CUDA(offs.alloc(size_t(n) * 4));
    }
    GSR_CUDA(launchEncodeDegrees(ea, degrees.as<uint8_t>(), compact ? sizes.as<uint32_t>() : nullptr, 0));
    if (compact) {
        DevBuf total;
        GSR_CUDA(total.alloc(4));
        const int rc = gsr_scan(sizes.as<uint32_t>(), nullptr, offs.as<uint32_t>(), total.as<uint32_t>(), n, GSR_SCAN_PLAIN, nullptr);
        if (rc) return rc;
        uint32_t t = 0;
        GSR_CUDA(cudaMemcpy(&t, total.p, 4, cudaMemcpyDeviceToHost));
        compactTotal = t;
        if (compactTotal >= (1ull << 30)) return fail(GSR_ERROR_INVALID_ARGUMENT, "variable SH: compacted data exceeds 2^30");
    }
    // cb: the k-means codebook of the SH-rest vectors, and every gaussian's entry
    DevBuf cbPoints, cbAssign;
    std::vector<float> centroids;
    const uint32_t restDims = (K - 1) * 3;
    if (cb && restDims > 0) {
        GSR_CUDA(cbPoints.alloc(size_t(n) * restDims * 4));
        GSR_CUDA(cbAssign.alloc(size_t(n) * 4));
        GSR_CUDA(launchCodebookPoints(ea, degrees.as<uint8_t>(), cbPoints.as<float>(), 0));
        const uint32_t size = std::clamp(options->codebook_size ? options->codebook_size : 4096u, 1u, 65536u);
        const uint32_t iters = options->codebook_iterations ? options->codebook_iterations : 10u;
        int rc = trainCodebook(cbPoints.as<float>(), n, restDims, size, iters, options->codebook_samples,
                               cbAssign.as<uint32_t>(), centroids, scene->codebook);
        if (rc) return rc;
        ea.cbIndex = cbAssign.as<uint32_t>();
    }
    size_t bytes[4] = {0, 0, 0, 0};
    if (layout == GSR_LAYOUT_SOA) {
        bytes[0] = bytes[1] = bytes[2] = size_t(n) * 16;
        bytes[3] = (compact ? size_t(compactTotal) : size_t(n) * K * 3) * 4;
        d.geometry = GSR_GEOMETRY_SOA_F32;
        d.color = GSR_COLOR_SOA_F32;
        d.variable_sh = variable ? GSR_VARIABLE_SH_COMPACT : GSR_VARIABLE_SH_OFF;
    } else if (layout == GSR_LAYOUT_SPLIT) {
        bytes[0] = size_t(n) * ea.geomWords * 4;
        bytes[1] = compact ? size_t(compactTotal) * 16 : size_t(n) * ea.colorWords * 4;
        d.geometry = ea.geometry;
        d.color = ea.color;
        d.geometry_stride = ea.geomWords / 4;
        d.color_stride = cb ? 0u : ea.colorWords / 4;  // cb: records packed two per 16 bytes
        d.variable_sh = !variable ? GSR_VARIABLE_SH_OFF : compact ? GSR_VARIABLE_SH_COMPACT : GSR_VARIABLE_SH_DEGREE_ONLY;
    } else {
        bytes[0] = size_t(n) * (ea.geomWords + ea.colorWords) * 4;
        d.geometry = ea.geometry;
        d.color = ea.color;
        d.geometry_stride = (ea.geomWords + ea.colorWords) / 4;
        d.color_stride = (ea.geomWords + ea.colorWords) / 4;
        d.color_offset = ea.geomWords / 4;
        d.variable_sh = variable ? GSR_VARIABLE_SH_DEGREE_ONLY : GSR_VARIABLE_SH_OFF;
    }
    std::vector<uint32_t> codebookWords;
    if (cb) {  // entries of (K - 1) * 3 fp32 words padded to 16 bytes (at least one entry)
        const uint32_t entryWords = std::max(4u, vec4sFor(restDims * 4) * 4);
        d.codebook_stride = entryWords / 4;
        const uint32_t entries = scene->codebook.entries;
        codebookWords.assign(size_t(std::max(entries, 1u)) * entryWords, 0u);
        for (uint32_t c = 0; c < entries; ++c)
            std::memcpy(&codebookWords[size_t(c) * entryWords], &centroids[size_t(c) * restDims], size_t(restDims) * 4);
        bytes[2] = codebookWords.size() * 4;
    }
    for (int b = 0; b < 4; ++b) {
        if (!bytes[b]) continue;
        GSR_CUDA(scene->buffers[b].alloc(bytes[b]));
        GSR_CUDA(cudaMemset(scene->buffers[b].p, 0, bytes[b]));
        ea.out[b] = scene->buffers[b].p;
        d.buffers[b] = scene->buffers[b].p;
        d.buffer_bytes[b] = bytes[b];
    }
    if (cb) GSR_CUDA(cudaMemcpy(scene->buffers[2].p, codebookWords.data(), bytes[2], cudaMemcpyHostToDevice));
    GSR_CUDA(launchEncodeRecords(ea, degrees.as<uint8_t>(), compact ? offs.as<uint32_t>() : nullptr, 0));
    GSR_CUDA(cudaDeviceSynchronize());
    *out = scene.release();
    return GSR_OK;
}

int gsr_scene_codebook_stats(const GsrScene* scene, GsrCodebookStats* out) {
    if (!scene || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = scene->codebook;
    return GSR_OK;
}

void gsr_compression_default(GsrCompression* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->format = GSR_FORMAT_F32;
    c->layout = GSR_LAYOUT_SOA;
    c->max_sh_degree = 3;
    c->sh_threshold = -1.0f;
    c->codebook_size = 4096;
    c->codebook_iterations = 10;
}

int gsr_scene_get_desc(const GsrScene* scene, GsrSceneDesc* out) {
    if (!scene || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = scene->desc;
    return GSR_OK;
}

int gsr_scene_read_buffer(const GsrScene* scene, uint32_t b, void* host, uint64_t bytes) {
    if (!scene || b > 3 || !host) return fail(GSR_ERROR_INVALID_ARGUMENT, "bad argument");
    if (bytes != scene->desc.buffer_bytes[b]) return fail(GSR_ERROR_INVALID_ARGUMENT, "size %llu != %llu",
                                                          (unsigned long long)bytes, (unsigned long long)scene->desc.buffer_bytes[b]);
    if (bytes) GSR_CUDA(cudaMemcpy(host, scene->buffers[b].p, bytes, cudaMemcpyDeviceToHost));
    return GSR_OK;
}

void gsr_scene_destroy(GsrScene* scene) { delete scene; }

// ---- renderer ----------------------------------------------------------------------------------
int gsr_renderer_create(const GsrSceneDesc* scene, const GsrSettings* settings, GsrRenderer** out) {
    if (!scene || !settings || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int rc = validateScene(*scene);
    if (rc) return rc;
    if (settings->tile_size != 8 && settings->tile_size != 16 && settings->tile_size != 32)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "--tile-size must be 8, 16 or 32 (8 x 8, 16 x 16 or 32 x 8 tiles)");
    if (settings->bounds > GSR_BOUNDS_CUTOFF_ONLY) return fail(GSR_ERROR_INVALID_ARGUMENT, "bounds %u", settings->bounds);
    if (settings->output_format > GSR_OUTPUT_RGBA8)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "output format %u", settings->output_format);
    auto r = std::make_unique<GsrRenderer>();
    r->scene = *scene;
    r->settings = *settings;
    r->settings.max_sh_degree = std::clamp(settings->max_sh_degree, 0, 3);
    r->settings.frames_in_flight = std::max(settings->frames_in_flight, 1u);
    r->evalDegree = std::min(scene->sh_degree, r->settings.max_sh_degree);
    rc = deviceTables(&r->logf);
    if (rc) return rc;
    rc = staticScanReady(nullptr);  // gsr_scan_static's scratch and kernels on this device
    if (rc) return rc;
    if (settings->list_mode > GSR_LIST_GLOBAL) return fail(GSR_ERROR_INVALID_ARGUMENT, "list mode %u", settings->list_mode);
    if (settings->sort_window > 64)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "sort window %u (at most 64)", settings->sort_window);
    if (settings->render_splat > GSR_RENDER_SPLAT_P24)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "render splat mode %u", settings->render_splat);
    if (settings->raster_schedule > GSR_RASTER_PERSISTENT)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "raster schedule %u", settings->raster_schedule);
    if (settings->raster_gather > GSR_GATHER_TMA ||
        (settings->raster_gather == GSR_GATHER_TMA &&
         (settings->render_splat != GSR_RENDER_SPLAT_FULL || settings->sort_window > 0 || settings->tile_stats)))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "raster gather %u (TMA: full records, no sort window, no tile stats)",
                    settings->raster_gather);
    if (settings->tile_stats > 1 || (settings->tile_stats && settings->sort_window > 0))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "tile_stats %u (0 or 1, not with sort_window)", settings->tile_stats);
    if (settings->sort_digit_bits != 0 && (settings->sort_digit_bits < 7 || settings->sort_digit_bits > 9))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "sort digit bits %u (7, 8 or 9)", settings->sort_digit_bits);
    if (settings->color_decode > GSR_DECODE_TCGEN05)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "colour decode %u", settings->color_decode);
    GSR_CUDA(r->control.alloc(sizeof(DeviceControl)));
    GSR_CUDA(cudaMemset(r->control.p, 0, sizeof(DeviceControl)));
    GSR_CUDA(r->plan.alloc(sizeof(SortPlan)));
    GSR_CUDA(cudaMemset(r->plan.p, 0, sizeof(SortPlan)));
    GSR_CUDA(r->depthPlan.alloc(sizeof(SortPlan)));
    GSR_CUDA(cudaMemset(r->depthPlan.p, 0, sizeof(SortPlan)));
    for (uint32_t k = 0; k < r->settings.frames_in_flight; ++k) {
        auto s = std::make_unique<GsrRenderer::Slot>();
        GSR_CUDA(cudaMallocHost(&s->host, sizeof(GsrControl)));
        std::memset(s->host, 0, sizeof(GsrControl));
        GSR_CUDA(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
        r->slots.push_back(std::move(s));
    }
    rc = r->ensureViews(1);
    if (rc) return rc;
    for (auto& e : r->ev) GSR_CUDA(cudaEventCreate(&e));
    GSR_CUDA(cudaEventCreateWithFlags(&r->imageCopied, cudaEventDisableTiming));
    for (auto& e : r->hostDone) GSR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *out = r.release();
    return GSR_OK;
}

int gsr_renderer_resize(GsrRenderer* r, uint32_t width, uint32_t height) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    return r->resize(width, height);
}

int gsr_render_splat_camera(GsrRenderer* r, const GsrSplatCamera* camera, void* stream) {
    if (!r || !camera) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    return r->render(*camera, static_cast<cudaStream_t>(stream));
}

int gsr_render(GsrRenderer* r, const GsrCamera* camera, void* stream) {
    if (!r || !camera) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    GsrSplatCamera cam;
    splatCamera(*camera, cam);
    return r->render(cam, static_cast<cudaStream_t>(stream));
}

int gsr_renderer_image(GsrRenderer* r, const void** rgba, const void** rgb8, uint32_t* width, uint32_t* height) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (rgba) *rgba = r->image.p;
    if (rgb8) *rgb8 = r->rgb8.p;
    if (width) *width = r->width;
    if (height) *height = r->height;
    return GSR_OK;
}

namespace {
// The frame's images to `host` (RGB8 when kept, else the output format): part by part on the
// renderer's copy stream after each part's rasterizer launch when the frame ran in parts, else
// one copy on `s`; then both streams are synchronized.
int copyFrameToHost(GsrRenderer* r, void* host, uint64_t need, cudaStream_t s) {
    const bool rgb = r->rgb8.p != nullptr;
    const size_t bpp = rgb ? 3 : r->imageBytes();
    const unsigned char* src = rgb ? r->rgb8.as<unsigned char>() : r->image.as<unsigned char>();
    if (r->lastSplit) {
        if (!r->copyStream) GSR_CUDA(cudaStreamCreateWithFlags(&r->copyStream, cudaStreamNonBlocking));
        for (size_t j = 0; j < r->parts.size(); ++j) {
            const size_t off = size_t(r->parts[j].pixelOffset) * bpp, len = size_t(r->parts[j].pixels) * bpp;
            GSR_CUDA(cudaStreamWaitEvent(r->copyStream, r->lastSlot->viewDone[j], 0));
            GSR_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(host) + off, src + off, len, cudaMemcpyDeviceToHost,
                                     r->copyStream));
        }
        GSR_CUDA(cudaStreamSynchronize(r->copyStream));
    } else {
        GSR_CUDA(cudaMemcpyAsync(host, src, need, cudaMemcpyDeviceToHost, s));
    }
    GSR_CUDA(cudaStreamSynchronize(s));
    return GSR_OK;
}
}  // namespace

int gsr_render_to_host(GsrRenderer* r, const GsrCamera* camera, void* host, uint64_t bytes, void* stream) {
    if (!r || !camera || !host) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    r->hostCopies = true;
    int rc = gsr_render(r, camera, stream);
    r->hostCopies = false;
    if (rc) return rc;
    const bool rgb = r->rgb8.p != nullptr;
    const uint64_t need = uint64_t(r->width) * r->height * (rgb ? 3 : r->imageBytes());
    if (bytes != need) return fail(GSR_ERROR_INVALID_ARGUMENT, "host buffer %llu bytes, image needs %llu",
                                   (unsigned long long)bytes, (unsigned long long)need);
    return copyFrameToHost(r, host, need, static_cast<cudaStream_t>(stream));
}

int gsr_renderer_last_stats(GsrRenderer* r, GsrControl* out, uint64_t* frameIndex) {
    if (!r || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    for (auto& s : r->slots) r->readSlot(*s);
    if (!r->lastStatsValid) return GSR_ERROR_NOT_READY;
    *out = r->lastStats;
    if (frameIndex) *frameIndex = r->lastStatsFrame;
    return GSR_OK;
}

int gsr_read_control(GsrRenderer* r, GsrControl* out) {
    if (!r || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    GSR_CUDA(cudaDeviceSynchronize());
    GSR_CUDA(cudaMemcpy(out, &r->control.as<DeviceControl>()->c, sizeof(GsrControl), cudaMemcpyDeviceToHost));
    if (out->status & GSR_CONTROL_TIMEOUT) {
        fail(GSR_ERROR_DEVICE_TIMEOUT, "device wait %u gave up", out->timeout_where);
        return GSR_ERROR_DEVICE_TIMEOUT;
    }
    return GSR_OK;
}

int gsr_read_list(GsrRenderer* r, uint32_t* keysLo, uint32_t* keysHi, uint32_t* values, uint32_t n, uint32_t* rangesOut,
                  uint32_t rangesWords) {
    if (!r || !r->list) return fail(GSR_ERROR_INVALID_ARGUMENT, "no list");
    GSR_CUDA(cudaDeviceSynchronize());
    GsrControl c;
    GSR_CUDA(cudaMemcpy(&c, &r->control.as<DeviceControl>()->c, sizeof(c), cudaMemcpyDeviceToHost));
    n = std::min(n, c.entries);
    const uint32_t b = c.sorted_buffer & 1u;
    SortPlan plan;
    GSR_CUDA(cudaMemcpy(&plan, r->plan.p, sizeof(plan), cudaMemcpyDeviceToHost));
    if (n && (keysLo || keysHi || (values && plan.packed))) {
        std::vector<uint64_t> k(n);
        GSR_CUDA(cudaMemcpy(k.data(), r->list->keys[b].p, size_t(n) * 8, cudaMemcpyDeviceToHost));
        // packed words: (((tile << W) | depth mod 2^W) << indexBits) | index; the depth bits above
        // W are those of the frame's smallest depth (equal in every key)
        const uint32_t W = plan.lowBits, ib = plan.indexBits;
        const uint32_t lowMask = W >= 32 ? 0xFFFFFFFFu : ((1u << W) - 1u);
        // binning entries carry no depth bits: the depth comes from the gaussian's record
        std::vector<uint32_t> recDepth;  // depth bits per (view, gaussian) record
        if (r->binning() && keysLo) {
            const size_t records = size_t(r->scene.count) * r->views.size();
            recDepth.resize(records);
            if (r->settings.render_splat == GSR_RENDER_SPLAT_FULL) {
                std::vector<DevSplat48> rec(records);
                GSR_CUDA(cudaMemcpy(rec.data(), r->splats.p, records * 48, cudaMemcpyDeviceToHost));
                for (size_t k = 0; k < records; ++k) recDepth[k] = rec[k].depthBits;
            } else {
                GSR_CUDA(cudaMemcpy(recDepth.data(), r->depths.p, records * 4, cudaMemcpyDeviceToHost));
            }
        }
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t lo, hi;
            if (plan.packed) {
                lo = (c.depth_min_bits & ~lowMask) | (uint32_t(k[i] >> ib) & lowMask);
                hi = uint32_t(k[i] >> (ib + W));
                const uint32_t g = uint32_t(k[i] & ((1ull << ib) - 1ull));
                if (values) values[i] = g;
                if (!recDepth.empty()) {
                    size_t view = 0;  // the view holding frame tile hi
                    while (view + 1 < r->views.size() && r->views[view + 1].tile_base <= hi) ++view;
                    const size_t at = view * r->scene.count + g;
                    lo = at < recDepth.size() ? recDepth[at] : 0u;
                }
            } else {
                lo = uint32_t(k[i]);
                hi = uint32_t(k[i] >> 32);
            }
            if (keysLo) keysLo[i] = lo;
            if (keysHi) keysHi[i] = hi;
        }
    }
    if (n && values && !plan.packed)
        GSR_CUDA(cudaMemcpy(values, r->list->values[b].p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    if (rangesOut) {
        const uint32_t words = std::min<uint32_t>(rangesWords, r->totalTiles * 2);
        GSR_CUDA(cudaMemcpy(rangesOut, r->ranges.p, size_t(words) * 4, cudaMemcpyDeviceToHost));
    }
    return GSR_OK;
}

int gsr_read_splats(GsrRenderer* r, void* splatsOut, uint32_t* tileCountsOut, uint32_t n) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (splatsOut && r->settings.render_splat != GSR_RENDER_SPLAT_FULL)
        return fail(GSR_ERROR_UNSUPPORTED, "packed render splats: read them with gsr_read_packed_splats");
    GSR_CUDA(cudaDeviceSynchronize());
    n = std::min(n, r->scene.count);
    if (splatsOut) GSR_CUDA(cudaMemcpy(splatsOut, r->splats.p, size_t(n) * 48, cudaMemcpyDeviceToHost));
    if (tileCountsOut) GSR_CUDA(cudaMemcpy(tileCountsOut, r->tileCounts.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    return GSR_OK;
}

int gsr_read_packed_splats(GsrRenderer* r, uint32_t* words, uint32_t* rectsOut, uint32_t* depthsOut,
                           uint32_t* tileCountsOut, uint32_t n) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (r->settings.render_splat == GSR_RENDER_SPLAT_FULL)
        return fail(GSR_ERROR_UNSUPPORTED, "full render splats: read them with gsr_read_splats");
    GSR_CUDA(cudaDeviceSynchronize());
    n = std::min(n, r->scene.count);
    if (words) GSR_CUDA(cudaMemcpy(words, r->packedSplats.p, size_t(n) * r->packedWords() * 4, cudaMemcpyDeviceToHost));
    if (rectsOut) GSR_CUDA(cudaMemcpy(rectsOut, r->rects.p, size_t(n) * 8, cudaMemcpyDeviceToHost));
    if (depthsOut) GSR_CUDA(cudaMemcpy(depthsOut, r->depths.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    if (tileCountsOut) GSR_CUDA(cudaMemcpy(tileCountsOut, r->tileCounts.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    return GSR_OK;
}

int gsr_read_image(GsrRenderer* r, float* rgba, uint8_t* rgb) { return gsr_read_view_image(r, 0, rgba, rgb); }

int gsr_read_tile_stats(GsrRenderer* r, uint32_t* stats, uint32_t tiles, uint64_t* testedPairs) {
    if (!r || !stats) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    if (!r->settings.tile_stats || !r->tileStats.p) return fail(GSR_ERROR_INVALID_ARGUMENT, "renderer built without tile_stats");
    if (tiles != r->totalTiles) return fail(GSR_ERROR_INVALID_ARGUMENT, "tiles %u != the frame's %u", tiles, r->totalTiles);
    GSR_CUDA(cudaDeviceSynchronize());
    GSR_CUDA(cudaMemcpy(stats, r->tileStats.p, size_t(tiles) * kTileStatWords * 4, cudaMemcpyDeviceToHost));
    if (testedPairs) GSR_CUDA(cudaMemcpy(testedPairs, r->testedPairs.p, 8, cudaMemcpyDeviceToHost));
    return GSR_OK;
}

int gsr_render_views(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* stream) {
    if (!r || !cameras) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    return r->renderViews(cameras, views, static_cast<cudaStream_t>(stream));
}

int gsr_render_views_to_host(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* host, uint64_t bytes,
                             void* stream) {
    if (!r || !cameras || !host) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    r->hostCopies = true;
    int rc = gsr_render_views(r, cameras, views, stream);
    r->hostCopies = false;
    if (rc) return rc;
    const bool rgb = r->rgb8.p != nullptr;
    const uint64_t need = r->totalPixels * (rgb ? 3 : r->imageBytes());
    if (bytes != need) return fail(GSR_ERROR_INVALID_ARGUMENT, "host buffer %llu bytes, the views need %llu",
                                   (unsigned long long)bytes, (unsigned long long)need);
    return copyFrameToHost(r, host, need, static_cast<cudaStream_t>(stream));
}

int gsr_render_views_to_host_async(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* host,
                                   uint64_t bytes, void* stream, uint64_t* ticket) {
    if (!r || !cameras || !host || !ticket) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    r->hostCopies = true;
    r->hostAsync = true;
    int rc = gsr_render_views(r, cameras, views, stream);
    r->hostCopies = false;
    r->hostAsync = false;
    if (rc) return rc;
    const bool rgb = r->rgb8.p != nullptr;
    const uint64_t need = r->totalPixels * (rgb ? 3 : r->imageBytes());
    if (bytes != need) return fail(GSR_ERROR_INVALID_ARGUMENT, "host buffer %llu bytes, the views need %llu",
                                   (unsigned long long)bytes, (unsigned long long)need);
    if (!r->copyStream) GSR_CUDA(cudaStreamCreateWithFlags(&r->copyStream, cudaStreamNonBlocking));
    const unsigned char* src = rgb ? r->rgb8.as<unsigned char>() : r->image.as<unsigned char>();
    // the frame was rasterized whole (no view-by-view split): its image once the frame is done
    GSR_CUDA(cudaStreamWaitEvent(r->copyStream, r->lastSlot->done, 0));
    GSR_CUDA(cudaMemcpyAsync(host, src, need, cudaMemcpyDeviceToHost, r->copyStream));
    GSR_CUDA(cudaEventRecord(r->imageCopied, r->copyStream));
    const uint64_t t = r->hostTickets++;
    GSR_CUDA(cudaEventRecord(r->hostDone[t % GsrRenderer::kHostTickets], r->copyStream));
    *ticket = t;
    return GSR_OK;
}

int gsr_renderer_host_wait(GsrRenderer* r, uint64_t ticket) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (ticket >= r->hostTickets) return fail(GSR_ERROR_INVALID_ARGUMENT, "ticket %llu was not issued", (unsigned long long)ticket);
    // a ticket older than the ring waits for a later one (copies complete in order)
    GSR_CUDA(cudaEventSynchronize(r->hostDone[ticket % GsrRenderer::kHostTickets]));
    return GSR_OK;
}

int gsr_renderer_view_layout(GsrRenderer* r, uint32_t view, GsrViewLayout* out, uint32_t* views) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (views) *views = uint32_t(r->views.size());
    if (out) {
        if (view >= r->views.size()) return fail(GSR_ERROR_INVALID_ARGUMENT, "view %u of %zu", view, r->views.size());
        *out = r->views[view];
    }
    return GSR_OK;
}

int gsr_renderer_view_image(GsrRenderer* r, uint32_t view, const void** rgba, const void** rgb8) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (view >= r->views.size()) return fail(GSR_ERROR_INVALID_ARGUMENT, "view %u of %zu", view, r->views.size());
    const uint64_t base = r->views[view].pixel_base;
    if (rgba) *rgba = r->image.as<unsigned char>() + base * r->imageBytes();
    if (rgb8) *rgb8 = r->rgb8.p ? r->rgb8.as<unsigned char>() + base * 3 : nullptr;
    return GSR_OK;
}

int gsr_read_view_image(GsrRenderer* r, uint32_t view, float* rgba, uint8_t* rgb) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (view >= r->views.size()) return fail(GSR_ERROR_INVALID_ARGUMENT, "view %u of %zu", view, r->views.size());
    GSR_CUDA(cudaDeviceSynchronize());
    const GsrViewLayout& v = r->views[view];
    const size_t pixels = size_t(v.width) * v.height;
    if (rgba) {
        const uint32_t bpp = r->imageBytes();
        if (bpp == 16) {
            GSR_CUDA(cudaMemcpy(rgba, r->image.as<unsigned char>() + v.pixel_base * 16, pixels * 16, cudaMemcpyDeviceToHost));
        } else {
            std::vector<unsigned char> raw(pixels * bpp);
            GSR_CUDA(cudaMemcpy(raw.data(), r->image.as<unsigned char>() + v.pixel_base * bpp, raw.size(),
                                cudaMemcpyDeviceToHost));
            for (size_t k = 0; k < pixels * 4; ++k) {
                if (bpp == 8) {
                    uint16_t h;
                    std::memcpy(&h, &raw[k * 2], 2);
                    rgba[k] = halfToFloat(h);
                } else {
                    rgba[k] = float(raw[k]) / 255.0f;
                }
            }
        }
    }
    if (rgb) {
        if (!r->rgb8.p) return fail(GSR_ERROR_INVALID_ARGUMENT, "rgb8 output is off");
        GSR_CUDA(cudaMemcpy(rgb, r->rgb8.as<unsigned char>() + v.pixel_base * 3, pixels * 3, cudaMemcpyDeviceToHost));
    }
    return GSR_OK;
}

int gsr_renderer_set_timing(GsrRenderer* r, int enabled) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    r->timing = enabled != 0;
    return GSR_OK;
}

int gsr_renderer_pass_times(GsrRenderer* r, float* ms, const char** names, uint32_t capacity, uint32_t* count) {
    static const char* kGlobal[] = {"reset + preprocess + scan + duplicate", "tile sort (total)", "tile ranges",
                                    "render tiles", "control readback"};
    static const char* kBinning[] = {"reset + preprocess (depth keys)", "depth sort (total)",
                                     "scan + duplicate (depth order)", "tile sort (total)", "tile ranges",
                                     "render tiles", "control readback"};
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (!r->timed || r->evCount < 2) return GSR_ERROR_NOT_READY;
    const uint32_t passes = uint32_t(r->evCount - 1);
    const char** kNames = passes == 7 ? kBinning : kGlobal;
    if (passes != 7 && passes != 5) return fail(GSR_ERROR_UNSUPPORTED, "pass events %u", passes);
    GSR_CUDA(cudaEventSynchronize(r->ev[passes]));
    const uint32_t n = std::min<uint32_t>(capacity, passes);
    for (uint32_t i = 0; i < n; ++i) {
        float t = 0.0f;
        GSR_CUDA(cudaEventElapsedTime(&t, r->ev[i], r->ev[i + 1]));
        if (ms) ms[i] = t;
        if (names) names[i] = kNames[i];
    }
    if (count) *count = n;
    return GSR_OK;
}

int gsr_renderer_capacity(GsrRenderer* r, uint32_t* capacity, uint32_t* maxCapacity, uint32_t* resizes) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (capacity) *capacity = r->list ? r->list->capacity : 0;
    if (maxCapacity) *maxCapacity = r->maxCapacity;
    if (resizes) *resizes = r->listResizes;
    return GSR_OK;
}

int gsr_renderer_kernel_launches(GsrRenderer* r, uint64_t* count) {
    if (!r || !count) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *count = r->kernelLaunches;
    return GSR_OK;
}

int gsr_renderer_debug_force_timeout(GsrRenderer* r, uint32_t iterations) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    r->forceTimeout = iterations;
    return GSR_OK;
}

void gsr_renderer_destroy(GsrRenderer* r) {
    if (!r) return;
    cudaDeviceSynchronize();
    delete r;
}

// ---- the learned colour stage -------------------------------------------------------------------
void gsr_color_model_options_default(GsrColorModelOptions* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->directions = 64;
    o->batch = 65536;
    o->steps = 2000;
    o->learning_rate = 1e-3f;
    o->seed = 1;
    o->gate = 2.0f / 255.0f;
    o->sh_degree = -1;
}

namespace {
// Initial weights: uniform(-b, b) with b = sqrt(6 / fan_in) before a ReLU and sqrt(3 / fan_in)
// otherwise, biases 0; drawn from a 64-bit LCG seeded with the options' seed.
void initColorParams(uint32_t seed, std::vector<float>& p) {
    p.assign(kColorModelParams, 0.0f);
    uint64_t st = 0x9E3779B97F4A7C15ull ^ (uint64_t(seed) * 0xD1B54A32D192ED03ull);
    auto uni = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return float((st >> 40) & 0xFFFFFF) / 16777216.0f * 2.0f - 1.0f;
    };
    struct Layer { uint32_t offset, in, out; bool relu; };
    // encoder W1 [48][64], W2 [64][8]; decoder W1 [11][32], W2 [32][32], W3 [32][3]
    const Layer layers[] = {{0, 48, 64, true}, {48 * 64 + 64, 64, 8, false}, {48 * 64 + 64 + 64 * 8 + 8, 11, 32, true},
                            {48 * 64 + 64 + 64 * 8 + 8 + 11 * 32 + 32, 32, 32, true},
                            {48 * 64 + 64 + 64 * 8 + 8 + 11 * 32 + 32 + 32 * 32 + 32, 32, 3, false}};
    for (const Layer& L : layers) {
        const float b = std::sqrt((L.relu ? 6.0f : 3.0f) / float(L.in));
        for (uint32_t e = 0; e < L.in * L.out; ++e) p[L.offset + e] = b * uni();
    }
}
}  // namespace

namespace {
// `steps` more Adam steps of the model on the scene's SH colour (from the model's state), then
// the latents of every gaussian and the gate; the statistics cover every step taken so far.
int trainColorModel(const GsrSceneDesc& scene, GsrColorModel& m, uint32_t steps) {
    const GsrColorModelOptions& o = m.options;
    const uint32_t n = scene.count, blocks = o.batch / colorTrainBatchMultiple();
    DevBuf sh, degrees, partials, lossDev, counters;
    GSR_CUDA(sh.alloc(size_t(n) * 48 * 4));
    GSR_CUDA(degrees.alloc(n));
    GSR_CUDA(partials.alloc(size_t(blocks) * (kColorModelParams + 1) * 4));
    GSR_CUDA(lossDev.alloc(size_t(std::max(steps, 1u)) * 4));
    GSR_CUDA(counters.alloc(8));
    GSR_CUDA(cudaMemset(counters.p, 0, 8));
    cudaStream_t s = nullptr;
    GSR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    };
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    if (ce == cudaSuccess) ce = cudaEventRecord(e0, s);
    if (ce == cudaSuccess)
        ce = launchShDecode(sceneArgs(scene), scene.geometry, scene.color, n, m.degree, sh.as<float>(), degrees.as<uint8_t>(), s);
    for (uint32_t k = 0; ce == cudaSuccess && k < steps; ++k)
        ce = launchColorTrainStep(sh.as<float>(), degrees.as<uint8_t>(), n, o.directions, o.seed, o.batch,
                                  m.params.as<float>(), m.mom.as<float>(), m.vel.as<float>(), partials.as<float>(),
                                  m.stepDev.as<uint32_t>(), o.learning_rate, lossDev.as<float>(), m.step, m.step + steps, s);
    if (ce == cudaSuccess)
        ce = launchColorEncode(sh.as<float>(), m.params.as<float>(), m.latents.as<uint4>(), m.decoder.as<DecoderWeights>(), n, s);
    if (ce == cudaSuccess)
        ce = launchColorGate(sh.as<float>(), degrees.as<uint8_t>(), n, o.directions, m.decoder.as<DecoderWeights>(),
                             m.latents.as<uint4>(), o.gate, counters.as<uint32_t>(), counters.as<uint32_t>() + 1, s);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    cleanup();
    if (ce != cudaSuccess) return cudaFail(ce, "colour model training");
    const size_t before = m.loss.size();
    m.loss.resize(before + steps);
    if (steps) GSR_CUDA(cudaMemcpy(m.loss.data() + before, lossDev.p, size_t(steps) * 4, cudaMemcpyDeviceToHost));
    m.step += steps;
    uint32_t cnt[2];
    GSR_CUDA(cudaMemcpy(cnt, counters.p, 8, cudaMemcpyDeviceToHost));
    GsrColorModelStats& st = m.stats;
    st.gaussians = n;
    st.fallback = cnt[0];
    std::memcpy(&st.max_error_kept, &cnt[1], 4);
    st.steps = m.step;
    st.sh_degree = m.degree;
    st.first_loss = m.loss.empty() ? 0.0f : m.loss.front();
    st.final_loss = m.loss.empty() ? 0.0f : m.loss.back();
    st.train_ms = ms;
    return GSR_OK;
}

// The model's device buffers for n gaussians.
int allocColorModel(GsrColorModel& m, uint32_t n) {
    GSR_CUDA(m.params.alloc(size_t(kColorModelParams) * 4));
    GSR_CUDA(m.mom.alloc(size_t(kColorModelParams) * 4));
    GSR_CUDA(m.vel.alloc(size_t(kColorModelParams) * 4));
    GSR_CUDA(m.stepDev.alloc(8));
    GSR_CUDA(m.latents.alloc(size_t(n) * 16));
    GSR_CUDA(m.decoder.alloc(kDecoderWeightsBytes));
    return GSR_OK;
}
}  // namespace

int gsr_color_model_train(const GsrSceneDesc* scene, const GsrColorModelOptions* options, GsrColorModel** out) {
    if (!scene || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int rc = validateScene(*scene);
    if (rc) return rc;
    GsrColorModelOptions o;
    gsr_color_model_options_default(&o);
    if (options) o = *options;
    const uint32_t mult = colorTrainBatchMultiple();
    if (o.directions == 0 || o.directions > 4096) return fail(GSR_ERROR_INVALID_ARGUMENT, "directions %u", o.directions);
    if (o.batch == 0 || o.batch % mult || o.batch > (1u << 24))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "batch %u (a multiple of %u, at most 2^24)", o.batch, mult);
    if (o.steps == 0 || !(o.learning_rate > 0.0f) || !(o.gate >= 0.0f))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "steps %u, learning rate %g, gate %g", o.steps, o.learning_rate, o.gate);
    auto m = std::make_unique<GsrColorModel>();
    m->count = scene->count;
    m->degree = o.sh_degree < 0 ? scene->sh_degree : std::min(o.sh_degree, scene->sh_degree);
    m->options = o;
    rc = allocColorModel(*m, scene->count);
    if (rc) return rc;
    std::vector<float> p0;
    initColorParams(o.seed, p0);
    GSR_CUDA(cudaMemcpy(m->params.p, p0.data(), p0.size() * 4, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemset(m->mom.p, 0, m->mom.bytes));
    GSR_CUDA(cudaMemset(m->vel.p, 0, m->vel.bytes));
    GSR_CUDA(cudaMemset(m->stepDev.p, 0, 8));
    rc = trainColorModel(*scene, *m, o.steps);
    if (rc) return rc;
    *out = m.release();
    return GSR_OK;
}

int gsr_color_model_resume(const GsrSceneDesc* scene, GsrColorModel* model, uint32_t steps) {
    if (!scene || !model) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    int rc = validateScene(*scene);
    if (rc) return rc;
    if (scene->count != model->count || model->degree > scene->sh_degree)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "colour model of %u gaussians (degree %d) for a scene of %u (degree %d)",
                    model->count, model->degree, scene->count, scene->sh_degree);
    GSR_CUDA(cudaDeviceSynchronize());  // renderers using the model finish their frames first
    return trainColorModel(*scene, *model, steps);
}

int gsr_color_model_save(const GsrColorModel* model, const char* path) {
    if (!model || !path) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    GSR_CUDA(cudaDeviceSynchronize());
    std::vector<float> params(kColorModelParams), m(kColorModelParams), v(kColorModelParams);
    std::vector<uint16_t> latents(size_t(model->count) * 8);
    GSR_CUDA(cudaMemcpy(params.data(), model->params.p, params.size() * 4, cudaMemcpyDeviceToHost));
    GSR_CUDA(cudaMemcpy(m.data(), model->mom.p, m.size() * 4, cudaMemcpyDeviceToHost));
    GSR_CUDA(cudaMemcpy(v.data(), model->vel.p, v.size() * 4, cudaMemcpyDeviceToHost));
    GSR_CUDA(cudaMemcpy(latents.data(), model->latents.p, latents.size() * 2, cudaMemcpyDeviceToHost));
    GsrColorModelCheckpoint ck{};
    ck.count = model->count;
    ck.sh_degree = model->degree;
    ck.step = model->step;
    ck.loss_count = uint32_t(model->loss.size());
    ck.options = model->options;
    ck.stats = model->stats;
    ck.params = params.data();
    ck.adam_m = m.data();
    ck.adam_v = v.data();
    ck.loss = const_cast<float*>(model->loss.data());
    ck.latents = latents.data();
    return gsr_color_model_file_write(path, &ck);
}

int gsr_color_model_load(const GsrSceneDesc* scene, const char* path, GsrColorModel** out) {
    if (!scene || !path || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int rc = validateScene(*scene);
    if (rc) return rc;
    GsrColorModelCheckpoint ck{};
    rc = gsr_color_model_file_read(path, &ck);  // the sizes
    if (rc) return rc;
    if (ck.count != scene->count || ck.sh_degree < 0 || ck.sh_degree > scene->sh_degree)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "%s: a model of %u gaussians (degree %d) for a scene of %u (degree %d)", path,
                    ck.count, ck.sh_degree, scene->count, scene->sh_degree);
    std::vector<float> params(kColorModelParams), m(kColorModelParams), v(kColorModelParams), loss(ck.loss_count);
    std::vector<uint16_t> latents(size_t(ck.count) * 8);
    ck.params = params.data();
    ck.adam_m = m.data();
    ck.adam_v = v.data();
    ck.loss = loss.data();
    ck.latents = latents.data();
    rc = gsr_color_model_file_read(path, &ck);
    if (rc) return rc;
    auto model = std::make_unique<GsrColorModel>();
    model->count = ck.count;
    model->degree = ck.sh_degree;
    model->options = ck.options;
    model->stats = ck.stats;
    model->step = ck.step;
    model->loss = std::move(loss);
    rc = allocColorModel(*model, ck.count);
    if (rc) return rc;
    const uint32_t stepWords[2] = {ck.step, 0u};
    GSR_CUDA(cudaMemcpy(model->params.p, params.data(), params.size() * 4, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(model->mom.p, m.data(), m.size() * 4, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(model->vel.p, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(model->stepDev.p, stepWords, 8, cudaMemcpyHostToDevice));
    GSR_CUDA(cudaMemcpy(model->latents.p, latents.data(), latents.size() * 2, cudaMemcpyHostToDevice));
    GSR_CUDA(launchPackDecoder(model->params.as<float>(), model->decoder.as<DecoderWeights>(), nullptr));
    GSR_CUDA(cudaDeviceSynchronize());
    *out = model.release();
    return GSR_OK;
}

int gsr_color_model_stats(const GsrColorModel* model, GsrColorModelStats* out) {
    if (!model || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    *out = model->stats;
    return GSR_OK;
}

int gsr_color_model_read(const GsrColorModel* model, uint16_t* latents, float* params, float* lossPerStep) {
    if (!model) return fail(GSR_ERROR_INVALID_ARGUMENT, "null model");
    GSR_CUDA(cudaDeviceSynchronize());
    if (latents) GSR_CUDA(cudaMemcpy(latents, model->latents.p, size_t(model->count) * 16, cudaMemcpyDeviceToHost));
    if (params) GSR_CUDA(cudaMemcpy(params, model->params.p, size_t(kColorModelParams) * 4, cudaMemcpyDeviceToHost));
    if (lossPerStep) std::memcpy(lossPerStep, model->loss.data(), model->loss.size() * 4);
    return GSR_OK;
}

int gsr_renderer_set_color_model(GsrRenderer* r, const GsrColorModel* model) {
    if (!r) return fail(GSR_ERROR_INVALID_ARGUMENT, "null renderer");
    if (model) {
        if (model->count != r->scene.count)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "colour model of %u gaussians for a scene of %u", model->count,
                        r->scene.count);
        if (model->degree != r->evalDegree)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "colour model learned SH degree %d, the renderer evaluates %d",
                        model->degree, r->evalDegree);
    }
    GSR_CUDA(cudaDeviceSynchronize());
    // a model whose gate kept no gaussian colours every one by SH: the plain path gives the same
    // records without reading the latents
    const bool use = model && model->stats.fallback < model->count;
    r->colorLatents = use ? model->latents.as<uint4>() : nullptr;
    r->colorDecoder = use ? model->decoder.as<DecoderWeights>() : nullptr;
    ++r->layoutVersion;  // captured frames hold the old pointers
    return GSR_OK;
}

void gsr_color_model_destroy(GsrColorModel* model) {
    if (!model) return;
    cudaDeviceSynchronize();
    delete model;
}

// ---- autotuner ------------------------------------------------------------------------------
int gsr_autotune_space(const GsrSceneDesc* scene, const GsrSettings* settings, const GsrColorModel* model,
                       const GsrSplatCamera* cameras, uint32_t count, const GsrTuneSpace* space, uint32_t frames,
                       GsrTuneResult* out) {
    if (!scene || !settings || !cameras || !space || !out) return fail(GSR_ERROR_INVALID_ARGUMENT, "null argument");
    if (count == 0 || frames == 0 || !space->views_per_frame || space->views_per_frame_count == 0)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "nothing to tune");
    std::memset(out, 0, sizeof(*out));
    // the knobs' value lists (a missing list keeps the settings' value; both schedules by default)
    auto listOf = [](const uint32_t* v, uint32_t n, std::vector<uint32_t> fallback) {
        return v && n ? std::vector<uint32_t>(v, v + n) : fallback;
    };
    const std::vector<uint32_t> depths = listOf(space->views_per_frame, space->views_per_frame_count, {});
    const std::vector<uint32_t> schedules =
        listOf(space->raster_schedules, space->raster_schedule_count, {GSR_RASTER_PER_TILE, GSR_RASTER_PERSISTENT});
    const std::vector<uint32_t> tiles = listOf(space->tile_sizes, space->tile_size_count, {settings->tile_size});
    const std::vector<uint32_t> digits =
        listOf(space->sort_digit_bits, space->sort_digit_bits_count, {settings->sort_digit_bits});
    if (uint64_t(depths.size()) * schedules.size() * tiles.size() * digits.size() > GSR_TUNE_MAX_CANDIDATES)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "more than %u candidates", GSR_TUNE_MAX_CANDIDATES);
    for (uint32_t d : depths)
        if (d == 0 || d > count || d > GSR_MAX_VIEWS)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "views per frame %u (1..%u)", d, std::min(count, GSR_MAX_VIEWS));
    for (uint32_t sc : schedules)
        if (sc != GSR_RASTER_PER_TILE && sc != GSR_RASTER_PERSISTENT)
            return fail(GSR_ERROR_INVALID_ARGUMENT, "raster schedule %u", sc);
    cudaStream_t s = nullptr;
    GSR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = GSR_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = fail(GSR_ERROR_CUDA, "events");
    for (uint32_t tile : tiles)
        for (uint32_t bits : digits)
            for (uint32_t d : depths)
                for (uint32_t sc : schedules) {
                    if (rc) break;
                    GsrSettings st = *settings;
                    st.raster_schedule = sc;
                    st.tile_size = tile;
                    st.sort_digit_bits = bits;
                    GsrRenderer* r = nullptr;
                    rc = gsr_renderer_create(scene, &st, &r);
                    if (rc) break;
                    if (model) rc = gsr_renderer_set_color_model(r, model);
                    const uint32_t frameCount = count / d;  // whole frames of consecutive cameras
                    auto frame = [&](uint32_t k) { return r->renderViews(cameras + size_t(k % frameCount) * d, d, s); };
                    // warm-up: the layout, then frames until the adaptive list has kept its
                    // capacity for three frames (its statistics arrive frames_in_flight frames late)
                    uint32_t stable = 0, last = 0, k = 0;
                    for (; rc == GSR_OK && k < 24 && stable < 3; ++k) {
                        rc = frame(k);
                        if (rc == GSR_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(GSR_ERROR_CUDA, "warm-up");
                        const uint32_t cap = r->list ? r->list->capacity : 0;
                        stable = cap == last ? stable + 1 : 0;
                        last = cap;
                    }
                    if (rc == GSR_OK && cudaEventRecord(e0, s) != cudaSuccess) rc = fail(GSR_ERROR_CUDA, "event");
                    for (uint32_t j = 0; rc == GSR_OK && j < frames; ++j) rc = frame(k + j);
                    float ms = 0.0f;
                    if (rc == GSR_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                         cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                        rc = fail(GSR_ERROR_CUDA, "timing");
                    gsr_renderer_destroy(r);
                    if (rc) break;
                    GsrTuneCandidate& c = out->table[out->candidates++];
                    c.views_per_frame = d;
                    c.raster_schedule = sc;
                    c.tile_size = tile;
                    c.sort_digit_bits = bits ? bits : 8u;
                    c.ms_per_frame = ms / float(frames);
                    c.views_per_s = ms > 0.0f ? float(frames) * float(d) / (ms * 1e-3f) : 0.0f;
                    if (c.views_per_s > out->views_per_s) {
                        out->views_per_s = c.views_per_s;
                        out->views_per_frame = d;
                        out->raster_schedule = sc;
                        out->tile_size = tile;
                        out->sort_digit_bits = c.sort_digit_bits;
                    }
                }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return rc;
}

int gsr_autotune(const GsrSceneDesc* scene, const GsrSettings* settings, const GsrColorModel* model,
                 const GsrSplatCamera* cameras, uint32_t count, const uint32_t* depths, uint32_t depthCount,
                 uint32_t frames, GsrTuneResult* out) {
    if (!depths || depthCount == 0) return fail(GSR_ERROR_INVALID_ARGUMENT, "nothing to tune");
    GsrTuneSpace space{};
    space.views_per_frame = depths;
    space.views_per_frame_count = depthCount;
    return gsr_autotune_space(scene, settings, model, cameras, count, &space, frames, out);
}

// ---- primitives ----------------------------------------------------------------------------
int gsr_scan(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count, uint32_t mode,
             void* stream) {
    if (mode > GSR_SCAN_GATHER || (count && (!in || !out)) || (mode == GSR_SCAN_GATHER && count && !index))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "scan arguments");
    int rc = staticScanReady(nullptr);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf ctl, status;
    const uint32_t blocks = (count + kScanBlockItems - 1) / kScanBlockItems;
    GSR_CUDA(ctl.alloc(sizeof(DeviceControl)));
    GSR_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(DeviceControl), s));
    GSR_CUDA(status.alloc(size_t(std::max(blocks, 1u)) * 8));
    GSR_CUDA(cudaMemsetAsync(status.p, 0, status.bytes, s));
    GSR_CUDA(launchFrameBegin(ctl.as<DeviceControl>(), count, 0, nullptr, 0, nullptr, 0, s));
    GSR_CUDA(launchScan(in, index, out, total, count, mode, status.as<uint64_t>(), ctl.as<DeviceControl>(), s));
    GSR_CUDA(cudaStreamSynchronize(s));  // the scratch is freed on return
    DeviceControl c;
    GSR_CUDA(cudaMemcpy(&c, ctl.p, sizeof(c), cudaMemcpyDeviceToHost));
    if (c.c.status & GSR_CONTROL_TIMEOUT) return fail(GSR_ERROR_DEVICE_TIMEOUT, "scan look-back timed out");
    return GSR_OK;
}

int gsr_scan_static(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
                    uint32_t mode, void* stream) {
    if (mode > GSR_SCAN_GATHER || (count && (!in || !out)) || (mode == GSR_SCAN_GATHER && count && !index))
        return fail(GSR_ERROR_INVALID_ARGUMENT, "scan arguments");
    if (count > GSR_SCAN_STATIC_MAX_COUNT)
        return fail(GSR_ERROR_INVALID_ARGUMENT, "gsr_scan_static: count %u exceeds the static scratch limit of %u items",
                    count, GSR_SCAN_STATIC_MAX_COUNT);
    void* base = nullptr;
    int rc = staticScanReady(&base);
    if (rc) return rc;
    if (count == 0) return GSR_OK;  // the set-up call: the scratch and the kernels are ready
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceControl* ctl = static_cast<DeviceControl*>(base);
    uint64_t* status = reinterpret_cast<uint64_t*>(static_cast<unsigned char*>(base) + kStaticScanCtlBytes);
    const uint32_t blocks = (count + kScanBlockItems - 1) / kScanBlockItems;
    static_assert(kStaticScanCtlBytes + size_t((GSR_SCAN_STATIC_MAX_COUNT + kScanBlockItems - 1) / kScanBlockItems) * 8 <=
                      kStaticScanScratchBytes, "the look-back words of the largest count fit the array");
    // what must start at zero: the look-back words here, the block tickets in frame begin
    GSR_CUDA(cudaMemsetAsync(status, 0, size_t(blocks) * 8, s));
    GSR_CUDA(launchFrameBegin(ctl, count, 0, nullptr, 0, nullptr, 0, s));
    GSR_CUDA(launchScan(in, index, out, total, count, mode, status, ctl, s));
    uint32_t st = 0;
    GSR_CUDA(cudaMemcpyAsync(&st, &ctl->c.status, sizeof(st), cudaMemcpyDeviceToHost, s));
    GSR_CUDA(cudaStreamSynchronize(s));
    if (st & GSR_CONTROL_TIMEOUT) return fail(GSR_ERROR_DEVICE_TIMEOUT, "scan look-back timed out");
    return GSR_OK;
}

int gsr_sort_pairs(uint32_t* keysLo, uint32_t* keysHi, uint32_t* values, uint32_t count, uint32_t keyBits, void* stream) {
    if (keyBits == 0 || keyBits > 64 || (!keysHi && keyBits > 32)) return fail(GSR_ERROR_INVALID_ARGUMENT, "key_bits %u", keyBits);
    if (count == 0) return GSR_OK;
    if (!keysLo || !values) return fail(GSR_ERROR_INVALID_ARGUMENT, "null keys/values");
    const int ready = staticScanReady(nullptr);
    if (ready) return ready;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t passes = (keyBits + 7) / 8;
    const uint32_t maxTiles = (count + kSortTile - 1) / kSortTile;
    DevBuf ctl, plan, status, k0, k1, v1;
    GSR_CUDA(ctl.alloc(sizeof(DeviceControl)));
    GSR_CUDA(plan.alloc(sizeof(SortPlan)));
    GSR_CUDA(status.alloc(size_t(passes) * maxTiles * 256 * 8));
    GSR_CUDA(k0.alloc(size_t(count) * 8));
    GSR_CUDA(k1.alloc(size_t(count) * 8));
    GSR_CUDA(v1.alloc(size_t(count) * 4));
    GSR_CUDA(cudaMemsetAsync(ctl.p, 0, ctl.bytes, s));
    GSR_CUDA(cudaMemsetAsync(plan.p, 0, plan.bytes, s));
    GSR_CUDA(cudaMemsetAsync(status.p, 0, status.bytes, s));
    GSR_CUDA(launchFrameBegin(ctl.as<DeviceControl>(), count, count, nullptr, 0, plan.as<SortPlan>(), 0, s));
    GSR_CUDA(launchSetEntries(ctl.as<DeviceControl>(), count, s));
    GSR_CUDA(launchPack64(keysLo, keysHi, k0.as<uint64_t>(), count, s));
    SortArgs sa{};
    sa.keys[0] = k0.as<uint64_t>();
    sa.keys[1] = k1.as<uint64_t>();
    sa.values[0] = values;
    sa.values[1] = v1.as<uint32_t>();
    sa.status = status.as<uint64_t>();
    sa.maxTiles = maxTiles;
    sa.plan = plan.as<SortPlan>();
    sa.ctl = ctl.as<DeviceControl>();
    sa.passesLaunched = passes;
    sa.frameMode = 0;
    sa.fixedLowBits = 32;
    sa.fixedKeyBits = keyBits;
    GSR_CUDA(launchSort(sa, 148 * 4, s));
    GSR_CUDA(cudaStreamSynchronize(s));
    DeviceControl c;
    GSR_CUDA(cudaMemcpy(&c, ctl.p, sizeof(c), cudaMemcpyDeviceToHost));
    const uint32_t b = c.c.sorted_buffer & 1u;
    GSR_CUDA(launchUnpack64(b ? k1.as<uint64_t>() : k0.as<uint64_t>(), keysLo, keysHi, count, s));
    if (b) GSR_CUDA(cudaMemcpyAsync(values, v1.p, size_t(count) * 4, cudaMemcpyDeviceToDevice, s));
    GSR_CUDA(cudaStreamSynchronize(s));
    if (c.c.status & GSR_CONTROL_TIMEOUT) return fail(GSR_ERROR_DEVICE_TIMEOUT, "sort look-back timed out");
    if (c.c.status & GSR_CONTROL_BOUNDS) return fail(GSR_ERROR_CUDA, "sort scatter index out of range");
    return GSR_OK;
}

int gsr_debug_logf_table(float* outDevice, void* stream) {
    if (!outDevice) return fail(GSR_ERROR_INVALID_ARGUMENT, "null output");
    LogfFixups t;
    const int rc = deviceTables(&t);
    if (rc) return rc;
    GSR_CUDA(launchLogfTable(outDevice, t, static_cast<cudaStream_t>(stream)));
    return GSR_OK;
}

}  // extern "C"
