// Host-side scene input: the 3DGS PLY loader (src/scene/ply_loader.h:1-120) and the INRIA
// training cameras (src/scene/training_cameras.h:1-44), restated for this library. The decoded
// arrays are the activated SoA layout that gsr_scene_create() uploads and encodes on the GPU:
// posAlpha / scales / rotations as float4[N], SH as float[N * K * 3] RGB triplets.
//
// Floating point: every activation is the same float expression as the reference's decode
// (ply_loader.cpp:127-150) evaluated with this machine's C library (expf, sqrtf), with no
// contraction into FMA, so the arrays are bit-identical to the reference loader's.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace gsr::io {

// A malformed file (the reference's PlyError); I/O failures are std::runtime_error.
class FormatError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

enum class PlyFormat : uint32_t { BinaryLittleEndian = 0, BinaryBigEndian = 1, Ascii = 2 };
enum class PlyScalar : uint32_t { Int8 = 0, UInt8, Int16, UInt16, Int32, UInt32, Float32, Float64 };
uint32_t scalarBytes(PlyScalar type);

struct PlyProperty {
    std::string name;
    PlyScalar type = PlyScalar::Float32;
    bool list = false;
    uint32_t offset = 0;  // byte offset in the element's record (scalar properties)
};

struct PlyElement {
    std::string name;
    uint64_t count = 0;
    std::vector<PlyProperty> properties;
    uint32_t stride = 0;  // bytes of one record: every scalar property, known or not
    bool hasList = false;
    const PlyProperty* find(std::string_view property) const;
};

struct PlyHeader {
    PlyFormat format = PlyFormat::BinaryLittleEndian;
    std::vector<PlyElement> elements;
    std::vector<std::string> comments;
    size_t headerBytes = 0;  // the payload starts here
};

// The header at the start of `bytes` (parsePlyHeaderPrefix, ply_loader.cpp:208-283): nullopt
// while no end_header line has arrived and `final` is false; FormatError on bad syntax.
std::optional<PlyHeader> parsePlyHeader(std::string_view bytes, bool final);
// 0/9/24/45 f_rest properties -> SH degree 0..3, else -1.
int shDegreeForRestCount(size_t restCount);

struct SceneStats {  // gsr::SceneStats (gaussian_scene.h:47-61)
    float bboxMin[3] = {0, 0, 0}, bboxMax[3] = {0, 0, 0};
    float robustMin[3] = {0, 0, 0}, robustMax[3] = {0, 0, 0};  // 1st / 99th percentile per axis
    float alphaMin = 0, alphaMax = 0, alphaMean = 0;
    uint32_t alphaBelowVisible = 0;
    float sigmaMin = 0, sigmaMax = 0, sigmaMaxMedian = 0;
    float quatNormMin = 0, quatNormMax = 0;
    uint32_t zeroQuaternions = 0;
    uint64_t nonFiniteValues = 0;
};

struct LoadTimings {
    double mapMs = 0, headerMs = 0, decodeMs = 0, statsMs = 0, totalMs = 0;
};

// gsr::GaussianScene (gaussian_scene.h:71-101): activated arrays + the raw file values.
struct HostScene {
    std::string sourcePath;
    uint32_t count = 0;
    int shDegree = 0;
    std::vector<float> posAlpha;     // float4[N]: mean, sigmoid(opacity)
    std::vector<float> scales;       // float4[N]: exp(log scale), 0
    std::vector<float> rotations;    // float4[N]: normalized (w, x, y, z)
    std::vector<float> sh;           // float[N * K * 3]
    std::vector<float> rawOpacity;   // [N]
    std::vector<float> rawLogScale;  // float3[N]
    std::vector<float> rawRotation;  // float4[N]
    SceneStats stats;
    LoadTimings timings;
    std::vector<std::string> comments;
    std::vector<std::string> warnings;

    uint32_t coeffsPerChannel() const { return uint32_t((shDegree + 1) * (shDegree + 1)); }
    void resize(size_t n);
};

// loadGaussianPly (ply_loader.cpp:439-503): from a file (its name prefixes the messages) or
// from bytes in memory. Throws FormatError or std::runtime_error.
HostScene loadPly(const std::string& path);
HostScene loadPly(const uint8_t* bytes, size_t size, const std::string& name);
// computeSceneStats (gaussian_scene.cpp:30-99).
void computeSceneStats(HostScene& scene);

// PlyStreamDecoder (ply_loader.h:82-117): bytes pushed in order, in chunks of any size; the
// header is parsed as soon as it is complete, then complete records are decoded in batches.
class PlyStream {
public:
    using HeaderFn = std::function<void(const HostScene& info)>;
    using BatchFn = std::function<void(uint32_t first, const HostScene& batch)>;
    PlyStream(std::string name, uint64_t totalBytes, HeaderFn onHeader, BatchFn onBatch, uint32_t batchCapacity);
    ~PlyStream();
    PlyStream(const PlyStream&) = delete;
    PlyStream& operator=(const PlyStream&) = delete;
    void push(const uint8_t* bytes, size_t size);  // FormatError; std::logic_error after an error or finish
    void finish();
    bool headerParsed() const;
    bool finished() const;
    uint64_t bytesReceived() const;
    uint64_t recordsDecoded() const;
    const HostScene& info() const;

private:
    struct State;
    std::unique_ptr<State> s_;
};

// TrainingCamera (training_cameras.h:17-32); cameraToWorld is column-major (column c at [3c]).
struct TrainingCamera {
    int id = 0;
    std::string imageName;
    uint32_t width = 0, height = 0;
    float position[3] = {0, 0, 0};
    float cameraToWorld[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float fx = 0, fy = 0;
};
std::vector<TrainingCamera> loadTrainingCameras(const std::string& path);
float fovYDeg(const TrainingCamera& camera);
void meanCameraUp(const TrainingCamera* cameras, size_t count, float up[3]);
void cameraFocusPoint(const TrainingCamera* cameras, size_t count, float point[3]);

}  // namespace gsr::io
