// The 3DGS PLY loader (src/scene/ply_loader.cpp) and the scene statistics
// (src/scene/gaussian_scene.cpp:11-99), restated. Same accepted files, same error and warning
// texts, and the same decoded values bit for bit; the structure is this library's own: the file
// is memory-mapped, the header is parsed into a per-record field table, and the records are
// decoded by all host threads into the SoA arrays that gsr_scene_create() takes.
#include "scene_io.h"

#include <algorithm>
#include <chrono>
#include <charconv>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace gsr::io {

namespace {

using Clock = std::chrono::steady_clock;
double msSince(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

// Headers of real files are about 1.5 KB; a longer one is not a 3DGS file.
constexpr size_t kMaxHeaderBytes = size_t(1) << 20;

bool scalarFromName(std::string_view s, PlyScalar& t) {
    // the classic PLY names and their sized aliases
    static const struct {
        const char* name;
        PlyScalar type;
    } kNames[] = {{"char", PlyScalar::Int8},      {"int8", PlyScalar::Int8},       {"uchar", PlyScalar::UInt8},
                  {"uint8", PlyScalar::UInt8},    {"short", PlyScalar::Int16},     {"int16", PlyScalar::Int16},
                  {"ushort", PlyScalar::UInt16},  {"uint16", PlyScalar::UInt16},   {"int", PlyScalar::Int32},
                  {"int32", PlyScalar::Int32},    {"uint", PlyScalar::UInt32},     {"uint32", PlyScalar::UInt32},
                  {"float", PlyScalar::Float32},  {"float32", PlyScalar::Float32}, {"double", PlyScalar::Float64},
                  {"float64", PlyScalar::Float64}};
    for (const auto& e : kNames)
        if (s == e.name) {
            t = e.type;
            return true;
        }
    return false;
}

// whitespace (space, tab) separated words of one header line
std::vector<std::string_view> words(std::string_view line) {
    std::vector<std::string_view> out;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
        size_t j = i;
        while (j < line.size() && line[j] != ' ' && line[j] != '\t') ++j;
        if (j > i) out.push_back(line.substr(i, j - i));
        i = j;
    }
    return out;
}

template <typename T>
bool parseWhole(std::string_view s, T& v) {
    const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
    return r.ec == std::errc() && r.ptr == s.data() + s.size();
}

template <typename T>
T readAs(const uint8_t* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));  // records are packed: no alignment
    return v;
}

float toFloat(const uint8_t* p, PlyScalar t) {
    switch (t) {
        case PlyScalar::Int8: return float(readAs<int8_t>(p));
        case PlyScalar::UInt8: return float(readAs<uint8_t>(p));
        case PlyScalar::Int16: return float(readAs<int16_t>(p));
        case PlyScalar::UInt16: return float(readAs<uint16_t>(p));
        case PlyScalar::Int32: return float(readAs<int32_t>(p));
        case PlyScalar::UInt32: return float(readAs<uint32_t>(p));
        case PlyScalar::Float32: return readAs<float>(p);
        case PlyScalar::Float64: return float(readAs<double>(p));
    }
    return 0.0f;
}

// NaN or infinity: all exponent bits set
inline bool nonFinite(float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return (b & 0x7F800000u) == 0x7F800000u;
}

struct Field {
    uint32_t offset = 0;
    PlyScalar type = PlyScalar::Float32;
};

// What the header says about the vertex records once the 3DGS checks have passed.
struct VertexPlan {
    Field pos[3], dc[3], opacity, scale[3], rot[4];
    std::vector<Field> rest;  // f_rest_0 .. f_rest_{n-1} in file (channel-major) order
    uint32_t stride = 0;
    bool allFloat = true;
    int shDegree = 0;
    uint64_t count = 0;
    uint64_t vertexOffset = 0;   // file offset of the first vertex record
    uint64_t trailingBytes = 0;  // list-free elements after `vertex`
    bool trailingUnknown = false;
    std::vector<std::string> warnings;
};

// planVertexDecode (ply_loader.cpp:300-401). `fileSize` bounds the elements stored before
// `vertex` (UINT64_MAX while a stream's size is unknown).
VertexPlan planVertices(const PlyHeader& h, const std::string& file, uint64_t fileSize) {
    if (h.format == PlyFormat::Ascii)
        throw FormatError(file + ": ASCII PLY is not supported (3DGS files are binary_little_endian; "
                                 "re-export as binary)");
    if (h.format == PlyFormat::BinaryBigEndian)
        throw FormatError(file + ": binary_big_endian PLY is not supported (expected binary_little_endian)");
    for (const PlyElement& e : h.elements) {
        bool quantized = e.name == "chunk";
        for (const PlyProperty& p : e.properties) quantized = quantized || p.name.compare(0, 7, "packed_") == 0;
        if (quantized)
            throw FormatError(file + ": this is a PlayCanvas compressed PLY (element 'chunk' / packed_* properties), "
                                     "not a standard 3DGS PLY. Decompress it first (e.g. @playcanvas/splat-transform).");
    }
    VertexPlan plan;
    plan.vertexOffset = h.headerBytes;
    const PlyElement* vertex = nullptr;
    for (const PlyElement& e : h.elements) {
        if (e.name == "vertex") {
            vertex = &e;
            continue;
        }
        if (!vertex) {
            if (e.hasList) throw FormatError(file + ": element '" + e.name + "' with list properties precedes 'vertex'");
            const uint64_t left = fileSize - std::min<uint64_t>(plan.vertexOffset, fileSize);
            if (e.stride != 0 && e.count > left / e.stride)
                throw FormatError(file + ": file is truncated inside element '" + e.name + "'");
            plan.vertexOffset += e.count * e.stride;
        } else if (e.hasList) {
            plan.trailingUnknown = true;
        } else {
            plan.trailingBytes += e.count * e.stride;
        }
        plan.warnings.push_back("skipped element '" + e.name + "' (" + std::to_string(e.count) + " records)");
    }
    if (!vertex) throw FormatError(file + ": no 'vertex' element");
    if (vertex->hasList) throw FormatError(file + ": 'vertex' element has list properties (not a 3DGS file)");
    if (vertex->count == 0) throw FormatError(file + ": 'vertex' element is empty (0 gaussians)");
    if (vertex->count > UINT32_MAX) throw FormatError(file + ": too many gaussians");
    plan.count = vertex->count;
    plan.stride = vertex->stride;

    auto need = [&](const char* name) {
        const PlyProperty* p = vertex->find(name);
        if (!p) throw FormatError(file + ": missing required property '" + name + "'");
        plan.allFloat = plan.allFloat && p->type == PlyScalar::Float32;
        return Field{p->offset, p->type};
    };
    static const char* const kPos[3] = {"x", "y", "z"}, *const kDc[3] = {"f_dc_0", "f_dc_1", "f_dc_2"};
    static const char* const kScale[3] = {"scale_0", "scale_1", "scale_2"};
    static const char* const kRot[4] = {"rot_0", "rot_1", "rot_2", "rot_3"};
    for (int c = 0; c < 3; ++c) plan.pos[c] = need(kPos[c]);
    for (int c = 0; c < 3; ++c) plan.dc[c] = need(kDc[c]);
    plan.opacity = need("opacity");
    for (int c = 0; c < 3; ++c) plan.scale[c] = need(kScale[c]);
    for (int c = 0; c < 4; ++c) plan.rot[c] = need(kRot[c]);

    // f_rest_<j>: the count sets the degree; the indices must be exactly 0..n-1
    std::vector<const PlyProperty*> rest;
    for (const PlyProperty& p : vertex->properties) {
        if (p.name.compare(0, 7, "f_rest_") != 0) continue;
        size_t j = 0;
        if (!parseWhole(std::string_view(p.name).substr(7), j))
            throw FormatError(file + ": bad SH property name '" + p.name + "'");
        if (j >= rest.size()) rest.resize(j + 1, nullptr);
        if (rest[j]) throw FormatError(file + ": duplicate property '" + p.name + "'");
        rest[j] = &p;
    }
    size_t present = 0;
    for (const PlyProperty* p : rest) present += p != nullptr;
    if (present != rest.size())
        throw FormatError(file + ": f_rest_* indices are not contiguous (highest index " + std::to_string(rest.size() - 1) +
                          ", but only " + std::to_string(present) + " present)");
    plan.shDegree = shDegreeForRestCount(present);
    if (plan.shDegree < 0)
        throw FormatError(file + ": unexpected number of f_rest_* properties: " + std::to_string(present) +
                          " (expected 0, 9, 24 or 45 for SH degree 0..3)");
    for (const PlyProperty* p : rest) {
        plan.rest.push_back({p->offset, p->type});
        plan.allFloat = plan.allFloat && p->type == PlyScalar::Float32;
    }
    return plan;
}

// checkPayloadSize (ply_loader.cpp:405-422)
void checkPayload(const VertexPlan& plan, uint64_t fileSize, const std::string& file, std::vector<std::string>& warnings) {
    const uint64_t avail = fileSize > plan.vertexOffset ? fileSize - plan.vertexOffset : 0;
    const uint64_t need = plan.count * plan.stride;
    if (avail < need)
        throw FormatError(file + ": file is truncated: header declares " + std::to_string(plan.count) + " gaussians x " +
                          std::to_string(plan.stride) + " bytes = " + std::to_string(need) +
                          " bytes of vertex data, but only " + std::to_string(avail) + " bytes follow the header (" +
                          std::to_string(avail / plan.stride) + " complete records)");
    if (!plan.trailingUnknown && avail > need + plan.trailingBytes)
        warnings.push_back(std::to_string(avail - need - plan.trailingBytes) +
                           " unexpected trailing bytes after the last element");
    if (!plan.trailingUnknown && avail < need + plan.trailingBytes)
        warnings.push_back("elements after 'vertex' are truncated (ignored)");
}

void valueWarnings(HostScene& s, bool allFloat) {
    if (s.stats.nonFiniteValues)
        s.warnings.push_back(std::to_string(s.stats.nonFiniteValues) + " NaN/Inf values in the file");
    if (s.stats.zeroQuaternions)
        s.warnings.push_back(std::to_string(s.stats.zeroQuaternions) + " zero-length quaternions replaced by identity");
    if (!allFloat) s.warnings.push_back("non-float32 properties converted to float");
}

struct DecodeCounters {
    uint64_t nonFinite = 0;
    uint32_t zeroQuats = 0;
};

// Records [0, n) at `records` into scene entries [first, first + n): the raw values, the
// activations of gaussian_model.py (sigmoid opacity, exp scale, normalized rotation) as the
// reference evaluates them (ply_loader.cpp:127-150), and the SH transpose from the file's
// channel-major f_rest[c (K-1) + k-1] to RGB triplets sh[k][c].
template <bool kAllFloat>
void decodeRecords(const VertexPlan& plan, const uint8_t* records, size_t n, HostScene& s, size_t first,
                   DecodeCounters& ctr) {
    const uint32_t K = s.coeffsPerChannel();
    for (size_t r = 0; r < n; ++r) {
        const uint8_t* rec = records + r * plan.stride;
        auto get = [&](const Field& f) {
            const float v = kAllFloat ? readAs<float>(rec + f.offset) : toFloat(rec + f.offset, f.type);
            ctr.nonFinite += nonFinite(v) ? 1u : 0u;
            return v;
        };
        const size_t i = first + r;
        const float px = get(plan.pos[0]), py = get(plan.pos[1]), pz = get(plan.pos[2]);
        const float op = get(plan.opacity);
        float ls[3], q[4];
        for (int c = 0; c < 3; ++c) ls[c] = get(plan.scale[c]);
        for (int c = 0; c < 4; ++c) q[c] = get(plan.rot[c]);
        s.rawOpacity[i] = op;
        for (int c = 0; c < 3; ++c) s.rawLogScale[i * 3 + c] = ls[c];
        for (int c = 0; c < 4; ++c) s.rawRotation[i * 4 + c] = q[c];

        const float e = std::exp(-op);
        const float alpha = 1.0f / (1.0f + e);
        float* pa = &s.posAlpha[i * 4];
        pa[0] = px;
        pa[1] = py;
        pa[2] = pz;
        pa[3] = alpha;
        float* sc = &s.scales[i * 4];
        for (int c = 0; c < 3; ++c) sc[c] = std::exp(ls[c]);
        sc[3] = 0.0f;
        // |q|^2 in GLM 1.0.1's vec4 dot order: (x x + y y) + (z z + w w)
        const float n2 = (q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]);
        float* ro = &s.rotations[i * 4];
        if (n2 > 1e-24f && !nonFinite(n2)) {
            const float len = std::sqrt(n2);
            for (int c = 0; c < 4; ++c) ro[c] = q[c] / len;
        } else {
            ro[0] = 1.0f;
            ro[1] = ro[2] = ro[3] = 0.0f;
            ++ctr.zeroQuats;
        }
        float* out = &s.sh[i * K * 3];
        for (int c = 0; c < 3; ++c) out[c] = get(plan.dc[c]);
        for (uint32_t k = 1; k < K; ++k)
            for (uint32_t c = 0; c < 3; ++c) out[k * 3 + c] = get(plan.rest[c * (K - 1) + (k - 1)]);
    }
}

void decode(const VertexPlan& plan, const uint8_t* records, size_t n, HostScene& s, size_t first, DecodeCounters& ctr) {
    if (plan.allFloat) decodeRecords<true>(plan, records, n, s, first, ctr);
    else decodeRecords<false>(plan, records, n, s, first, ctr);
}

uint32_t hostThreads() { return std::max(1u, std::thread::hardware_concurrency()); }

// k-th smallest (k = floor(p (n - 1))) of the finite values, as sorted[k]
float percentileOf(std::vector<float>& v, double p) {
    if (v.empty()) return 0.0f;
    const size_t k = size_t(p * double(v.size() - 1));
    std::nth_element(v.begin(), v.begin() + std::ptrdiff_t(k), v.end());
    return v[k];
}

// The file's bytes: read-only mapping of the whole file.
struct FileBytes {
    const uint8_t* data = nullptr;
    size_t size = 0;
    void* map = nullptr;
    explicit FileBytes(const std::string& path) {
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("Cannot open file: " + path);
        struct stat st {};
        if (::fstat(fd, &st) != 0) {
            ::close(fd);
            throw std::runtime_error("Cannot read file: " + path);
        }
        size = size_t(st.st_size);
        if (size > 0) {
            map = ::mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (map == MAP_FAILED) {
                map = nullptr;
                ::close(fd);
                throw std::runtime_error("Cannot read file: " + path);
            }
            ::madvise(map, size, MADV_SEQUENTIAL);
            data = static_cast<const uint8_t*>(map);
        }
        ::close(fd);
    }
    ~FileBytes() {
        if (map) ::munmap(map, size);
    }
    FileBytes(const FileBytes&) = delete;
    FileBytes& operator=(const FileBytes&) = delete;
};

std::string baseName(const std::string& path) {
    const size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? path : path.substr(slash + 1);
}

}  // namespace

uint32_t scalarBytes(PlyScalar t) {
    switch (t) {
        case PlyScalar::Int8:
        case PlyScalar::UInt8: return 1;
        case PlyScalar::Int16:
        case PlyScalar::UInt16: return 2;
        case PlyScalar::Int32:
        case PlyScalar::UInt32:
        case PlyScalar::Float32: return 4;
        case PlyScalar::Float64: return 8;
    }
    return 0;
}

const PlyProperty* PlyElement::find(std::string_view property) const {
    for (const PlyProperty& p : properties)
        if (p.name == property) return &p;
    return nullptr;
}

int shDegreeForRestCount(size_t restCount) {
    // restCount = 3 ((d + 1)^2 - 1)
    for (int d = 0; d <= 3; ++d)
        if (restCount == size_t(3 * ((d + 1) * (d + 1) - 1))) return d;
    return -1;
}

std::optional<PlyHeader> parsePlyHeader(std::string_view bytes, bool final) {
    PlyHeader h;
    const std::string_view window = bytes.substr(0, std::min(bytes.size(), kMaxHeaderBytes));
    size_t pos = 0, lineNo = 0;
    bool haveFormat = false;
    for (;;) {
        const size_t eol = window.find('\n', pos);
        if (eol == std::string_view::npos) {
            if (!final && bytes.size() < kMaxHeaderBytes) return std::nullopt;  // more bytes to come
            throw FormatError(lineNo == 0 ? "not a PLY file (empty or no header)"
                                          : "PLY header has no 'end_header' line (file truncated or not a PLY)");
        }
        std::string_view line = bytes.substr(pos, eol - pos);
        if (!line.empty() && line.back() == '\r') line.remove_suffix(1);  // CRLF headers
        pos = eol + 1;
        ++lineNo;
        const std::string at = "PLY header line " + std::to_string(lineNo) + ": ";
        if (lineNo == 1) {
            if (line != "ply") throw FormatError("not a PLY file (first line is not 'ply')");
            continue;
        }
        const std::vector<std::string_view> w = words(line);
        if (w.empty()) continue;
        const std::string_view key = w[0];
        if (key == "end_header") {
            if (!haveFormat) throw FormatError("PLY header has no 'format' line");
            h.headerBytes = pos;
            return h;
        }
        if (key == "comment" || key == "obj_info") {
            h.comments.emplace_back(line.size() > key.size() + 1 ? line.substr(key.size() + 1) : std::string_view());
        } else if (key == "format") {
            if (w.size() < 2) throw FormatError(at + "malformed 'format' line");
            if (w[1] == "binary_little_endian") h.format = PlyFormat::BinaryLittleEndian;
            else if (w[1] == "binary_big_endian") h.format = PlyFormat::BinaryBigEndian;
            else if (w[1] == "ascii") h.format = PlyFormat::Ascii;
            else throw FormatError(at + "unknown format '" + std::string(w[1]) + "'");
            haveFormat = true;
        } else if (key == "element") {
            if (w.size() != 3) throw FormatError(at + "malformed 'element' line");
            PlyElement e;
            e.name = std::string(w[1]);
            if (!parseWhole(w[2], e.count)) throw FormatError(at + "bad element count '" + std::string(w[2]) + "'");
            h.elements.push_back(std::move(e));
        } else if (key == "property") {
            if (h.elements.empty()) throw FormatError(at + "'property' before any 'element'");
            PlyElement& e = h.elements.back();
            PlyProperty p;
            if (w.size() == 5 && w[1] == "list") {
                PlyScalar countType, itemType;
                if (!scalarFromName(w[2], countType) || !scalarFromName(w[3], itemType))
                    throw FormatError(at + "unknown list types");
                p.list = true;
                p.name = std::string(w[4]);
                e.hasList = true;
            } else if (w.size() == 3) {
                if (!scalarFromName(w[1], p.type))
                    throw FormatError(at + "unknown property type '" + std::string(w[1]) + "'");
                p.name = std::string(w[2]);
                p.offset = e.stride;  // unknown names count towards the record size too
                e.stride += scalarBytes(p.type);
            } else {
                throw FormatError(at + "malformed 'property' line");
            }
            e.properties.push_back(std::move(p));
        } else {
            throw FormatError(at + "unknown keyword '" + std::string(key) + "'");
        }
    }
}

void HostScene::resize(size_t n) {
    count = uint32_t(n);
    posAlpha.resize(n * 4);
    scales.resize(n * 4);
    rotations.resize(n * 4);
    sh.resize(n * coeffsPerChannel() * 3);
    rawOpacity.resize(n);
    rawLogScale.resize(n * 3);
    rawRotation.resize(n * 4);
}

void computeSceneStats(HostScene& scene) {
    SceneStats& s = scene.stats;
    s = SceneStats{};
    const size_t n = scene.count;
    if (n == 0) return;
    // positions and opacity (computePositionStats); non-finite values are left out
    const float inf = std::numeric_limits<float>::infinity();
    float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
    float aMin = inf, aMax = -inf;
    double aSum = 0.0;
    uint32_t aLow = 0;
    std::vector<float> axis[3];
    for (auto& a : axis) a.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        const float* pa = &scene.posAlpha[i * 4];
        if (std::isfinite(pa[0]) && std::isfinite(pa[1]) && std::isfinite(pa[2])) {
            for (int c = 0; c < 3; ++c) {
                lo[c] = pa[c] < lo[c] ? pa[c] : lo[c];
                hi[c] = hi[c] < pa[c] ? pa[c] : hi[c];
                axis[c].push_back(pa[c]);
            }
        }
        if (std::isfinite(pa[3])) {
            aMin = std::min(aMin, pa[3]);
            aMax = std::max(aMax, pa[3]);
            aSum += pa[3];
            if (pa[3] < 1.0f / 255.0f) ++aLow;
        }
    }
    for (int c = 0; c < 3; ++c) {
        s.bboxMin[c] = lo[c];
        s.bboxMax[c] = hi[c];
        s.robustMin[c] = percentileOf(axis[c], 0.01f);
        s.robustMax[c] = percentileOf(axis[c], 1.0 - 0.01f);
    }
    s.alphaMin = aMin;
    s.alphaMax = aMax;
    s.alphaMean = float(aSum / double(n));
    s.alphaBelowVisible = aLow;
    // scales and raw quaternion lengths
    float sMin = inf, sMax = -inf, qMin = inf, qMax = -inf;
    std::vector<float> maxSigma;
    maxSigma.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        const float* sg = &scene.scales[i * 4];
        if (std::isfinite(sg[0]) && std::isfinite(sg[1]) && std::isfinite(sg[2])) {
            // std::min / std::max over a list keep the first of equal values
            float mn = sg[0], mx = sg[0];
            for (int c = 1; c < 3; ++c) {
                if (sg[c] < mn) mn = sg[c];
                if (mx < sg[c]) mx = sg[c];
            }
            sMin = std::min(sMin, mn);
            sMax = std::max(sMax, mx);
            maxSigma.push_back(mx);
        }
        const float* q = &scene.rawRotation[i * 4];
        const float qn = std::sqrt((q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]));
        if (std::isfinite(qn)) {
            qMin = std::min(qMin, qn);
            qMax = std::max(qMax, qn);
        }
    }
    s.sigmaMin = sMin;
    s.sigmaMax = sMax;
    s.sigmaMaxMedian = percentileOf(maxSigma, 0.5);
    s.quatNormMin = qMin;
    s.quatNormMax = qMax;
}

HostScene loadPly(const uint8_t* bytes, size_t size, const std::string& file) {
    const auto t0 = Clock::now();
    HostScene scene;
    scene.sourcePath = file;
    const auto tHeader = Clock::now();
    std::optional<PlyHeader> header;
    try {
        header = parsePlyHeader(std::string_view(reinterpret_cast<const char*>(bytes), size), true);
    } catch (const FormatError& e) {
        throw FormatError(file + ": " + e.what());
    }
    scene.comments = header->comments;
    const VertexPlan plan = planVertices(*header, file, size);
    scene.warnings = plan.warnings;
    checkPayload(plan, size, file, scene.warnings);
    scene.shDegree = plan.shDegree;
    scene.timings.headerMs = msSince(tHeader);

    const auto tDecode = Clock::now();
    const size_t n = size_t(plan.count);
    scene.resize(n);
    const uint8_t* records = bytes + plan.vertexOffset;
    // contiguous ranges, one per host thread (16384 records at least per thread)
    const size_t threads = std::clamp<size_t>(n / 16384, 1, hostThreads());
    std::vector<DecodeCounters> ctr(threads);
    if (threads == 1) {
        decode(plan, records, n, scene, 0, ctr[0]);
    } else {
        std::vector<std::thread> pool;
        for (size_t t = 0; t < threads; ++t) {
            const size_t b = n * t / threads, e = n * (t + 1) / threads;
            pool.emplace_back([&, t, b, e] { decode(plan, records + b * plan.stride, e - b, scene, b, ctr[t]); });
        }
        for (auto& th : pool) th.join();
    }
    scene.timings.decodeMs = msSince(tDecode);

    const auto tStats = Clock::now();
    computeSceneStats(scene);
    for (const DecodeCounters& c : ctr) {
        scene.stats.nonFiniteValues += c.nonFinite;
        scene.stats.zeroQuaternions += c.zeroQuats;
    }
    valueWarnings(scene, plan.allFloat);
    scene.timings.statsMs = msSince(tStats);
    scene.timings.totalMs = msSince(t0);
    return scene;
}

HostScene loadPly(const std::string& path) {
    const auto t0 = Clock::now();
    FileBytes f(path);
    const double mapMs = msSince(t0);
    HostScene scene = loadPly(f.data, f.size, baseName(path));
    scene.sourcePath = path;
    scene.timings.mapMs = mapMs;
    scene.timings.totalMs = msSince(t0);
    return scene;
}

// ---- the streaming decoder (ply_loader.cpp:507-678) -------------------------------------------
struct PlyStream::State {
    std::string file;
    uint64_t totalBytes = 0;  // 0: unknown
    uint32_t batchCapacity = 1;
    HeaderFn onHeader;
    BatchFn onBatch;
    uint64_t received = 0;
    std::string headerText;  // the first bytes, until the header parses
    bool headerDone = false, done = false, failed = false;
    PlyHeader header;
    VertexPlan plan;
    uint64_t vertexEnd = 0;
    std::vector<uint8_t> pending;  // whole records waiting for a batch decode
    size_t pendingBytes = 0;
    uint64_t decoded = 0;
    HostScene batch, info;
    DecodeCounters counters;
    Clock::time_point start = Clock::now();
    double decodeMs = 0.0;

    void beginPayload() {
        headerDone = true;
        info.comments = header.comments;
        // with the total size known, a truncated file fails before any record is decoded
        plan = planVertices(header, file, totalBytes ? totalBytes : UINT64_MAX);
        if (totalBytes) {
            std::vector<std::string> later;  // reported by finish()
            checkPayload(plan, totalBytes, file, later);
        }
        const uint64_t vertexBytes = plan.count * plan.stride;
        vertexEnd = plan.vertexOffset > UINT64_MAX - vertexBytes ? UINT64_MAX : plan.vertexOffset + vertexBytes;
        info.count = uint32_t(plan.count);
        info.shDegree = plan.shDegree;
        info.timings.headerMs = msSince(start);
        pending.resize(size_t(std::min<uint64_t>(plan.count, batchCapacity)) * plan.stride);
        batch.shDegree = plan.shDegree;
        batch.comments = header.comments;
        if (onHeader) onHeader(info);
    }

    // the bytes [fileOffset, fileOffset + size) of the file; only vertex records are kept
    void payload(const uint8_t* data, size_t size, uint64_t fileOffset) {
        const uint64_t b = std::max<uint64_t>(fileOffset, plan.vertexOffset);
        const uint64_t e = std::min<uint64_t>(fileOffset + size, vertexEnd);
        for (uint64_t at = b; at < e;) {
            const size_t take = size_t(std::min<uint64_t>(e - at, pending.size() - pendingBytes));
            std::memcpy(pending.data() + pendingBytes, data + (at - fileOffset), take);
            pendingBytes += take;
            at += take;
            if (pendingBytes == pending.size()) flush();
        }
        if (fileOffset + size >= vertexEnd && pendingBytes > 0) flush();  // the last, partial batch
    }

    void flush() {
        const size_t m = pendingBytes / plan.stride;
        const auto t0 = Clock::now();
        batch.resize(m);
        decode(plan, pending.data(), m, batch, 0, counters);
        decodeMs += msSince(t0);
        if (onBatch) onBatch(uint32_t(decoded), batch);
        decoded += m;
        pendingBytes = 0;
    }
};

PlyStream::PlyStream(std::string name, uint64_t totalBytes, HeaderFn onHeader, BatchFn onBatch, uint32_t batchCapacity)
    : s_(std::make_unique<State>()) {
    s_->file = std::move(name);
    s_->totalBytes = totalBytes;
    s_->batchCapacity = std::max(1u, batchCapacity);
    s_->onHeader = std::move(onHeader);
    s_->onBatch = std::move(onBatch);
    s_->info.sourcePath = s_->file;
}

PlyStream::~PlyStream() = default;
bool PlyStream::headerParsed() const { return s_->headerDone; }
bool PlyStream::finished() const { return s_->done; }
uint64_t PlyStream::bytesReceived() const { return s_->received; }
uint64_t PlyStream::recordsDecoded() const { return s_->decoded; }
const HostScene& PlyStream::info() const { return s_->info; }

void PlyStream::push(const uint8_t* bytes, size_t size) {
    State& s = *s_;
    if (s.failed || s.done) throw std::logic_error("PlyStreamDecoder::push after an error or finish()");
    try {
        size_t used = 0;
        if (!s.headerDone) {
            // collect at most kMaxHeaderBytes; try the header whenever a line has ended
            used = std::min(size, kMaxHeaderBytes - std::min(kMaxHeaderBytes, s.headerText.size()));
            const size_t before = s.headerText.size();
            s.headerText.append(reinterpret_cast<const char*>(bytes), used);
            s.received += used;
            const bool full = s.headerText.size() >= kMaxHeaderBytes;
            if (full || s.headerText.find('\n', before) != std::string::npos) {
                std::optional<PlyHeader> h;
                try {
                    h = parsePlyHeader(s.headerText, full);
                } catch (const FormatError& e) {
                    throw FormatError(s.file + ": " + e.what());
                }
                if (h) {
                    s.header = std::move(*h);
                    s.beginPayload();
                    const size_t hb = s.header.headerBytes;  // collected bytes past end_header are payload
                    s.payload(reinterpret_cast<const uint8_t*>(s.headerText.data()) + hb, s.headerText.size() - hb, hb);
                    s.headerText = std::string();
                }
            }
        }
        if (s.headerDone && used < size) {
            s.payload(bytes + used, size - used, s.received);
            s.received += size - used;
        }
    } catch (...) {
        s.failed = true;
        throw;
    }
}

void PlyStream::finish() {
    State& s = *s_;
    if (s.failed || s.done) throw std::logic_error("PlyStreamDecoder::finish after an error or finish()");
    try {
        if (!s.headerDone) {
            try {
                parsePlyHeader(s.headerText, true);  // throws: no complete header arrived
            } catch (const FormatError& e) {
                throw FormatError(s.file + ": " + e.what());
            }
            throw FormatError(s.file + ": incomplete PLY header");
        }
        if (s.totalBytes && s.received != s.totalBytes)
            throw std::runtime_error(s.file + ": stream ended after " + std::to_string(s.received) + " of " +
                                     std::to_string(s.totalBytes) + " bytes");
        // the whole-file checks with the real size: the same errors and warnings
        s.plan = planVertices(s.header, s.file, s.received);
        s.info.warnings = s.plan.warnings;
        checkPayload(s.plan, s.received, s.file, s.info.warnings);
        s.info.stats.nonFiniteValues = s.counters.nonFinite;
        s.info.stats.zeroQuaternions = s.counters.zeroQuats;
        valueWarnings(s.info, s.plan.allFloat);
        s.info.timings.decodeMs = s.decodeMs;
        s.info.timings.totalMs = msSince(s.start);
        s.done = true;
    } catch (...) {
        s.failed = true;
        throw;
    }
}

}  // namespace gsr::io
