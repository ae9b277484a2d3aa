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

// A header is read from at most this many bytes (3DGS headers are a few KB).
constexpr size_t kMaxHeaderBytes = size_t(1) << 20;

// ---- scalars -----------------------------------------------------------------------------------
struct ScalarName {
    std::string_view name;
    PlyScalar type;
};
// the PLY specification's type names and their sized spellings
constexpr ScalarName kScalarNames[] = {
    {"char", PlyScalar::Int8},      {"uchar", PlyScalar::UInt8},    {"short", PlyScalar::Int16},
    {"ushort", PlyScalar::UInt16},  {"int", PlyScalar::Int32},      {"uint", PlyScalar::UInt32},
    {"float", PlyScalar::Float32},  {"double", PlyScalar::Float64}, {"int8", PlyScalar::Int8},
    {"uint8", PlyScalar::UInt8},    {"int16", PlyScalar::Int16},    {"uint16", PlyScalar::UInt16},
    {"int32", PlyScalar::Int32},    {"uint32", PlyScalar::UInt32},  {"float32", PlyScalar::Float32},
    {"float64", PlyScalar::Float64}};

std::optional<PlyScalar> scalarNamed(std::string_view s) {
    const auto it = std::find_if(std::begin(kScalarNames), std::end(kScalarNames),
                                 [&](const ScalarName& n) { return n.name == s; });
    if (it == std::end(kScalarNames)) return std::nullopt;
    return it->type;
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

bool startsWith(std::string_view s, std::string_view prefix) { return s.substr(0, prefix.size()) == prefix; }

// ---- the 3DGS vertex schema ---------------------------------------------------------------------
// The attributes the renderer reads from a vertex record, in the order a missing one is reported.
enum Attr : int { kPosX = 0, kDcR = 3, kOpacity = 6, kScale0 = 7, kRotW = 10, kAttrCount = 14 };
constexpr std::string_view kAttrNames[kAttrCount] = {"x",       "y",       "z",       "f_dc_0", "f_dc_1",
                                                     "f_dc_2",  "opacity", "scale_0", "scale_1", "scale_2",
                                                     "rot_0",   "rot_1",   "rot_2",   "rot_3"};
constexpr std::string_view kShRestPrefix = "f_rest_";

struct Field {
    uint32_t offset = 0;
    PlyScalar type = PlyScalar::Float32;
};

// Where a file's 3DGS records are and how one of them is read.
struct VertexSource {
    uint64_t first = 0;         // file offset of record 0
    uint64_t records = 0;
    uint32_t recordBytes = 0;
    Field attr[kAttrCount];
    std::vector<Field> shRest;  // f_rest_0 .. in index (channel-major) order
    int shDegree = 0;
    bool float32Only = true;    // every field the decode reads is float32
    uint64_t bytesAfter = 0;    // bytes of the list-free elements that follow the vertex records
    bool listsAfter = false;    // an element with list properties follows (its size is unknown)
    std::vector<std::string> notes;  // one warning per skipped element
};

// ---- what the element list says, before any judgement ------------------------------------------
struct ElementSurvey {
    const PlyElement* vertex = nullptr;        // the element the records are read with
    size_t firstVertex = SIZE_MAX;             // index of the first element named 'vertex'
    const PlyElement* listBefore = nullptr;    // the first element with lists stored before the records
    const PlyElement* overrunBefore = nullptr; // the first element before the records longer than the file
    uint64_t recordsAt = 0;
    uint64_t bytesAfter = 0;
    bool listsAfter = false;
    bool compressed = false;                   // PlayCanvas quantized layout
    std::vector<std::string> skipped;
};

ElementSurvey surveyElements(const PlyHeader& h, uint64_t fileSize) {
    ElementSurvey v;
    v.recordsAt = h.headerBytes;
    for (size_t i = 0; i < h.elements.size(); ++i) {
        const PlyElement& e = h.elements[i];
        v.compressed = v.compressed || e.name == "chunk" ||
                       std::any_of(e.properties.begin(), e.properties.end(),
                                   [](const PlyProperty& p) { return startsWith(p.name, "packed_"); });
        if (e.name == "vertex") {
            v.vertex = &e;  // a later 'vertex' element is the one the records are read with
            v.firstVertex = std::min(v.firstVertex, i);
            continue;
        }
        v.skipped.push_back("skipped element '" + e.name + "' (" + std::to_string(e.count) + " records)");
        if (v.firstVertex != SIZE_MAX) {  // stored after the vertex records
            if (e.hasList) v.listsAfter = true;
            else v.bytesAfter += e.count * e.stride;
            continue;
        }
        if (v.listBefore || v.overrunBefore) continue;  // the first offender decides
        if (e.hasList) {
            v.listBefore = &e;
            continue;
        }
        const uint64_t room = fileSize - std::min<uint64_t>(v.recordsAt, fileSize);
        if (e.stride != 0 && e.count > room / e.stride) {  // (count x stride would overflow first)
            v.overrunBefore = &e;
            continue;
        }
        v.recordsAt += e.count * e.stride;
    }
    return v;
}

// ---- the acceptance rules, in the order they are checked ----------------------------------------
struct HeaderRule {
    bool (*broken)(const PlyHeader&, const ElementSurvey&);
    std::string (*explain)(const ElementSurvey&);
};
const HeaderRule kHeaderRules[] = {
    {[](const PlyHeader& h, const ElementSurvey&) { return h.format == PlyFormat::Ascii; },
     [](const ElementSurvey&) -> std::string {
         return "ASCII PLY is not supported (3DGS files are binary_little_endian; re-export as binary)";
     }},
    {[](const PlyHeader& h, const ElementSurvey&) { return h.format == PlyFormat::BinaryBigEndian; },
     [](const ElementSurvey&) -> std::string {
         return "binary_big_endian PLY is not supported (expected binary_little_endian)";
     }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.compressed; },
     [](const ElementSurvey&) -> std::string {
         return "this is a PlayCanvas compressed PLY (element 'chunk' / packed_* properties), not a standard "
                "3DGS PLY. Decompress it first (e.g. @playcanvas/splat-transform).";
     }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.listBefore != nullptr; },
     [](const ElementSurvey& v) { return "element '" + v.listBefore->name + "' with list properties precedes 'vertex'"; }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.overrunBefore != nullptr; },
     [](const ElementSurvey& v) { return "file is truncated inside element '" + v.overrunBefore->name + "'"; }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.vertex == nullptr; },
     [](const ElementSurvey&) -> std::string { return "no 'vertex' element"; }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.vertex->hasList; },
     [](const ElementSurvey&) -> std::string { return "'vertex' element has list properties (not a 3DGS file)"; }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.vertex->count == 0; },
     [](const ElementSurvey&) -> std::string { return "'vertex' element is empty (0 gaussians)"; }},
    {[](const PlyHeader&, const ElementSurvey& v) { return v.vertex->count > UINT32_MAX; },
     [](const ElementSurvey&) -> std::string { return "too many gaussians"; }},
};

// Binds the schema's attributes and the SH-rest properties of the vertex element.
void bindAttributes(const PlyElement& vertex, const std::string& file, VertexSource& src) {
    for (int a = 0; a < kAttrCount; ++a) {
        const PlyProperty* p = vertex.find(kAttrNames[a]);
        if (!p) throw FormatError(file + ": missing required property '" + std::string(kAttrNames[a]) + "'");
        src.attr[a] = Field{p->offset, p->type};
        src.float32Only = src.float32Only && p->type == PlyScalar::Float32;
    }
    // f_rest_<j>: indices 0..n-1 exactly once each; n sets the degree
    std::vector<std::pair<size_t, const PlyProperty*>> rest;
    for (const PlyProperty& p : vertex.properties) {
        if (!startsWith(p.name, kShRestPrefix)) continue;
        size_t j = 0;
        if (!parseWhole(std::string_view(p.name).substr(kShRestPrefix.size()), j))
            throw FormatError(file + ": bad SH property name '" + p.name + "'");
        if (std::any_of(rest.begin(), rest.end(), [&](const auto& r) { return r.first == j; }))
            throw FormatError(file + ": duplicate property '" + p.name + "'");
        rest.emplace_back(j, &p);
    }
    std::sort(rest.begin(), rest.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const size_t highest = rest.empty() ? 0 : rest.back().first;
    if (!rest.empty() && highest + 1 != rest.size())
        throw FormatError(file + ": f_rest_* indices are not contiguous (highest index " + std::to_string(highest) +
                          ", but only " + std::to_string(rest.size()) + " present)");
    src.shDegree = shDegreeForRestCount(rest.size());
    if (src.shDegree < 0)
        throw FormatError(file + ": unexpected number of f_rest_* properties: " + std::to_string(rest.size()) +
                          " (expected 0, 9, 24 or 45 for SH degree 0..3)");
    for (const auto& r : rest) {
        src.shRest.push_back(Field{r.second->offset, r.second->type});
        src.float32Only = src.float32Only && r.second->type == PlyScalar::Float32;
    }
}

// The header judged for 3DGS use (loadGaussianPly's checks, ply_loader.cpp:300-401: the same
// files are accepted and the same texts name the first problem). `fileSize` is UINT64_MAX while a
// stream's size is unknown.
VertexSource locateVertices(const PlyHeader& h, const std::string& file, uint64_t fileSize) {
    const ElementSurvey survey = surveyElements(h, fileSize);
    for (const HeaderRule& rule : kHeaderRules)
        if (rule.broken(h, survey)) throw FormatError(file + ": " + rule.explain(survey));
    VertexSource src;
    src.first = survey.recordsAt;
    src.records = survey.vertex->count;
    src.recordBytes = survey.vertex->stride;
    src.bytesAfter = survey.bytesAfter;
    src.listsAfter = survey.listsAfter;
    src.notes = survey.skipped;
    bindAttributes(*survey.vertex, file, src);
    return src;
}

// The payload against the header (checkPayloadSize, ply_loader.cpp:405-422): too few bytes for
// the records is an error; bytes that the elements after the records do not explain are warnings.
void checkPayload(const VertexSource& src, uint64_t fileSize, const std::string& file,
                  std::vector<std::string>& warnings) {
    const uint64_t follow = fileSize > src.first ? fileSize - src.first : 0;
    const uint64_t wanted = src.records * src.recordBytes;
    if (follow < wanted)
        throw FormatError(file + ": file is truncated: header declares " + std::to_string(src.records) +
                          " gaussians x " + std::to_string(src.recordBytes) + " bytes = " + std::to_string(wanted) +
                          " bytes of vertex data, but only " + std::to_string(follow) +
                          " bytes follow the header (" + std::to_string(follow / src.recordBytes) +
                          " complete records)");
    if (src.listsAfter) return;  // the size of what follows is unknown: nothing to compare
    const uint64_t explained = wanted + src.bytesAfter;
    if (follow > explained) warnings.push_back(std::to_string(follow - explained) + " unexpected trailing bytes after the last element");
    if (follow < explained) warnings.push_back("elements after 'vertex' are truncated (ignored)");
}

void valueWarnings(HostScene& s, bool float32Only) {
    if (s.stats.nonFiniteValues)
        s.warnings.push_back(std::to_string(s.stats.nonFiniteValues) + " NaN/Inf values in the file");
    if (s.stats.zeroQuaternions)
        s.warnings.push_back(std::to_string(s.stats.zeroQuaternions) + " zero-length quaternions replaced by identity");
    if (!float32Only) s.warnings.push_back("non-float32 properties converted to float");
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
void decodeRecords(const VertexSource& src, const uint8_t* records, size_t n, HostScene& s, size_t first,
                   DecodeCounters& ctr) {
    const uint32_t K = s.coeffsPerChannel();
    for (size_t r = 0; r < n; ++r) {
        const uint8_t* rec = records + r * src.recordBytes;
        auto get = [&](const Field& f) {
            const float v = kAllFloat ? readAs<float>(rec + f.offset) : toFloat(rec + f.offset, f.type);
            ctr.nonFinite += nonFinite(v) ? 1u : 0u;
            return v;
        };
        const size_t i = first + r;
        const float px = get(src.attr[kPosX]), py = get(src.attr[kPosX + 1]), pz = get(src.attr[kPosX + 2]);
        const float op = get(src.attr[kOpacity]);
        float ls[3], q[4];
        for (int c = 0; c < 3; ++c) ls[c] = get(src.attr[kScale0 + c]);
        for (int c = 0; c < 4; ++c) q[c] = get(src.attr[kRotW + c]);
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
        for (int c = 0; c < 3; ++c) out[c] = get(src.attr[kDcR + c]);
        for (uint32_t k = 1; k < K; ++k)
            for (uint32_t c = 0; c < 3; ++c) out[k * 3 + c] = get(src.shRest[c * (K - 1) + (k - 1)]);
    }
}

void decode(const VertexSource& src, const uint8_t* records, size_t n, HostScene& s, size_t first, DecodeCounters& ctr) {
    if (src.float32Only) decodeRecords<true>(src, records, n, s, first, ctr);
    else decodeRecords<false>(src, records, n, s, first, ctr);
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

namespace {

// One header line split into its words (spaces and tabs separate them).
struct HeaderLine {
    std::string_view text;  // without the line end
    std::vector<std::string_view> word;
    std::string where;      // "PLY header line <n>: ", the prefix of a syntax error on it
};

void splitWords(HeaderLine& l) {
    constexpr std::string_view kBlank = " \t";
    for (size_t b = l.text.find_first_not_of(kBlank); b != std::string_view::npos;
         b = l.text.find_first_not_of(kBlank, b)) {
        const size_t e = std::min(l.text.find_first_of(kBlank, b), l.text.size());
        l.word.push_back(l.text.substr(b, e - b));
        b = e;
    }
}

// What the header lines build.
struct HeaderBuilder {
    PlyHeader header;
    bool haveFormat = false;
};

void onComment(HeaderBuilder& b, const HeaderLine& l) {
    const size_t skip = l.word[0].size() + 1;  // the keyword and one separator
    b.header.comments.emplace_back(l.text.size() > skip ? l.text.substr(skip) : std::string_view());
}

void onFormat(HeaderBuilder& b, const HeaderLine& l) {
    static const std::pair<std::string_view, PlyFormat> kFormats[] = {
        {"binary_little_endian", PlyFormat::BinaryLittleEndian},
        {"binary_big_endian", PlyFormat::BinaryBigEndian},
        {"ascii", PlyFormat::Ascii}};
    if (l.word.size() < 2) throw FormatError(l.where + "malformed 'format' line");
    const auto it = std::find_if(std::begin(kFormats), std::end(kFormats), [&](const auto& f) { return f.first == l.word[1]; });
    if (it == std::end(kFormats)) throw FormatError(l.where + "unknown format '" + std::string(l.word[1]) + "'");
    b.header.format = it->second;
    b.haveFormat = true;
}

void onElement(HeaderBuilder& b, const HeaderLine& l) {
    if (l.word.size() != 3) throw FormatError(l.where + "malformed 'element' line");
    PlyElement e;
    e.name = std::string(l.word[1]);
    if (!parseWhole(l.word[2], e.count)) throw FormatError(l.where + "bad element count '" + std::string(l.word[2]) + "'");
    b.header.elements.push_back(std::move(e));
}

void onProperty(HeaderBuilder& b, const HeaderLine& l) {
    if (b.header.elements.empty()) throw FormatError(l.where + "'property' before any 'element'");
    PlyElement& e = b.header.elements.back();
    PlyProperty p;
    const size_t n = l.word.size();
    if (n == 5 && l.word[1] == "list") {  // property list <count type> <item type> <name>
        if (!scalarNamed(l.word[2]) || !scalarNamed(l.word[3])) throw FormatError(l.where + "unknown list types");
        p.list = true;
        e.hasList = true;
    } else if (n == 3) {  // property <type> <name>; every scalar counts towards the record, named or not
        const std::optional<PlyScalar> t = scalarNamed(l.word[1]);
        if (!t) throw FormatError(l.where + "unknown property type '" + std::string(l.word[1]) + "'");
        p.type = *t;
        p.offset = e.stride;
        e.stride += scalarBytes(p.type);
    } else {
        throw FormatError(l.where + "malformed 'property' line");
    }
    p.name = std::string(l.word[n - 1]);
    e.properties.push_back(std::move(p));
}

using LineHandler = void (*)(HeaderBuilder&, const HeaderLine&);
const std::pair<std::string_view, LineHandler> kHeaderKeywords[] = {
    {"comment", onComment}, {"obj_info", onComment}, {"format", onFormat},
    {"element", onElement}, {"property", onProperty}};

}  // namespace

std::optional<PlyHeader> parsePlyHeader(std::string_view bytes, bool final) {
    // lines are searched for in the first kMaxHeaderBytes bytes only
    const std::string_view window = bytes.substr(0, std::min(bytes.size(), kMaxHeaderBytes));
    HeaderBuilder b;
    size_t next = 0;
    for (size_t lineNo = 1;; ++lineNo) {
        const size_t eol = window.find('\n', next);
        if (eol == std::string_view::npos) {
            if (!final && bytes.size() < kMaxHeaderBytes) return std::nullopt;  // more bytes to come
            throw FormatError(lineNo == 1 ? "not a PLY file (empty or no header)"
                                          : "PLY header has no 'end_header' line (file truncated or not a PLY)");
        }
        HeaderLine l;
        l.text = bytes.substr(next, eol - next);
        if (!l.text.empty() && l.text.back() == '\r') l.text.remove_suffix(1);  // CRLF line ends
        next = eol + 1;
        if (lineNo == 1) {
            if (l.text != "ply") throw FormatError("not a PLY file (first line is not 'ply')");
            continue;
        }
        l.where = "PLY header line " + std::to_string(lineNo) + ": ";
        splitWords(l);
        if (l.word.empty()) continue;
        if (l.word[0] == "end_header") {
            if (!b.haveFormat) throw FormatError("PLY header has no 'format' line");
            b.header.headerBytes = next;
            return std::move(b.header);
        }
        const auto h = std::find_if(std::begin(kHeaderKeywords), std::end(kHeaderKeywords),
                                    [&](const auto& k) { return k.first == l.word[0]; });
        if (h == std::end(kHeaderKeywords)) throw FormatError(l.where + "unknown keyword '" + std::string(l.word[0]) + "'");
        h->second(b, l);
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
    const VertexSource src = locateVertices(*header, file, size);
    scene.warnings = src.notes;
    checkPayload(src, size, file, scene.warnings);
    scene.shDegree = src.shDegree;
    scene.timings.headerMs = msSince(tHeader);

    const auto tDecode = Clock::now();
    const size_t n = size_t(src.records);
    scene.resize(n);
    const uint8_t* records = bytes + src.first;
    // contiguous ranges, one per host thread (16384 records at least per thread)
    const size_t threads = std::clamp<size_t>(n / 16384, 1, hostThreads());
    std::vector<DecodeCounters> ctr(threads);
    if (threads == 1) {
        decode(src, records, n, scene, 0, ctr[0]);
    } else {
        std::vector<std::thread> pool;
        for (size_t t = 0; t < threads; ++t) {
            const size_t b = n * t / threads, e = n * (t + 1) / threads;
            pool.emplace_back([&, t, b, e] { decode(src, records + b * src.recordBytes, e - b, scene, b, ctr[t]); });
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
    valueWarnings(scene, src.float32Only);
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
    VertexSource src;
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
        src = locateVertices(header, file, totalBytes ? totalBytes : UINT64_MAX);
        if (totalBytes) {
            std::vector<std::string> later;  // reported by finish()
            checkPayload(src, totalBytes, file, later);
        }
        const uint64_t vertexBytes = src.records * src.recordBytes;
        vertexEnd = src.first > UINT64_MAX - vertexBytes ? UINT64_MAX : src.first + vertexBytes;
        info.count = uint32_t(src.records);
        info.shDegree = src.shDegree;
        info.timings.headerMs = msSince(start);
        pending.resize(size_t(std::min<uint64_t>(src.records, batchCapacity)) * src.recordBytes);
        batch.shDegree = src.shDegree;
        batch.comments = header.comments;
        if (onHeader) onHeader(info);
    }

    // the bytes [fileOffset, fileOffset + size) of the file; only vertex records are kept
    void payload(const uint8_t* data, size_t size, uint64_t fileOffset) {
        const uint64_t b = std::max<uint64_t>(fileOffset, src.first);
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
        const size_t m = pendingBytes / src.recordBytes;
        const auto t0 = Clock::now();
        batch.resize(m);
        decode(src, pending.data(), m, batch, 0, counters);
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
        s.src = locateVertices(s.header, s.file, s.received);
        s.info.warnings = s.src.notes;
        checkPayload(s.src, s.received, s.file, s.info.warnings);
        s.info.stats.nonFiniteValues = s.counters.nonFinite;
        s.info.stats.zeroQuaternions = s.counters.zeroQuats;
        valueWarnings(s.info, s.src.float32Only);
        s.info.timings.decodeMs = s.decodeMs;
        s.info.timings.totalMs = msSince(s.start);
        s.done = true;
    } catch (...) {
        s.failed = true;
        throw;
    }
}

}  // namespace gsr::io
