// Checkpoint files of the learned colour stage (no reference counterpart): the host-only writer
// and reader of the versioned binary layout that include/gsr_b200.h documents. The device side
// (gsr_color_model_save / load / resume) lives with the model in renderer.cpp.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gsr_b200.h"

namespace gsr {
void setLastError(const std::string& message);
}

namespace {

constexpr char kMagic[8] = {'G', 'S', 'R', 'C', 'L', 'R', 'M', '\0'};
static_assert(sizeof(GsrColorModelOptions) == 48 && sizeof(GsrColorModelStats) == 48, "the file's header blocks");

// The fixed part after the magic: version, count, degree, step, loss count, parameter count.
struct FileHeader {
    uint32_t version, count;
    int32_t shDegree;
    uint32_t step, lossCount, params;
    GsrColorModelOptions options;
    GsrColorModelStats stats;
};
static_assert(sizeof(FileHeader) == 24 + 48 + 48, "no padding in the header");

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), table-driven.
uint32_t crc32(const uint8_t* p, size_t n, uint32_t crc = 0) {
    static const auto table = [] {
        std::vector<uint32_t> t(256);
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[i] = c;
        }
        return t;
    }();
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return ~crc;
}

int failWith(int status, const std::string& message) {
    gsr::setLastError(message);
    return status;
}

uint64_t payloadBytes(const FileHeader& h) {
    return uint64_t(h.params) * 4 * 3 + uint64_t(h.lossCount) * 4 + uint64_t(h.count) * 16;
}

}  // namespace

extern "C" {

int gsr_color_model_file_write(const char* path, const GsrColorModelCheckpoint* ck) {
    if (!path || !ck || !ck->params || !ck->adam_m || !ck->adam_v || (ck->loss_count && !ck->loss) ||
        (ck->count && !ck->latents))
        return failWith(GSR_ERROR_INVALID_ARGUMENT, "checkpoint: null argument");
    FileHeader h{};
    h.version = GSR_COLOR_MODEL_FILE_VERSION;
    h.count = ck->count;
    h.shDegree = ck->sh_degree;
    h.step = ck->step;
    h.lossCount = ck->loss_count;
    h.params = GSR_COLOR_MODEL_PARAMS;
    h.options = ck->options;
    h.stats = ck->stats;
    std::vector<uint8_t> bytes(sizeof(kMagic) + sizeof(h) + payloadBytes(h) + 4);
    uint8_t* at = bytes.data();
    auto put = [&](const void* src, size_t n) {
        if (n) std::memcpy(at, src, n);
        at += n;
    };
    put(kMagic, sizeof(kMagic));
    put(&h, sizeof(h));
    put(ck->params, size_t(h.params) * 4);
    put(ck->adam_m, size_t(h.params) * 4);
    put(ck->adam_v, size_t(h.params) * 4);
    put(ck->loss, size_t(h.lossCount) * 4);
    put(ck->latents, size_t(h.count) * 16);
    const uint32_t crc = crc32(bytes.data(), size_t(at - bytes.data()));
    put(&crc, 4);
    FILE* f = std::fopen(path, "wb");
    if (!f) return failWith(GSR_ERROR_IO, std::string("cannot write ") + path);
    const size_t written = std::fwrite(bytes.data(), 1, bytes.size(), f);
    const bool closed = std::fclose(f) == 0;
    if (written != bytes.size() || !closed) return failWith(GSR_ERROR_IO, std::string("cannot write ") + path);
    return GSR_OK;
}

int gsr_color_model_file_read(const char* path, GsrColorModelCheckpoint* ck) {
    if (!path || !ck) return failWith(GSR_ERROR_INVALID_ARGUMENT, "checkpoint: null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return failWith(GSR_ERROR_IO, std::string("cannot open ") + path);
    std::vector<uint8_t> bytes;
    uint8_t buf[1 << 16];
    for (size_t n; (n = std::fread(buf, 1, sizeof(buf), f)) > 0;) bytes.insert(bytes.end(), buf, buf + n);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) return failWith(GSR_ERROR_IO, std::string("cannot read ") + path);
    const std::string name(path);
    if (bytes.size() < sizeof(kMagic) + sizeof(FileHeader) + 4 || std::memcmp(bytes.data(), kMagic, sizeof(kMagic)) != 0)
        return failWith(GSR_ERROR_FORMAT, name + ": not a colour model checkpoint");
    FileHeader h;
    std::memcpy(&h, bytes.data() + sizeof(kMagic), sizeof(h));
    if (h.version != GSR_COLOR_MODEL_FILE_VERSION)
        return failWith(GSR_ERROR_FORMAT, name + ": checkpoint version " + std::to_string(h.version) + " (this library reads " +
                                              std::to_string(GSR_COLOR_MODEL_FILE_VERSION) + ")");
    if (h.params != GSR_COLOR_MODEL_PARAMS)
        return failWith(GSR_ERROR_FORMAT, name + ": " + std::to_string(h.params) + " parameters (expected " +
                                              std::to_string(GSR_COLOR_MODEL_PARAMS) + ")");
    const uint64_t want = sizeof(kMagic) + sizeof(FileHeader) + payloadBytes(h) + 4;
    if (bytes.size() != want)
        return failWith(GSR_ERROR_FORMAT, name + ": " + std::to_string(bytes.size()) + " bytes, the header declares " +
                                              std::to_string(want));
    uint32_t stored;
    std::memcpy(&stored, bytes.data() + bytes.size() - 4, 4);
    if (crc32(bytes.data(), bytes.size() - 4) != stored) return failWith(GSR_ERROR_FORMAT, name + ": checksum mismatch");
    ck->count = h.count;
    ck->sh_degree = h.shDegree;
    ck->step = h.step;
    ck->loss_count = h.lossCount;
    ck->options = h.options;
    ck->stats = h.stats;
    const uint8_t* at = bytes.data() + sizeof(kMagic) + sizeof(h);
    auto get = [&](void* dst, size_t n) {
        if (dst && n) std::memcpy(dst, at, n);
        at += n;
    };
    get(ck->params, size_t(h.params) * 4);
    get(ck->adam_m, size_t(h.params) * 4);
    get(ck->adam_v, size_t(h.params) * 4);
    get(ck->loss, size_t(h.lossCount) * 4);
    get(ck->latents, size_t(h.count) * 16);
    return GSR_OK;
}

}  // extern "C"
