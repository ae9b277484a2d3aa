// C ABI of the host-side scene input (PLY loader, PLY stream decoder, PLY header parser, training
// cameras): exceptions become GsrStatus codes with the message in gsr_last_error_message().
#include <algorithm>
#include <cstring>
#include <new>

#include "gsr_b200.h"
#include "scene_io.h"

namespace gsr {
void setLastError(const std::string& message);  // renderer.cpp
}

struct GsrLoadedScene {
    gsr::io::HostScene own;
    const gsr::io::HostScene* view = nullptr;  // a stream's header info or batch (not owned)
    const gsr::io::HostScene& scene() const { return view ? *view : own; }
};

struct GsrPlyHeader {
    gsr::io::PlyHeader header;
};

struct GsrPlyStream {
    std::unique_ptr<gsr::io::PlyStream> stream;
    GsrLoadedScene infoView, batchView;
};

namespace {

template <typename Fn>
int guarded(Fn&& fn) {
    try {
        return fn();
    } catch (const gsr::io::FormatError& e) {
        gsr::setLastError(e.what());
        return GSR_ERROR_FORMAT;
    } catch (const std::bad_alloc&) {
        gsr::setLastError("out of host memory");
        return GSR_ERROR_OUT_OF_MEMORY;
    } catch (const std::logic_error& e) {
        gsr::setLastError(e.what());
        return GSR_ERROR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        gsr::setLastError(e.what());
        return GSR_ERROR_IO;
    }
}

int nullArgument(const char* what) {
    gsr::setLastError(std::string("null argument: ") + what);
    return GSR_ERROR_INVALID_ARGUMENT;
}

void fillStats(const gsr::io::SceneStats& s, GsrSceneStats& o) {
    for (int c = 0; c < 3; ++c) {
        o.bbox_min[c] = s.bboxMin[c];
        o.bbox_max[c] = s.bboxMax[c];
        o.robust_min[c] = s.robustMin[c];
        o.robust_max[c] = s.robustMax[c];
    }
    o.alpha_min = s.alphaMin;
    o.alpha_max = s.alphaMax;
    o.alpha_mean = s.alphaMean;
    o.alpha_below_visible = s.alphaBelowVisible;
    o.sigma_min = s.sigmaMin;
    o.sigma_max = s.sigmaMax;
    o.sigma_max_median = s.sigmaMaxMedian;
    o.quat_norm_min = s.quatNormMin;
    o.quat_norm_max = s.quatNormMax;
    o.zero_quaternions = s.zeroQuaternions;
    o.non_finite_values = s.nonFiniteValues;
}

const float* dataOrNull(const std::vector<float>& v) { return v.empty() ? nullptr : v.data(); }

void toC(const gsr::io::TrainingCamera& c, GsrTrainingCamera& o) {
    std::memset(&o, 0, sizeof(o));
    o.id = c.id;
    o.width = c.width;
    o.height = c.height;
    std::memcpy(o.position, c.position, sizeof(o.position));
    std::memcpy(o.camera_to_world, c.cameraToWorld, sizeof(o.camera_to_world));
    o.fx = c.fx;
    o.fy = c.fy;
    const size_t n = std::min(c.imageName.size(), size_t(GSR_IMAGE_NAME_CAPACITY - 1));
    std::memcpy(o.image_name, c.imageName.data(), n);
}

gsr::io::TrainingCamera fromC(const GsrTrainingCamera& c) {
    gsr::io::TrainingCamera o;
    o.id = c.id;
    o.width = c.width;
    o.height = c.height;
    std::memcpy(o.position, c.position, sizeof(o.position));
    std::memcpy(o.cameraToWorld, c.camera_to_world, sizeof(o.cameraToWorld));
    o.fx = c.fx;
    o.fy = c.fy;
    return o;
}

}  // namespace

extern "C" {

int gsr_ply_load(const char* path, GsrLoadedScene** out) {
    if (!path || !out) return nullArgument("path/out");
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<GsrLoadedScene>();
        s->own = gsr::io::loadPly(std::string(path));
        *out = s.release();
        return int(GSR_OK);
    });
}

int gsr_ply_load_memory(const void* bytes, size_t size, const char* name, GsrLoadedScene** out) {
    if ((!bytes && size) || !name || !out) return nullArgument("bytes/name/out");
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<GsrLoadedScene>();
        s->own = gsr::io::loadPly(static_cast<const uint8_t*>(bytes), size, std::string(name));
        *out = s.release();
        return int(GSR_OK);
    });
}

int gsr_loaded_scene_info(const GsrLoadedScene* scene, GsrLoadedSceneInfo* info) {
    if (!scene || !info) return nullArgument("scene/info");
    const gsr::io::HostScene& s = scene->scene();
    std::memset(info, 0, sizeof(*info));
    info->count = s.count;
    info->sh_degree = s.shDegree;
    info->comment_count = uint32_t(s.comments.size());
    info->warning_count = uint32_t(s.warnings.size());
    fillStats(s.stats, info->stats);
    info->timings.map_ms = s.timings.mapMs;
    info->timings.header_ms = s.timings.headerMs;
    info->timings.decode_ms = s.timings.decodeMs;
    info->timings.stats_ms = s.timings.statsMs;
    info->timings.total_ms = s.timings.totalMs;
    return GSR_OK;
}

int gsr_loaded_scene_arrays(const GsrLoadedScene* scene, GsrLoadedSceneArrays* a) {
    if (!scene || !a) return nullArgument("scene/arrays");
    const gsr::io::HostScene& s = scene->scene();
    a->pos_alpha = dataOrNull(s.posAlpha);
    a->scales = dataOrNull(s.scales);
    a->rotations = dataOrNull(s.rotations);
    a->sh = dataOrNull(s.sh);
    a->raw_opacity = dataOrNull(s.rawOpacity);
    a->raw_log_scale = dataOrNull(s.rawLogScale);
    a->raw_rotation = dataOrNull(s.rawRotation);
    return GSR_OK;
}

int gsr_loaded_scene_host(const GsrLoadedScene* scene, GsrHostScene* host) {
    if (!scene || !host) return nullArgument("scene/host");
    const gsr::io::HostScene& s = scene->scene();
    host->count = s.count;
    host->sh_degree = s.shDegree;
    host->pos_alpha = dataOrNull(s.posAlpha);
    host->scales = dataOrNull(s.scales);
    host->rotations = dataOrNull(s.rotations);
    host->sh = dataOrNull(s.sh);
    return GSR_OK;
}

const char* gsr_loaded_scene_comment(const GsrLoadedScene* scene, uint32_t index) {
    if (!scene || index >= scene->scene().comments.size()) return nullptr;
    return scene->scene().comments[index].c_str();
}

const char* gsr_loaded_scene_warning(const GsrLoadedScene* scene, uint32_t index) {
    if (!scene || index >= scene->scene().warnings.size()) return nullptr;
    return scene->scene().warnings[index].c_str();
}

const char* gsr_loaded_scene_source(const GsrLoadedScene* scene) {
    return scene ? scene->scene().sourcePath.c_str() : nullptr;
}

void gsr_loaded_scene_destroy(GsrLoadedScene* scene) { delete scene; }

int gsr_ply_sh_degree_from_rest_count(uint64_t rest_count) { return gsr::io::shDegreeForRestCount(size_t(rest_count)); }

int gsr_ply_parse_header(const void* bytes, size_t size, int final_bytes, GsrPlyHeader** out) {
    if ((!bytes && size) || !out) return nullArgument("bytes/out");
    *out = nullptr;
    return guarded([&] {
        auto h = gsr::io::parsePlyHeader(std::string_view(static_cast<const char*>(bytes), size), final_bytes != 0);
        if (!h) {
            gsr::setLastError("the header is not complete yet");
            return int(GSR_ERROR_NOT_READY);
        }
        *out = new GsrPlyHeader{std::move(*h)};
        return int(GSR_OK);
    });
}

int gsr_ply_header_info(const GsrPlyHeader* h, uint32_t* format, uint32_t* element_count, uint32_t* comment_count,
                        uint64_t* header_bytes) {
    if (!h) return nullArgument("header");
    if (format) *format = uint32_t(h->header.format);
    if (element_count) *element_count = uint32_t(h->header.elements.size());
    if (comment_count) *comment_count = uint32_t(h->header.comments.size());
    if (header_bytes) *header_bytes = h->header.headerBytes;
    return GSR_OK;
}

int gsr_ply_header_element(const GsrPlyHeader* h, uint32_t index, GsrPlyElementInfo* info) {
    if (!h || !info) return nullArgument("header/info");
    if (index >= h->header.elements.size()) {
        gsr::setLastError("element index out of range");
        return GSR_ERROR_INVALID_ARGUMENT;
    }
    const gsr::io::PlyElement& e = h->header.elements[index];
    info->name = e.name.c_str();
    info->count = e.count;
    info->stride = e.stride;
    info->has_list = e.hasList ? 1u : 0u;
    info->property_count = uint32_t(e.properties.size());
    return GSR_OK;
}

int gsr_ply_header_property(const GsrPlyHeader* h, uint32_t element, uint32_t property, GsrPlyPropertyInfo* info) {
    if (!h || !info) return nullArgument("header/info");
    if (element >= h->header.elements.size() || property >= h->header.elements[element].properties.size()) {
        gsr::setLastError("element or property index out of range");
        return GSR_ERROR_INVALID_ARGUMENT;
    }
    const gsr::io::PlyProperty& p = h->header.elements[element].properties[property];
    info->name = p.name.c_str();
    info->type = uint32_t(p.type);
    info->is_list = p.list ? 1u : 0u;
    info->offset = p.offset;
    return GSR_OK;
}

const char* gsr_ply_header_comment(const GsrPlyHeader* h, uint32_t index) {
    if (!h || index >= h->header.comments.size()) return nullptr;
    return h->header.comments[index].c_str();
}

void gsr_ply_header_destroy(GsrPlyHeader* h) { delete h; }

int gsr_ply_stream_create(const char* name, uint64_t total_bytes, GsrPlyHeaderCallback on_header,
                          GsrPlyBatchCallback on_batch, void* user, uint32_t batch_capacity, GsrPlyStream** out) {
    if (!name || !out) return nullArgument("name/out");
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<GsrPlyStream>();
        GsrPlyStream* raw = s.get();
        auto headerFn = [raw, on_header, user](const gsr::io::HostScene& info) {
            raw->infoView.view = &info;
            if (on_header) on_header(user, &raw->infoView);
        };
        auto batchFn = [raw, on_batch, user](uint32_t first, const gsr::io::HostScene& batch) {
            raw->batchView.view = &batch;
            if (on_batch) on_batch(user, first, &raw->batchView);
        };
        s->stream = std::make_unique<gsr::io::PlyStream>(std::string(name), total_bytes, headerFn, batchFn,
                                                         batch_capacity ? batch_capacity : 16384u);
        s->infoView.view = &s->stream->info();
        *out = s.release();
        return int(GSR_OK);
    });
}

int gsr_ply_stream_push(GsrPlyStream* s, const void* bytes, size_t size) {
    if (!s || (!bytes && size)) return nullArgument("stream/bytes");
    return guarded([&] {
        s->stream->push(static_cast<const uint8_t*>(bytes), size);
        return int(GSR_OK);
    });
}

int gsr_ply_stream_finish(GsrPlyStream* s) {
    if (!s) return nullArgument("stream");
    return guarded([&] {
        s->stream->finish();
        return int(GSR_OK);
    });
}

int gsr_ply_stream_state(const GsrPlyStream* s, uint32_t* header_parsed, uint32_t* finished, uint64_t* bytes_received,
                         uint64_t* records_decoded) {
    if (!s) return nullArgument("stream");
    if (header_parsed) *header_parsed = s->stream->headerParsed() ? 1u : 0u;
    if (finished) *finished = s->stream->finished() ? 1u : 0u;
    if (bytes_received) *bytes_received = s->stream->bytesReceived();
    if (records_decoded) *records_decoded = s->stream->recordsDecoded();
    return GSR_OK;
}

const GsrLoadedScene* gsr_ply_stream_info(const GsrPlyStream* s) {
    if (!s) return nullptr;
    return &s->infoView;
}

void gsr_ply_stream_destroy(GsrPlyStream* s) { delete s; }

int gsr_training_cameras_load(const char* path, GsrTrainingCamera* cameras, uint32_t capacity, uint32_t* count) {
    if (!path || !count || (!cameras && capacity)) return nullArgument("path/cameras/count");
    return guarded([&] {
        const std::vector<gsr::io::TrainingCamera> cams = gsr::io::loadTrainingCameras(std::string(path));
        *count = uint32_t(cams.size());
        for (uint32_t k = 0; k < capacity && k < cams.size(); ++k) toC(cams[k], cameras[k]);
        return int(GSR_OK);
    });
}

float gsr_training_camera_fov_y_deg(const GsrTrainingCamera* camera) {
    return camera ? gsr::io::fovYDeg(fromC(*camera)) : 0.0f;
}

int gsr_training_cameras_mean_up(const GsrTrainingCamera* cameras, uint32_t count, float up[3]) {
    if ((!cameras && count) || !up) return nullArgument("cameras/up");
    std::vector<gsr::io::TrainingCamera> c;
    for (uint32_t k = 0; k < count; ++k) c.push_back(fromC(cameras[k]));
    gsr::io::meanCameraUp(c.data(), c.size(), up);
    return GSR_OK;
}

int gsr_training_cameras_focus_point(const GsrTrainingCamera* cameras, uint32_t count, float point[3]) {
    if ((!cameras && count) || !point) return nullArgument("cameras/point");
    std::vector<gsr::io::TrainingCamera> c;
    for (uint32_t k = 0; k < count; ++k) c.push_back(fromC(cameras[k]));
    gsr::io::cameraFocusPoint(c.data(), c.size(), point);
    return GSR_OK;
}

}  // extern "C"
