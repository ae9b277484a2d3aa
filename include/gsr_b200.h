/* gsr_b200.h - C ABI of the B200 (sm_100a) splat-tiles frame path.
 *
 * A drop-in for the reference renderer's `splat-tiles` path (gsr::SplatTileRenderer,
 * src/render/splat_tile_renderer.h:143-290, behind gsr::Renderer, src/render/renderer.h:59-72),
 * with the scene buffers of gsr::GpuScene (src/render/gpu_scene.h:42-78) and the camera of
 * gsr::FrameInput (src/render/renderer.h:28-52). Plain C types only: device memory is passed
 * as pointers, CUDA streams as opaque handles (cudaStream_t), sizes as integers.
 *
 * Errors are returned as GsrStatus codes (never exceptions); gsr_error_string() names them and
 * gsr_last_error_message() gives the detail of the calling thread's last failure. One
 * renderer handle is used from one host thread at a time; work is stream-ordered on the
 * stream passed to gsr_render(). The scene memory stays owned by the caller (or by a
 * GsrScene handle); every other buffer is owned by the renderer.
 */
#ifndef GSR_B200_H
#define GSR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSR_ABI_VERSION 2

typedef enum GsrStatus {
    GSR_OK = 0,
    GSR_ERROR_INVALID_ARGUMENT = 1, /* std::runtime_error for invalid settings (splat_tile_renderer.cpp:139-152) */
    GSR_ERROR_UNSUPPORTED = 2,      /* a format/option this build does not implement */
    GSR_ERROR_CUDA = 3,             /* a CUDA runtime call failed (VK_CHECK in the reference) */
    GSR_ERROR_OUT_OF_MEMORY = 4,
    GSR_ERROR_DEVICE_TIMEOUT = 5,   /* a bounded device-side wait gave up (GsrControl.status) */
    GSR_ERROR_NOT_READY = 6,        /* nothing to report yet (e.g. no completed frame) */
    GSR_ERROR_FORMAT = 7,           /* a malformed input file (PlyError, src/scene/ply_loader.h:29-32) */
    GSR_ERROR_IO = 8                /* a file could not be opened or read (std::runtime_error) */
} GsrStatus;

/* ---- scene (gsr::GpuScene, src/render/gpu_scene.h:42-78) ------------------------------ */
typedef enum GsrSceneFormat { GSR_FORMAT_F32 = 0, GSR_FORMAT_F16 = 1, GSR_FORMAT_Q8 = 2, GSR_FORMAT_CB = 3 } GsrSceneFormat;
typedef enum GsrSceneLayout { GSR_LAYOUT_SOA = 0, GSR_LAYOUT_SPLIT = 1, GSR_LAYOUT_AOS = 2 } GsrSceneLayout;
/* GeometryEncoding / ColorEncoding / VariableSh (src/scene/scene_compression.h:73-89). */
typedef enum GsrGeometryEncoding { GSR_GEOMETRY_SOA_F32 = 0, GSR_GEOMETRY_RECORD_F32 = 1, GSR_GEOMETRY_RECORD_F16 = 2 } GsrGeometryEncoding;
typedef enum GsrColorEncoding {
    GSR_COLOR_SOA_F32 = 0, GSR_COLOR_RECORD_F32 = 1, GSR_COLOR_RECORD_F16 = 2, GSR_COLOR_Q8 = 3, GSR_COLOR_CODEBOOK = 4
} GsrColorEncoding;
typedef enum GsrVariableSh { GSR_VARIABLE_SH_OFF = 0, GSR_VARIABLE_SH_DEGREE_ONLY = 1, GSR_VARIABLE_SH_COMPACT = 2 } GsrVariableSh;

/* The scene as the preprocess reads it: the 4 storage buffers of GpuScene's binding table
 * (gpu_scene.h:4-17) as DEVICE pointers, plus the format fields that the reference passes as
 * specialization constants 0-7 (shaders/scene_decode.glsl:31-40). Strides/offsets are in
 * 16-byte units, as there.
 *   soa   : buffers = posAlpha float4[N], scales float4[N], rotations float4[N], sh float[N*K*3]
 *   split : buffers = geometry records, colour records, -, -
 *   aos   : buffers = records, (same), -, - */
typedef struct GsrSceneDesc {
    uint32_t count;            /* N */
    int32_t sh_degree;         /* stored degree (0..3) */
    uint32_t sh_coeffs;        /* stored K = (sh_degree + 1)^2 */
    uint32_t format;           /* GsrSceneFormat (informational) */
    uint32_t layout;           /* GsrSceneLayout */
    uint32_t geometry;         /* GsrGeometryEncoding */
    uint32_t color;            /* GsrColorEncoding */
    uint32_t geometry_stride;  /* uvec4 per geometry record (0 for soa) */
    uint32_t color_stride;     /* uvec4 per colour record */
    uint32_t color_offset;     /* uvec4 offset of the colour record (aos) */
    uint32_t codebook_stride;  /* uvec4 per codebook entry (cb) */
    uint32_t variable_sh;      /* GsrVariableSh */
    const void* buffers[4];    /* device pointers, 16-byte aligned */
    uint64_t buffer_bytes[4];
} GsrSceneDesc;

/* Host-side activated scene (gsr::GaussianScene's GPU arrays, src/scene/gaussian_scene.h:71-102). */
typedef struct GsrHostScene {
    uint32_t count;
    int32_t sh_degree;
    const float* pos_alpha;  /* float4[N] */
    const float* scales;     /* float4[N] */
    const float* rotations;  /* float4[N] (w, x, y, z) */
    const float* sh;         /* float[N * K * 3] */
} GsrHostScene;

/* gsr::CompressionOptions (src/scene/scene_compression.h:76-86). The codebook fields configure
 * the cb format's k-means; 0 selects the reference's default (4096 entries, 10 iterations). */
typedef struct GsrCompression {
    uint32_t format;              /* GsrSceneFormat (f32, f16, q8, cb) */
    uint32_t layout;              /* GsrSceneLayout (soa only with f32) */
    int32_t max_sh_degree;        /* drop stored bands above this */
    float sh_threshold;           /* per-gaussian SH degree threshold in 1/255 (< 0: off) */
    uint32_t codebook_size;       /* cb: codebook entries (1..65536; 0 = 4096) */
    uint32_t codebook_iterations; /* cb: Lloyd iterations on the training sample (0 = 10) */
    uint32_t codebook_samples;    /* cb: training sample size (0 = min(N, 32 x entries)) */
    uint32_t reserved;
} GsrCompression;
/* The reference's defaults: f32, soa, degree 3, threshold off, 4096 entries, 10 iterations. */
void gsr_compression_default(GsrCompression* options);

/* CodebookStats (scene_compression.h:91-101) of a cb scene's k-means (entries 0 for other formats).
 * The assignment passes run on the GPU; the update and the statistics on the host. */
typedef struct GsrCodebookStats {
    uint32_t entries;        /* codebook size used (<= requested, <= N) */
    uint32_t dimensions;     /* (K - 1) * 3 */
    uint32_t samples;        /* training sample size */
    uint32_t iterations;     /* Lloyd iterations run */
    uint32_t empty_reseeded; /* empty clusters re-seeded over all iterations */
    uint32_t pad;
    double train_ms, assign_ms, total_ms;
    double sample_mse, full_mse; /* mean squared error per coefficient (sample, all gaussians) */
} GsrCodebookStats;

typedef struct GsrScene GsrScene;

/* GpuScene::upload (src/render/gpu_scene.cpp): encodes on the GPU (encodeScene,
 * src/scene/scene_compression.cpp:150-380, f32/f16/q8 in soa/split/aos, variable SH degree)
 * and keeps the encoded buffers in device memory owned by the handle. */
int gsr_scene_create(const GsrHostScene* host, const GsrCompression* options, GsrScene** out);
/* The cb format (encodeScene's codebook path, scene_compression.cpp:250-273, 309-314, 340-377):
 * fp16 geometry records, an 8-byte colour record (h(dc.r, dc.g), h(dc.b) | index << 16; two per
 * 16 bytes in the split layout) and the codebook of SH-rest vectors (fp32, entries padded to 16
 * bytes) from the reference's k-means (kmeans.cpp): the same sample, initial centroids, Lloyd
 * updates, re-seeding and final assignment, with the nearest-centroid searches computed on the
 * GPU in the reference's own arithmetic (the AVX2 kernel's fused multiply-adds), so the codebook
 * and the indices equal the reference's on a host with AVX2 and FMA. */
int gsr_scene_codebook_stats(const GsrScene* scene, GsrCodebookStats* out);
/* The descriptor of a GsrScene, to pass to gsr_renderer_create. */
int gsr_scene_get_desc(const GsrScene* scene, GsrSceneDesc* out);
/* Copies encoded buffer b (0..3) to host memory (tests): bytes = buffer_bytes[b]. */
int gsr_scene_read_buffer(const GsrScene* scene, uint32_t b, void* host, uint64_t bytes);
void gsr_scene_destroy(GsrScene* scene);

/* ---- settings (SplatSettings src/render/splat_draw.h:31-37 + TileSettings
 *      src/render/splat_tile_renderer.h:96-114) ------------------------------------------ */
typedef enum GsrTileBounds { GSR_BOUNDS_RECT = 0, GSR_BOUNDS_TIGHT = 1, GSR_BOUNDS_CUTOFF_ONLY = 2 } GsrTileBounds;
/* The rasterizer's output image (C, 1 - T) per pixel: the render target of SplatTargetFormat
 * (splat_draw.h:26; the reference's default is rgba16f), optionally with the 8-bit RGB image
 * lround(clamp(C, 0, 1) * 255) that the reference's PNG writer makes (image_io.cpp:55-56).
 * RGBA16F stores each channel as fp16 rounded to nearest even; RGBA8 as lround(clamp(v, 0, 1) * 255). */
typedef enum GsrOutputFormat {
    GSR_OUTPUT_RGBA32F = 0,          /* float4 per pixel */
    GSR_OUTPUT_RGBA32F_AND_RGB8 = 1, /* float4 + uint8 x 3 */
    GSR_OUTPUT_RGBA16F = 2,          /* half4 per pixel */
    GSR_OUTPUT_RGBA16F_AND_RGB8 = 3, /* half4 + uint8 x 3 */
    GSR_OUTPUT_RGBA8 = 4             /* uint8 x 4 per pixel */
} GsrOutputFormat;

typedef struct GsrSettings {
    uint32_t bounds;                   /* GsrTileBounds; reference default tight (cli.h) */
    uint32_t tile_size;                /* the binning and render tiles: 16 (INRIA's 16 x 16, the
                                          reference's default), 8 (8 x 8) or 32 (32 x 8, as many
                                          pixels as 16 x 16 in a wider, lower tile) */
    uint32_t budget_mb;                /* list memory incl. sort scratch; default 256 */
    uint32_t adaptive_list;            /* 1: capacity follows the measured entry count */
    uint32_t adaptive_initial_entries; /* 0: max(4 N, 1 M) */
    int32_t max_sh_degree;             /* bands evaluated (<= stored) */
    uint32_t output_format;            /* GsrOutputFormat */
    uint32_t frames_in_flight;         /* control readback slots (default 2) */
    uint32_t use_graph;                /* 1: launch each frame as a captured CUDA graph */
    uint32_t raster_schedule;          /* GsrRasterSchedule (no reference counterpart) */
    uint32_t list_mode;                /* GsrListMode (TileSettings' sort mode, cli.h:28) */
    uint32_t render_splat;             /* GsrRenderSplat (TileSettings::renderSplat, cli.h:34) */
    uint32_t sort_window;              /* StopThePop per-pixel window K (TileSettings::sortWindow, cli.h:46):
                                          0 = off (the list's order), 1..64 */
    uint32_t sort_digit_bits;          /* radix digit width of the depth and list sorts: 7, 8 or 9 bits
                                          a pass; 0 = 8 (the reference's GpuRadixSort digits,
                                          gpu_radix_sort.h:38-122). The depth keys are the depth
                                          offsets from the frame's nearest record (24 bits on a
                                          1080p orbit: 3 passes of 8 bits); 9 bits sort keys of
                                          25-27 bits in 3 passes where 8 bits need 4 */
    uint32_t tile_stats;               /* 1: the instrumented rasterizer with per-tile statistics
                                          (TileSettings::stats, splat_tile_renderer.h:102); not with
                                          sort_window; read with gsr_read_tile_stats */
    uint32_t raster_gather;            /* GsrRasterGather: how the rasterizer stages each batch of records */
    uint32_t color_decode;             /* GsrColorDecode: where the learned colour's decoder runs */
} GsrSettings;

/* Where the learned colour stage decodes (latent, view direction) -> RGB (no reference
 * counterpart). The images agree to the last bits of FP32 (the bias is added after the
 * products in the tcgen05 pre-pass, into the accumulator before them in the fused decode). */
typedef enum GsrColorDecode {
    GSR_DECODE_DEFAULT = 0, /* the build's default (GSR_DECODE_FUSED) */
    GSR_DECODE_FUSED = 1,   /* inside the preprocess: each warp decodes its 32 gaussians with chained
                               mma.sync.m16n8k16 BF16 products in registers */
    GSR_DECODE_TCGEN05 = 2  /* a pre-pass kernel on the fifth-generation tensor cores: tcgen05.mma over
                               128-gaussian tiles with FP32 accumulators in tensor memory; the colours
                               (16 B per view and gaussian) are read by the preprocess */
} GsrColorDecode;

/* How the rasterizer brings a batch of records into shared memory (no reference counterpart; the
 * reference's workgroup fetches them cooperatively, tile_render.comp:281-400). The images are
 * the same either way. */
typedef enum GsrRasterGather {
    GSR_GATHER_DEFAULT = 0, /* the build's default (GSR_GATHER_CP_ASYNC) */
    GSR_GATHER_CP_ASYNC = 1, /* every thread copies its record with 16-byte cp.async */
    GSR_GATHER_TMA = 2       /* one warp gathers four records per TMA instruction (cp.async.bulk.tensor
                                tile::gather4 over a 2-D tensor map of the record array), completed on
                                an mbarrier; full records, no sort window, no tile statistics, and
                                fewer than 2^31 records (else the cp.async gather runs) */
} GsrRasterGather;

/* The per-entry record that key emission and the rasterizer read (RenderSplatMode,
 * splat_tile_renderer.h:87-92; layouts of shaders/render_splat.glsl). Packed records keep the
 * tile rectangle (2 x u32: minX | minY << 16, maxX | maxY << 16) and the depth bits in arrays of
 * their own. Colour is fp16 in both packed forms; P24 also stores the conic (x 2^12) and the
 * opacity in fp16 and counts the covered tiles with those decoded values, so the list can
 * differ from FULL where a splat's cutoff ellipse changes under the rounding. */
typedef enum GsrRenderSplat {
    GSR_RENDER_SPLAT_FULL = 0, /* the 48-byte ProjectedSplat */
    GSR_RENDER_SPLAT_P32 = 1,  /* 32 bytes: cx, cy, a, b | c, opacity, h(r, g), h(b) | radius << 16 */
    GSR_RENDER_SPLAT_P24 = 2   /* 24 bytes: cx, cy | h(a S, b S), h(c S, opacity) | h(r, g), h(b) | radius << 16, S = 2^12 */
} GsrRenderSplat;

/* How the (tile, depth) list is built and sorted; both give the same list, entry for entry,
 * when it fits the capacity (test_tile_raster.cpp:459-464). */
typedef enum GsrListMode {
    GSR_LIST_BINNING = 0,  /* the default (TileSortMode::Binning, splat_tile_renderer.h:76): visible
                              splats sorted by depth, emission in that order, a stable sort by tile
                              alone; a list over the capacity is truncated in depth order */
    GSR_LIST_GLOBAL = 1    /* INRIA's scheme (TileSortMode::Global): emission in index order, one sort
                              of (tile, depth) keys; a list over the capacity is truncated in index order */
} GsrListMode;

/* How the rasterizer's blocks are given the frame's tiles. */
typedef enum GsrRasterSchedule {
    GSR_RASTER_AUTO = 0,       /* one block per tile for one view, the work queue for several */
    GSR_RASTER_PER_TILE = 1,   /* one block per tile (the reference's dispatch of T workgroups) */
    GSR_RASTER_PERSISTENT = 2  /* a fixed grid of blocks takes (view, tile) items from a queue */
} GsrRasterSchedule;

/* Reference defaults for this path (cli.h:28-50): tight bounds, 16-px tiles, 256 MB, adaptive. */
void gsr_settings_default(GsrSettings* s);

/* ---- camera (FrameInput view/proj/model, renderer.h:28-52) ------------------------------ */
typedef struct GsrCamera {
    float view[16];   /* world -> eye, column-major, -z forward, +y up */
    float proj[16];   /* Vulkan perspective (y flipped); only proj[0][0], proj[1][1] are used */
    float model[16];  /* data -> world */
    uint32_t width, height;
} GsrCamera;

/* gsr::SplatCamera (src/splat/splat_math.h:43-50) as splatCameraFromViewer computes it. */
typedef struct GsrSplatCamera {
    float view_inria[16];
    float position[3];
    uint32_t width, height;
    float tan_half_fov_x, tan_half_fov_y, focal_x, focal_y;
    uint32_t tiles_x, tiles_y;
} GsrSplatCamera;

/* splatCameraFromViewer (src/splat/splat_math.cpp:29-42). */
int gsr_splat_camera_from_viewer(const GsrCamera* camera, GsrSplatCamera* out);
/* glm::lookAt (RH) and glm::perspective (RH, depth 0..1) with the Vulkan y flip, as the
 * reference's viewer camera builds them (src/app/camera.cpp:41-45). Column-major outputs. */
void gsr_look_at(const float eye[3], const float center[3], const float up[3], float view[16]);
void gsr_perspective_vk(float fovy_radians, float aspect, float z_near, float z_far, float proj[16]);

/* ---- the control block (TileControl, splat_tile_renderer.h:117-128 + extensions) -------- */
typedef enum GsrControlStatus {
    GSR_CONTROL_OK = 0,
    GSR_CONTROL_TIMEOUT = 1,         /* a bounded device-side wait hit its iteration limit (a look-back,
                                        or a preprocess block's wait for its staged SH, which can leave
                                        that bulk copy writing shared memory after the block ended):
                                        the frame's records, list and image are untrusted, and
                                        gsr_read_control reports GSR_ERROR_DEVICE_TIMEOUT */
    GSR_CONTROL_BOUNDS = 2,          /* an index check failed; the access was skipped */
    GSR_CONTROL_KEY_RANGE = 4        /* the sort key did not fit the planned bits */
} GsrControlStatus;

typedef struct GsrControl {
    /* the reference's 80-byte TileControl, same order */
    uint32_t gaussian_count;         /* N */
    uint32_t visible;                /* V (visible splats; = cull_counts[0]) */
    uint32_t duplicates;             /* M, unclamped */
    uint32_t entries;                /* min(M, capacity) */
    uint32_t cull_counts[8];         /* per CullReason: visible, near, singular, off-screen, low opacity */
    uint32_t overflow;               /* M - entries */
    uint32_t ranges_groups[3];       /* ceil(entries / 256), 1, 1 */
    uint32_t coverage_mismatch;      /* splats whose written tiles != their count (always 0) */
    uint32_t pad[3];
    /* extensions of this build */
    uint32_t status;                 /* GsrControlStatus bits */
    uint32_t timeout_where;          /* id of the wait that gave up */
    uint32_t epoch;                  /* frame counter of the device-side look-back flags */
    uint32_t sort_passes;            /* radix passes that moved data */
    uint32_t key_bits;               /* significant bits of the (tile | depth) key */
    uint32_t depth_low_bits;         /* depth bits that vary across the frame's keys */
    uint32_t depth_min_bits, depth_max_bits;
    uint32_t tile_max;               /* largest tile id emitted */
    uint32_t sorted_buffer;          /* which list buffer holds the sorted result */
    uint32_t capacity;               /* list capacity of this frame */
    uint32_t packed_entries;         /* 1: entries were single 64-bit words (tile|depth|index) */
    uint32_t index_bits;             /* bits of the gaussian index in a packed entry */
    uint32_t ext_pad[3];
} GsrControl;

/* ---- the renderer (SplatTileRenderer) ---------------------------------------------------- */
typedef struct GsrRenderer GsrRenderer;

/* SplatTileRenderer::init (splat_tile_renderer.cpp:127-...): validates the settings and the
 * scene format, allocates the per-gaussian buffers and the list. The scene memory must stay
 * valid until gsr_renderer_destroy. */
int gsr_renderer_create(const GsrSceneDesc* scene, const GsrSettings* settings, GsrRenderer** out);
/* onRenderTargetsChanged (splat_tile_renderer.cpp:537-...): (re)creates the per-tile and
 * image buffers for a width x height target. gsr_render calls it on a size change. */
int gsr_renderer_resize(GsrRenderer* r, uint32_t width, uint32_t height);
/* render (splat_tile_renderer.cpp:624-833): the whole frame, enqueued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream). The image stays in renderer-owned device
 * memory (gsr_renderer_image); nothing is synchronized. */
int gsr_render(GsrRenderer* r, const GsrCamera* camera, void* stream);
/* The same frame from a precomputed SplatCamera (tests that share one camera with the oracle). */
int gsr_render_splat_camera(GsrRenderer* r, const GsrSplatCamera* camera, void* stream);
/* Device pointers of the last frame's outputs: rgba = the output image (C, 1 - T) in the settings'
 * format (float4, half4 or uint8 x 4 per pixel), rgb8 = uint8[W*H*3] (lround(clamp(C, 0, 1) *
 * 255), NULL unless an _AND_RGB8 format). */
int gsr_renderer_image(GsrRenderer* r, const void** rgba, const void** rgb8, uint32_t* width, uint32_t* height);
/* The end-to-end call for host callers: render and copy the RGB8 image (or the output image in
 * its format when rgb8 output is off) into `host` (pinned or pageable; `bytes` must match), then
 * synchronize `stream`. */
int gsr_render_to_host(GsrRenderer* r, const GsrCamera* camera, void* host, uint64_t bytes, void* stream);

/* ---- batched views (no reference counterpart: the reference renders one camera per frame) ---
 * One frame renders `views` cameras of any sizes together: every per-gaussian kernel runs over
 * (view, gaussian), the list keys carry the frame tile = the view's tile base + the tile in the
 * view (the view in the key's high bits), ONE sort orders every view's entries, and the
 * rasterizer walks (view, tile) items (GsrSettings.raster_schedule). Each view's image, list
 * and ranges equal those of the same camera rendered alone, bit for bit. The control block
 * sums over the views (gaussian_count = views * N). gsr_render is the one-view case; the
 * single-view accessors (gsr_renderer_image, gsr_read_image) address view 0, and
 * gsr_read_list returns frame tile ids and the ranges of every frame tile. */
#define GSR_MAX_VIEWS 4096u
typedef struct GsrViewLayout {
    uint32_t width, height, tiles_x, tiles_y;
    uint32_t tile_base;    /* first frame tile of the view */
    uint32_t pad;
    uint64_t pixel_base;   /* first pixel of the view in the frame's image buffers */
} GsrViewLayout;
/* Renders cameras[0..views) (each with its own width/height) as one frame; a new set of sizes
 * re-creates the per-tile and image buffers (synchronizing, like gsr_renderer_resize). */
int gsr_render_views(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* stream);
/* The layout of the current frame's view `view`, and the number of views. */
int gsr_renderer_view_layout(GsrRenderer* r, uint32_t view, GsrViewLayout* out, uint32_t* views);
/* Device pointers of view `view`'s outputs (rgba float4[W*H], rgb8 uint8[W*H*3] or NULL). */
int gsr_renderer_view_image(GsrRenderer* r, uint32_t view, const void** rgba, const void** rgb8);
/* ---- the learned colour stage (no reference counterpart) ----------------------------------
 * Each gaussian's SH coefficients (48 floats) are encoded to an 8-dim fp16 latent (16 bytes) and
 * one small MLP decodes (latent, view direction) to RGB inside the preprocess, on the tensor
 * cores (BF16 operands, FP32 accumulation): encoder 48 -> 64 -> 8, decoder (8 + 3) -> 32 -> 32 ->
 * 3 with a sigmoid output. Training runs on the device with hand-written forward, backward and
 * Adam kernels on (gaussian, direction) pairs whose targets are the plain SH colours. A
 * gaussian whose decoded colour is more than `gate` (max over channels and its training
 * directions) from its SH colour falls back to the SH evaluation, which stays the judge. */
typedef struct GsrColorModel GsrColorModel;
typedef struct GsrColorModelOptions {
    uint32_t directions;   /* view directions per gaussian (uniform on the sphere); default 64 */
    uint32_t batch;        /* (gaussian, direction) pairs per step, a multiple of 256; default 65536 */
    uint32_t steps;        /* Adam steps; default 2000 */
    float learning_rate;   /* default 1e-3 (beta1 0.9, beta2 0.999, eps 1e-8) */
    uint32_t seed;         /* initial weights and the pair draws; default 1 */
    float gate;            /* max channel error kept; default 2/255 */
    int32_t sh_degree;     /* the SH colour it learns: -1 = the scene's degree */
    uint32_t reserved[5];
} GsrColorModelOptions;
typedef struct GsrColorModelStats {
    uint32_t gaussians;
    uint32_t fallback;       /* gaussians that keep the SH colour */
    uint32_t steps;
    int32_t sh_degree;
    float first_loss;        /* mean squared error per channel of the first and the last step */
    float final_loss;
    float max_error_kept;    /* largest max-channel error among the gaussians decoded by the MLP */
    float train_ms;          /* device time of decode + training + encoding + gate */
    uint32_t reserved[4];
} GsrColorModelStats;
void gsr_color_model_options_default(GsrColorModelOptions* options);
/* Trains a colour model for the scene (synchronous; the scene must stay valid while it runs). */
int gsr_color_model_train(const GsrSceneDesc* scene, const GsrColorModelOptions* options, GsrColorModel** out);
int gsr_color_model_stats(const GsrColorModel* model, GsrColorModelStats* out);
/* Host copies: latents (count x 8 fp16 bits; a NaN last half marks a fallback gaussian), the fp32
 * parameters (5195 floats, encoder W1 [48][64], b1, W2 [64][8], b2, decoder W1 [11][32], b1,
 * W2 [32][32], b2, W3 [32][3], b3) and the per-step loss. Any pointer may be NULL. */
int gsr_color_model_read(const GsrColorModel* model, uint16_t* latents, float* params, float* loss_per_step);
/* Makes the renderer colour visible gaussians with the model (NULL: SH colour again). The model
 * must stay valid while the renderer uses it and must match the renderer's scene and degree. */
int gsr_renderer_set_color_model(GsrRenderer* r, const GsrColorModel* model);
void gsr_color_model_destroy(GsrColorModel* model);

/* ---- colour model checkpoints (no reference counterpart: its renderer keeps no trained state) --
 * A checkpoint file holds everything a training run has made: the fp32 parameters, Adam's first
 * and second moments, the steps taken, the options (seed, learning rate, batch, directions,
 * gate), the statistics, the loss of every step and the per-gaussian latents (fp16 bits, NaN in
 * the last half for the gaussians kept on SH). Layout, little-endian, version 1:
 *   "GSRCLRM\0" | u32 version | u32 count | i32 sh_degree | u32 step | u32 loss_count | u32 params
 *   | GsrColorModelOptions (48 B) | GsrColorModelStats (48 B) | f32 params[params] | f32 m[params]
 *   | f32 v[params] | f32 loss[loss_count] | u16 latents[count * 8] | u32 CRC-32 (IEEE, of every
 *   byte before it).
 * Reading checks the magic, the version, the sizes against the file length and the CRC, and
 * reports GSR_ERROR_FORMAT for a file that fails any of them, GSR_ERROR_IO when it cannot be
 * read or written. */
#define GSR_COLOR_MODEL_PARAMS 5195u
#define GSR_COLOR_MODEL_FILE_VERSION 1u
typedef struct GsrColorModelCheckpoint {
    uint32_t count;               /* gaussians */
    int32_t sh_degree;            /* the SH degree the model learned */
    uint32_t step;                /* Adam steps taken */
    uint32_t loss_count;          /* entries of loss */
    GsrColorModelOptions options;
    GsrColorModelStats stats;
    float* params;                /* [GSR_COLOR_MODEL_PARAMS], in gsr_color_model_read's order */
    float* adam_m;                /* [GSR_COLOR_MODEL_PARAMS] */
    float* adam_v;                /* [GSR_COLOR_MODEL_PARAMS] */
    float* loss;                  /* [loss_count] mean squared error per channel of each step */
    uint16_t* latents;            /* [count * 8] */
} GsrColorModelCheckpoint;
/* Host only (no device needed): writes / reads a checkpoint file. Reading with NULL arrays
 * fills the sizes and the header fields only, so the caller can size the arrays. */
int gsr_color_model_file_write(const char* path, const GsrColorModelCheckpoint* checkpoint);
int gsr_color_model_file_read(const char* path, GsrColorModelCheckpoint* checkpoint);
/* Saves a trained model to a checkpoint file. */
int gsr_color_model_save(const GsrColorModel* model, const char* path);
/* A model from a checkpoint file for `scene` (the count and the learned degree must match);
 * the decoder is packed from the parameters, the latents are the file's. */
int gsr_color_model_load(const GsrSceneDesc* scene, const char* path, GsrColorModel** out);
/* Continues training for `steps` more Adam steps from the model's parameters, moments and step
 * counter with its options, then encodes the latents and applies the gate again. A run cut into
 * pieces this way (with save and load between them) gives the same model bit for bit as one run
 * of all the steps. */
int gsr_color_model_resume(const GsrSceneDesc* scene, GsrColorModel* model, uint32_t steps);

/* ---- autotuner (no reference counterpart) -------------------------------------------------
 * Times each candidate of a search space on the caller's cameras with renderers of the given
 * settings (and colour model, or NULL) and returns the fastest. The knobs: views per frame, the
 * rasterizer schedule (one block per tile, or a persistent (view, tile) queue), the tile shape
 * (16 x 16, the reference's tiles, or 8 x 8) and the radix digit width of the list sort.
 * Synchronous; allocates and frees its own renderers. */
#define GSR_TUNE_MAX_CANDIDATES 64u
typedef struct GsrTuneCandidate {
    uint32_t views_per_frame;
    uint32_t raster_schedule;  /* GSR_RASTER_PER_TILE or GSR_RASTER_PERSISTENT */
    float views_per_s;         /* device time over whole frames of consecutive cameras */
    float ms_per_frame;
    uint32_t tile_size;        /* binning / render tiles: 16, 8 or 32 (32 x 8) */
    uint32_t sort_digit_bits;  /* digit width of the list's radix sort */
} GsrTuneCandidate;
typedef struct GsrTuneResult {
    uint32_t views_per_frame;  /* the fastest candidate */
    uint32_t raster_schedule;
    float views_per_s;
    uint32_t candidates;       /* entries of table */
    uint32_t tile_size;
    uint32_t sort_digit_bits;
    GsrTuneCandidate table[GSR_TUNE_MAX_CANDIDATES];
} GsrTuneResult;
/* The search space: a NULL list (or a zero count) keeps the settings' value for that knob, except
 * raster_schedules, where it means both schedules. Candidates beyond GSR_TUNE_MAX_CANDIDATES are
 * refused (GSR_ERROR_INVALID_ARGUMENT). */
typedef struct GsrTuneSpace {
    const uint32_t* views_per_frame;  /* each 1..min(count, GSR_MAX_VIEWS) */
    uint32_t views_per_frame_count;
    const uint32_t* raster_schedules; /* GSR_RASTER_PER_TILE / GSR_RASTER_PERSISTENT */
    uint32_t raster_schedule_count;
    const uint32_t* tile_sizes;       /* 16 or 8 */
    uint32_t tile_size_count;
    const uint32_t* sort_digit_bits;  /* see GsrSettings.sort_digit_bits */
    uint32_t sort_digit_bits_count;
} GsrTuneSpace;
/* cameras[0..count) are rendered in frames of `views_per_frame` consecutive cameras; each
 * candidate gets warm-up frames until the adaptive list keeps its capacity, then `frames` timed
 * frames. */
int gsr_autotune_space(const GsrSceneDesc* scene, const GsrSettings* settings, const GsrColorModel* model,
                       const GsrSplatCamera* cameras, uint32_t count, const GsrTuneSpace* space, uint32_t frames,
                       GsrTuneResult* out);
/* gsr_autotune_space over views per frame x both schedules, the settings' tile size and digit width. */
int gsr_autotune(const GsrSceneDesc* scene, const GsrSettings* settings, const GsrColorModel* model,
                 const GsrSplatCamera* cameras, uint32_t count, const uint32_t* depths, uint32_t depth_count,
                 uint32_t frames, GsrTuneResult* out);

/* Synchronizes and copies view `view`'s images to the host (either pointer may be NULL); rgba
 * receives float4 per pixel whatever the output format (fp16 and 8-bit values converted exactly:
 * v / 255 for RGBA8). */
int gsr_read_view_image(GsrRenderer* r, uint32_t view, float* rgba, uint8_t* rgb8);
/* The end-to-end call for batched host callers: render the views and copy every view's RGB8
 * (or, when rgb8 output is off, the output format's) image into `host`, view after view at
 * pixel_base (`bytes` must match), then synchronize `stream`. With the per-tile raster schedule
 * and more than one view the frame rasterizes the views one launch each (in its own CUDA graph
 * when use_graph is on) and copies each view's image on a renderer-owned stream as soon as that
 * view is done, so the copies overlap the rasterization of the following views; the images are
 * the same. */
int gsr_render_views_to_host(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* host, uint64_t bytes,
                             void* stream);
/* The streaming form of gsr_render_views_to_host (no reference counterpart): returns once the
 * frame and its copies are enqueued, with a ticket; the images are in `host` after
 * gsr_renderer_host_wait(r, ticket). Until then `host` must stay allocated and untouched, so a
 * caller alternates between (at least) two host buffers. The next frame's preprocess and sorts
 * run while this frame's copies are in flight; its rasterization (that of any later frame) waits
 * for them. The frame is rasterized in one launch and its image copied whole after it (the
 * copies overlap the next frame's front, not this frame's rasterization). The images are those
 * of gsr_render_views_to_host. A layout change (other view sizes) waits for copies in flight. */
int gsr_render_views_to_host_async(GsrRenderer* r, const GsrSplatCamera* cameras, uint32_t views, void* host,
                                   uint64_t bytes, void* stream, uint64_t* ticket);
/* Blocks until the copies of `ticket` (and of every earlier ticket) are in host memory. */
int gsr_renderer_host_wait(GsrRenderer* r, uint64_t ticket);

/* lastStats / collectPending (splat_tile_renderer.h:167-181): the control block of the most
 * recent frame whose readback has completed (frames_in_flight frames late, no stall).
 * GSR_ERROR_NOT_READY if none yet. frame_index receives that frame's number. */
int gsr_renderer_last_stats(GsrRenderer* r, GsrControl* out, uint64_t* frame_index);
/* Synchronizes and reads the current control block (readBack's TileControl). */
int gsr_read_control(GsrRenderer* r, GsrControl* out);
/* readBack (splat_tile_renderer.h:184-185), GPU idle: the sorted list's first n entries
 * (keys_lo = depth bits, keys_hi = tile, values = gaussian) and 2 words per tile of ranges.
 * Any pointer may be NULL. n is clamped to the entry count. */
int gsr_read_list(GsrRenderer* r, uint32_t* keys_lo, uint32_t* keys_hi, uint32_t* values, uint32_t n,
                  uint32_t* ranges, uint32_t ranges_words);
/* readBackSplats (splat_tile_renderer.h:188): 48-byte ProjectedSplat records (visible
 * gaussians only are written by a frame; the rest keep older contents) and tile counts. */
int gsr_read_splats(GsrRenderer* r, void* splats, uint32_t* tile_counts, uint32_t n);
/* readBackPackedSplats (splat_tile_renderer.h:191-192), packed render splats only: the first n
 * gaussians' records (8 or 6 words each), rects (2 words) and depth bits; any pointer may be
 * NULL. GSR_ERROR_UNSUPPORTED with FULL records (gsr_read_splats reads those). */
int gsr_read_packed_splats(GsrRenderer* r, uint32_t* words, uint32_t* rects, uint32_t* depths, uint32_t* tile_counts,
                           uint32_t n);
/* readBackImage (splat_tile_renderer.h:194): rgba float4[W*H] and/or rgb8 uint8[W*H*3]. */
int gsr_read_image(GsrRenderer* r, float* rgba, uint8_t* rgb8);
/* The per-tile counters of the last frame of a renderer created with tile_stats = 1, in the
 * reference's TileStat order (splat_tile_renderer.h:131-141), GSR_TILE_STAT_COUNT words per frame
 * tile: list length, entries fetched before the tile stopped, (pixel, splat) pairs evaluated
 * (entries a pixel visits until it terminates, all of them when it does not), pairs blended,
 * pixels terminated (T < 1e-4), lane slots of the blend loop (its warp iterations x 32), the
 * largest evaluated count of a pixel, pixels inside the image. tested_pairs (may be NULL)
 * receives the pairs this rasterizer computed alpha for (a pixel still blending and a record
 * whose cutoff ellipse meets that pixel's warp strip). Synchronizes; `tiles` must be the
 * frame's tile count over all views. */
#define GSR_TILE_STAT_COUNT 8u
int gsr_read_tile_stats(GsrRenderer* r, uint32_t* stats, uint32_t tiles, uint64_t* tested_pairs);
/* Per-pass device time of the last frame in ms (GpuProfiler scopes), when timing is on: 5 passes
 * in global mode, 7 in binning mode (its front as preprocess, depth sort, scan + emission). */
int gsr_renderer_set_timing(GsrRenderer* r, int enabled);
int gsr_renderer_pass_times(GsrRenderer* r, float* ms, const char** names, uint32_t capacity, uint32_t* count);
/* Capacity of the current list in entries, the budget's maximum, and list resizes so far. */
int gsr_renderer_capacity(GsrRenderer* r, uint32_t* capacity, uint32_t* max_capacity, uint32_t* resizes);
/* Kernels of this library that gsr_render has launched on this renderer so far. */
int gsr_renderer_kernel_launches(GsrRenderer* r, uint64_t* count);
/* Test hook: forces the look-back waits of the next frame to see no predecessor, and the
 * preprocess's waits for its staged SH to see no completion (those read the SH from global
 * memory instead), so that they run into their iteration limit and report GSR_CONTROL_TIMEOUT
 * (iterations = limit; timeout_where 1 scan, 2 sort, 4 SH staging). */
int gsr_renderer_debug_force_timeout(GsrRenderer* r, uint32_t iterations);
void gsr_renderer_destroy(GsrRenderer* r);

/* ---- primitives (GpuScan src/render/gpu_scan.h:25-76, GpuRadixSort
 *      src/render/gpu_radix_sort.h:38-122) ----------------------------------------------- */
typedef enum GsrScanMode { GSR_SCAN_PLAIN = 0, GSR_SCAN_NONZERO = 1, GSR_SCAN_GATHER = 2 } GsrScanMode;
/* Exclusive scan of `count` u32 (device pointers): out[j] = sum_{i<j} v(i), v(i) = in[i]
 * (plain), in[i] != 0 (non-zero flags) or in[index[i]] (gather); *total (device) = the sum.
 * The scratch (control block, look-back words) is allocated and freed per call, and the call
 * returns after the scan has finished on `stream`. */
int gsr_scan(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
             uint32_t mode, void* stream);
/* Stable LSD sort of (key, value) pairs by the low key_bits of the key, in place (device
 * pointers). keys_hi may be NULL (32-bit keys); with it the key is (keys_hi << 32 | keys_lo).
 * Bit-for-bit the order of a stable sort (DepthSorter::radixSortPairs for 32-bit keys). */
int gsr_sort_pairs(uint32_t* keys_lo, uint32_t* keys_hi, uint32_t* values, uint32_t count, uint32_t key_bits,
                   void* stream);

/* ---- allocation-free scan (no counterpart in the reference) ---------------------------- */
/* Largest count gsr_scan_static accepts. */
#define GSR_SCAN_STATIC_MAX_COUNT 16777216u
/* gsr_scan without any allocation, for callers that must not allocate device memory: recovery
 * code that runs after an allocation failed (device memory held by a resident scene), hooks of
 * a caching allocator that must not re-enter it, and streams that must not stall behind
 * cudaFree, which synchronizes the whole device.
 * Same arguments, results and errors as gsr_scan. The scratch (a 512-byte control block and
 * one look-back word per 2048 items) is a fixed 66,048-byte static device array of this
 * library, held on every device that loads it until the process exits; count above
 * GSR_SCAN_STATIC_MAX_COUNT (2^24) is rejected with GSR_ERROR_INVALID_ARGUMENT before anything
 * is launched. The call clears what must start at zero (the block tickets and the look-back
 * words) on `stream` and returns after the scan has finished there. Calls that overlap in time
 * on one device (two streams or two host threads) share the array and race: the caller
 * serializes them.
 * Set-up: with CUDA's lazy module loading, the array and the scan's kernels are loaded on a
 * device when first used, which can allocate device memory. This library does that loading
 * (and looks up the array's address) in every set-up call on a device: gsr_scene_create,
 * gsr_renderer_create, gsr_scan and gsr_sort_pairs; a caller that makes none of those first
 * calls gsr_scan_static once with count 0, which does only that. Make that first call before
 * any stream capture begins on the device. */
int gsr_scan_static(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
                    uint32_t mode, void* stream);

/* ---- scene input: 3DGS PLY files (src/scene/ply_loader.h:1-120) --------------------------
 * Host-side: the file is validated exactly as loadGaussianPly does (same accepted files, the
 * same error and warning texts) and decoded by all host threads into the activated SoA arrays
 * of gsr::GaussianScene: posAlpha = (x, y, z, sigmoid(opacity)), scales = (exp(scale_i), 0),
 * rotations = normalized (rot_0..rot_3) = (w, x, y, z), SH as RGB triplets per coefficient
 * (the file's channel-major f_rest transposed), bit-identical to the reference loader's.
 * gsr_loaded_scene_host() hands them to gsr_scene_create(). Errors: GSR_ERROR_FORMAT for a
 * malformed file, GSR_ERROR_IO when it cannot be read; the message names the problem. */
typedef struct GsrLoadedScene GsrLoadedScene;

/* gsr::SceneStats (src/scene/gaussian_scene.h:47-61). */
typedef struct GsrSceneStats {
    float bbox_min[3], bbox_max[3];
    float robust_min[3], robust_max[3]; /* per-axis 1st / 99th percentile: sorted[int(p (n - 1))] */
    float alpha_min, alpha_max, alpha_mean;
    uint32_t alpha_below_visible;       /* alpha < 1/255 */
    float sigma_min, sigma_max, sigma_max_median;
    float quat_norm_min, quat_norm_max; /* raw quaternion lengths */
    uint32_t zero_quaternions;          /* replaced by identity */
    uint64_t non_finite_values;         /* NaN/Inf in the decoded properties */
} GsrSceneStats;

/* gsr::LoadTimings (gaussian_scene.h:63-69). */
typedef struct GsrLoadTimings {
    double map_ms, header_ms, decode_ms, stats_ms, total_ms;
} GsrLoadTimings;

typedef struct GsrLoadedSceneInfo {
    uint32_t count;
    int32_t sh_degree;
    uint32_t comment_count; /* header comment lines */
    uint32_t warning_count; /* non-fatal issues (skipped elements, trailing bytes, NaN, ...) */
    GsrSceneStats stats;
    GsrLoadTimings timings;
} GsrLoadedSceneInfo;

/* Host arrays owned by the loaded scene (valid until gsr_loaded_scene_destroy). */
typedef struct GsrLoadedSceneArrays {
    const float* pos_alpha;     /* float4[N] */
    const float* scales;        /* float4[N] */
    const float* rotations;     /* float4[N] */
    const float* sh;            /* float[N * K * 3], K = (sh_degree + 1)^2 */
    const float* raw_opacity;   /* float[N]: the file's opacity (logit) */
    const float* raw_log_scale; /* float3[N]: the file's scale_0..2 (log sigma) */
    const float* raw_rotation;  /* float4[N]: the file's rot_0..3, unnormalized */
} GsrLoadedSceneArrays;

/* loadGaussianPly(path) (ply_loader.h:75-77): the file name prefixes the messages. */
int gsr_ply_load(const char* path, GsrLoadedScene** out);
/* loadGaussianPly(bytes, name) (ply_loader.h:78-80). */
int gsr_ply_load_memory(const void* bytes, size_t size, const char* name, GsrLoadedScene** out);
int gsr_loaded_scene_info(const GsrLoadedScene* scene, GsrLoadedSceneInfo* info);
int gsr_loaded_scene_arrays(const GsrLoadedScene* scene, GsrLoadedSceneArrays* arrays);
/* The activated arrays as a GsrHostScene, for gsr_scene_create(). */
int gsr_loaded_scene_host(const GsrLoadedScene* scene, GsrHostScene* host);
const char* gsr_loaded_scene_comment(const GsrLoadedScene* scene, uint32_t index);
const char* gsr_loaded_scene_warning(const GsrLoadedScene* scene, uint32_t index);
const char* gsr_loaded_scene_source(const GsrLoadedScene* scene);
void gsr_loaded_scene_destroy(GsrLoadedScene* scene);
/* shDegreeFromRestCount (ply_loader.h:72): 0/9/24/45 -> 0..3, else -1. */
int gsr_ply_sh_degree_from_rest_count(uint64_t rest_count);

/* parsePlyHeader / parsePlyHeaderPrefix (ply_loader.h:64-69): final_bytes = 0 returns
 * GSR_ERROR_NOT_READY while the end_header line has not arrived. Property types are
 * PlyScalar's order: int8, uint8, int16, uint16, int32, uint32, float32, float64. */
typedef struct GsrPlyHeader GsrPlyHeader;
typedef struct GsrPlyElementInfo {
    const char* name;
    uint64_t count;
    uint32_t stride; /* bytes per record: every scalar property */
    uint32_t has_list;
    uint32_t property_count;
} GsrPlyElementInfo;
typedef struct GsrPlyPropertyInfo {
    const char* name;
    uint32_t type;
    uint32_t is_list;
    uint32_t offset; /* byte offset in the record (scalar properties) */
} GsrPlyPropertyInfo;
int gsr_ply_parse_header(const void* bytes, size_t size, int final_bytes, GsrPlyHeader** out);
/* format: 0 binary_little_endian, 1 binary_big_endian, 2 ascii. */
int gsr_ply_header_info(const GsrPlyHeader* header, uint32_t* format, uint32_t* element_count, uint32_t* comment_count,
                        uint64_t* header_bytes);
int gsr_ply_header_element(const GsrPlyHeader* header, uint32_t index, GsrPlyElementInfo* info);
int gsr_ply_header_property(const GsrPlyHeader* header, uint32_t element, uint32_t property, GsrPlyPropertyInfo* info);
const char* gsr_ply_header_comment(const GsrPlyHeader* header, uint32_t index);
void gsr_ply_header_destroy(GsrPlyHeader* header);

/* PlyStreamDecoder (ply_loader.h:82-117): bytes pushed in order in chunks of any size; the header
 * callback runs once the header has passed its checks (info: count, degree, comments), the batch
 * callback with each decoded batch of up to batch_capacity gaussians (0: 16384) as gaussians
 * [first, first + batch count), valid during the call. The batches concatenated equal
 * gsr_ply_load's arrays bit for bit, and a bad file fails with the same message. finish() runs
 * the size checks and fills the info's warnings and NaN / zero-quaternion counters. After an
 * error, push and finish return GSR_ERROR_INVALID_ARGUMENT. */
typedef struct GsrPlyStream GsrPlyStream;
typedef void (*GsrPlyHeaderCallback)(void* user, const GsrLoadedScene* info);
typedef void (*GsrPlyBatchCallback)(void* user, uint32_t first, const GsrLoadedScene* batch);
int gsr_ply_stream_create(const char* name, uint64_t total_bytes, GsrPlyHeaderCallback on_header,
                          GsrPlyBatchCallback on_batch, void* user, uint32_t batch_capacity, GsrPlyStream** out);
int gsr_ply_stream_push(GsrPlyStream* stream, const void* bytes, size_t size);
int gsr_ply_stream_finish(GsrPlyStream* stream);
int gsr_ply_stream_state(const GsrPlyStream* stream, uint32_t* header_parsed, uint32_t* finished,
                         uint64_t* bytes_received, uint64_t* records_decoded);
const GsrLoadedScene* gsr_ply_stream_info(const GsrPlyStream* stream);
void gsr_ply_stream_destroy(GsrPlyStream* stream);

/* ---- scene input: INRIA training cameras (src/scene/training_cameras.h:1-44) ------------- */
#define GSR_IMAGE_NAME_CAPACITY 256
typedef struct GsrTrainingCamera {
    int32_t id;
    uint32_t width, height;
    float position[3];        /* camera centre, data space */
    float camera_to_world[9]; /* column-major; the columns are the camera's right, down, forward axes */
    float fx, fy;             /* focal lengths in pixels */
    char image_name[GSR_IMAGE_NAME_CAPACITY]; /* NUL-terminated (truncated) */
} GsrTrainingCamera;
/* loadTrainingCameras (cameras.json): *count = the cameras in the file; the first `capacity`
 * are written. GSR_ERROR_IO with "Cannot open cameras file: ..." or "Invalid cameras file ...". */
int gsr_training_cameras_load(const char* path, GsrTrainingCamera* cameras, uint32_t capacity, uint32_t* count);
/* TrainingCamera::fovYDeg: 2 atan(height / (2 fy)) in degrees. */
float gsr_training_camera_fov_y_deg(const GsrTrainingCamera* camera);
/* meanCameraUp: the normalized mean of -down over the cameras ((0, -1, 0) if it vanishes). */
int gsr_training_cameras_mean_up(const GsrTrainingCamera* cameras, uint32_t count, float up[3]);
/* cameraFocusPoint: the least-squares point nearest every optical axis (the centroid when the
 * axes are parallel). */
int gsr_training_cameras_focus_point(const GsrTrainingCamera* cameras, uint32_t count, float point[3]);

/* ---- diagnostics ------------------------------------------------------------------------ */
const char* gsr_error_string(int status);
const char* gsr_last_error_message(void);
int gsr_abi_version(void);
/* Device: computes the kernel's 2 ln(255 o) threshold log for every float x in [1, 255] into
 * out (device, 67,043,329 floats), so tests can compare it with the C library's logf. */
int gsr_debug_logf_table(float* out_device, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSR_B200_H */
