// Kernel argument blocks and launch entry points shared between the CUDA translation units
// and the host renderer (renderer.cpp).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "gsr_types.h"

namespace gsr {

// One-time launch set-up (function attributes, grid sizes) is per device: the slot of the
// current device in a launcher's table. The slots are atomics, so host threads that render on
// the same device at once may both do the set-up (it is idempotent) without a data race.
template <class T>
inline std::atomic<T>& perDevice(std::atomic<T> (&table)[64]) {
    int dev = 0;
    cudaGetDevice(&dev);
    return table[dev & 63];
}

struct DevCameraArgs {  // = DevCamera (splat_math.cuh)
    float v[16];
    float pos[3];
    uint32_t width, height;
    float tanHalfFovX, tanHalfFovY, focalX, focalY;
    uint32_t tilesX, tilesY;
};

// One view of a frame. A frame renders views [0, viewCount) of its launch together: view v's
// tiles are the frame's tiles [tileBase, tileBase + tilesX * tilesY) (the "global" tile id, so
// the view sits in the high bits of every list key) and its pixels start at pixelBase in the
// image buffers. Per-gaussian arrays (records, tile counts, offsets) are indexed v * N + g.
struct DevView {
    uint32_t tileBase;
    uint32_t tilesX, tilesY;  // the binning / render tiles of the view (tile_size pixels)
    uint32_t width, height;
    uint32_t pad;
    uint64_t pixelBase;
};
static_assert(sizeof(DevView) == 32, "DevView layout");

// The learned colour stage's decoder for the tensor cores (mlp.cuh); the host needs its size and
// the parameter count only.
struct DecoderWeights;
constexpr size_t kDecoderWeightsBytes = 32 * 16 * 2 + 32 * 32 * 2 + 8 * 32 * 2 + (32 + 32 + 8) * 4;
constexpr uint32_t kColorModelParams = 5195;

struct SceneArgs {
    const uint4* b0;     // soa posAlpha | geometry records | aos records
    const uint4* b1;     // soa scales   | colour records   | aos records
    const uint4* b2;     // soa rotations
    const float* shSoa;  // soa sh float[]
    uint32_t geometryStride, colorStride, colorOffset;
    uint32_t storedCoeffs;  // K
    uint32_t codebookStride;  // cb: 16-byte units per codebook entry (b2 = the codebook)
    uint32_t codebookLast;    // cb: the last entry the codebook buffer holds (indices clamp to it)
    uint32_t variableSh;    // GsrVariableSh
};

// Arguments of the per-gaussian kernels of the frame's front (preprocess, scan, key emission).
struct FrontArgs {
    const DevCameraArgs* cam;  // device copies of the views' SplatCameras [viewCount] (written by the frame itself)
    const DevView* views;      // [viewCount]
    uint32_t viewCount;        // V (grid.y of the per-gaussian kernels)
    uint32_t totalTiles;       // tiles of all views = the sentinel tile id
    SceneArgs scene;
    uint32_t count;       // N
    int evalDegree;       // min(stored degree, max_sh_degree)
    uint32_t bounds;      // GsrTileBounds
    int binSize;          // the bins: 16 or 8 (S x S), 32 (32 x 8)
    uint32_t capacity;    // list entries
    void* splats;         // DevSplat[V * N] (full render records)
    uint32_t renderSplat; // kRenderSplatFull / P32 / P24
    void* packed;         // packed render records [V * N] (8 or 6 words), P32 / P24
    uint2* rects;         // [V * N] packed tile rectangles, P32 / P24
    float4* rayDepth;     // [V * N * 3] StopThePop ray-depth parameters of visible gaussians, or null
    uint32_t* depths;     // [V * N] depth bits, P32 / P24
    float4* hints;        // [V * N] cutoff-ellipse terms of visible gaussians (coverageHint), tight/cutoff bounds,
                          // or rows 0-3 of their runs (span hints)
    uint4* spanRows;      // [V * N] rows 3-6 of span hints with more than 3 rows
    uint32_t* tileCounts; // [V * N]
    uint32_t* offsets;    // [V * N] exclusive scan of tileCounts
    uint64_t* keys;       // [capacity] (tile << 32 | depth bits), view-major index order
    uint32_t* values;     // [capacity]
    uint64_t* scanStatus; // [ceil(V * N / 2048)] look-back words of the scan over the counts
    // binning mode (the reference's default list construction): the records ordered by
    // (depth, record index), a packed word per record, sorted on the device
    uint32_t binning;
    uint32_t shStaged;                    // soa SH3 scenes: each block's SH copied to shared memory by one bulk copy
    uint64_t* depthKeys[2];               // [V * N] (depth mod 2^W, or the no-tile sentinel) << recordBits | record
    const struct SortPlan* depthPlan;     // its sort's plan (which buffer holds the result)
    uint32_t recordBits;                  // bits of a record index (V * N - 1)
    uint32_t depthViewShift;              // the view's field in the depth words, above the depth bits
                                          // (0: none; the depth sort then orders all views together)
    const uint4* latents;                 // learned colour: fp16 latents [N] (null: SH colour)
    const struct DecoderWeights* decoder; // learned colour: the tensor-core decoder (mlp.cuh)
    float4* decoded;                      // tcgen05 decode: kept gaussians' colours [viewCount][N]
                                          // (null: the preprocess decodes with mma.sync)
    DeviceControl* ctl;
    LogfFixups logf;
};

// Sort plan written by the histogram kernel's last block.
constexpr int kMaxSortPasses = 10;  // 64 key bits in 7-bit digits
constexpr int kMaxSortBins = 512;   // digits of up to 9 bits
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
// binning mode's depth sort (frameMode 2): 4096-key tiles, its status array sized by them
constexpr int kDepthSortItems = 16;
constexpr int kDepthSortTile = kSortThreads * kDepthSortItems;
struct SortPlan {
    uint32_t passes;        // significant 8-bit digits of the virtual key
    uint32_t lowBits;       // W: low key bits kept below the high word
    uint32_t keyBits;
    uint32_t packed;        // entries are single words (vkey << indexBits | index), see KeyLayout
    uint32_t indexBits;
    uint32_t active[kMaxSortPasses];
    uint32_t inBuffer[kMaxSortPasses];
    uint32_t digitBits;     // digit width of the passes (7, 8 or 9)
    uint32_t depthBits;     // the depth sort: bits of (depth bits - depthMin) over the frame's visible records
    uint32_t depthMin;      // the depth sort: the frame's smallest visible depth bits
    uint32_t digitBase[kMaxSortPasses][kMaxSortBins];
    uint32_t hist[kMaxSortPasses][kMaxSortBins];
    uint32_t sortedBuffer;  // the buffer that holds the result (active passes mod 2)
};

struct SortArgs {
    uint64_t* keys[2];
    uint32_t* values[2];
    uint64_t* status;      // [passes][maxTiles][1 << digitBits]
    uint32_t maxTiles;     // ceil(capacity / kSortTile); the depth sort: ceil(count / kDepthSortTile)
    SortPlan* plan;
    DeviceControl* ctl;
    uint32_t passesLaunched;
    // plan source: frameMode = 1 derives the low bits from the frame's depth range and the high
    // bits from the largest tile id (binning = 1: tile-only keys, no depth bits); 2 = the depth
    // words of binning mode (the depth bits above a record index of indexBits, each view's run
    // sorted by their offset from the frame's smallest visible depth bits); 0 uses
    // fixedLowBits/fixedKeyBits (standalone sort).
    uint32_t frameMode;
    uint32_t fixedLowBits, fixedKeyBits;
    uint32_t tileCount, count;  // frame mode: the grid's tiles and N (for the entry layout)
    uint32_t binning;
    uint32_t indexBits;         // frameMode 2: bits of the record index
    uint32_t digitBits;         // 7, 8 or 9 bits a pass
    // frameMode 2: the records are `segments` runs of segLength (one view's records each, in view
    // order), sorted each on its own: tiles never straddle two runs (tile t is tile t mod
    // ceil(segLength / tile) of run t / ceil(segLength / tile)), a run's first tile starts its
    // look-back chains, and its digits start at the run's first record. segHist / segBase:
    // [segments][passesLaunched][1 << digitBits] digit counts (zeroed by frameBegin) and bases.
    uint32_t segments, segLength;
    uint32_t* segHist;
    uint32_t* segBase;
};

struct RenderArgs {
    const void* splats;       // DevSplat[V * N] (full render records)
    uint32_t renderSplat;     // kRenderSplatFull / P32 / P24
    const void* packed;       // packed render records [V * N], P32 / P24
    const float4* rayDepth;   // [V * N * 3] StopThePop ray-depth parameters (sortWindow > 0)
    const DevCameraArgs* cam; // the frame's cameras [viewCount] (focal lengths of the pixel rays)
    uint32_t sortWindow;      // StopThePop window K, 0 = off
    uint32_t tileSize;        // the render tile: 16 (INRIA), 8 or 32 (32 x 8) pixels
    uint32_t bounds;          // GsrTileBounds of the list (32 x 8 tiles clip splats to their 16-px rectangle)
    const uint32_t* values[2];
    const uint64_t* keys[2];
    uint32_t* ranges;         // uint2 per tile of the frame (all views)
    void* image;              // per view W*H at the view's pixelBase: float4, half4 or uchar4 (imageFormat)
    uint32_t imageFormat;     // 0: float4, 1: half4 (fp16 round to nearest even), 2: uchar4 (lround(clamp(v) 255))
    uint8_t* rgb8;            // per view W*H*3 at 3 * pixelBase, or null
    const DevView* views;     // [viewCount]
    uint32_t viewCount;
    uint32_t totalTiles;
    uint32_t persistent;      // 1: a fixed grid takes (view, tile) work items from a queue
    uint32_t tileOffset;      // per-tile schedule: the launch's first frame tile
    uint32_t tileLaunch;      // per-tile schedule: the launch's tiles (0: every tile of the frame)
    uint32_t count;           // N: gaussian indices read from the list are checked against it
    DeviceControl* ctl;
    const SortPlan* plan;     // the entry layout (packed words or key/value arrays)
    const void* splatMap;     // host copy of the CUtensorMap over the full records: the TMA gather (null: cp.async)
    uint32_t* tileStats;      // the stats build: kTileStatWords per frame tile (null: the plain build)
    unsigned long long* testedPairs;  // the stats build: pairs the kernel tested, summed over the frame
};

// The stats build's words per tile (TileStat, splat_tile_renderer.h:131-141).
constexpr uint32_t kTileStatListLength = 0, kTileStatFetched = 1, kTileStatEvaluated = 2, kTileStatBlended = 3,
                   kTileStatTerminated = 4, kTileStatLaneSlots = 5, kTileStatMaxDepth = 6, kTileStatPixels = 7,
                   kTileStatWords = 8;

// ---- launchers (return cudaGetLastError()) ---------------------------------------------------
cudaError_t launchFrameBegin(DeviceControl* ctl, uint32_t count, uint32_t capacity, uint32_t* ranges,
                             uint32_t rangeWords, SortPlan* plan, uint32_t forceTimeout, cudaStream_t s,
                             SortPlan* plan2 = nullptr, uint32_t* clearWords = nullptr, uint32_t clearCount = 0);
cudaError_t launchFront(const FrontArgs& a, uint32_t geometry, uint32_t color, cudaStream_t s);
// Binning mode, split around the depth sort: preprocess + the depth keys, then (after the sort of
// the depth keys) the scan of the counts in depth order and the emission in that order.
cudaError_t launchFrontBinningKeys(const FrontArgs& a, uint32_t geometry, uint32_t color, cudaStream_t s);
cudaError_t launchFrontBinningEmit(const FrontArgs& a, cudaStream_t s);
// The learned colour's decode as a pre-pass on the tcgen05 tensor cores: every kept gaussian's
// colour for every view of the frame into a.decoded (before the preprocess, which reads them).
cudaError_t launchDecodeColoursTc(const FrontArgs& a, uint32_t geometry, cudaStream_t s);
cudaError_t launchSort(const SortArgs& a, uint32_t histBlocks, cudaStream_t s);
cudaError_t launchRanges(const RenderArgs& a, uint32_t capacity, cudaStream_t s);
cudaError_t launchRender(const RenderArgs& a, cudaStream_t s);
cudaError_t launchLogfTable(float* out, LogfFixups t, cudaStream_t s);
// Exclusive scan (decoupled look-back, 2048 items per block); with setupCapacity != 0 the last
// block also writes the frame's entries = min(total, capacity), overflow and ranges groups.
// Gather source of the scan in binning mode: in[word & mask] for the sorted packed words.
struct ScanGather {
    const uint64_t* words[2];
    const struct SortPlan* plan;  // plan->sortedBuffer picks the words
    uint64_t mask;
};
constexpr uint32_t kScanGatherSorted = 8;  // internal scan mode next to GsrScanMode's
cudaError_t launchScan(const uint32_t* in, const uint32_t* index, uint32_t* out, uint32_t* total, uint32_t count,
                       uint32_t mode, uint64_t* status, DeviceControl* ctl, cudaStream_t s, uint32_t setupCapacity = 0,
                       uint32_t waitSite = kWaitStandaloneScan, const ScanGather* gather = nullptr);
// ---- the learned colour stage (k_mlp.cu; decoded SH from k_front.cu) -------------------------
// Decoded SH coefficients [count][48] (zeros past each gaussian's evaluated degree) and degrees.
cudaError_t launchShDecode(const SceneArgs& scene, uint32_t geometry, uint32_t color, uint32_t count, int evalDegree,
                           float* out, uint8_t* degrees, cudaStream_t s);
// One training step (batch pairs, a multiple of colorTrainBatchMultiple()): forward/backward
// partial sums, then Adam; step = {step counter, scratch counter} advanced on the device.
cudaError_t launchColorTrainStep(const float* sh, const uint8_t* degrees, uint32_t count, uint32_t dirs, uint32_t seed,
                                 uint32_t batch, float* params, float* m, float* v, float* partials, uint32_t* step,
                                 float lr, float* lossOut, uint32_t lossBase, uint32_t maxSteps, cudaStream_t s);
// The tensor-core decoder packed from the fp32 parameters.
cudaError_t launchPackDecoder(const float* params, struct DecoderWeights* decoder, cudaStream_t s);
uint32_t colorTrainBatchMultiple();
// Latents of every gaussian and the packed decoder from the trained parameters.
cudaError_t launchColorEncode(const float* sh, const float* params, uint4* latents, struct DecoderWeights* decoder,
                              uint32_t count, cudaStream_t s);
// Marks gaussians whose decoded colour is more than `gate` from the SH colour on their directions.
cudaError_t launchColorGate(const float* sh, const uint8_t* degrees, uint32_t count, uint32_t dirs,
                            const struct DecoderWeights* decoder, uint4* latents, float gate, uint32_t* fallbackCount,
                            uint32_t* maxErrorBits, cudaStream_t s);

// Device address of the static scratch of gsr_scan_static (kStaticScanScratchBytes) on the
// current device.
cudaError_t staticScanScratch(void** base);
// Load the code of the kernels gsr_scan_static launches on the current device (cudaFuncGetAttributes).
cudaError_t loadScanKernel();
cudaError_t loadFrameBeginKernel();
cudaError_t launchPack64(const uint32_t* lo, const uint32_t* hi, uint64_t* out, uint32_t n, cudaStream_t s);
cudaError_t launchUnpack64(const uint64_t* in, uint32_t* lo, uint32_t* hi, uint32_t n, cudaStream_t s);
cudaError_t launchSetEntries(DeviceControl* ctl, uint32_t count, cudaStream_t s);

}  // namespace gsr
