// Types and constants shared by the host renderer and the kernels (host-safe: no device code).
#pragma once

#include <cstddef>
#include <cstdint>

#include "gsr_b200.h"

namespace gsr {

constexpr int kTileSize = 16;                  // INRIA BLOCK_X = BLOCK_Y (splat_math.h:32)
constexpr uint32_t kCullReasonCount = 5;       // Visible, NearPlane, SingularCov, OffScreen, LowOpacity
constexpr uint32_t kCullVisible = 0, kCullNear = 1, kCullSingular = 2, kCullOffScreen = 3, kCullLowOpacity = 4;
constexpr uint32_t kBoundsRect = 0, kBoundsTight = 1, kBoundsCutoff = 2;

// Iteration limit of every device-side wait; on expiry the kernel records
// GSR_CONTROL_TIMEOUT + where, stops waiting and finishes (the frame is then invalid).
constexpr uint32_t kSpinLimit = 1u << 22;
enum WaitSite : uint32_t {
    kWaitScan = 1,
    kWaitSort = 2,
    kWaitStandaloneScan = 3,
    kWaitShStage = 4,
    kWaitGather = 5,
    kWaitDecode = 6,  // the tensor-core colour decode's MMA completions
};

constexpr int kControlTickets = 32;
constexpr uint32_t kListSortTickets = 1, kDepthSortTickets = 16;

// The per-frame control block in device memory (GsrControl in gsr_b200.h) plus scratch
// counters that only the kernels use.
struct DeviceControl {
    GsrControl c;
    // block tickets: [1 + p] list sort pass p, [12] scans, [13] the rasterizer's tile queue,
    // [16 + p] depth sort pass p (binning mode)
    uint32_t tickets[kControlTickets];
    uint32_t histDone[2];       // blocks of the histogram kernels that have finished (list, depth sort)
    uint32_t forceTimeout;      // test hook: look-back waits see no predecessor for this many spins
    uint32_t pad[5];
};

// Items of one block of the exclusive scan (scanKernel: 256 threads x kScanItems); the scan's
// grid, its look-back words and the static scratch below are all sized by it.
constexpr uint32_t kScanBlockItems = 2048;

// Layout of the static scratch of gsr_scan_static: the control block, then one look-back word
// per scan block of the largest accepted count.
constexpr size_t kStaticScanCtlBytes = 512;
constexpr size_t kStaticScanScratchBytes =
    kStaticScanCtlBytes + size_t((GSR_SCAN_STATIC_MAX_COUNT + kScanBlockItems - 1) / kScanBlockItems) * 8;
static_assert(sizeof(DeviceControl) <= kStaticScanCtlBytes, "the control block fits its slot");
static_assert(kStaticScanScratchBytes == 66048, "the size the header states");

// The C library's logf fixup table on the device (see libcLogf in gsr_device.cuh).
struct LogfFixups {
    const uint32_t* entries;       // ((x_bits - base) << 1) | up, sorted
    const uint32_t* bucketStart;   // per 1024-input bucket
    const uint32_t* groups;        // one bit per 8 consecutive inputs (word = off >> 8, bit = (off >> 3) & 31):
                                   // set when one of them holds a fixup (most inputs are answered by it)
    uint32_t base, last, count;
};

}  // namespace gsr
