// Arguments of the GPU scene encoder (k_encode.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gsr_b200.h"

namespace gsr {

struct EncodeArgs {
    const float4* pa;   // source posAlpha [n]
    const float4* sc;   // source scales [n]
    const float4* ro;   // source rotations [n]
    const float* sh;    // source sh [n * srcK * 3]
    uint32_t n, srcK;   // count, source K
    uint32_t K;         // stored K after max_sh_degree
    int degree;         // stored degree
    int variable;       // per-gaussian degree on
    float threshold255;
    uint32_t layout, geometry, color;
    uint32_t geomWords, colorWords;  // record words (fixed-size records)
    const uint32_t* cbIndex;         // cb: the codebook entry of every gaussian (null: entry 0)
    void* out[4];
};

cudaError_t launchEncodeDegrees(const EncodeArgs& a, uint8_t* degrees, uint32_t* sizes, cudaStream_t s);
cudaError_t launchEncodeRecords(const EncodeArgs& a, const uint8_t* degrees, const uint32_t* offsets, cudaStream_t s);

// The cb format's k-means on the device (kmeans.cpp): the SH-rest vectors (K - 1) * 3 of every
// gaussian (non-finite values as 0), a gather of the training sample, and the nearest centroid
// of `count` points (ties to the lowest index) with max(0, |x|^2 + min_j (|c_j|^2 - 2 x.c_j)).
cudaError_t launchCodebookPoints(const EncodeArgs& a, const uint8_t* degrees, float* points, cudaStream_t s);
cudaError_t launchCodebookGather(const float* points, uint32_t dims, const uint32_t* index, uint32_t count, float* out,
                                 cudaStream_t s);
cudaError_t launchNearestCentroid(const float* points, uint32_t count, uint32_t dims, const float* centroids,
                                  const float* norm2, uint32_t k, uint32_t* assignment, float* sqDist, cudaStream_t s);

}  // namespace gsr
