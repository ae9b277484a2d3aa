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
    void* out[4];
};

cudaError_t launchEncodeDegrees(const EncodeArgs& a, uint8_t* degrees, uint32_t* sizes, cudaStream_t s);
cudaError_t launchEncodeRecords(const EncodeArgs& a, const uint8_t* degrees, const uint32_t* offsets, cudaStream_t s);

}  // namespace gsr
