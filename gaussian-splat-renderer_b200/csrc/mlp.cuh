// The learned colour stage (no reference counterpart): a per-gaussian 8-dim fp16 latent, encoded
// from the gaussian's 48 SH coefficients, and one small MLP that decodes (latent, view direction)
// to RGB in place of the SH evaluation.
//
//   encoder  48 -> 64 (ReLU) -> 8                      (training and latent encoding only)
//   decoder  (8 latent + 3 direction) -> 32 (ReLU) -> 32 (ReLU) -> 3 (sigmoid)
//
// The decoder runs inside the preprocess on the tensor cores: one warp decodes the colours of
// its 32 gaussians as three chained mma.sync.m16n8k16 BF16 products with FP32 accumulation (the
// accumulator fragment of one layer is, after ReLU and BF16 rounding, the A fragment of the
// next). The matrices are tiny (K <= 32, N <= 32), so the stage is bound by the latent reads,
// not by tensor throughput. A gaussian whose decoded colour is more than the gate away from its
// SH colour on the training directions keeps the SH path: its latent's last half is NaN.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "kernels.cuh"

namespace gsr {

constexpr int kMlpIn = 11, kMlpHidden = 32, kMlpOut = 3, kMlpLatent = 8;
constexpr int kEncIn = 48, kEncHidden = 64;

// Parameter offsets (floats) in the fp32 master array (row-major W[in][out]).
struct MlpLayout {
    static constexpr int kEncW1 = 0;                                 // [48][64]
    static constexpr int kEncB1 = kEncW1 + kEncIn * kEncHidden;      // [64]
    static constexpr int kEncW2 = kEncB1 + kEncHidden;               // [64][8]
    static constexpr int kEncB2 = kEncW2 + kEncHidden * kMlpLatent;  // [8]
    static constexpr int kDecW1 = kEncB2 + kMlpLatent;               // [11][32]
    static constexpr int kDecB1 = kDecW1 + kMlpIn * kMlpHidden;      // [32]
    static constexpr int kDecW2 = kDecB1 + kMlpHidden;               // [32][32]
    static constexpr int kDecB2 = kDecW2 + kMlpHidden * kMlpHidden;  // [32]
    static constexpr int kDecW3 = kDecB2 + kMlpHidden;               // [32][3]
    static constexpr int kDecB3 = kDecW3 + kMlpHidden * kMlpOut;     // [3]
    static constexpr int kCount = kDecB3 + kMlpOut;                  // 5195
};

// The decoder for the tensor cores: each weight matrix transposed to [n][k] BF16 (k padded to a
// multiple of 16, n to a multiple of 8) so that a B fragment register is two consecutive k of
// one column; biases fp32, padded.
struct DecoderWeights {
    __nv_bfloat16 w1[32][16];  // [n][k], k = 0..10 used
    __nv_bfloat16 w2[32][32];
    __nv_bfloat16 w3[8][32];   // n = 0..2 used
    float b1[32], b2[32], b3[8];
};

static_assert(sizeof(DecoderWeights) == kDecoderWeightsBytes, "the host allocates kDecoderWeightsBytes");
static_assert(MlpLayout::kCount == int(kColorModelParams), "the host's parameter count");

__device__ __forceinline__ float bf16Round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t packBf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mmaBf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float sigmoidF(float x) { return 1.0f / (1.0f + __expf(-x)); }

// Decodes the colours of the warp's 32 rows; all 32 lanes call it. feat = the lane's row
// (latent 8, direction 3), stage = this warp's 32 x 16 BF16 staging area and out4 its 32 x 4
// fp32 result area in shared memory. Rows of lanes that need no colour may hold anything.
__device__ __forceinline__ void mlpDecodeWarp(const DecoderWeights& W, const float (&feat)[kMlpIn],
                                              __nv_bfloat16 (*stage)[16], float (*out4)[4], float (&rgb)[3]) {
    const uint32_t lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int k = 0; k < 16; ++k) stage[lane][k] = __float2bfloat16_rn(k < kMlpIn ? feat[k] : 0.0f);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t*>(&stage[r0][tig * 2]);
        a[1] = *reinterpret_cast<const uint32_t*>(&stage[r1][tig * 2]);
        a[2] = *reinterpret_cast<const uint32_t*>(&stage[r0][tig * 2 + 8]);
        a[3] = *reinterpret_cast<const uint32_t*>(&stage[r1][tig * 2 + 8]);
        // layer 1: 16 -> 32
        float c1[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int col = nt * 8 + tig * 2;
            c1[nt][0] = W.b1[col]; c1[nt][1] = W.b1[col + 1]; c1[nt][2] = W.b1[col]; c1[nt][3] = W.b1[col + 1];
            const int n = nt * 8 + g;
            mmaBf16(c1[nt], a, *reinterpret_cast<const uint32_t*>(&W.w1[n][tig * 2]),
                    *reinterpret_cast<const uint32_t*>(&W.w1[n][tig * 2 + 8]));
        }
        uint32_t a2[2][4];
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
            a2[kb][0] = packBf16(fmaxf(c1[2 * kb][0], 0.0f), fmaxf(c1[2 * kb][1], 0.0f));
            a2[kb][1] = packBf16(fmaxf(c1[2 * kb][2], 0.0f), fmaxf(c1[2 * kb][3], 0.0f));
            a2[kb][2] = packBf16(fmaxf(c1[2 * kb + 1][0], 0.0f), fmaxf(c1[2 * kb + 1][1], 0.0f));
            a2[kb][3] = packBf16(fmaxf(c1[2 * kb + 1][2], 0.0f), fmaxf(c1[2 * kb + 1][3], 0.0f));
        }
        // layer 2: 32 -> 32
        float c2[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int col = nt * 8 + tig * 2;
            c2[nt][0] = W.b2[col]; c2[nt][1] = W.b2[col + 1]; c2[nt][2] = W.b2[col]; c2[nt][3] = W.b2[col + 1];
            const int n = nt * 8 + g;
#pragma unroll
            for (int kb = 0; kb < 2; ++kb)
                mmaBf16(c2[nt], a2[kb], *reinterpret_cast<const uint32_t*>(&W.w2[n][kb * 16 + tig * 2]),
                        *reinterpret_cast<const uint32_t*>(&W.w2[n][kb * 16 + tig * 2 + 8]));
        }
        uint32_t a3[2][4];
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
            a3[kb][0] = packBf16(fmaxf(c2[2 * kb][0], 0.0f), fmaxf(c2[2 * kb][1], 0.0f));
            a3[kb][1] = packBf16(fmaxf(c2[2 * kb][2], 0.0f), fmaxf(c2[2 * kb][3], 0.0f));
            a3[kb][2] = packBf16(fmaxf(c2[2 * kb + 1][0], 0.0f), fmaxf(c2[2 * kb + 1][1], 0.0f));
            a3[kb][3] = packBf16(fmaxf(c2[2 * kb + 1][2], 0.0f), fmaxf(c2[2 * kb + 1][3], 0.0f));
        }
        // layer 3: 32 -> 8 (3 used)
        float c3[4];
        const int col = tig * 2;
        c3[0] = W.b3[col]; c3[1] = W.b3[col + 1]; c3[2] = W.b3[col]; c3[3] = W.b3[col + 1];
#pragma unroll
        for (int kb = 0; kb < 2; ++kb)
            mmaBf16(c3, a3[kb], *reinterpret_cast<const uint32_t*>(&W.w3[g][kb * 16 + tig * 2]),
                    *reinterpret_cast<const uint32_t*>(&W.w3[g][kb * 16 + tig * 2 + 8]));
        if (tig < 2) {
            out4[r0][col] = c3[0];
            out4[r0][col + 1] = c3[1];
            out4[r1][col] = c3[2];
            out4[r1][col + 1] = c3[3];
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < kMlpOut; ++c) rgb[c] = sigmoidF(out4[lane][c]);
    __syncwarp();  // the staging areas may be reused by the caller's next decode
}

// The fallback marker: a latent whose last half is NaN keeps the SH colour.
__device__ __forceinline__ bool latentIsFallback(const uint4& q) { return __hisnan(__ushort_as_half(uint16_t(q.w >> 16))); }

}  // namespace gsr
