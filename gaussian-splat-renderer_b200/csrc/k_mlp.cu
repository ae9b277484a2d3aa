// Training and encoding of the learned colour stage (mlp.cuh); no reference counterpart. The
// plain SH evaluation (evalSH, splat_math.cpp:129-151) is the teacher, the judge of every
// gaussian (the fallback gate) and the colour of the gaussians that fail the gate.
//
// Samples are (gaussian g, direction j < dirs) pairs; direction j of gaussian g is a uniform
// point on the sphere from a hash of (g, j), the same in training and in the gate. A training
// step draws `batch` pairs from a hash of (seed, step, k), so the run is reproducible bit for bit.
//
//   trainStep   on the tensor cores: a 128-thread block takes 256 samples in chunks of 64, each
//               warp 16 of them. Forward (BF16 weights and activations, FP32 accumulation, the
//               latent rounded to fp16 then BF16 as the tensor-core decode sees it), loss and
//               backward (straight through the roundings) are mma.sync.m16n8k16 products whose
//               fragments come from shared memory by ldmatrix; the weight gradients are products
//               over the chunk's samples (activations transposed by ldmatrix.trans), kept in
//               registers across the chunks and written once as the block's partial sums (no
//               atomics: the run is reproducible bit for bit)
//   adamStep    one thread per parameter: the batch gradient from the partial sums, Adam
//   encode      latents of every gaussian (fp32 encoder, stored fp16)
//   gate        per gaussian, the tensor-core decode on its directions against the SH colour;
//               max channel error above the gate -> fallback (the latent's last half = NaN)
#include "kernels.cuh"
#include "mlp.cuh"
#include "splat_math.cuh"

namespace gsr {

namespace {

// The tensor-core training step: blocks of 4 warps, chunks of 64 samples (16 per warp), 4
// chunks (256 samples) a block. Row strides of the shared-memory matrices are K + 8 BF16 so
// that the 8 rows an ldmatrix reads fall into distinct banks.
constexpr int kTcWarps = 4, kTcThreads = kTcWarps * 32, kTcChunk = kTcWarps * 16, kTcChunks = 4;
constexpr int kTcBlockSamples = kTcChunk * kTcChunks;
constexpr int S48 = kEncIn + 8, S64 = kEncHidden + 8, S32 = kMlpHidden + 8, S16 = 16 + 8;

struct alignas(16) TrainSmem {
    // forward operands [n][k] (the weight matrices transposed), backward operands [n][k] = W[in][out]
    __nv_bfloat16 wt1e[kEncHidden][S48], wt2e[8][S64], wt1d[kMlpHidden][S16], wt2d[kMlpHidden][S32], wt3d[8][S32];
    __nv_bfloat16 wb3[kMlpHidden][S16], wb2[kMlpHidden][S32], wb1[kMlpLatent][S32], wb2e[kEncHidden][S16];
    // the chunk's activations and gradients, one row per sample
    __nv_bfloat16 x[kTcChunk][S48], h[kTcChunk][S64], in[kTcChunk][S16], a1[kTcChunk][S32], a2[kTcChunk][S32];
    __nv_bfloat16 dO[kTcChunk][S16], dA2[kTcChunk][S32], dA1[kTcChunk][S32], dZ[kTcChunk][S16], dH[kTcChunk][S64];
    float b1e[kEncHidden], b2e[8], b1d[kMlpHidden], b2d[kMlpHidden], b3d[8];
    float tgt[kTcChunk][4];
    float lossWarp[kTcWarps];
};

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) {
    return mix32(a * 0x9E3779B1u ^ mix32(b + 0x85EBCA77u) ^ mix32(c * 0xC2B2AE3Du + 0x27D4EB2Fu));
}
__device__ __forceinline__ float unit01(uint32_t h) { return float(h >> 8) * (1.0f / 16777216.0f); }

// Direction j of gaussian g: uniform on the sphere.
__device__ __forceinline__ void sampleDirection(uint32_t g, uint32_t j, float d[3]) {
    const float z = 1.0f - 2.0f * unit01(hash3(g, j, 0x51u));
    const float phi = 6.283185307179586f * unit01(hash3(g, j, 0xA7u));
    const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    d[0] = r * cosf(phi);
    d[1] = r * sinf(phi);
    d[2] = z;
}

__device__ __forceinline__ float latentRound(float z) { return bf16Round(__half2float(__float2half_rn(z))); }

struct TrainArgs {
    const float* sh;         // [N][48] decoded coefficients (zeros past the gaussian's degree)
    const uint8_t* degrees;  // [N]
    uint32_t count;
    uint32_t dirs;           // directions per gaussian
    uint32_t seed;
    const float* params;     // fp32 masters [kCount]
    float* partials;         // [blocks][kCount + 1] (the last float: the block's loss sum)
    const uint32_t* step;    // current step (device counter, advanced by adamStep)
};

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smemAddr(p)));
}
__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smemAddr(p)));
}
__device__ __forceinline__ void ldsm2(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(smemAddr(p)));
}
__device__ __forceinline__ void ldsm2t(uint32_t& r0, uint32_t& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(smemAddr(p)));
}

// One warp's 16 rows (rb..rb+15) of act (row-major, stride SA) times B ([n][k], stride SB):
// c[nt] += rows x B for n-tiles nt (columns 8 nt .. 8 nt + 7), K = 16 KSTEPS.
template <int KSTEPS, int NTILES, int SA, int SB>
__device__ __forceinline__ void rowsTimes(float (&c)[NTILES][4], const __nv_bfloat16 (*act)[SA], int rb,
                                          const __nv_bfloat16 (*B)[SB]) {
    const int lane = threadIdx.x & 31, j = lane >> 3, i = lane & 7;
#pragma unroll
    for (int ks = 0; ks < KSTEPS; ++ks) {
        uint32_t a[4];
        ldsm4(a, &act[rb + (j & 1) * 8 + i][ks * 16 + (j >> 1) * 8]);
#pragma unroll
        for (int nt = 0; nt < NTILES; ++nt) {
            uint32_t b0, b1;
            ldsm2(b0, b1, &B[nt * 8 + i][ks * 16 + (j & 1) * 8]);
            mmaBf16(c[nt], a, b0, b1);
        }
    }
}

// c (16 x 8 tile) -> BF16 rows of out; op applied per element with its column
template <int S, typename Op>
__device__ __forceinline__ void storeTile(__nv_bfloat16 (*out)[S], int rb, int n0, const float (&c)[4], Op op) {
    const int lane = threadIdx.x & 31, g = lane >> 2, col = n0 + (lane & 3) * 2;
    *reinterpret_cast<uint32_t*>(&out[rb + g][col]) = packBf16(op(c[0], rb + g, col), op(c[1], rb + g, col + 1));
    *reinterpret_cast<uint32_t*>(&out[rb + g + 8][col]) = packBf16(op(c[2], rb + g + 8, col), op(c[3], rb + g + 8, col + 1));
}

// The chunk's weight-gradient tiles (16 x 8 each): dW1e 48 x 64 (3 x 8 tiles), dW2e 64 x 8
// (4 x 1), dW1d 16 x 32 (1 x 4; rows 11..15 are padding), dW2d 32 x 32 (2 x 4), dW3d 32 x 8
// (2 x 1); tile t goes to warp t mod 4.
constexpr int kGradTiles = 24 + 4 + 4 + 8 + 2;
constexpr int kTilesPerWarp = (kGradTiles + kTcWarps - 1) / kTcWarps;
struct GradTile {
    int mat, m0, n0;
};
__device__ __forceinline__ GradTile gradTile(int t) {
    if (t < 24) return {0, (t / 8) * 16, (t % 8) * 8};
    t -= 24;
    if (t < 4) return {1, t * 16, 0};
    t -= 4;
    if (t < 4) return {2, 0, t * 8};
    t -= 4;
    if (t < 8) return {3, (t / 4) * 16, (t % 4) * 8};
    t -= 8;
    return {4, t * 16, 0};
}

// acc += act^T (rows m0.., the chunk's samples as K) x grad (columns n0..n0+7)
template <int SA, int SG>
__device__ __forceinline__ void gradTimes(float (&acc)[4], const __nv_bfloat16 (*act)[SA], int m0,
                                          const __nv_bfloat16 (*grad)[SG], int n0) {
    const int lane = threadIdx.x & 31, j = lane >> 3, i = lane & 7;
#pragma unroll
    for (int ks = 0; ks < kTcChunk / 16; ++ks) {
        uint32_t a[4], b0, b1;
        ldsm4t(a, &act[ks * 16 + (j >> 1) * 8 + i][m0 + (j & 1) * 8]);
        ldsm2t(b0, b1, &grad[ks * 16 + (j & 1) * 8 + i][n0]);
        mmaBf16(acc, a, b0, b1);
    }
}

__global__ void __launch_bounds__(kTcThreads) trainStepKernel(const __grid_constant__ TrainArgs a) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smemRaw);
    using L = MlpLayout;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tig = lane & 3;
    const float* P = a.params;
    auto bf = [](float v) { return __float2bfloat16_rn(v); };
    // weights in both layouts (padding zero), biases, and the constant zero columns
    for (int e = tid; e < kEncHidden * S48; e += kTcThreads) {
        const int o = e / S48, i = e % S48;
        S.wt1e[o][i] = bf(i < kEncIn ? P[L::kEncW1 + i * kEncHidden + o] : 0.0f);
    }
    for (int e = tid; e < 8 * S64; e += kTcThreads) {
        const int o = e / S64, i = e % S64;
        S.wt2e[o][i] = bf(i < kEncHidden ? P[L::kEncW2 + i * kMlpLatent + o] : 0.0f);
    }
    for (int e = tid; e < kMlpHidden * S16; e += kTcThreads) {
        const int o = e / S16, i = e % S16;
        S.wt1d[o][i] = bf(i < kMlpIn ? P[L::kDecW1 + i * kMlpHidden + o] : 0.0f);
        S.wb3[o][i] = bf(i < kMlpOut ? P[L::kDecW3 + o * kMlpOut + i] : 0.0f);
    }
    for (int e = tid; e < kMlpHidden * S32; e += kTcThreads) {
        const int r = e / S32, c = e % S32;
        S.wt2d[r][c] = bf(c < kMlpHidden ? P[L::kDecW2 + c * kMlpHidden + r] : 0.0f);
        S.wb2[r][c] = bf(c < kMlpHidden ? P[L::kDecW2 + r * kMlpHidden + c] : 0.0f);
    }
    for (int e = tid; e < 8 * S32; e += kTcThreads) {
        const int r = e / S32, c = e % S32;
        S.wt3d[r][c] = bf(r < kMlpOut && c < kMlpHidden ? P[L::kDecW3 + c * kMlpOut + r] : 0.0f);
        S.wb1[r][c] = bf(c < kMlpHidden ? P[L::kDecW1 + r * kMlpHidden + c] : 0.0f);  // the latent rows of W1d
    }
    for (int e = tid; e < kEncHidden * S16; e += kTcThreads) {
        const int r = e / S16, c = e % S16;
        S.wb2e[r][c] = bf(c < kMlpLatent ? P[L::kEncW2 + r * kMlpLatent + c] : 0.0f);
    }
    for (int e = tid; e < kEncHidden; e += kTcThreads) S.b1e[e] = P[L::kEncB1 + e];
    for (int e = tid; e < kMlpHidden; e += kTcThreads) {
        S.b1d[e] = P[L::kDecB1 + e];
        S.b2d[e] = P[L::kDecB2 + e];
    }
    if (tid < 8) {
        S.b2e[tid] = P[L::kEncB2 + tid];
        S.b3d[tid] = tid < kMlpOut ? P[L::kDecB3 + tid] : 0.0f;
    }
    for (int e = tid; e < kTcChunk * 8; e += kTcThreads) {
        const int r = e / 8, c = 8 + e % 8;
        S.in[r][c] = bf(0.0f);  // columns 11..15 stay zero (8..10 are rewritten per chunk)
        S.dO[r][c] = bf(0.0f);
        S.dZ[r][c] = bf(0.0f);
    }
    __syncthreads();

    const uint32_t step = *a.step;
    const int rb = warp * 16;
    float acc[kTilesPerWarp][4];
#pragma unroll
    for (int q = 0; q < kTilesPerWarp; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.0f;
    float bsum[2] = {0.0f, 0.0f};  // bias gradients of columns tid and tid + 128 of [dH | dZ | dA1 | dA2 | dO]
    float loss = 0.0f;
    for (int chunk = 0; chunk < kTcChunks; ++chunk) {
        // ---- the chunk's samples: (gaussian, direction), SH coefficients and the SH colour
        if (tid < kTcChunk) {
            const uint32_t k = blockIdx.x * kTcBlockSamples + chunk * kTcChunk + tid;
            const uint32_t gs = uint32_t((uint64_t(hash3(a.seed, step, k)) * a.count) >> 32);
            const uint32_t jd = hash3(a.seed ^ 0x5bd1e995u, step, k) % a.dirs;
            float dir[3], target[3];
            sampleDirection(gs, jd, dir);
            const float* shg = a.sh + size_t(gs) * kEncIn;
            evalSH(int(a.degrees[gs]), shg, dir[0], dir[1], dir[2], target);
            const float4* sh4 = reinterpret_cast<const float4*>(shg);
#pragma unroll
            for (int q = 0; q < kEncIn / 4; ++q) {
                const float4 v = __ldg(&sh4[q]);
                *reinterpret_cast<uint32_t*>(&S.x[tid][4 * q]) = packBf16(v.x, v.y);
                *reinterpret_cast<uint32_t*>(&S.x[tid][4 * q + 2]) = packBf16(v.z, v.w);
            }
            for (int c = 0; c < 3; ++c) {
                S.in[tid][kMlpLatent + c] = bf(dir[c]);
                S.tgt[tid][c] = target[c];
            }
        }
        __syncthreads();
        // ---- forward, each warp its 16 rows
        {
            float c[8][4];
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int col = nt * 8 + tig * 2;
                c[nt][0] = c[nt][2] = S.b1e[col];
                c[nt][1] = c[nt][3] = S.b1e[col + 1];
            }
            rowsTimes<3, 8>(c, S.x, rb, S.wt1e);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) storeTile(S.h, rb, nt * 8, c[nt], [](float v, int, int) { return fmaxf(v, 0.0f); });
        }
        __syncwarp();
        {
            float c[1][4];
            c[0][0] = c[0][2] = S.b2e[tig * 2];
            c[0][1] = c[0][3] = S.b2e[tig * 2 + 1];
            rowsTimes<4, 1>(c, S.h, rb, S.wt2e);
            storeTile(S.in, rb, 0, c[0], [](float v, int, int) { return latentRound(v); });
        }
        __syncwarp();
        {
            float c[4][4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int col = nt * 8 + tig * 2;
                c[nt][0] = c[nt][2] = S.b1d[col];
                c[nt][1] = c[nt][3] = S.b1d[col + 1];
            }
            rowsTimes<1, 4>(c, S.in, rb, S.wt1d);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) storeTile(S.a1, rb, nt * 8, c[nt], [](float v, int, int) { return fmaxf(v, 0.0f); });
        }
        __syncwarp();
        {
            float c[4][4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int col = nt * 8 + tig * 2;
                c[nt][0] = c[nt][2] = S.b2d[col];
                c[nt][1] = c[nt][3] = S.b2d[col + 1];
            }
            rowsTimes<2, 4>(c, S.a1, rb, S.wt2d);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) storeTile(S.a2, rb, nt * 8, c[nt], [](float v, int, int) { return fmaxf(v, 0.0f); });
        }
        __syncwarp();
        {
            float c[1][4];
            c[0][0] = c[0][2] = S.b3d[tig * 2];
            c[0][1] = c[0][3] = S.b3d[tig * 2 + 1];
            rowsTimes<2, 1>(c, S.a2, rb, S.wt3d);
            // sigmoid, squared error against the SH colour, d loss / d pre-sigmoid
            storeTile(S.dO, rb, 0, c[0], [&](float v, int row, int col) {
                if (col >= kMlpOut) return 0.0f;
                const float y = 1.0f / (1.0f + expf(-v));
                const float e = y - S.tgt[row - 0][col];
                loss += e * e;
                return 2.0f * e * y * (1.0f - y);
            });
        }
        __syncwarp();
        // ---- backward (activations are post-ReLU: > 0 means the unit was active)
        auto activeIn = [](const __nv_bfloat16(*act)[S32]) {
            return [act](float v, int row, int col) { return __bfloat162float(act[row][col]) > 0.0f ? v : 0.0f; };
        };
        {
            float c[4][4] = {};
            rowsTimes<1, 4>(c, S.dO, rb, S.wb3);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) storeTile(S.dA2, rb, nt * 8, c[nt], activeIn(S.a2));
        }
        __syncwarp();
        {
            float c[4][4] = {};
            rowsTimes<2, 4>(c, S.dA2, rb, S.wb2);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) storeTile(S.dA1, rb, nt * 8, c[nt], activeIn(S.a1));
        }
        __syncwarp();
        {
            float c[1][4] = {};
            rowsTimes<2, 1>(c, S.dA1, rb, S.wb1);  // straight through the latent's roundings
            storeTile(S.dZ, rb, 0, c[0], [](float v, int, int) { return v; });
        }
        __syncwarp();
        {
            float c[8][4] = {};
            rowsTimes<1, 8>(c, S.dZ, rb, S.wb2e);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
                storeTile(S.dH, rb, nt * 8, c[nt],
                          [&](float v, int row, int col) { return __bfloat162float(S.h[row][col]) > 0.0f ? v : 0.0f; });
        }
        __syncthreads();
        // ---- the chunk's weight gradients (tiles of this warp) and bias gradients
#pragma unroll
        for (int q = 0; q < kTilesPerWarp; ++q) {
            const int t = warp + q * kTcWarps;
            if (t >= kGradTiles) break;
            const GradTile gt = gradTile(t);
            switch (gt.mat) {
                case 0: gradTimes(acc[q], S.x, gt.m0, S.dH, gt.n0); break;
                case 1: gradTimes(acc[q], S.h, gt.m0, S.dZ, gt.n0); break;
                case 2: gradTimes(acc[q], S.in, gt.m0, S.dA1, gt.n0); break;
                case 3: gradTimes(acc[q], S.a1, gt.m0, S.dA2, gt.n0); break;
                default: gradTimes(acc[q], S.a2, gt.m0, S.dO, gt.n0); break;
            }
        }
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
            const int col = tid + h2 * kTcThreads;
            float sum = 0.0f;
            for (int r = 0; r < kTcChunk; ++r) {
                const __nv_bfloat16 v = col < 64    ? S.dH[r][col]
                                        : col < 72  ? S.dZ[r][col - 64]
                                        : col < 104 ? S.dA1[r][col - 72]
                                        : col < 136 ? S.dA2[r][col - 104]
                                        : col < 139 ? S.dO[r][col - 136]
                                                    : __float2bfloat16_rn(0.0f);
                sum += __bfloat162float(v);
            }
            bsum[h2] += sum;
        }
        __syncthreads();  // the next chunk overwrites the rows
    }
    // ---- the block's partial sums
    float* part = a.partials + size_t(blockIdx.x) * (L::kCount + 1);
#pragma unroll
    for (int q = 0; q < kTilesPerWarp; ++q) {
        const int t = warp + q * kTcWarps;
        if (t >= kGradTiles) break;
        const GradTile gt = gradTile(t);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int m = gt.m0 + g + (e >> 1) * 8, n = gt.n0 + tig * 2 + (e & 1);
            int p = -1;
            if (gt.mat == 0) p = L::kEncW1 + m * kEncHidden + n;
            else if (gt.mat == 1) p = L::kEncW2 + m * kMlpLatent + n;
            else if (gt.mat == 2) p = m < kMlpIn ? L::kDecW1 + m * kMlpHidden + n : -1;
            else if (gt.mat == 3) p = L::kDecW2 + m * kMlpHidden + n;
            else p = n < kMlpOut ? L::kDecW3 + m * kMlpOut + n : -1;
            if (p >= 0) part[p] = acc[q][e];
        }
    }
#pragma unroll
    for (int h2 = 0; h2 < 2; ++h2) {
        const int col = tid + h2 * kTcThreads;
        const int p = col < 64 ? L::kEncB1 + col : col < 72 ? L::kEncB2 + col - 64 : col < 104 ? L::kDecB1 + col - 72
                      : col < 136 ? L::kDecB2 + col - 104 : col < 139 ? L::kDecB3 + col - 136 : -1;
        if (p >= 0) part[p] = bsum[h2];
    }
    for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    if (lane == 0) S.lossWarp[warp] = loss;
    __syncthreads();
    if (tid == 0) {
        float sum = 0.0f;
        for (int w = 0; w < kTcWarps; ++w) sum += S.lossWarp[w];
        part[L::kCount] = sum;
    }
}

struct AdamArgs {
    float* params;
    float* m;
    float* v;
    const float* partials;
    uint32_t blocks;   // partial sums per parameter
    float invBatch;
    float lr, beta1, beta2, eps;
    uint32_t* step;    // advanced here (t = step + 1 in the bias corrections)
    float* lossOut;    // mean squared error per pair of steps lossBase .. maxSteps - 1
    uint32_t lossBase;
    uint32_t maxSteps;
};

__global__ void adamStepKernel(const __grid_constant__ AdamArgs a) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t step = *a.step;
    if (p <= uint32_t(MlpLayout::kCount)) {
        float g = 0.0f;
        for (uint32_t b = 0; b < a.blocks; ++b) g += a.partials[size_t(b) * (MlpLayout::kCount + 1) + p];
        g *= a.invBatch;
        if (p == uint32_t(MlpLayout::kCount)) {
            if (step >= a.lossBase && step < a.maxSteps) a.lossOut[step - a.lossBase] = g / 3.0f;  // per channel
        } else {
            const float t = float(step + 1);
            const float m = a.beta1 * a.m[p] + (1.0f - a.beta1) * g;
            const float v = a.beta2 * a.v[p] + (1.0f - a.beta2) * g * g;
            a.m[p] = m;
            a.v[p] = v;
            const float mh = m / (1.0f - powf(a.beta1, t));
            const float vh = v / (1.0f - powf(a.beta2, t));
            a.params[p] -= a.lr * mh / (sqrtf(vh) + a.eps);
        }
    }
    __syncthreads();
    // the step counter advances once every parameter of this launch has read it: the last
    // block to finish (grid-wide) bumps it
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(a.step + 1, 1u);
        if (done == gridDim.x - 1) {
            a.step[1] = 0;
            __threadfence();
            atomicAdd(a.step, 1u);
        }
    }
}

// Latents of every gaussian (one thread per gaussian), stored as fp16: the encoder with the
// training's roundings (BF16 coefficients, weights and hidden units, FP32 sums).
__global__ void __launch_bounds__(128) encodeLatentsKernel(const float* __restrict__ sh, const float* __restrict__ params,
                                                           uint4* __restrict__ latents, uint32_t count) {
    __shared__ float W[MlpLayout::kDecW1];  // the encoder part
    for (int p = threadIdx.x; p < MlpLayout::kDecW1; p += blockDim.x)
        W[p] = (p >= MlpLayout::kEncB1 && p < MlpLayout::kEncW2) || p >= MlpLayout::kEncB2 ? params[p] : bf16Round(params[p]);
    __syncthreads();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= count) return;
    using L = MlpLayout;
    float x[kEncIn];
    for (int i = 0; i < kEncIn; ++i) x[i] = bf16Round(sh[size_t(g) * kEncIn + i]);
    float z[kMlpLatent];
    for (int o = 0; o < kMlpLatent; ++o) z[o] = W[L::kEncB2 + o];
    for (int hdn = 0; hdn < kEncHidden; ++hdn) {
        float v = W[L::kEncB1 + hdn];
        for (int i = 0; i < kEncIn; ++i) v += x[i] * W[L::kEncW1 + i * kEncHidden + hdn];
        v = bf16Round(fmaxf(v, 0.0f));
        for (int o = 0; o < kMlpLatent; ++o) z[o] += v * W[L::kEncW2 + hdn * kMlpLatent + o];
    }
    uint32_t w[4];
    for (int q = 0; q < 4; ++q)
        w[q] = uint32_t(__half_as_ushort(__float2half_rn(z[2 * q]))) |
               (uint32_t(__half_as_ushort(__float2half_rn(z[2 * q + 1]))) << 16);
    latents[g] = make_uint4(w[0], w[1], w[2], w[3]);
}

// The tensor-core decoder weights from the fp32 masters.
__global__ void packDecoderKernel(const float* __restrict__ params, DecoderWeights* out) {
    using L = MlpLayout;
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
        const int n = e / 16, k = e % 16;
        out->w1[n][k] = __float2bfloat16_rn(k < kMlpIn ? params[L::kDecW1 + k * kMlpHidden + n] : 0.0f);
    }
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int n = e / 32, k = e % 32;
        out->w2[n][k] = __float2bfloat16_rn(params[L::kDecW2 + k * kMlpHidden + n]);
    }
    for (int e = threadIdx.x; e < 8 * 32; e += blockDim.x) {
        const int n = e / 32, k = e % 32;
        out->w3[n][k] = __float2bfloat16_rn(n < kMlpOut ? params[L::kDecW3 + k * kMlpOut + n] : 0.0f);
    }
    for (int e = threadIdx.x; e < 32; e += blockDim.x) {
        out->b1[e] = params[L::kDecB1 + e];
        out->b2[e] = params[L::kDecB2 + e];
    }
    for (int e = threadIdx.x; e < 8; e += blockDim.x) out->b3[e] = e < kMlpOut ? params[L::kDecB3 + e] : 0.0f;
}

// The gate: one warp per gaussian at a time, 32 directions per decode.
struct GateArgs {
    const float* sh;
    const uint8_t* degrees;
    uint32_t count, dirs;
    const DecoderWeights* decoder;
    uint4* latents;          // fallback gaussians get the NaN marker
    float gate;              // max channel error allowed
    uint32_t* fallbackCount;
    uint32_t* maxErrorBits;  // max over the kept gaussians (float bits, non-negative)
};

constexpr int kGateWarps = 8;
__global__ void __launch_bounds__(kGateWarps * 32) gateKernel(const __grid_constant__ GateArgs a) {
    __shared__ DecoderWeights W;
    __shared__ __nv_bfloat16 stage[kGateWarps][32][16];
    __shared__ float out4[kGateWarps][32][4];
    for (int e = threadIdx.x; e < int(sizeof(DecoderWeights) / 4); e += blockDim.x)
        reinterpret_cast<uint32_t*>(&W)[e] = reinterpret_cast<const uint32_t*>(a.decoder)[e];
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t warpsTotal = gridDim.x * kGateWarps;
    uint32_t fallbacks = 0, keptMax = 0;
    for (uint32_t g = blockIdx.x * kGateWarps + warp; g < a.count; g += warpsTotal) {
        const uint4 q = a.latents[g];
        float feat[kMlpIn];
        const uint32_t qw[4] = {q.x, q.y, q.z, q.w};
        for (int i = 0; i < kMlpLatent; ++i)
            feat[i] = __half2float(__ushort_as_half(uint16_t(qw[i >> 1] >> (16 * (i & 1)))));
        float err = 0.0f;
        bool nan = false;
        for (uint32_t j0 = 0; j0 < a.dirs; j0 += 32) {
            const uint32_t j = j0 + lane;
            float dir[3];
            sampleDirection(g, j < a.dirs ? j : 0u, dir);
            for (int c = 0; c < 3; ++c) feat[kMlpLatent + c] = dir[c];
            float rgb[3], ref[3];
            mlpDecodeWarp(W, feat, stage[warp], out4[warp], rgb);
            evalSH(int(a.degrees[g]), a.sh + size_t(g) * kEncIn, dir[0], dir[1], dir[2], ref);
            if (j < a.dirs) {
                for (int c = 0; c < 3; ++c) {
                    const float d = fabsf(rgb[c] - ref[c]);
                    nan |= d != d;
                    err = fmaxf(err, d);
                }
            }
        }
        // non-negative floats order like their bits
        err = __uint_as_float(__reduce_max_sync(0xFFFFFFFFu, __float_as_uint(err)));
        const bool fail = __any_sync(0xFFFFFFFFu, nan) || !(err <= a.gate);
        if (lane == 0) {
            if (fail) {
                uint4 m = q;
                m.w = (m.w & 0xFFFFu) | 0x7E000000u;  // half NaN in the last slot
                a.latents[g] = m;
                ++fallbacks;
            } else {
                keptMax = max(keptMax, __float_as_uint(err));
            }
        }
    }
    if (lane == 0) {
        if (fallbacks) atomicAdd(a.fallbackCount, fallbacks);
        atomicMax(a.maxErrorBits, keptMax);
    }
}

}  // namespace

cudaError_t launchColorTrainStep(const float* sh, const uint8_t* degrees, uint32_t count, uint32_t dirs, uint32_t seed,
                                 uint32_t batch, float* params, float* m, float* v, float* partials, uint32_t* step,
                                 float lr, float* lossOut, uint32_t lossBase, uint32_t maxSteps, cudaStream_t s) {
    static std::atomic<bool> configuredOn[64] = {};
    std::atomic<bool>& configured = perDevice(configuredOn);
    const int smem = int(sizeof(TrainSmem));
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(trainStepKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const uint32_t blocks = batch / kTcBlockSamples;
    TrainArgs ta{sh, degrees, count, dirs, seed, params, partials, step};
    trainStepKernel<<<blocks, kTcThreads, smem, s>>>(ta);
    AdamArgs aa{params, m, v, partials, blocks, 1.0f / float(batch), lr, 0.9f, 0.999f, 1e-8f, step, lossOut, lossBase,
                maxSteps};
    adamStepKernel<<<(MlpLayout::kCount + 1 + 255) / 256, 256, 0, s>>>(aa);
    return cudaGetLastError();
}

cudaError_t launchColorEncode(const float* sh, const float* params, uint4* latents, DecoderWeights* decoder,
                              uint32_t count, cudaStream_t s) {
    encodeLatentsKernel<<<(count + 127) / 128, 128, 0, s>>>(sh, params, latents, count);
    packDecoderKernel<<<1, 256, 0, s>>>(params, decoder);
    return cudaGetLastError();
}

cudaError_t launchPackDecoder(const float* params, DecoderWeights* decoder, cudaStream_t s) {
    packDecoderKernel<<<1, 256, 0, s>>>(params, decoder);
    return cudaGetLastError();
}

cudaError_t launchColorGate(const float* sh, const uint8_t* degrees, uint32_t count, uint32_t dirs,
                            const DecoderWeights* decoder, uint4* latents, float gate, uint32_t* fallbackCount,
                            uint32_t* maxErrorBits, cudaStream_t s) {
    GateArgs ga{sh, degrees, count, dirs, decoder, latents, gate, fallbackCount, maxErrorBits};
    gateKernel<<<148 * 8, kGateWarps * 32, 0, s>>>(ga);
    return cudaGetLastError();
}

uint32_t colorTrainBatchMultiple() { return kTcBlockSamples; }

}  // namespace gsr
