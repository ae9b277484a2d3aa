// Training and encoding of the learned colour stage (mlp.cuh); no reference counterpart. The
// plain SH evaluation (evalSH, splat_math.cpp:129-151) is the teacher, the judge of every
// gaussian (the fallback gate) and the colour of the gaussians that fail the gate.
//
// Samples are (gaussian g, direction j < dirs) pairs; direction j of gaussian g is a uniform
// point on the sphere from a hash of (g, j), the same in training and in the gate. A training
// step draws `batch` pairs from a hash of (seed, step, k), so the run is reproducible bit for bit.
//
//   trainStep   one thread per sample: forward (BF16-rounded weights and decoder activations, the
//               latent rounded to fp16 then BF16, as the tensor-core decode sees them), loss,
//               backward (straight through the roundings); then the block's weight gradients
//               over its 64 samples, written as the block's partial sums (no atomics)
//   adamStep    one thread per parameter: the batch gradient from the partial sums, Adam
//   encode      latents of every gaussian (fp32 encoder, stored fp16)
//   gate        per gaussian, the tensor-core decode on its directions against the SH colour;
//               max channel error above the gate -> fallback (the latent's last half = NaN)
#include "kernels.cuh"
#include "mlp.cuh"
#include "splat_math.cuh"

namespace gsr {

namespace {

constexpr int kTrainThreads = 64;
constexpr int kActStride = kTrainThreads + 1;  // per-sample vectors stored [element][sample], padded
// per-sample vectors kept for the weight gradients
constexpr int kOffX = 0, kOffH = kOffX + kEncIn, kOffIn = kOffH + kEncHidden, kOffA1 = kOffIn + kMlpIn,
              kOffA2 = kOffA1 + kMlpHidden, kOffDH = kOffA2 + kMlpHidden, kOffDZ = kOffDH + kEncHidden,
              kOffDA1 = kOffDZ + kMlpLatent, kOffDA2 = kOffDA1 + kMlpHidden, kOffDO = kOffDA2 + kMlpHidden,
              kActRows = kOffDO + kMlpOut;
constexpr int kTrainSmemFloats = MlpLayout::kCount + 1 + kActRows * kActStride;

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

__global__ void __launch_bounds__(kTrainThreads) trainStepKernel(const __grid_constant__ TrainArgs a) {
    extern __shared__ float sm[];
    float* W = sm;                                   // BF16-rounded weights (encoder fp32)
    float* act = sm + MlpLayout::kCount + 1;         // [kActRows][kActStride]
    const uint32_t s = threadIdx.x;
    using L = MlpLayout;
    for (int p = s; p < L::kCount; p += kTrainThreads)
        W[p] = p >= L::kDecW1 ? bf16Round(a.params[p]) : a.params[p];
    __syncthreads();
    auto A = [&](int row) -> float& { return act[row * kActStride + s]; };
    const uint32_t step = *a.step;
    const uint32_t k = blockIdx.x * kTrainThreads + s;
    const uint32_t h = hash3(a.seed, step, k);
    const uint32_t g = uint32_t((uint64_t(h) * a.count) >> 32);
    const uint32_t j = hash3(a.seed ^ 0x5bd1e995u, step, k) % a.dirs;
    float dir[3];
    sampleDirection(g, j, dir);
    float target[3];
    const float* shg = a.sh + size_t(g) * kEncIn;
    evalSH(int(a.degrees[g]), shg, dir[0], dir[1], dir[2], target);
    // ---- forward
    for (int i = 0; i < kEncIn; ++i) A(kOffX + i) = shg[i];
    for (int o = 0; o < kEncHidden; ++o) {
        float v = W[L::kEncB1 + o];
        for (int i = 0; i < kEncIn; ++i) v += A(kOffX + i) * W[L::kEncW1 + i * kEncHidden + o];
        A(kOffH + o) = fmaxf(v, 0.0f);
    }
    for (int o = 0; o < kMlpLatent; ++o) {
        float v = W[L::kEncB2 + o];
        for (int i = 0; i < kEncHidden; ++i) v += A(kOffH + i) * W[L::kEncW2 + i * kMlpLatent + o];
        A(kOffIn + o) = latentRound(v);
    }
    for (int c = 0; c < 3; ++c) A(kOffIn + kMlpLatent + c) = bf16Round(dir[c]);
    for (int o = 0; o < kMlpHidden; ++o) {
        float v = W[L::kDecB1 + o];
        for (int i = 0; i < kMlpIn; ++i) v += A(kOffIn + i) * W[L::kDecW1 + i * kMlpHidden + o];
        A(kOffA1 + o) = bf16Round(fmaxf(v, 0.0f));
    }
    for (int o = 0; o < kMlpHidden; ++o) {
        float v = W[L::kDecB2 + o];
        for (int i = 0; i < kMlpHidden; ++i) v += A(kOffA1 + i) * W[L::kDecW2 + i * kMlpHidden + o];
        A(kOffA2 + o) = bf16Round(fmaxf(v, 0.0f));
    }
    float loss = 0.0f;
    for (int o = 0; o < kMlpOut; ++o) {
        float v = W[L::kDecB3 + o];
        for (int i = 0; i < kMlpHidden; ++i) v += A(kOffA2 + i) * W[L::kDecW3 + i * kMlpOut + o];
        const float y = 1.0f / (1.0f + expf(-v));
        const float e = y - target[o];
        loss += e * e;
        A(kOffDO + o) = 2.0f * e * y * (1.0f - y);  // d loss / d pre-sigmoid
    }
    // ---- backward (activations are post-ReLU: > 0 means the unit was active)
    for (int i = 0; i < kMlpHidden; ++i) {
        float v = 0.0f;
        for (int o = 0; o < kMlpOut; ++o) v += W[L::kDecW3 + i * kMlpOut + o] * A(kOffDO + o);
        A(kOffDA2 + i) = A(kOffA2 + i) > 0.0f ? v : 0.0f;
    }
    for (int i = 0; i < kMlpHidden; ++i) {
        float v = 0.0f;
        for (int o = 0; o < kMlpHidden; ++o) v += W[L::kDecW2 + i * kMlpHidden + o] * A(kOffDA2 + o);
        A(kOffDA1 + i) = A(kOffA1 + i) > 0.0f ? v : 0.0f;
    }
    for (int i = 0; i < kMlpLatent; ++i) {
        float v = 0.0f;
        for (int o = 0; o < kMlpHidden; ++o) v += W[L::kDecW1 + i * kMlpHidden + o] * A(kOffDA1 + o);
        A(kOffDZ + i) = v;  // straight through the fp16/BF16 roundings of the latent
    }
    for (int i = 0; i < kEncHidden; ++i) {
        float v = 0.0f;
        for (int o = 0; o < kMlpLatent; ++o) v += W[L::kEncW2 + i * kMlpLatent + o] * A(kOffDZ + o);
        A(kOffDH + i) = A(kOffH + i) > 0.0f ? v : 0.0f;
    }
    // the block's loss sum
    for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    __syncthreads();
    float* part = a.partials + size_t(blockIdx.x) * (L::kCount + 1);
    if ((s & 31) == 0) atomicAdd(&part[L::kCount], loss);  // two warps; the slot is zeroed below first
    // ---- weight gradients of the block: parameter p sums over the block's samples
    for (int p = s; p < L::kCount; p += kTrainThreads) {
        int u = -1, v = -1;  // rows of the two factors (u = -1: a bias, the factor is 1)
        if (p < L::kEncB1) { u = kOffX + (p - L::kEncW1) / kEncHidden; v = kOffDH + (p - L::kEncW1) % kEncHidden; }
        else if (p < L::kEncW2) { v = kOffDH + (p - L::kEncB1); }
        else if (p < L::kEncB2) { u = kOffH + (p - L::kEncW2) / kMlpLatent; v = kOffDZ + (p - L::kEncW2) % kMlpLatent; }
        else if (p < L::kDecW1) { v = kOffDZ + (p - L::kEncB2); }
        else if (p < L::kDecB1) { u = kOffIn + (p - L::kDecW1) / kMlpHidden; v = kOffDA1 + (p - L::kDecW1) % kMlpHidden; }
        else if (p < L::kDecW2) { v = kOffDA1 + (p - L::kDecB1); }
        else if (p < L::kDecB2) { u = kOffA1 + (p - L::kDecW2) / kMlpHidden; v = kOffDA2 + (p - L::kDecW2) % kMlpHidden; }
        else if (p < L::kDecW3) { v = kOffDA2 + (p - L::kDecB2); }
        else if (p < L::kDecB3) { u = kOffA2 + (p - L::kDecW3) / kMlpOut; v = kOffDO + (p - L::kDecW3) % kMlpOut; }
        else { v = kOffDO + (p - L::kDecB3); }
        float sum = 0.0f;
        const float* vr = act + v * kActStride;
        if (u < 0) {
            for (int t = 0; t < kTrainThreads; ++t) sum += vr[t];
        } else {
            const float* ur = act + u * kActStride;
            for (int t = 0; t < kTrainThreads; ++t) sum += ur[t] * vr[t];
        }
        part[p] = sum;
    }
}

__global__ void zeroLossSlotsKernel(float* partials, uint32_t blocks) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < blocks) partials[size_t(b) * (MlpLayout::kCount + 1) + MlpLayout::kCount] = 0.0f;
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
    float* lossOut;    // [steps] mean squared error per pair of each step
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
            if (step < a.maxSteps) a.lossOut[step] = g / 3.0f;  // per channel
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

// Latents of every gaussian: the fp32 encoder (one thread per gaussian), stored as fp16.
__global__ void __launch_bounds__(128) encodeLatentsKernel(const float* __restrict__ sh, const float* __restrict__ params,
                                                           uint4* __restrict__ latents, uint32_t count) {
    __shared__ float W[MlpLayout::kDecW1];  // the encoder part
    for (int p = threadIdx.x; p < MlpLayout::kDecW1; p += blockDim.x) W[p] = params[p];
    __syncthreads();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= count) return;
    using L = MlpLayout;
    float x[kEncIn];
    for (int i = 0; i < kEncIn; ++i) x[i] = sh[size_t(g) * kEncIn + i];
    float z[kMlpLatent];
    for (int o = 0; o < kMlpLatent; ++o) z[o] = W[L::kEncB2 + o];
    for (int hdn = 0; hdn < kEncHidden; ++hdn) {
        float v = W[L::kEncB1 + hdn];
        for (int i = 0; i < kEncIn; ++i) v += x[i] * W[L::kEncW1 + i * kEncHidden + hdn];
        v = fmaxf(v, 0.0f);
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
                                 float lr, float* lossOut, uint32_t maxSteps, cudaStream_t s) {
    static std::atomic<bool> configuredOn[64] = {};
    std::atomic<bool>& configured = perDevice(configuredOn);
    const int smem = kTrainSmemFloats * 4;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(trainStepKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const uint32_t blocks = batch / kTrainThreads;
    zeroLossSlotsKernel<<<(blocks + 255) / 256, 256, 0, s>>>(partials, blocks);
    TrainArgs ta{sh, degrees, count, dirs, seed, params, partials, step};
    trainStepKernel<<<blocks, kTrainThreads, smem, s>>>(ta);
    AdamArgs aa{params, m, v, partials, blocks, 1.0f / float(batch), lr, 0.9f, 0.999f, 1e-8f, step, lossOut, maxSteps};
    adamStepKernel<<<(MlpLayout::kCount + 1 + 255) / 256, 256, 0, s>>>(aa);
    return cudaGetLastError();
}

cudaError_t launchColorEncode(const float* sh, const float* params, uint4* latents, DecoderWeights* decoder,
                              uint32_t count, cudaStream_t s) {
    encodeLatentsKernel<<<(count + 127) / 128, 128, 0, s>>>(sh, params, latents, count);
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

uint32_t colorTrainBatchMultiple() { return kTrainThreads; }

}  // namespace gsr
