// mlp.cu — inference (BF16 tensor cores, FP32 accumulate) and online training (FP32 forward /
// backward, deterministic reductions, Adam) of the warm-start MLP described in mlp.cuh.
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "dfsph_common.cuh"

namespace dfsph {

namespace {

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low 16 bits) = lo
    return *reinterpret_cast<uint32_t*>(&v);
}

// D += A (16x16, row) * B (16x8, col) with BF16 inputs and FP32 accumulation.
__device__ __forceinline__ void mma_bf16_16x8x16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-memory row strides (32-bit words) chosen so that the 8 row-groups of a fragment load hit
// distinct banks.
constexpr int kS1 = 12;  // W1: 16 BF16 = 8 words per row, padded
constexpr int kS2 = 36;  // W2 / W3: 64 BF16 = 32 words per row, padded

// One warp evaluates 16 particles per iteration: layer 1 (K = 16 with 5 real inputs), layer 2
// (K = 64), layer 3 (N = 8 with 2 real outputs). The FP32 accumulator fragment of an m16n8 tile is
// exactly the BF16 A-fragment layout of the next layer's k-chunk, so activations stay in registers.
__global__ void __launch_bounds__(128) mlp_forward_kernel(const uint16_t* __restrict__ w1b,
                                                          const uint16_t* __restrict__ w2b,
                                                          const uint16_t* __restrict__ w3b,
                                                          const float* __restrict__ params,
                                                          const MlpScales* __restrict__ scales,
                                                          const float* __restrict__ features, uint32_t n,
                                                          float* __restrict__ pred) {
    DFSPH_PDL_ENTER;
    __shared__ uint32_t sW1[kMlpHidden * kS1];
    __shared__ uint32_t sW2[kMlpHidden * kS2];
    __shared__ uint32_t sW3[8 * kS2];
    __shared__ float sB1[kMlpHidden], sB2[kMlpHidden], sB3[8], sIn[kMlpIn];
    const uint32_t* w1 = reinterpret_cast<const uint32_t*>(w1b);
    const uint32_t* w2 = reinterpret_cast<const uint32_t*>(w2b);
    const uint32_t* w3 = reinterpret_cast<const uint32_t*>(w3b);
    for (int t = threadIdx.x; t < kMlpHidden * 8; t += blockDim.x) sW1[(t / 8) * kS1 + t % 8] = w1[t];
    for (int t = threadIdx.x; t < kMlpHidden * 32; t += blockDim.x) sW2[(t / 32) * kS2 + t % 32] = w2[t];
    for (int t = threadIdx.x; t < 8 * 32; t += blockDim.x) sW3[(t / 32) * kS2 + t % 32] = w3[t];
    for (int t = threadIdx.x; t < kMlpHidden; t += blockDim.x) {
        sB1[t] = params[kB1 + t];
        sB2[t] = params[kB2 + t];
    }
    if (threadIdx.x < 8) sB3[threadIdx.x] = threadIdx.x < kMlpOut ? params[kB3 + threadIdx.x] : 0.0f;
    if (threadIdx.x < kMlpIn) sIn[threadIdx.x] = scales->in_scale[threadIdx.x];
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    for (uint32_t tile = (blockIdx.x * 4 + warp) * 16; tile < n; tile += gridDim.x * 4 * 16) {
        const uint32_t r0 = tile + g, r1 = tile + g + 8;
        float x00 = 0.f, x01 = 0.f, x10 = 0.f, x11 = 0.f;
        if (r0 < n) {
            const float2 f = *reinterpret_cast<const float2*>(features + (size_t)r0 * kMlpIn + 2 * q);
            x00 = f.x * sIn[2 * q];
            x01 = f.y * sIn[2 * q + 1];
        }
        if (r1 < n) {
            const float2 f = *reinterpret_cast<const float2*>(features + (size_t)r1 * kMlpIn + 2 * q);
            x10 = f.x * sIn[2 * q];
            x11 = f.y * sIn[2 * q + 1];
        }
        const uint32_t a0 = pack_bf16x2(x00, x01), a1 = pack_bf16x2(x10, x11);
        uint32_t h1[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4];
            c[0] = c[2] = sB1[8 * nt + 2 * q];
            c[1] = c[3] = sB1[8 * nt + 2 * q + 1];
            const uint32_t* row = sW1 + (8 * nt + g) * kS1;
            mma_bf16_16x8x16(c, a0, a1, 0u, 0u, row[q], row[4 + q]);
#pragma unroll
            for (int e = 0; e < 4; ++e) c[e] = fmaxf(c[e], 0.0f);
            h1[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16x2(c[0], c[1]);
            h1[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16x2(c[2], c[3]);
        }
        uint32_t h2[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4];
            c[0] = c[2] = sB2[8 * nt + 2 * q];
            c[1] = c[3] = sB2[8 * nt + 2 * q + 1];
            const uint32_t* row = sW2 + (8 * nt + g) * kS2;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                mma_bf16_16x8x16(c, h1[kk][0], h1[kk][1], h1[kk][2], h1[kk][3], row[8 * kk + q], row[8 * kk + 4 + q]);
#pragma unroll
            for (int e = 0; e < 4; ++e) c[e] = fmaxf(c[e], 0.0f);
            h2[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16x2(c[0], c[1]);
            h2[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16x2(c[2], c[3]);
        }
        float c[4];
        c[0] = c[2] = sB3[2 * q];
        c[1] = c[3] = sB3[2 * q + 1];
        const uint32_t* row = sW3 + g * kS2;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma_bf16_16x8x16(c, h2[kk][0], h2[kk][1], h2[kk][2], h2[kk][3], row[8 * kk + q], row[8 * kk + 4 + q]);
        if (q == 0) {  // columns 0 and 1 are the two outputs
            if (r0 < n) *reinterpret_cast<float2*>(pred + 2 * (size_t)r0) = make_float2(c[0], c[1]);
            if (r1 < n) *reinterpret_cast<float2*>(pred + 2 * (size_t)r1) = make_float2(c[2], c[3]);
        }
    }
}

__global__ void mlp_pack_kernel(const float* __restrict__ params, uint16_t* __restrict__ w1b,
                                uint16_t* __restrict__ w2b, uint16_t* __restrict__ w3b) {
    DFSPH_PDL_ENTER;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    auto bf = [](float v) {
        __nv_bfloat16 b = __float2bfloat16_rn(v);
        return *reinterpret_cast<uint16_t*>(&b);
    };
    if (t < kMlpHidden * 16) {
        const int j = t / 16, k = t % 16;
        w1b[t] = bf(k < kMlpIn ? params[kW1 + j * kMlpIn + k] : 0.0f);
    }
    if (t < kMlpHidden * kMlpHidden) w2b[t] = bf(params[kW2 + t]);
    if (t < 8 * kMlpHidden) {
        const int o = t / kMlpHidden, j = t % kMlpHidden;
        w3b[t] = bf(o < kMlpOut ? params[kW3 + o * kMlpHidden + j] : 0.0f);
    }
}

// Training block: 128 samples. Dynamic shared memory holds the FP32 weights, the batch and the
// activations / gradients of every sample; each thread runs one sample's forward and backward
// pass, then the block sums every parameter's gradient over its samples in sample order and
// writes one partial per block (plus the block's loss sum at index kMlpParams).
constexpr int kHp = kMlpHidden + 1;  // padded activation row
__global__ void __launch_bounds__(kTrainBlock) mlp_train_partials_kernel(const float* __restrict__ params,
                                                                        const MlpScales* __restrict__ scales,
                                                                        const float* __restrict__ x,
                                                                        const float* __restrict__ tgt, uint32_t batch,
                                                                        float* __restrict__ partials) {
    DFSPH_PDL_ENTER;
    extern __shared__ float sm[];
    float* W1 = sm;                                 // [64][8]
    float* B1 = W1 + kMlpHidden * kMlpIn;           // [64]
    float* W2 = B1 + kMlpHidden;                    // [64][64]
    float* B2 = W2 + kMlpHidden * kMlpHidden;       // [64]
    float* W3 = B2 + kMlpHidden;                    // [2][64]
    float* B3 = W3 + kMlpOut * kMlpHidden;          // [2] (+2 pad)
    float* X = B3 + 4;                              // [128][8]
    float* DY = X + kTrainBlock * kMlpIn;           // [128][2]
    float* LS = DY + kTrainBlock * kMlpOut;         // [128]
    float* H1 = LS + kTrainBlock;                   // [128][65]
    float* H2 = H1 + kTrainBlock * kHp;
    float* G1 = H2 + kTrainBlock * kHp;
    float* G2 = G1 + kTrainBlock * kHp;
    const int t = threadIdx.x;
    for (int p = t; p < kMlpParams; p += blockDim.x) sm[p] = params[p];
    const uint32_t s = blockIdx.x * kTrainBlock + t;
    const bool valid = s < batch;
    for (int i = 0; i < kMlpIn; ++i) X[t * kMlpIn + i] = valid ? x[(size_t)s * kMlpIn + i] * scales->in_scale[i] : 0.0f;
    __syncthreads();
    // forward
    for (int j = 0; j < kMlpHidden; ++j) {
        float a = B1[j];
        for (int i = 0; i < kMlpIn; ++i) a += W1[j * kMlpIn + i] * X[t * kMlpIn + i];
        H1[t * kHp + j] = fmaxf(a, 0.0f);
    }
    for (int j = 0; j < kMlpHidden; ++j) {
        float a = B2[j];
        for (int k = 0; k < kMlpHidden; ++k) a += W2[j * kMlpHidden + k] * H1[t * kHp + k];
        H2[t * kHp + j] = fmaxf(a, 0.0f);
    }
    float loss = 0.0f;
    for (int o = 0; o < kMlpOut; ++o) {
        float y = B3[o];
        for (int j = 0; j < kMlpHidden; ++j) y += W3[o * kMlpHidden + j] * H2[t * kHp + j];
        const float r = valid ? y - tgt[(size_t)s * kMlpOut + o] : 0.0f;
        loss += r * r;
        DY[t * kMlpOut + o] = 2.0f * r / (float)batch;  // d(mean over samples of sum over outputs)
    }
    LS[t] = loss;
    // backward
    for (int j = 0; j < kMlpHidden; ++j) {
        float a = 0.0f;
        for (int o = 0; o < kMlpOut; ++o) a += W3[o * kMlpHidden + j] * DY[t * kMlpOut + o];
        G2[t * kHp + j] = H2[t * kHp + j] > 0.0f ? a : 0.0f;
    }
    for (int k = 0; k < kMlpHidden; ++k) {
        float a = 0.0f;
        for (int j = 0; j < kMlpHidden; ++j) a += W2[j * kMlpHidden + k] * G2[t * kHp + j];
        G1[t * kHp + k] = H1[t * kHp + k] > 0.0f ? a : 0.0f;
    }
    __syncthreads();
    float* out = partials + (size_t)blockIdx.x * (kMlpParams + 1);
    for (int p = t; p < kMlpParams; p += blockDim.x) {
        float acc = 0.0f;
        if (p < kB1) {
            const int j = p / kMlpIn, i = p % kMlpIn;
            for (int u = 0; u < kTrainBlock; ++u) acc += G1[u * kHp + j] * X[u * kMlpIn + i];
        } else if (p < kW2) {
            const int j = p - kB1;
            for (int u = 0; u < kTrainBlock; ++u) acc += G1[u * kHp + j];
        } else if (p < kB2) {
            const int j = (p - kW2) / kMlpHidden, k = (p - kW2) % kMlpHidden;
            for (int u = 0; u < kTrainBlock; ++u) acc += G2[u * kHp + j] * H1[u * kHp + k];
        } else if (p < kW3) {
            const int j = p - kB2;
            for (int u = 0; u < kTrainBlock; ++u) acc += G2[u * kHp + j];
        } else if (p < kB3) {
            const int o = (p - kW3) / kMlpHidden, j = (p - kW3) % kMlpHidden;
            for (int u = 0; u < kTrainBlock; ++u) acc += DY[u * kMlpOut + o] * H2[u * kHp + j];
        } else {
            const int o = p - kB3;
            for (int u = 0; u < kTrainBlock; ++u) acc += DY[u * kMlpOut + o];
        }
        out[p] = acc;
    }
    if (t == 0) {
        float l = 0.0f;
        for (int u = 0; u < kTrainBlock; ++u) l += LS[u];
        out[kMlpParams] = l;
    }
}

// Sums the block partials in block order (deterministic) and optionally applies Adam.
__global__ void mlp_reduce_adam_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                       float* __restrict__ grad, const float* __restrict__ partials, int blocks,
                                       uint32_t batch, int adam, float lr, float beta1, float beta2, float eps,
                                       int step, double* __restrict__ loss) {
    DFSPH_PDL_ENTER;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kMlpParams) return;
    double acc = 0.0;
    for (int b = 0; b < blocks; ++b) acc += (double)partials[(size_t)b * (kMlpParams + 1) + p];
    if (p == kMlpParams) {
        *loss = acc / (double)batch;
        return;
    }
    const float gp = (float)acc;
    grad[p] = gp;
    if (adam) {
        const float mp = beta1 * m[p] + (1.0f - beta1) * gp;
        const float vp = beta2 * v[p] + (1.0f - beta2) * gp * gp;
        m[p] = mp;
        v[p] = vp;
        const float mh = mp / (1.0f - powf(beta1, (float)step));
        const float vh = vp / (1.0f - powf(beta2, (float)step));
        params[p] -= lr * mh / (sqrtf(vh) + eps);
    }
}

// splitmix64 hash of (seed, index) mapped to [-1, 1).
__device__ __forceinline__ float hash_uniform(uint32_t seed, uint32_t i) {
    unsigned long long z = ((unsigned long long)seed << 32) + i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((z >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
}

__global__ void mlp_init_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                uint32_t seed) {
    DFSPH_PDL_ENTER;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float val = 0.0f;
    if (p < kB1) {
        const int i = p % kMlpIn;
        val = i < 5 ? hash_uniform(seed, p) * sqrtf(6.0f / 5.0f) : 0.0f;  // He-uniform, 5 real inputs
    } else if (p >= kW2 && p < kB2) {
        val = hash_uniform(seed, p) * sqrtf(6.0f / (float)kMlpHidden);
    }
    params[p] = val;  // biases and the output layer start at zero: the first predictions are the base
    m[p] = 0.0f;
    v[p] = 0.0f;
}

}  // namespace

size_t mlp_partials_floats(uint32_t max_batch) {
    const size_t blocks = (max_batch + kTrainBlock - 1) / kTrainBlock;
    return blocks * (kMlpParams + 1);
}

void launch_mlp_forward(const MlpDev& m, const float* features, uint32_t n, float* pred, cudaStream_t s) {
    if (!n) return;
    uint32_t tiles = (n + 63) / 64;
    if (tiles > 148 * 16) tiles = 148 * 16;
    launch_pdl(mlp_forward_kernel, tiles, 128, 0, s, m.w1_bf16, m.w2_bf16, m.w3_bf16, m.params, m.scales, features, n, pred);
}

void launch_mlp_pack(const MlpDev& m, cudaStream_t s) {
    launch_pdl(mlp_pack_kernel, (kMlpHidden * kMlpHidden + 255) / 256, 256, 0, s, m.params, m.w1_bf16, m.w2_bf16, m.w3_bf16);
}

static size_t train_smem_bytes() {
    return sizeof(float) * (kMlpParams + 2 + kTrainBlock * kMlpIn + kTrainBlock * kMlpOut + kTrainBlock +
                            4 * kTrainBlock * kHp);
}

void launch_mlp_train_step(const MlpDev& m, const float* x, const float* t, uint32_t batch, int adam, float lr,
                           float beta1, float beta2, float eps, int step, cudaStream_t s) {
    if (!batch) return;
    const int blocks = (int)((batch + kTrainBlock - 1) / kTrainBlock);
    const size_t smem = train_smem_bytes();
    // per device and idempotent: set on every call (the caller may switch devices)
    cudaFuncSetAttribute(mlp_train_partials_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_pdl(mlp_train_partials_kernel, blocks, kTrainBlock, smem, s, m.params, m.scales, x, t, batch, m.partials);
    launch_pdl(mlp_reduce_adam_kernel, (kMlpParams + 1 + 255) / 256, 256, 0, s, m.params, m.adam_m, m.adam_v, m.grad,
                                                                        m.partials, blocks, batch, adam, lr, beta1,
                                                                        beta2, eps, step, m.loss);
}

void launch_mlp_init(const MlpDev& m, uint32_t seed, cudaStream_t s) {
    launch_pdl(mlp_init_kernel, (kMlpParams + 255) / 256, 256, 0, s, m.params, m.adam_m, m.adam_v, seed);
}

}  // namespace dfsph
