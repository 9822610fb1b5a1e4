// mlp.cu — inference (BF16 tensor cores, FP32 accumulate) and online training (FP32 forward /
// backward, deterministic reductions, Adam) of the warm-start MLP described in mlp.cuh.
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "mma_phases.h"
#include "dfsph_common.cuh"

namespace dfsph {

namespace {

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low 16 bits) = lo
    return *reinterpret_cast<uint32_t*>(&v);
}

// ---- inference on the 5th-generation tensor cores (tcgen05) -------------------------------------
// One CTA of 128 threads evaluates tiles of 128 particles (the MMA's M): thread t owns particle row t
// of the tile. Operands sit in shared memory in the canonical K-major, unswizzled UMMA layout
// (core matrices of 8 rows x 16 bytes; LBO = byte distance between the two 8-element K halves of
// one MMA's K = 16, SBO = distance between 8-row groups); one thread issues the MMAs, whose FP32
// accumulators live in tensor memory (TMEM); each warp reads its 32 rows back with tcgen05.ld, adds
// the bias, applies ReLU and stores the BF16 activations as the next layer's A operand.
//   layer 1: [128 x 16] x [16 x 64]   (5 inputs + zero padding)  -> TMEM columns 0..63
//   layer 2: [128 x 64] x [64 x 64]   (4 MMAs of K = 16)         -> TMEM columns 64..127
//   layer 3: [128 x 64] x [64 x 16]   (2 outputs + zero padding) -> TMEM columns 0..15
constexpr int kMmaM = 128;
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kSA = 0;                    // A operand: 128 x 64 BF16 = 16 KB
constexpr uint32_t kSW1 = kSA + 16384;         // 64 x 16 BF16 = 2 KB
constexpr uint32_t kSW2 = kSW1 + 2048;         // 64 x 64 BF16 = 8 KB
constexpr uint32_t kSW3 = kSW2 + 8192;         // 16 x 64 BF16 = 2 KB
constexpr uint32_t kSBias = kSW3 + 2048;       // b1[64], b2[64], b3[2], in_scale[8] (FP32)
constexpr uint32_t kSBar = kSBias + 1024;      // mbarrier (8 B) + TMEM address slot (4 B)
// Dynamic shared memory per CTA: the operands plus padding up to 56 KB, so that at most four CTAs
// share an SM and their four 128-column TMEM allocations fit the SM's 512 columns (no CTA ever waits
// in tcgen05.alloc).
constexpr uint32_t kMlpSmem = 56 * 1024;
constexpr uint32_t kMmaWaitLimit = 1u << 22;   // bounded mbarrier waits (a give-up raises a status bit)

// Byte offset of element (r, k) of a K-major operand with 8-row groups of kchunks 16-byte chunks.
__device__ __forceinline__ uint32_t umma_off(uint32_t r, uint32_t k, uint32_t kchunks) {
    return (r >> 3) * (kchunks * 128u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (sm_100 layout): start address, LBO, SBO in 16-byte units,
// version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__device__ __forceinline__ uint32_t umma_idesc(uint32_t m, uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Waits for the mbarrier phase `parity`; false if the wait gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kMmaWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bias + ReLU of 64 accumulator columns of this thread's row (TMEM column `col`), stored as BF16
// row r of the 128 x 64 A operand.
__device__ __forceinline__ void epilogue64(uint32_t taddr_row, uint32_t col, const float* bias, unsigned char* sa,
                                           uint32_t r) {
#pragma unroll
    for (int c0 = 0; c0 < 64; c0 += 16) {
        float v[16];
        tmem_ld16(taddr_row + col + c0, v);
        tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 16; h += 8) {
            uint4 chunk;
            chunk.x = pack_bf16x2(fmaxf(v[h + 0] + bias[c0 + h + 0], 0.f), fmaxf(v[h + 1] + bias[c0 + h + 1], 0.f));
            chunk.y = pack_bf16x2(fmaxf(v[h + 2] + bias[c0 + h + 2], 0.f), fmaxf(v[h + 3] + bias[c0 + h + 3], 0.f));
            chunk.z = pack_bf16x2(fmaxf(v[h + 4] + bias[c0 + h + 4], 0.f), fmaxf(v[h + 5] + bias[c0 + h + 5], 0.f));
            chunk.w = pack_bf16x2(fmaxf(v[h + 6] + bias[c0 + h + 6], 0.f), fmaxf(v[h + 7] + bias[c0 + h + 7], 0.f));
            *reinterpret_cast<uint4*>(sa + umma_off(r, c0 + h, 8)) = chunk;
        }
    }
}

__global__ void __launch_bounds__(kMmaM) mlp_forward_kernel(const uint16_t* __restrict__ w1b,
                                                            const uint16_t* __restrict__ w2b,
                                                            const uint16_t* __restrict__ w3b,
                                                            const float* __restrict__ params,
                                                            const MlpScales* __restrict__ scales,
                                                            const float* __restrict__ features, uint32_t n,
                                                            float* __restrict__ pred, uint32_t* __restrict__ status) {
    DFSPH_PDL_ENTER;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sa = smem + kSA;
    float* sb1 = reinterpret_cast<float*>(smem + kSBias);
    float* sb2 = sb1 + 64;
    float* sb3 = sb2 + 64;
    float* sin = sb3 + 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kSBar + 8);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t bar_addr = s_base + kSBar;

    // weights into the UMMA layout (B operands are [N][K], K-major)
    for (uint32_t t = tid; t < 64 * 2; t += kMmaM) {  // W1: 64 rows x 2 chunks (K = 16)
        const uint32_t r = t >> 1, c = t & 1;
        *reinterpret_cast<uint4*>(smem + kSW1 + umma_off(r, 8 * c, 2)) =
            *reinterpret_cast<const uint4*>(w1b + r * 16 + 8 * c);
    }
    for (uint32_t t = tid; t < 64 * 8; t += kMmaM) {  // W2: 64 rows x 8 chunks
        const uint32_t r = t >> 3, c = t & 7;
        *reinterpret_cast<uint4*>(smem + kSW2 + umma_off(r, 8 * c, 8)) =
            *reinterpret_cast<const uint4*>(w2b + r * 64 + 8 * c);
    }
    for (uint32_t t = tid; t < 16 * 8; t += kMmaM) {  // W3: 16 rows (8 stored, the rest zero) x 8 chunks
        const uint32_t r = t >> 3, c = t & 7;
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(smem + kSW3 + umma_off(r, 8 * c, 8)) =
            r < 8 ? *reinterpret_cast<const uint4*>(w3b + r * 64 + 8 * c) : z;
    }
    if (tid < 64) {
        sb1[tid] = params[kB1 + tid];
        sb2[tid] = params[kB2 + tid];
    }
    if (tid < kMlpOut) sb3[tid] = params[kB3 + tid];
    if (tid < kMlpIn) sin[tid] = scales->in_scale[tid];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_addr) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // TMEM for the accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_base + kSBar + 8),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t trow = tmem + ((warp * 32u) << 16);  // this warp's 32 TMEM lanes
    const uint32_t idesc64 = umma_idesc(kMmaM, 64), idesc16 = umma_idesc(kMmaM, 16);
    MmaPhases ph;  // tid 0's copy decides the drain below
    bool ok = true;

    for (uint32_t tile = blockIdx.x; tile * kMmaM < n && ok; tile += gridDim.x) {
        const uint32_t row = tile * kMmaM + tid;
        // layer-1 operand: the scaled features, K padded to 16
        {
            float x[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (row < n) {
                const float4 f0 = *reinterpret_cast<const float4*>(features + (size_t)row * kMlpIn);
                const float4 f1 = *reinterpret_cast<const float4*>(features + (size_t)row * kMlpIn + 4);
                x[0] = f0.x * sin[0]; x[1] = f0.y * sin[1]; x[2] = f0.z * sin[2]; x[3] = f0.w * sin[3];
                x[4] = f1.x * sin[4]; x[5] = f1.y * sin[5]; x[6] = f1.z * sin[6]; x[7] = f1.w * sin[7];
            }
            uint4 c0;
            c0.x = pack_bf16x2(x[0], x[1]);
            c0.y = pack_bf16x2(x[2], x[3]);
            c0.z = pack_bf16x2(x[4], x[5]);
            c0.w = pack_bf16x2(x[6], x[7]);
            *reinterpret_cast<uint4*>(sa + umma_off(tid, 0, 2)) = c0;
            *reinterpret_cast<uint4*>(sa + umma_off(tid, 8, 2)) = make_uint4(0u, 0u, 0u, 0u);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            umma_bf16(tmem + 0, umma_desc(s_base + kSA, 128, 256), umma_desc(s_base + kSW1, 128, 256), idesc64, 0);
            umma_commit(bar_addr);
        }
        {
            ph.committed();
            const bool done = mbar_wait(bar_addr, ph.phase);
            ph.waited(done);
            ok = __all_sync(0xFFFFFFFFu, done);  // warp-uniform for tcgen05.ld
        }
        tc_fence_after();
        if (ok) epilogue64(trow, 0, sb1, sa, tid);  // layer-1 activations -> A operand (K = 64)
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_fence_after();
            for (uint32_t k = 0; k < 4; ++k)
                umma_bf16(tmem + 64, umma_desc(s_base + kSA + 256 * k, 128, 1024),
                          umma_desc(s_base + kSW2 + 256 * k, 128, 1024), idesc64, k > 0);
            umma_commit(bar_addr);
        }
        if (ok) {
            ph.committed();
            const bool done = mbar_wait(bar_addr, ph.phase);
            ph.waited(done);
            ok = __all_sync(0xFFFFFFFFu, done);
        }
        tc_fence_after();
        if (ok) epilogue64(trow, 64, sb2, sa, tid);  // layer-2 activations -> A operand
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_fence_after();
            for (uint32_t k = 0; k < 4; ++k)
                umma_bf16(tmem + 0, umma_desc(s_base + kSA + 256 * k, 128, 1024),
                          umma_desc(s_base + kSW3 + 256 * k, 128, 1024), idesc16, k > 0);
            umma_commit(bar_addr);
        }
        if (ok) {
            ph.committed();
            const bool done = mbar_wait(bar_addr, ph.phase);
            ph.waited(done);
            ok = __all_sync(0xFFFFFFFFu, done);
        }
        tc_fence_after();
        if (ok) {
            float v[16];
            tmem_ld16(trow, v);
            tmem_wait_ld();
            if (row < n) *reinterpret_cast<float2*>(pred + 2 * (size_t)row) = make_float2(v[0] + sb3[0], v[1] + sb3[1]);
        }
        tc_fence_before();
        __syncthreads();
        ok = __syncthreads_and(ok);
    }
    if (!ok && tid == 0) atomicOr(status, DFSPH_ST_MMA_TIMEOUT);
    // A wait that gave up leaves at most one MMA group in flight: the one thread 0 committed and did
    // not see complete. Give it the same bounded time before the tensor memory is freed.
    uint32_t drain_parity;
    if (tid == 0 && ph.drain(drain_parity)) mbar_wait(bar_addr, drain_parity);
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
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

void launch_mlp_forward(const MlpDev& m, const float* features, uint32_t n, float* pred, uint32_t* status,
                        cudaStream_t s) {
    if (!n) return;
    cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMlpSmem);
    uint32_t tiles = (n + kMmaM - 1) / kMmaM;
    if (tiles > 148 * 4) tiles = 148 * 4;  // persistent CTAs, at most four per SM (see kMlpSmem)
    launch_pdl(mlp_forward_kernel, tiles, kMmaM, kMlpSmem, s, m.w1_bf16, m.w2_bf16, m.w3_bf16, m.params, m.scales,
               features, n, pred, status);
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
