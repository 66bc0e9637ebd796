// mlp_tc.cu - the preconditioner MLP's inference layers on the 5th-generation
// tensor cores (tcgen05, sm_100a).
//
// One layer: Y[rows x nout] = act(X[rows x K] W^T + b), X and W in BF16, FP32
// accumulation in tensor memory.  A CTA of four warps owns 128 rows and all
// (up to) 256 outputs: it stages its X tile and the whole W in shared memory
// in the canonical no-swizzle K-major layout of the MMA operands (8-row x
// 16-byte core matrices, contiguous 128 bytes each; core matrices adjacent in
// M/N are 128 bytes apart (SBO), adjacent in K 16 * rows bytes apart (LBO)),
// one thread issues the K/16 MMAs (M = 128, N = 256, K = 16 each) into a
// 256-column TMEM accumulator and commits them to an mbarrier, and each warp
// reads its 32 rows back (tcgen05.ld 32x32b) for bias, ReLU and the store.
// The wait on the mbarrier is bounded: on time-out the CTA records an error
// flag, frees its tensor memory and returns.
//
// Layer sizes of the network (144 -> 256 -> 256 -> 225): K in {144, 256}
// (multiples of 16), nout <= 256 (W zero-padded to 256 rows).
#include <cuda_bf16.h>

#include "rf_kernels.h"

namespace rf {
namespace {

constexpr int kTcRows = 128;   // rows of X per CTA (MMA M)
constexpr int kTcN = 256;      // MMA N (outputs, zero-padded)
constexpr int kTcThreads = 128;
constexpr long long kTcSpinLimit = 1LL << 26;   // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, no swizzle, K-major (tcgen05 format:
// start address, LBO and SBO in 16-byte units; version 1 at bits 46-47)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;   // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
// N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcRows >> 4) << 24);

// byte offset of element (row, k) in the canonical layout of an operand with
// `rows` rows: core matrix (row / 8, k / 8) at ((k / 8) * rows / 8 + row / 8) * 128
__device__ __forceinline__ uint32_t core_offset(int row, int kc, int rows) {
    return (uint32_t)((kc * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16);
}

template <typename TX, typename TY>
__global__ void __launch_bounds__(kTcThreads, 1) mlp_layer_tc_kernel(const TX *__restrict__ X, int rows, int K,
                                                                     const __nv_bfloat16 *__restrict__ W,
                                                                     const float *__restrict__ bias, int nout,
                                                                     int relu, TY *__restrict__ Y, int ldy,
                                                                     int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    unsigned char *sX = smem;                                   // kTcRows x K bf16
    unsigned char *sW = smem + (size_t)kTcRows * K * 2;         // kTcN x K bf16
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * kTcRows;
    const int kcs = K / 8;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_bar)));
    }
    // stage X (converted to BF16) and W: one 16-byte core-matrix row per item
    for (int it = tid; it < kTcRows * kcs; it += kTcThreads) {
        const int r = it / kcs, kc = it - r * kcs;
        const int gr = row0 + r;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gr < rows) {
            const TX *src = X + (int64_t)gr * K + kc * 8;
            __nv_bfloat162 h[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn((float)src[2 * e], (float)src[2 * e + 1]);
            v = *reinterpret_cast<uint4 *>(h);
        }
        *reinterpret_cast<uint4 *>(sX + core_offset(r, kc, kTcRows)) = v;
    }
    for (int it = tid; it < kTcN * kcs; it += kTcThreads) {
        const int r = it / kcs, kc = it - r * kcs;
        const uint4 v = *reinterpret_cast<const uint4 *>(W + (int64_t)r * K + kc * 8);
        *reinterpret_cast<uint4 *>(sW + core_offset(r, kc, kTcN)) = v;
    }
    // make the generic-proxy stores visible to the tensor cores (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = s_tmem;
    if (tid == 0) {
        const uint32_t xa = smem_u32(sX), wa = smem_u32(sW);
        const uint32_t lbo_x = 16u * kTcRows, lbo_w = 16u * kTcN;
        for (int ks = 0; ks < K / 16; ++ks) {
            const uint64_t ad = umma_desc(xa + 2u * ks * lbo_x, lbo_x, 128u);
            const uint64_t bd = umma_desc(wa + 2u * ks * lbo_w, lbo_w, 128u);
            const uint32_t acc = ks > 0 ? 1u : 0u;
            asm volatile(
                "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_u32(&s_bar))
                     : "memory");
    }
    // bounded wait for the MMAs (phase 0 of the barrier)
    bool done = false;
    for (long long spin = 0; spin < kTcSpinLimit && !done; ++spin) {
        uint32_t ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(&s_bar)), "r"(0u)
            : "memory");
        done = ok != 0;
    }
    if (!done) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int r = row0 + warp * 32 + lane;   // this thread's row: TMEM lane 32 warp + lane
        for (int c0 = 0; c0 < kTcN; c0 += 32) {
            uint32_t v[32];
            const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (r < rows) {
#pragma unroll
                for (int e = 0; e < 32; ++e) {
                    const int c = c0 + e;
                    if (c < nout) {
                        float y = __uint_as_float(v[e]) + bias[c];
                        if (relu) y = fmaxf(y, 0.f);
                        Y[(int64_t)r * ldy + c] = (TY)y;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcN));
}

// W (nout x K, FP32, row-major) -> BF16 rows padded with zeros to kTcN
__global__ void pad_weights_kernel(const float *__restrict__ w, int nout, int K, __nv_bfloat16 *__restrict__ out) {
    const int64_t tot = (int64_t)kTcN * K;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / K);
        out[e] = __float2bfloat16_rn(r < nout ? w[e] : 0.f);
    }
}

template <typename TX, typename TY>
cudaError_t launch_layer(const TX *X, int rows, int K, const __nv_bfloat16 *W, const float *bias, int nout, int relu,
                         TY *Y, int ldy, int *err, cudaStream_t st) {
    if (K % 16 != 0 || K > 256 || nout > kTcN || rows < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)(kTcRows + kTcN) * K * 2;
    auto kern = mlp_layer_tc_kernel<TX, TY>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(rows + kTcRows - 1) / kTcRows, kTcThreads, smem, st>>>(X, rows, K, W, bias, nout, relu, Y, ldy, err);
    return cudaGetLastError();
}

}  // namespace

int mlp_tc_padded_rows() { return kTcN; }

cudaError_t mlp_tc_pad_weights(const float *w, int nout, int K, __nv_bfloat16 *out, cudaStream_t st) {
    if (nout > kTcN) return cudaErrorInvalidValue;
    pad_weights_kernel<<<256, 256, 0, st>>>(w, nout, K, out);
    return cudaGetLastError();
}

cudaError_t mlp_tc_forward(const __nv_bfloat16 *W1, const float *b1, const __nv_bfloat16 *W2, const float *b2,
                           const __nv_bfloat16 *W3, const float *b3, int rows, int nin, int nhid, int nout,
                           const float *X, __nv_bfloat16 *H1, __nv_bfloat16 *H2, float *O, int *err, cudaStream_t st) {
    cudaError_t e = launch_layer<float, __nv_bfloat16>(X, rows, nin, W1, b1, nhid, 1, H1, nhid, err, st);
    if (e == cudaSuccess) e = launch_layer<__nv_bfloat16, __nv_bfloat16>(H1, rows, nhid, W2, b2, nhid, 1, H2, nhid, err, st);
    if (e == cudaSuccess) e = launch_layer<__nv_bfloat16, float>(H2, rows, nhid, W3, b3, nout, 0, O, nout, err, st);
    return e;
}

}  // namespace rf
