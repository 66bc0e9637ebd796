// linalg.cu - K2 streaming matrix-vector product and K5 Krylov-vector kernels.
//
// Reference: the GMRES of lib/viennacl/linalg/gmres.hpp:168-339 with
// vec_mul_col_kernel (matrix_operations_col.hpp:1251-1278, launched
// <<<128,128>>>) and the inner_prod/norm kernels of vector_operations.hpp;
// the Fortran path uses dgemv (coeffs_and_vels.f90:483,492).
//
// GEMV.  A is column-major.  A CTA of 256 threads owns a tile of 256*VEC
// consecutive rows (VEC = 16 bytes / element size) and a contiguous range of
// columns; every column contributes one 16-byte streaming load per thread
// (fully coalesced 4 KB per CTA and column).  Column ranges split the matrix
// so that the grid fills every SM several times; per-split partial sums are
// added in a fixed order by a second kernel (deterministic, no atomics).
//
// Reductions.  Dot products and norms use one pass with a per-block partial,
// and the last block to finish (ticket counter, no spinning) adds the
// partials in block order and writes the scalar to device memory.
#include <algorithm>

#include "rf_kernels.h"

namespace rf {

namespace {

// 16 bytes of A per thread and column: raw() issues the streaming load,
// get() converts the raw bits to the accumulation type.  The GEMV issues all
// loads of an unrolled column group before converting any, so that every
// load is in flight at once.
template <typename S>
struct Vec16;
template <>
struct Vec16<double> {
    static constexpr int kVec = 2;
    __device__ __forceinline__ static uint4 raw(const double *p, int64_t) {
        return __ldcs(reinterpret_cast<const uint4 *>(p));
    }
    template <typename ACC>
    __device__ __forceinline__ static void get(const uint4 &t, ACC *v) {
        v[0] = (ACC)__hiloint2double((int)t.y, (int)t.x);
        v[1] = (ACC)__hiloint2double((int)t.w, (int)t.z);
    }
};
template <>
struct Vec16<float> {
    static constexpr int kVec = 4;
    __device__ __forceinline__ static uint4 raw(const float *p, int64_t) {
        return __ldcs(reinterpret_cast<const uint4 *>(p));
    }
    template <typename ACC>
    __device__ __forceinline__ static void get(const uint4 &t, ACC *v) {
        v[0] = (ACC)__uint_as_float(t.x);
        v[1] = (ACC)__uint_as_float(t.y);
        v[2] = (ACC)__uint_as_float(t.z);
        v[3] = (ACC)__uint_as_float(t.w);
    }
};
template <>
struct Vec16<__nv_bfloat16> {
    static constexpr int kVec = 8;
    __device__ __forceinline__ static uint4 raw(const __nv_bfloat16 *p, int64_t) {
        return __ldcs(reinterpret_cast<const uint4 *>(p));
    }
    template <typename ACC>
    __device__ __forceinline__ static void get(const uint4 &t, ACC *v) {
        const uint32_t w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // bf16 -> fp32 is a 16-bit shift
            v[2 * k] = (ACC)__uint_as_float(w[k] << 16);
            v[2 * k + 1] = (ACC)__uint_as_float(w[k] & 0xffff0000u);
        }
    }
};

// split FP32 storage: 8 bytes of each plane per thread and column (4 rows);
// the FP32 words are rebuilt after all loads of a column group are issued
template <>
struct Vec16<SplitF32> {
    static constexpr int kVec = 4;
    __device__ __forceinline__ static uint4 raw(const SplitF32 *p, int64_t plane) {
        const uint2 h = __ldcs(reinterpret_cast<const uint2 *>(p));
        const uint2 l = __ldcs(reinterpret_cast<const uint2 *>(p + plane));
        return make_uint4(h.x, h.y, l.x, l.y);
    }
    template <typename ACC>
    __device__ __forceinline__ static void get(const uint4 &t, ACC *v) {
        v[0] = (ACC)__uint_as_float(split_join(t.x & 0xffffu, t.z & 0xffffu));
        v[1] = (ACC)__uint_as_float(split_join(t.x >> 16, t.z >> 16));
        v[2] = (ACC)__uint_as_float(split_join(t.y & 0xffffu, t.w & 0xffffu));
        v[3] = (ACC)__uint_as_float(split_join(t.y >> 16, t.w >> 16));
    }
};

constexpr int kGemvThreads = 256;
constexpr int kGemvUnroll = 8;

// FP32 accumulation: eight resident CTAs per SM (32 registers), the streaming
// loads of 64 warps per SM; the stop test alone made the compiler take 40
// registers (six CTAs per SM) and the BF16 product ran 16 % slower.
template <typename ACC>
struct GemvMinBlocks {
    static constexpr int value = sizeof(ACC) == 4 ? 8 : 0;  // 0: no minimum
};

template <typename S, typename X, typename ACC>
__global__ void __launch_bounds__(kGemvThreads, GemvMinBlocks<ACC>::value) gemv_partial_kernel(const S *__restrict__ A, int64_t lda, int64_t m,
                                                                    int64_t k, const X *__restrict__ x,
                                                                    int64_t cols_per_split, ACC *__restrict__ work,
                                                                    int64_t mpad, const int *__restrict__ stop,
                                                                    int64_t plane) {
    pdl_wait();
    if (stop && *stop) return;  // a speculatively queued product of a finished solve
    constexpr int VEC = Vec16<S>::kVec;
    const int64_t row = ((int64_t)blockIdx.x * kGemvThreads + threadIdx.x) * VEC;
    const int64_t c0 = (int64_t)blockIdx.y * cols_per_split;
    const int64_t c1 = min(k, c0 + cols_per_split);
    ACC acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = (ACC)0;
    if (row < lda) {
        const S *p = A + c0 * lda + row;
        int64_t c = c0;
        for (; c + kGemvUnroll <= c1; c += kGemvUnroll) {
            uint4 raw[kGemvUnroll];
            ACC xv[kGemvUnroll];
#pragma unroll
            for (int u = 0; u < kGemvUnroll; ++u) raw[u] = Vec16<S>::raw(p + (int64_t)u * lda, plane);
#pragma unroll
            for (int u = 0; u < kGemvUnroll; ++u) xv[u] = (ACC)__ldg(x + c + u);
#pragma unroll
            for (int u = 0; u < kGemvUnroll; ++u) {
                ACC a[VEC];
                Vec16<S>::get(raw[u], a);
#pragma unroll
                for (int v = 0; v < VEC; ++v) acc[v] += a[v] * xv[u];
            }
            p += (int64_t)kGemvUnroll * lda;
        }
        for (; c < c1; ++c) {
            ACC a[VEC];
            Vec16<S>::get(Vec16<S>::raw(p, plane), a);
            const ACC xv = (ACC)__ldg(x + c);
#pragma unroll
            for (int v = 0; v < VEC; ++v) acc[v] += a[v] * xv;
            p += lda;
        }
        ACC *w = work + (int64_t)blockIdx.y * mpad + row;
#pragma unroll
        for (int v = 0; v < VEC; ++v) w[v] = acc[v];
    }
    (void)m;
}

template <typename ACC, typename Y>
__global__ void gemv_reduce_kernel(const ACC *__restrict__ work, int splits, int64_t mpad, int64_t m, Y *y,
                                   const Y *r, const int *__restrict__ stop) {
    pdl_wait();
    if (stop && *stop) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    ACC s = (ACC)0;
    for (int t = 0; t < splits; ++t) s += work[(int64_t)t * mpad + i];
    if (r) y[i] = (Y)((ACC)r[i] - s);
    else y[i] = (Y)s;
}

// Resident CTAs of one instance on the whole GPU (queried once per instance).
template <typename S, typename X, typename ACC>
int gemv_slots(int sm_count) {
    static int occ = 0;
    if (occ == 0) {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, gemv_partial_kernel<S, X, ACC>, kGemvThreads, 0) !=
                cudaSuccess ||
            o < 1)
            o = 1;
        occ = o;
    }
    return sm_count * occ;
}

// Column splits: a few full waves of resident CTAs, so that the last, partial
// wave costs little; at least 64 columns per split.
// BF16 (8 elements per load) prefers 4 waves: its many row-tile-narrow splits
// otherwise write and re-read ~80 MB of partial sums per product at M = 4000
// (measured 1.029 vs 1.096 ms; FP32 and FP64 are best at 8).
int gemv_splits(int64_t m, int64_t k, int vec, int slots) {
    const int waves = vec >= 8 ? 4 : 8;
    const int64_t tiles = (m + (int64_t)kGemvThreads * vec - 1) / ((int64_t)kGemvThreads * vec);
    int64_t splits = ((int64_t)waves * slots + tiles - 1) / tiles;
    const int64_t max_by_cols = k / 64 > 0 ? k / 64 : 1;
    if (splits > max_by_cols) splits = max_by_cols;
    if (splits < 1) splits = 1;
    return (int)splits;
}

template <typename S, typename X, typename ACC>
int64_t gemv_work_elems_of(int64_t m, int sm_count) {
    constexpr int VEC = Vec16<S>::kVec;
    const int64_t tiles = (m + (int64_t)kGemvThreads * VEC - 1) / ((int64_t)kGemvThreads * VEC);
    const int64_t mpad = tiles * kGemvThreads * VEC;
    return (int64_t)gemv_splits(m, m, VEC, gemv_slots<S, X, ACC>(sm_count)) * mpad;
}

}  // namespace

int64_t gemv_work_elems(int64_t m, int sm_count, int elem_bytes) {
    // the largest split buffer over the instances that read elements of this size
    if (elem_bytes == 8) return gemv_work_elems_of<double, double, double>(m, sm_count);
    if (elem_bytes == 4)
        return std::max({gemv_work_elems_of<float, double, double>(m, sm_count),
                         gemv_work_elems_of<float, float, float>(m, sm_count),
                         gemv_work_elems_of<SplitF32, double, double>(m, sm_count),
                         gemv_work_elems_of<SplitF32, float, float>(m, sm_count)});
    return std::max(gemv_work_elems_of<__nv_bfloat16, float, float>(m, sm_count),
                    gemv_work_elems_of<__nv_bfloat16, double, double>(m, sm_count));
}

template <typename S, typename X, typename ACC, typename Y>
cudaError_t launch_gemv(const S *A, int64_t lda, int64_t m, int64_t k, const X *x, Y *y, const Y *r, ACC *work,
                        int64_t work_elems, int sm_count, cudaStream_t st, const int *stop, int64_t plane) {
    constexpr int VEC = Vec16<S>::kVec;
    const int64_t tiles = (lda + (int64_t)kGemvThreads * VEC - 1) / ((int64_t)kGemvThreads * VEC);
    const int64_t mpad = tiles * kGemvThreads * VEC;
    int splits = gemv_splits(m, k, VEC, gemv_slots<S, X, ACC>(sm_count));
    while (splits > 1 && (int64_t)splits * mpad > work_elems) --splits;
    if ((int64_t)splits * mpad > work_elems) return cudaErrorInvalidValue;
    const int64_t cps = (k + splits - 1) / splits;
    dim3 grid((unsigned)tiles, (unsigned)splits);
    cudaError_t e = launch_pdl(gemv_partial_kernel<S, X, ACC>, grid, dim3(kGemvThreads), 0, st, A, lda, m, k, x, cps,
                               work, mpad, stop, plane);
    if (e != cudaSuccess) return e;
    return launch_pdl(gemv_reduce_kernel<ACC, Y>, dim3((unsigned)((m + 255) / 256)), dim3(256), 0, st,
                      static_cast<const ACC *>(work), splits, mpad, m, y, r, stop);
}

template cudaError_t launch_gemv<double, double, double, double>(const double *, int64_t, int64_t, int64_t,
                                                                 const double *, double *, const double *,
                                                                 double *, int64_t, int, cudaStream_t, const int *, int64_t);
template cudaError_t launch_gemv<float, double, double, double>(const float *, int64_t, int64_t, int64_t,
                                                                const double *, double *, const double *,
                                                                double *, int64_t, int, cudaStream_t, const int *, int64_t);
template cudaError_t launch_gemv<float, float, float, float>(const float *, int64_t, int64_t, int64_t,
                                                             const float *, float *, const float *, float *,
                                                             int64_t, int, cudaStream_t, const int *, int64_t);
template cudaError_t launch_gemv<__nv_bfloat16, float, float, float>(const __nv_bfloat16 *, int64_t, int64_t,
                                                                     int64_t, const float *, float *,
                                                                     const float *, float *, int64_t, int,
                                                                     cudaStream_t, const int *, int64_t);
template cudaError_t launch_gemv<__nv_bfloat16, double, double, double>(const __nv_bfloat16 *, int64_t, int64_t,
                                                                        int64_t, const double *, double *,
                                                                        const double *, double *, int64_t, int,
                                                                        cudaStream_t, const int *, int64_t);
template cudaError_t launch_gemv<SplitF32, double, double, double>(const SplitF32 *, int64_t, int64_t, int64_t,
                                                                   const double *, double *, const double *,
                                                                   double *, int64_t, int, cudaStream_t, const int *,
                                                                   int64_t);
template cudaError_t launch_gemv<SplitF32, float, float, float>(const SplitF32 *, int64_t, int64_t, int64_t,
                                                                const float *, float *, const float *, float *,
                                                                int64_t, int, cudaStream_t, const int *, int64_t);

// ---------------------------------------------------------------------------
// reductions

namespace {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    }
    return s;  // valid in thread 0
}

// The last block to finish adds all block partials in order.
__device__ __forceinline__ void finish_reduction(double blocksum, const RedBuf &rb, double *out, bool take_sqrt) {
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        rb.partials[blockIdx.x] = blocksum;
        __threadfence();
        const unsigned int ticket = atomicAdd(rb.counter, 1u);
        is_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        double s = 0.0;
        for (unsigned int b = 0; b < gridDim.x; ++b) s += __ldcg(rb.partials + b);
        *out = take_sqrt ? sqrt(s) : s;
        *rb.counter = 0u;
    }
}

inline int red_blocks(int64_t n, const RedBuf &rb) {
    int64_t b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
    if (b > rb.max_blocks) b = rb.max_blocks;
    if (b < 1) b = 1;
    return (int)b;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) mgs_step_kernel(int64_t n, T *w, const T *vprev,
                                                               const double *hprev, const T *v, double *out,
                                                               RedBuf rb) {
    __shared__ double sh[kRedThreads / 32];
    const double h = vprev ? *hprev : 0.0;
    double acc = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        T we = w[e];
        if (vprev) {
            we = (T)((double)we + (-h) * (double)vprev[e]);
            w[e] = we;
        }
        acc += (double)v[e] * (double)we;
    }
    const double s = block_sum(acc, sh);
    finish_reduction(s, rb, out, false);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) mgs_norm_kernel(int64_t n, T *w, const T *vprev,
                                                               const double *hprev, double *out, RedBuf rb) {
    __shared__ double sh[kRedThreads / 32];
    const double h = vprev ? *hprev : 0.0;
    double acc = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        T we = w[e];
        if (vprev) {
            we = (T)((double)we + (-h) * (double)vprev[e]);
            w[e] = we;
        }
        acc += (double)we * (double)we;
    }
    const double s = block_sum(acc, sh);
    finish_reduction(s, rb, out, true);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) dot_kernel(int64_t n, const T *a, const T *b, double *out,
                                                          RedBuf rb) {
    __shared__ double sh[kRedThreads / 32];
    double acc = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        acc += (double)a[e] * (double)b[e];
    const double s = block_sum(acc, sh);
    finish_reduction(s, rb, out, false);
}

template <typename TO, typename TI>
__global__ void scale_kernel(int64_t n, const TI *x, const double *den, double num, TO *y) {
    const double f = num / *den;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        y[e] = (TO)(f * (double)x[e]);
}

template <typename TO, typename TI>
__global__ void scale_h_kernel(int64_t n, const TI *x, double alpha, TO *y) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        y[e] = (TO)(alpha * (double)x[e]);
}

template <typename TV>
__global__ void combine_kernel(int64_t n, const double *x, const TV *V, int64_t ldv, const double *y, int k,
                               double *xcur) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += (double)V[(int64_t)c * ldv + e] * y[c];
        xcur[e] = (x ? x[e] : 0.0) + s;
    }
}

template <typename T>
__global__ void bmr_kernel(int64_t n, const T *b, T *r) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        r[e] = b[e] - r[e];
}

template <typename T>
__global__ void vy_kernel(int64_t n, const T *V, int64_t ldv, const double *y, int k, T *u) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += (double)V[(int64_t)c * ldv + e] * y[c];
        u[e] = (T)s;
    }
}

template <typename T>
__global__ void add_kernel(int64_t n, const T *x, const T *u, T *out) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = x[e] + u[e];
}

__global__ void axpy_d_kernel(int64_t n, double alpha, const double *x, double *y) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        y[e] += alpha * x[e];
}

__global__ void axpy_fd_kernel(int64_t n, double alpha, const float *d, double *x) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        x[e] += alpha * (double)d[e];
}

template <typename TO, typename TI>
__global__ void convert_kernel(int64_t n, const TI *x, TO *y) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        y[e] = (TO)x[e];
}

// out[r + c * rows] = A[row0 + r + c * lda] for r < rows, c < cols (FP64 copy
// of a row block of a column-major matrix in any storage precision)
template <typename T>
__global__ void gather_rows_kernel(const T *A, int64_t lda, int64_t row0, int64_t rows, int64_t cols,
                                   double *out, int64_t plane) {
    const int64_t tot = rows * cols;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / rows, r = e - c * rows;
        out[e] = load_entry<T>(A, row0 + r + c * lda, plane);
    }
}

// z_i = v_i + omega sum_{m < kp} B_{i,m} v_{j_m}.  A CTA owns kApplyFibers fibers:
// it first stages their neighbour lists and the neighbours' entries of v in
// shared memory (independent, coalesced loads), then one thread per output
// entry (i, r) runs over the blocks' rows; B row-major blocks, pstride blocks
// per fiber; j_m = knn[i * kstride + m] (negative: no neighbour).  FP64
// accumulation in a fixed order.  Needs nb <= 24 and kp <= 8.
constexpr int kApplyFibers = 16;
constexpr int kApplyMaxNb = 24;
constexpr int kApplyMaxKp = 8;
template <typename T>
__global__ void __launch_bounds__(kApplyFibers * kApplyMaxNb) pair_apply_kernel(
    int M, int nb, int kp, int pstride, const float *__restrict__ B, const int *__restrict__ knn, int kstride,
    double omega, const T *__restrict__ v, T *__restrict__ z, const int *__restrict__ stop) {
    pdl_wait();
    if (stop && *stop) return;
    __shared__ int s_j[kApplyFibers * kApplyMaxKp];
    __shared__ T s_v[kApplyFibers * kApplyMaxKp * kApplyMaxNb];
    const int f0 = blockIdx.x * kApplyFibers;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int t = tid; t < kApplyFibers * kp; t += nt) {
        const int f = t / kp, m = t - f * kp;
        s_j[t] = (f0 + f < M) ? knn[(int64_t)(f0 + f) * kstride + m] : -1;
    }
    __syncthreads();
    for (int t = tid; t < kApplyFibers * kp * nb; t += nt) {
        const int q = t / nb, c = t - q * nb;
        const int j = s_j[q];
        s_v[t] = j >= 0 ? v[(int64_t)j * nb + c] : (T)0;
    }
    __syncthreads();
    const int f = tid / nb, r = tid - f * nb;
    const int64_t i = f0 + f;
    if (f >= kApplyFibers || i >= M) return;
    double s = 0.0;
    for (int m = 0; m < kp; ++m) {
        const float *b = B + ((i * pstride + m) * nb + r) * nb;
        const T *vj = s_v + (f * kp + m) * nb;
        for (int c = 0; c < nb; ++c) s += (double)b[c] * (double)vj[c];
    }
    z[i * nb + r] = (T)fma(omega, s, (double)v[i * nb + r]);
}

inline unsigned grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 4096) b = 4096;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace

template <typename T>
cudaError_t launch_mgs_step(int64_t n, T *w, const T *vprev, const double *hprev, const T *v, double *out,
                            const RedBuf &rb, cudaStream_t st) {
    mgs_step_kernel<T><<<red_blocks(n, rb), kRedThreads, 0, st>>>(n, w, vprev, hprev, v, out, rb);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_mgs_norm(int64_t n, T *w, const T *vprev, const double *hprev, double *out, const RedBuf &rb,
                            cudaStream_t st) {
    mgs_norm_kernel<T><<<red_blocks(n, rb), kRedThreads, 0, st>>>(n, w, vprev, hprev, out, rb);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_dot(int64_t n, const T *a, const T *b, double *out, const RedBuf &rb, cudaStream_t st) {
    dot_kernel<T><<<red_blocks(n, rb), kRedThreads, 0, st>>>(n, a, b, out, rb);
    return cudaGetLastError();
}
template <typename TO, typename TI>
cudaError_t launch_scale(int64_t n, const TI *x, const double *den, double num, TO *y, cudaStream_t st) {
    scale_kernel<TO, TI><<<grid_for(n), 256, 0, st>>>(n, x, den, num, y);
    return cudaGetLastError();
}
template <typename TO, typename TI>
cudaError_t launch_scale_h(int64_t n, const TI *x, double alpha, TO *y, cudaStream_t st) {
    scale_h_kernel<TO, TI><<<grid_for(n), 256, 0, st>>>(n, x, alpha, y);
    return cudaGetLastError();
}
template cudaError_t launch_scale_h<float, double>(int64_t, const double *, double, float *, cudaStream_t);
template cudaError_t launch_scale_h<double, double>(int64_t, const double *, double, double *, cudaStream_t);

template <typename TV>
cudaError_t launch_combine(int64_t n, const double *x, const TV *V, int64_t ldv, const double *y, int k,
                           double *xcur, cudaStream_t st) {
    combine_kernel<TV><<<grid_for(n), 256, 0, st>>>(n, x, V, ldv, y, k, xcur);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_bmr(int64_t n, const T *b, T *r, cudaStream_t st) {
    bmr_kernel<T><<<grid_for(n), 256, 0, st>>>(n, b, r);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_vy(int64_t n, const T *V, int64_t ldv, const double *y, int k, T *u, cudaStream_t st) {
    vy_kernel<T><<<grid_for(n), 256, 0, st>>>(n, V, ldv, y, k, u);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_add(int64_t n, const T *x, const T *u, T *out, cudaStream_t st) {
    add_kernel<T><<<grid_for(n), 256, 0, st>>>(n, x, u, out);
    return cudaGetLastError();
}
template cudaError_t launch_bmr<double>(int64_t, const double *, double *, cudaStream_t);
template cudaError_t launch_bmr<float>(int64_t, const float *, float *, cudaStream_t);
template cudaError_t launch_vy<double>(int64_t, const double *, int64_t, const double *, int, double *, cudaStream_t);
template cudaError_t launch_vy<float>(int64_t, const float *, int64_t, const double *, int, float *, cudaStream_t);
template cudaError_t launch_add<double>(int64_t, const double *, const double *, double *, cudaStream_t);
template cudaError_t launch_add<float>(int64_t, const float *, const float *, float *, cudaStream_t);

cudaError_t launch_axpy_d(int64_t n, double alpha, const double *x, double *y, cudaStream_t st) {
    axpy_d_kernel<<<grid_for(n), 256, 0, st>>>(n, alpha, x, y);
    return cudaGetLastError();
}
cudaError_t launch_axpy_fd(int64_t n, double alpha, const float *d, double *x, cudaStream_t st) {
    axpy_fd_kernel<<<grid_for(n), 256, 0, st>>>(n, alpha, d, x);
    return cudaGetLastError();
}
template <typename TO, typename TI>
cudaError_t launch_convert(int64_t n, const TI *x, TO *y, cudaStream_t st) {
    convert_kernel<TO, TI><<<grid_for(n), 256, 0, st>>>(n, x, y);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_gather_rows(const T *A, int64_t lda, int64_t row0, int64_t rows, int64_t cols, double *out,
                               cudaStream_t st, int64_t plane) {
    gather_rows_kernel<T><<<grid_for(rows * cols), 256, 0, st>>>(A, lda, row0, rows, cols, out, plane);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_pair_apply(int M, int nb, int kp, int pstride, const float *B, const int *knn, int kstride,
                              double omega, const T *v, T *z, cudaStream_t st, const int *stop) {
    if (nb > kApplyMaxNb || kp > kApplyMaxKp) return cudaErrorInvalidValue;
    return launch_pdl(pair_apply_kernel<T>, dim3((unsigned)((M + kApplyFibers - 1) / kApplyFibers)),
                      dim3(kApplyFibers * nb), 0, st, M, nb, kp, pstride, B, knn, kstride, omega, v, z, stop);
}

template cudaError_t launch_mgs_step<double>(int64_t, double *, const double *, const double *, const double *,
                                             double *, const RedBuf &, cudaStream_t);
template cudaError_t launch_mgs_step<float>(int64_t, float *, const float *, const double *, const float *,
                                            double *, const RedBuf &, cudaStream_t);
template cudaError_t launch_mgs_norm<double>(int64_t, double *, const double *, const double *, double *,
                                             const RedBuf &, cudaStream_t);
template cudaError_t launch_mgs_norm<float>(int64_t, float *, const float *, const double *, double *,
                                            const RedBuf &, cudaStream_t);
template cudaError_t launch_dot<double>(int64_t, const double *, const double *, double *, const RedBuf &,
                                        cudaStream_t);
template cudaError_t launch_dot<float>(int64_t, const float *, const float *, double *, const RedBuf &,
                                       cudaStream_t);
template cudaError_t launch_scale<double, double>(int64_t, const double *, const double *, double, double *,
                                                  cudaStream_t);
template cudaError_t launch_scale<float, float>(int64_t, const float *, const double *, double, float *,
                                                cudaStream_t);
template cudaError_t launch_scale<float, double>(int64_t, const double *, const double *, double, float *,
                                                 cudaStream_t);
template cudaError_t launch_combine<double>(int64_t, const double *, const double *, int64_t, const double *,
                                            int, double *, cudaStream_t);
template cudaError_t launch_combine<float>(int64_t, const double *, const float *, int64_t, const double *, int,
                                           double *, cudaStream_t);
template cudaError_t launch_convert<float, double>(int64_t, const double *, float *, cudaStream_t);
template cudaError_t launch_convert<double, float>(int64_t, const float *, double *, cudaStream_t);
template cudaError_t launch_convert<double, __nv_bfloat16>(int64_t, const __nv_bfloat16 *, double *,
                                                           cudaStream_t);
template cudaError_t launch_gather_rows<double>(const double *, int64_t, int64_t, int64_t, int64_t, double *,
                                                cudaStream_t, int64_t);
template cudaError_t launch_gather_rows<float>(const float *, int64_t, int64_t, int64_t, int64_t, double *,
                                               cudaStream_t, int64_t);
template cudaError_t launch_gather_rows<__nv_bfloat16>(const __nv_bfloat16 *, int64_t, int64_t, int64_t, int64_t,
                                                       double *, cudaStream_t, int64_t);
template cudaError_t launch_gather_rows<SplitF32>(const SplitF32 *, int64_t, int64_t, int64_t, int64_t, double *,
                                                  cudaStream_t, int64_t);
template cudaError_t launch_pair_apply<double>(int, int, int, int, const float *, const int *, int, double,
                                               const double *, double *, cudaStream_t, const int *);
template cudaError_t launch_pair_apply<float>(int, int, int, int, const float *, const int *, int, double,
                                              const float *, float *, cudaStream_t, const int *);

}  // namespace rf
