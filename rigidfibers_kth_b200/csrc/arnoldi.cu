// arnoldi.cu - Arnoldi steps of the inner GMRES controlled on the device.
//
// The inner solves of the mixed-precision refinement stop on the Arnoldi
// estimate alone, so the whole GMRES(m) cycle can run without the host: the
// Gram-Schmidt coefficients, the Givens update of the Hessenberg column and
// the stop test happen in the kernels, and every kernel of the next step
// reads the stop flag first and returns at once when it is set.  The host
// then queues step j + 1 before it learns (from host-mapped memory) whether
// step j stopped: the GPU never waits for the host between steps, and a
// step queued after the stop costs a few empty launches.
//
// Orthogonalisation: classical Gram-Schmidt applied twice (CGS2), fused into
// three passes over the basis: (1) h1 = V^T w; (2) w -= V h1, h2 = V^T w;
// (3) w -= V h2, |w|.  The reference solver (dGMRES.f with icntl(5) = 0) uses
// modified Gram-Schmidt, one pass per basis vector; the FP64 GMRES of this
// library keeps that order (its iterates are compared with the oracle's),
// the inner solves of the refinement use CGS2: as stable, and three launches
// per step instead of j + 3.
//
// Reductions: per-block partial sums, and the last block to finish (ticket
// counter, no spinning) adds them in block order (deterministic).
#include <cmath>

#include "rf_kernels.h"

namespace rf {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int KM = kArnoldiMax;

// one element per thread: the passes are latency bound, more CTAs keep more
// loads in flight
inline int blocks_for(int64_t n, int max_blocks) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    return (int)b;
}

// Block sums of cnt per-thread values into part[k * gridDim.x + blockIdx.x];
// true in every thread of the last block to finish, which may then read all
// partials (with __ldcg).
template <int CMAX>
__device__ bool block_partials(const double (&v)[CMAX], int cnt, double *part, unsigned int *counter) {
    __shared__ double sh[kWarps][CMAX];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < CMAX; ++k) {
        if (k < cnt) {  // cnt is uniform: every lane takes part in the shuffles
            double s = v[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) sh[wid][k] = s;
        }
    }
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sh[w][threadIdx.x];
        part[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// the partials of value k summed by one warp (lane-strided over the blocks,
// then a fixed shuffle tree: the same order every run); valid in every lane
__device__ double warp_sum_partials(const double *part, int k, int lane) {
    double s = 0.0;
    for (unsigned int b = lane; b < gridDim.x; b += 32) s += __ldcg(part + (int64_t)k * gridDim.x + b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// LINPACK drotg semantics (fortran/blas_rot.f:117-146), as in the host solver
__device__ void rotg_d(double a, double b, double *c, double *s) {
    const double roe = (fabs(a) > fabs(b)) ? a : b;
    const double scale = fabs(a) + fabs(b);
    if (scale == 0.0) {
        *c = 1.0;
        *s = 0.0;
        return;
    }
    double r = scale * sqrt((a / scale) * (a / scale) + (b / scale) * (b / scale));
    r = copysign(1.0, roe) * r;
    *c = a / r;
    *s = b / r;
}

__device__ __forceinline__ void rot_d(double &x, double &y, double c, double s) {
    const double t = c * x + s * y;
    y = c * y - s * x;
    x = t;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) start_kernel(int64_t n, const T *__restrict__ r, ArnoldiCtrl *c,
                                                         double tol, int iter_max, int first, double *part,
                                                         unsigned int *counter, ArnoldiStat *stat) {
    double v[1] = {0.0};
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads) {
        const double x = (double)r[e];
        v[0] += x * x;
    }
    if (block_partials<1>(v, 1, part, counter) && threadIdx.x < 32) {
        const double beta = sqrt(warp_sum_partials(part, 0, threadIdx.x));
        if (threadIdx.x != 0) return;
        if (first) {
            c->bn = beta;
            c->itn = 0;
            c->tol = tol;
            c->iter_max = iter_max;
            c->bea = 1.0;
        }
        for (int i = 0; i <= KM; ++i) c->g[i] = 0.0;
        c->g[0] = beta;
        c->k = 0;
        c->hnext = beta;
        c->stop = isfinite(beta) ? (beta == 0.0 ? 1 : 0) : 3;
        if (beta == 0.0) c->bea = 0.0;
        volatile ArnoldiStat *out = stat;
        out->stop = c->stop;
        out->itn = c->itn;
        out->bea = c->bea;
        __threadfence_system();
        *counter = 0u;
    }
}

// out = w / hnext, unless the solve has stopped (or out is not needed)
template <typename T>
__global__ void scale_next_kernel(int64_t n, const T *__restrict__ w, T *__restrict__ out, const ArnoldiCtrl *c) {
    pdl_wait();
    if (c->stop) return;
    const double inv = 1.0 / c->hnext;
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads)
        out[e] = (T)((double)w[e] * inv);
}

// pass 1: h1 = V(:, 0:j1)^T w
template <typename T>
__global__ void __launch_bounds__(kThreads) cgs_dots_kernel(int64_t n, const T *__restrict__ w,
                                                            const T *__restrict__ V, int j1, ArnoldiCtrl *c,
                                                            double *part, unsigned int *counter) {
    pdl_wait();
    if (c->stop) return;
    double acc[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) acc[k] = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads) {
        const double we = (double)w[e];
#pragma unroll
        for (int k = 0; k < KM; ++k)
            if (k < j1) acc[k] += (double)V[(int64_t)k * n + e] * we;
    }
    if (block_partials<KM>(acc, j1, part, counter)) {
        const int lane = threadIdx.x & 31;
        for (int k = threadIdx.x >> 5; k < j1; k += kWarps) {
            const double s = warp_sum_partials(part, k, lane);
            if (lane == 0) c->h1[k] = s;
        }
        if (threadIdx.x == 0) *counter = 0u;
    }
}

// pass 2: w -= V h1, then h2 = V^T w (with the stored, rounded w)
template <typename T>
__global__ void __launch_bounds__(kThreads) cgs_update_dots_kernel(int64_t n, T *__restrict__ w,
                                                                   const T *__restrict__ V, int j1, ArnoldiCtrl *c,
                                                                   double *part, unsigned int *counter) {
    pdl_wait();
    if (c->stop) return;
    __shared__ double hs[KM];
    if ((int)threadIdx.x < j1) hs[threadIdx.x] = c->h1[threadIdx.x];
    __syncthreads();
    double acc[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) acc[k] = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads) {
        double vk[KM];
        double we = (double)w[e];
#pragma unroll
        for (int k = 0; k < KM; ++k)
            if (k < j1) {
                vk[k] = (double)V[(int64_t)k * n + e];
                we -= hs[k] * vk[k];
            }
        const T ws = (T)we;
        w[e] = ws;
        const double wr = (double)ws;
#pragma unroll
        for (int k = 0; k < KM; ++k)
            if (k < j1) acc[k] += vk[k] * wr;
    }
    if (block_partials<KM>(acc, j1, part, counter)) {
        const int lane = threadIdx.x & 31;
        for (int k = threadIdx.x >> 5; k < j1; k += kWarps) {
            const double s = warp_sum_partials(part, k, lane);
            if (lane == 0) c->h2[k] = s;
        }
        if (threadIdx.x == 0) *counter = 0u;
    }
}

// pass 3: w -= V h2, |w|; the last block forms Hessenberg column j = h1 + h2
// with |w| below it, applies the earlier rotations, makes rotation j, rotates
// g, and sets the stop flag and the step's outcome
template <typename T>
__global__ void __launch_bounds__(kThreads) cgs_update_norm_kernel(int64_t n, T *__restrict__ w,
                                                                   const T *__restrict__ V, int j, ArnoldiCtrl *c,
                                                                   ArnoldiStat *stat, double *part,
                                                                   unsigned int *counter) {
    pdl_wait();
    if (c->stop) return;
    const int j1 = j + 1;
    __shared__ double hs[KM];
    if ((int)threadIdx.x < j1) hs[threadIdx.x] = c->h2[threadIdx.x];
    __syncthreads();
    double v[1] = {0.0};
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads) {
        double we = (double)w[e];
#pragma unroll
        for (int k = 0; k < KM; ++k)
            if (k < j1) we -= hs[k] * (double)V[(int64_t)k * n + e];
        const T ws = (T)we;
        w[e] = ws;
        const double wr = (double)ws;
        v[0] += wr * wr;
    }
    if (block_partials<1>(v, 1, part, counter) && threadIdx.x < 32) {
        const double hn = sqrt(warp_sum_partials(part, 0, threadIdx.x));
        if (threadIdx.x != 0) return;
        double h[KM + 1];
        bool finite = isfinite(hn);
        for (int r = 0; r <= j; ++r) {
            h[r] = c->h1[r] + c->h2[r];
            finite = finite && isfinite(h[r]);
        }
        h[j + 1] = hn;
        for (int r = 0; r < j; ++r) rot_d(h[r], h[r + 1], c->cs[r], c->sn[r]);
        double cj, sj;
        rotg_d(h[j], h[j + 1], &cj, &sj);
        c->cs[j] = cj;
        c->sn[j] = sj;
        rot_d(c->g[j], c->g[j + 1], cj, sj);
        rot_d(h[j], h[j + 1], cj, sj);
        for (int r = 0; r <= j; ++r) c->H[r + j * KM] = h[r];
        c->hnext = hn;
        c->k = j + 1;
        c->itn += 1;
        const double bea = fabs(c->g[j + 1]) / c->bn;
        c->bea = bea;
        int stop = 0;
        if (!finite || !isfinite(bea)) stop = 3;
        else if (bea <= c->tol) stop = 1;
        else if (c->itn >= c->iter_max) stop = 2;
        c->stop = stop;
        volatile ArnoldiStat *out = stat + j;
        out->stop = stop;
        out->itn = c->itn;
        out->bea = bea;
        __threadfence_system();
        *counter = 0u;
    }
}

// y = H(0:k, 0:k)^-1 g(0:k)  (upper triangular, dtrsv 'U','N')
__global__ void lsq_kernel(ArnoldiCtrl *c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int k = c->k;
    for (int r = 0; r < k; ++r) c->y[r] = c->g[r];
    for (int col = k - 1; col >= 0; --col) {
        c->y[col] /= c->H[col + col * KM];
        for (int r = 0; r < col; ++r) c->y[r] -= c->y[col] * c->H[r + col * KM];
    }
}

// u = V(:, 0:k) y
template <typename T>
__global__ void vy_kernel(int64_t n, const T *__restrict__ V, const ArnoldiCtrl *c, T *__restrict__ u) {
    __shared__ double ys[KM];
    __shared__ int ks;
    if (threadIdx.x == 0) ks = c->k;
    if (threadIdx.x < KM) ys[threadIdx.x] = c->y[threadIdx.x];
    __syncthreads();
    const int k = ks;
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kThreads) {
        double s = 0.0;
        for (int q = 0; q < k; ++q) s += (double)V[(int64_t)q * n + e] * ys[q];
        u[e] = (T)s;
    }
}

}  // namespace

template <typename T>
cudaError_t launch_arnoldi_start(int64_t n, const T *r, T *V0, ArnoldiCtrl *c, double tol, int iter_max, int first,
                                 double *part, unsigned int *counter, int max_blocks, ArnoldiStat *stat,
                                 cudaStream_t st) {
    const int nb = blocks_for(n, max_blocks);
    start_kernel<T><<<nb, kThreads, 0, st>>>(n, r, c, tol, iter_max, first, part, counter, stat);
    scale_next_kernel<T><<<nb, kThreads, 0, st>>>(n, r, V0, c);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_arnoldi_orthogonalize(int64_t n, T *w, T *V, int j, int m, ArnoldiCtrl *c, ArnoldiStat *stat,
                                         double *part, unsigned int *counter, int max_blocks, cudaStream_t st) {
    if (j < 0 || j >= m || m > KM) return cudaErrorInvalidValue;
    const int nb = blocks_for(n, max_blocks);
    // each kernel waits (pdl_wait) for the previous one before touching memory
    cudaError_t e = launch_pdl(cgs_dots_kernel<T>, dim3(nb), dim3(kThreads), 0, st, n, static_cast<const T *>(w),
                               static_cast<const T *>(V), j + 1, c, part, counter);
    if (e == cudaSuccess)
        e = launch_pdl(cgs_update_dots_kernel<T>, dim3(nb), dim3(kThreads), 0, st, n, w, static_cast<const T *>(V),
                       j + 1, c, part, counter);
    if (e == cudaSuccess)
        e = launch_pdl(cgs_update_norm_kernel<T>, dim3(nb), dim3(kThreads), 0, st, n, w, static_cast<const T *>(V),
                       j, c, stat, part, counter);
    if (e == cudaSuccess && j + 1 < m)
        e = launch_pdl(scale_next_kernel<T>, dim3(nb), dim3(kThreads), 0, st, n, static_cast<const T *>(w),
                       V + (int64_t)(j + 1) * n, static_cast<const ArnoldiCtrl *>(c));
    return e;
}

template <typename T>
cudaError_t launch_arnoldi_combine(int64_t n, const T *V, ArnoldiCtrl *c, T *u, cudaStream_t st) {
    lsq_kernel<<<1, 32, 0, st>>>(c);
    vy_kernel<T><<<blocks_for(n, 1024), kThreads, 0, st>>>(n, V, c, u);
    return cudaGetLastError();
}

template cudaError_t launch_arnoldi_start<float>(int64_t, const float *, float *, ArnoldiCtrl *, double, int, int,
                                                 double *, unsigned int *, int, ArnoldiStat *, cudaStream_t);
template cudaError_t launch_arnoldi_start<double>(int64_t, const double *, double *, ArnoldiCtrl *, double, int, int,
                                                  double *, unsigned int *, int, ArnoldiStat *, cudaStream_t);
template cudaError_t launch_arnoldi_orthogonalize<float>(int64_t, float *, float *, int, int, ArnoldiCtrl *,
                                                         ArnoldiStat *, double *, unsigned int *, int, cudaStream_t);
template cudaError_t launch_arnoldi_orthogonalize<double>(int64_t, double *, double *, int, int, ArnoldiCtrl *,
                                                          ArnoldiStat *, double *, unsigned int *, int, cudaStream_t);
template cudaError_t launch_arnoldi_combine<float>(int64_t, const float *, ArnoldiCtrl *, float *, cudaStream_t);
template cudaError_t launch_arnoldi_combine<double>(int64_t, const double *, ArnoldiCtrl *, double *, cudaStream_t);

}  // namespace rf
