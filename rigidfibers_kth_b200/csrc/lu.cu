// lu.cu - the direct variant of the solve: dense LU factorisation with
// partial pivoting and the two triangular solves, FP64 on the device.
//
// Reference: LAPACK dgesv called by fortran/coeffs_and_vels.f90:62,158,333,514
// (the *_direct golden runs).  Blocked right-looking factorisation, panel
// width kLuNb:
//   lu_panel_kernel  one CTA factors the tall panel A[k:n, k:k+nb]: per column
//                    the pivot (first row of largest magnitude, as idamax),
//                    the row swap inside the panel, the scaling by the
//                    reciprocal pivot and the rank-1 update of the panel's
//                    remaining columns (dgetf2's steps);
//   lu_swap_kernel   the panel's row swaps applied to the trailing columns;
//   lu_trsm_kernel   U12 = L11^-1 A12, one thread per trailing column;
//   lu_gemm_kernel   A22 -= L21 U12, 64 x 64 tiles staged in shared memory.
// The swaps are not applied to the L columns left of a panel: the forward
// solve applies each panel's swaps to the right-hand side just before that
// panel's columns of L, which is the same elimination (LINPACK's order).
// Info as LAPACK: the first zero pivot (1-based), 0 when there is none.
#include <algorithm>

#include "rf_kernels.h"

namespace rf {
namespace {

constexpr int kLuNb = 32;
constexpr int kPanelThreads = 512;

__device__ __forceinline__ void argmax_merge(double &v, int64_t &i, double ov, int64_t oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

__global__ void __launch_bounds__(kPanelThreads) lu_panel_kernel(double *A, int64_t lda, int64_t n, int64_t k, int nb,
                                                                int *piv, int *info) {
    __shared__ double s_val[kPanelThreads / 32];
    __shared__ int64_t s_idx[kPanelThreads / 32];
    __shared__ int64_t s_piv;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int j = 0; j < nb; ++j) {
        const int64_t col = k + j;
        double *cj = A + col * lda;
        double best = -1.0;
        int64_t bi = n;
        for (int64_t r = col + tid; r < n; r += blockDim.x) argmax_merge(best, bi, fabs(cj[r]), r);
        for (int o = 16; o; o >>= 1)
            argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, o), __shfl_down_sync(0xffffffffu, bi, o));
        if (lane == 0) {
            s_val[warp] = best;
            s_idx[warp] = bi;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < nwarps ? s_val[lane] : -1.0;
            bi = lane < nwarps ? s_idx[lane] : n;
            for (int o = 16; o; o >>= 1)
                argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, o), __shfl_down_sync(0xffffffffu, bi, o));
            if (lane == 0) s_piv = bi < n ? bi : col;  // a column of NaN keeps its row
        }
        __syncthreads();
        const int64_t p = s_piv;
        if (tid == 0) piv[col] = (int)p;
        if (p != col && tid < nb) {
            double *c = A + (k + tid) * lda;
            const double t = c[col];
            c[col] = c[p];
            c[p] = t;
        }
        __syncthreads();
        const double d = cj[col];
        if (d == 0.0) {
            if (tid == 0 && *info == 0) *info = (int)(col + 1);
        } else {
            const double inv = 1.0 / d;
            for (int64_t r = col + 1 + tid; r < n; r += blockDim.x) cj[r] *= inv;
        }
        __syncthreads();
        for (int c = j + 1; c < nb; ++c) {
            double *cc = A + (k + c) * lda;
            const double u = cc[col];
            if (u != 0.0)
                for (int64_t r = col + 1 + tid; r < n; r += blockDim.x) cc[r] = fma(-cj[r], u, cc[r]);
        }
        __syncthreads();
    }
}

// The panel's swaps on columns [c0, n): one thread per column, in order.
__global__ void lu_swap_kernel(double *A, int64_t lda, int64_t n, int64_t k, int nb, int64_t c0, const int *piv) {
    const int64_t c = c0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n) return;
    double *col = A + c * lda;
    for (int j = 0; j < nb; ++j) {
        const int64_t p = piv[k + j];
        if (p != k + j) {
            const double t = col[k + j];
            col[k + j] = col[p];
            col[p] = t;
        }
    }
}

// U12 = L11^-1 A12 (L11 unit lower, nb x nb): one thread per trailing column.
__global__ void __launch_bounds__(128) lu_trsm_kernel(double *A, int64_t lda, int64_t n, int64_t k, int nb) {
    __shared__ double s_l[kLuNb][kLuNb + 1];
    for (int t = threadIdx.x; t < kLuNb * kLuNb; t += blockDim.x) {
        const int r = t % kLuNb, c = t / kLuNb;
        s_l[r][c] = (r < nb && c < nb) ? A[(k + c) * lda + k + r] : 0.0;
    }
    __syncthreads();
    const int64_t c = k + nb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n) return;
    double *col = A + c * lda + k;
    double x[kLuNb];
#pragma unroll
    for (int i = 0; i < kLuNb; ++i) x[i] = i < nb ? col[i] : 0.0;
#pragma unroll
    for (int i = 1; i < kLuNb; ++i) {
        double s = x[i];
#pragma unroll
        for (int p = 0; p < i; ++p) s = fma(-s_l[i][p], x[p], s);
        x[i] = s;
    }
#pragma unroll
    for (int i = 0; i < kLuNb; ++i)
        if (i < nb) col[i] = x[i];
}

// A22 -= L21 U12 over rows and columns [k + nb, n): 64 x 64 tiles, 256 threads,
// 4 x 4 entries per thread (rows tx + 16 i, columns ty + 16 j: consecutive
// threads touch consecutive rows of a column).
__global__ void __launch_bounds__(256) lu_gemm_kernel(double *A, int64_t lda, int64_t n, int64_t k, int nb) {
    __shared__ double s_a[kLuNb][64];      // L21 tile: [p][row]
    __shared__ double s_b[64][kLuNb + 1];  // U12 tile: [column][p]
    const int64_t base = k + nb;
    const int64_t r0 = base + blockIdx.x * 64, c0 = base + blockIdx.y * 64;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int t = tid; t < kLuNb * 64; t += 256) {
        const int p = t / 64, r = t % 64;
        s_a[p][r] = (p < nb && r0 + r < n) ? A[(k + p) * lda + r0 + r] : 0.0;
        const int cc = t / kLuNb, q = t % kLuNb;
        s_b[cc][q] = (q < nb && c0 + cc < n) ? A[(c0 + cc) * lda + k + q] : 0.0;
    }
    __syncthreads();
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 8
    for (int p = 0; p < kLuNb; ++p) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = s_a[p][tx + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = s_b[ty + 16 * j][p];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + ty + 16 * j;
        if (c >= n) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t r = r0 + tx + 16 * i;
            if (r < n) A[c * lda + r] -= acc[i][j];
        }
    }
}

// Forward solve, panel k: the panel's swaps on x, then the unit lower
// triangle L11 (one thread, nb <= 32 rows).
__global__ void lu_fwd_diag_kernel(const double *A, int64_t lda, int64_t k, int nb, const int *piv, double *x) {
    for (int j = 0; j < nb; ++j) {
        const int64_t p = piv[k + j];
        if (p != k + j) {
            const double t = x[k + j];
            x[k + j] = x[p];
            x[p] = t;
        }
    }
    for (int i = 1; i < nb; ++i) {
        double s = x[k + i];
        for (int p = 0; p < i; ++p) s = fma(-A[(k + p) * lda + k + i], x[k + p], s);
        x[k + i] = s;
    }
}

// Backward solve, panel k: the upper triangle U11 (one thread).
__global__ void lu_bwd_diag_kernel(const double *A, int64_t lda, int64_t k, int nb, double *x) {
    for (int i = nb - 1; i >= 0; --i) {
        double s = x[k + i];
        for (int p = i + 1; p < nb; ++p) s = fma(-A[(k + p) * lda + k + i], x[k + p], s);
        x[k + i] = s / A[(k + i) * lda + k + i];
    }
}

// x[r] -= sum_p A[r, k + p] x[k + p] for rows r in [r0, r1): the panel's
// columns applied to the rest of the right-hand side.
__global__ void lu_update_kernel(const double *A, int64_t lda, int64_t k, int nb, int64_t r0, int64_t r1, double *x) {
    const int64_t r = r0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= r1) return;
    double s = x[r];
    for (int p = 0; p < nb; ++p) s = fma(-A[(k + p) * lda + r], x[k + p], s);
    x[r] = s;
}

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

cudaError_t lu_factor(double *A, int64_t lda, int64_t n, int *piv, int *info, cudaStream_t st, int64_t *launches) {
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), st);
    for (int64_t k = 0; k < n && e == cudaSuccess; k += kLuNb) {
        const int nb = (int)std::min<int64_t>(kLuNb, n - k);
        lu_panel_kernel<<<1, kPanelThreads, 0, st>>>(A, lda, n, k, nb, piv, info);
        ++*launches;
        const int64_t rest = n - k - nb;
        if (rest > 0) {
            lu_swap_kernel<<<(unsigned)cdiv(rest, 128), 128, 0, st>>>(A, lda, n, k, nb, k + nb, piv);
            lu_trsm_kernel<<<(unsigned)cdiv(rest, 128), 128, 0, st>>>(A, lda, n, k, nb);
            lu_gemm_kernel<<<dim3((unsigned)cdiv(rest, 64), (unsigned)cdiv(rest, 64)), 256, 0, st>>>(A, lda, n, k, nb);
            *launches += 3;
        }
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t lu_solve(const double *A, int64_t lda, int64_t n, const int *piv, double *x, cudaStream_t st,
                     int64_t *launches) {
    cudaError_t e = cudaSuccess;
    for (int64_t k = 0; k < n && e == cudaSuccess; k += kLuNb) {
        const int nb = (int)std::min<int64_t>(kLuNb, n - k);
        lu_fwd_diag_kernel<<<1, 1, 0, st>>>(A, lda, k, nb, piv, x);
        ++*launches;
        if (k + nb < n) {
            lu_update_kernel<<<(unsigned)cdiv(n - k - nb, 256), 256, 0, st>>>(A, lda, k, nb, k + nb, n, x);
            ++*launches;
        }
        e = cudaGetLastError();
    }
    const int64_t last = ((n - 1) / kLuNb) * kLuNb;
    for (int64_t k = last; k >= 0 && e == cudaSuccess; k -= kLuNb) {
        const int nb = (int)std::min<int64_t>(kLuNb, n - k);
        lu_bwd_diag_kernel<<<1, 1, 0, st>>>(A, lda, k, nb, x);
        ++*launches;
        if (k > 0) {
            lu_update_kernel<<<(unsigned)cdiv(k, 256), 256, 0, st>>>(A, lda, k, nb, 0, k, x);
            ++*launches;
        }
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace rf
