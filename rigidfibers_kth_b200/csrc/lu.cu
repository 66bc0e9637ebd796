// lu.cu - the direct variant of the solve: dense LU factorisation with
// partial pivoting and the two triangular solves, FP64 on the device.
//
// Reference: LAPACK dgesv called by fortran/coeffs_and_vels.f90:62,158,333,514
// (the *_direct golden runs).  Blocked right-looking factorisation, panel
// width kLuNb = 64:
//   lu_panel_kernel  a cluster of 8 CTAs factors 8 columns of the tall
//                    panel A[k:n, k:k+nb]: per column the pivot (first row of
//                    largest magnitude, as idamax), the row swap across the
//                    panel, the scaling by the reciprocal pivot and the rank-1
//                    update of the 8 columns (dgetf2's steps; the last three
//                    and the next pivot search in one pass over the rows);
//   lu_panel_update_kernel  the 8 columns' update of the rest of the panel,
//                    over the whole GPU;
//   lu_swap_kernel   the panel's row swaps applied to the trailing columns;
//   lu_trsm_kernel   U12 = L11^-1 A12, one thread per trailing column;
//   cublasDgemm      A22 -= L21 U12, the rank-64 trailing update (a plain
//                    GEMM: most of the 2/3 n^3 flops).  The wider panel
//                    halves the passes over the trailing matrix that
//                    32-column panels needed.
// The swaps are not applied to the L columns left of a panel: the forward
// solve applies each panel's swaps to the right-hand side just before that
// panel's columns of L, which is the same elimination (LINPACK's order).
// Info as LAPACK: the first zero pivot (1-based), 0 when there is none.
#include <cooperative_groups.h>
#include <cublas_v2.h>

#include <algorithm>

#include "rf_kernels.h"

namespace rf {
namespace {

namespace cg = cooperative_groups;

constexpr int kLuNb = 64;
constexpr int kLuSub = 8;   // sub-panel width: the columns one CTA factors
constexpr int kPanelThreads = 512;
constexpr int kRowBatch = 2;  // rows per thread whose loads are issued together in the panel's passes
constexpr int kPanelCluster = 8;  // CTAs (SMs) that factor one sub-panel together

__device__ __forceinline__ void argmax_merge(double &v, int64_t &i, double ov, int64_t oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

// Block-wide first-maximum reduction of (value, row) pairs; every thread gets
// the row (and, in *vmax, the value).
__device__ __forceinline__ int64_t block_argmax(double best, int64_t bi, int64_t none, double *s_val,
                                                int64_t *s_idx, double *vmax) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int o = 16; o; o >>= 1)
        argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, o), __shfl_down_sync(0xffffffffu, bi, o));
    if (lane == 0) {
        s_val[warp] = best;
        s_idx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
        best = lane < nwarps ? s_val[lane] : -1.0;
        bi = lane < nwarps ? s_idx[lane] : none;
        for (int o = 16; o; o >>= 1)
            argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, o), __shfl_down_sync(0xffffffffu, bi, o));
        if (lane == 0) {
            s_idx[0] = bi;
            s_val[0] = best;
        }
    }
    __syncthreads();
    const int64_t r = s_idx[0];
    *vmax = s_val[0];
    __syncthreads();  // s_idx is reused by the next reduction
    return r;
}

// Sub-panel factorisation: columns [s0, s0 + sb) of the panel [k, k + nb),
// on one cluster of kPanelCluster CTAs (one per SM), the rows below the
// diagonal interleaved over all their threads.  One pass per column over
// those rows: scale the column by the reciprocal pivot, update the
// sub-panel's remaining columns (the pivot row's entries staged in shared
// memory) and, in the same pass, find the next column's pivot among the
// updated values.  Each CTA's candidate (value, row) goes to a slot in the
// shared memory of the cluster's first CTA, and every CTA merges the slots
// in the same way (first maximum: the same pivot as one CTA over all rows).
// Row swaps (by the first CTA) cover all nb columns of the panel, so its L
// is consistent.  Then U of the sub-panel's rows for the panel's columns
// right of it (unit lower sb x sb triangle, one thread per column).
// Every thread of the cluster passes the same 1 + 2 sb cluster barriers.
__global__ void __cluster_dims__(kPanelCluster, 1, 1) __launch_bounds__(kPanelThreads)
    lu_panel_kernel(double *A, int64_t lda, int64_t n, int64_t k, int nb, int64_t s0, int sb, int *piv, int *info) {
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();
    __shared__ double s_val[kPanelThreads / 32];
    __shared__ int64_t s_idx[kPanelThreads / 32];
    __shared__ double s_u[kLuSub];
    __shared__ double c_val[kPanelCluster];   // pivot candidates (the first CTA's copy is used)
    __shared__ int64_t c_idx[kPanelCluster];
    double *r_val = cluster.map_shared_rank(c_val, 0);
    int64_t *r_idx = cluster.map_shared_rank(c_idx, 0);
    const int tid = threadIdx.x;
    const int64_t g = (int64_t)rank * kPanelThreads + tid;  // this thread's offset among the cluster's rows
    constexpr int64_t kStride = (int64_t)kPanelCluster * kPanelThreads;
    // the cluster's first maximum; ends with the row pass's stores visible
    // to every CTA (fence, then the barrier)
    auto cluster_argmax = [&](double best, int64_t bi) -> int64_t {
        double v;
        const int64_t r = block_argmax(best, bi, n, s_val, s_idx, &v);
        if (tid == 0) {
            r_val[rank] = v;
            r_idx[rank] = r;
        }
        __threadfence();
        cluster.sync();
        double bv = -1.0;
        int64_t bidx = n;
        for (int q = 0; q < kPanelCluster; ++q) argmax_merge(bv, bidx, r_val[q], r_idx[q]);
        return bidx;
    };
    double best = -1.0;
    int64_t bi = n;
    for (int64_t r = s0 + g; r < n; r += kStride) argmax_merge(best, bi, fabs(A[s0 * lda + r]), r);
    int64_t p = cluster_argmax(best, bi);
    for (int j = 0; j < sb; ++j) {
        const int64_t col = s0 + j;
        if (p >= n) p = col;  // a column of NaN keeps its row
        if (rank == 0) {
            if (tid == 0) piv[col] = (int)p;
            if (p != col && tid < nb) {
                double *c = A + (k + tid) * lda;
                const double t = c[col];
                c[col] = c[p];
                c[p] = t;
            }
        }
        __threadfence();
        cluster.sync();  // the swapped rows, seen by every CTA
        double *cj = A + col * lda;
        const double d = cj[col];
        if (tid < sb) s_u[tid] = tid > j ? A[(s0 + tid) * lda + col] : 0.0;
        if (rank == 0 && d == 0.0 && tid == 0 && *info == 0) *info = (int)(col + 1);
        __syncthreads();
        const double inv = d != 0.0 ? 1.0 / d : 0.0;  // a zero pivot leaves a zero column (dgetf2)
        best = -1.0;
        bi = n;
        // kRowBatch rows per thread and round: all their loads are issued
        // before the stores (the stores of one row could otherwise hold back
        // the loads of the next); the pivot search is order-independent
        for (int64_t rb = col + 1 + g; rb < n; rb += (int64_t)kRowBatch * kStride) {
            double xs[kRowBatch], vs[kRowBatch][kLuSub];
#pragma unroll
            for (int u = 0; u < kRowBatch; ++u) {
                const int64_t r = rb + (int64_t)u * kStride;
                if (r < n) {
                    xs[u] = cj[r];
#pragma unroll
                    for (int c = 0; c < kLuSub; ++c)
                        if (c > j && c < sb) vs[u][c] = A[(s0 + c) * lda + r];
                }
            }
#pragma unroll
            for (int u = 0; u < kRowBatch; ++u) {
                const int64_t r = rb + (int64_t)u * kStride;
                if (r < n) {
                    const double x = d != 0.0 ? xs[u] * inv : xs[u];
                    cj[r] = x;
#pragma unroll
                    for (int c = 0; c < kLuSub; ++c)
                        if (c > j && c < sb) {
                            const double v = fma(-x, s_u[c], vs[u][c]);
                            A[(s0 + c) * lda + r] = v;
                            if (c == j + 1) argmax_merge(best, bi, fabs(v), r);
                        }
                }
            }
        }
        if (j + 1 < sb) {
            p = cluster_argmax(best, bi);
        } else {
            __threadfence();
            cluster.sync();  // every CTA's rows written before the U rows below read them
        }
    }
    // U rows of the sub-panel for the panel's columns right of it
    const int64_t c = s0 + sb + tid;
    if (rank == 0 && c < k + nb && c < n) {
        double *col = A + c * lda + s0;
        for (int i = 1; i < sb; ++i) {
            double v = col[i];
            for (int q = 0; q < i; ++q) v = fma(-A[(s0 + q) * lda + s0 + i], col[q], v);
            col[i] = v;
        }
    }
}

// The sub-panel's rank-sb update of the panel's columns right of it:
// A[r, c] -= sum_q A[r, s0 + q] A[s0 + q, c] for rows r >= s0 + sb and columns
// c in [s0 + sb, k + nb); one thread per row and group of kUpdCols columns
// (blockIdx.y), the U entries in shared memory.
constexpr int kUpdCols = 8;
constexpr int kUpdThreads = 128;
__global__ void __launch_bounds__(kUpdThreads) lu_panel_update_kernel(double *A, int64_t lda, int64_t n, int64_t k,
                                                                      int nb, int64_t s0, int sb) {
    __shared__ double s_uu[kUpdCols][kLuSub];
    const int64_t c0 = s0 + sb + (int64_t)blockIdx.y * kUpdCols;
    const int64_t c1 = std::min<int64_t>(std::min<int64_t>(k + nb, n), c0 + kUpdCols);
    const int nc = (int)(c1 - c0);
    for (int t = threadIdx.x; t < nc * sb; t += blockDim.x) {
        const int c = t / sb, q = t % sb;
        s_uu[c][q] = A[(c0 + c) * lda + s0 + q];
    }
    __syncthreads();
    const int64_t r = s0 + sb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    double l[kLuSub];
#pragma unroll
    for (int q = 0; q < kLuSub; ++q) l[q] = q < sb ? A[(s0 + q) * lda + r] : 0.0;
    for (int c = 0; c < nc; ++c) {
        double v = A[(c0 + c) * lda + r];
#pragma unroll
        for (int q = 0; q < kLuSub; ++q)
            if (q < sb) v = fma(-l[q], s_uu[c][q], v);
        A[(c0 + c) * lda + r] = v;
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

// Forward solve, panel k: the panel's swaps on x, then the unit lower
// triangle L11; one CTA of kLuNb threads.  The rows the swaps touch (the
// panel's nb rows and up to nb pivot rows below) are loaded at once, the
// swaps applied in order in shared memory and the rows written back; then
// L11 from shared memory, one column per step.
__global__ void __launch_bounds__(kLuNb) lu_fwd_diag_kernel(const double *A, int64_t lda, int64_t k, int nb,
                                                            const int *piv, double *x) {
    __shared__ double s_l[kLuNb][kLuNb + 1];
    __shared__ double s_x[2 * kLuNb];
    __shared__ int64_t s_p[kLuNb];
    __shared__ int s_slot[kLuNb];
    const int t = threadIdx.x;
    if (t < nb) {
        s_p[t] = piv[k + t];
        s_x[t] = x[k + t];
        for (int p = 0; p < nb; ++p) s_l[t][p] = A[(k + p) * lda + k + t];
    }
    __syncthreads();
    if (t < nb) {
        // slot of pivot row p_t: inside the panel its own row, below it the
        // slot of the first swap that names the same row
        const int64_t p = s_p[t];
        int slot = (int)(p - k);
        if (p >= k + nb) {
            slot = kLuNb + t;
            for (int q = 0; q < t; ++q)
                if (s_p[q] == p) {
                    slot = kLuNb + q;
                    break;
                }
            if (slot == kLuNb + t) s_x[slot] = x[p];
        }
        s_slot[t] = slot;
    }
    __syncthreads();
    if (t == 0)
        for (int q = 0; q < nb; ++q) {
            const int o = s_slot[q];
            if (o != q) {
                const double v = s_x[q];
                s_x[q] = s_x[o];
                s_x[o] = v;
            }
        }
    __syncthreads();
    if (t < nb && s_slot[t] == kLuNb + t) x[s_p[t]] = s_x[kLuNb + t];
    for (int p = 0; p + 1 < nb; ++p) {
        if (t > p && t < nb) s_x[t] = fma(-s_l[t][p], s_x[p], s_x[t]);
        __syncthreads();
    }
    if (t < nb) x[k + t] = s_x[t];
}

// Backward solve, panel k: the upper triangle U11, one CTA of kLuNb threads,
// U11 from shared memory, one column per step (last first).
__global__ void __launch_bounds__(kLuNb) lu_bwd_diag_kernel(const double *A, int64_t lda, int64_t k, int nb,
                                                            double *x) {
    __shared__ double s_u[kLuNb][kLuNb + 1];
    __shared__ double s_x[kLuNb];
    const int t = threadIdx.x;
    if (t < nb) {
        s_x[t] = x[k + t];
        for (int p = 0; p < nb; ++p) s_u[t][p] = A[(k + p) * lda + k + t];
    }
    __syncthreads();
    for (int p = nb - 1; p >= 0; --p) {
        if (t == p) s_x[p] = s_x[p] / s_u[p][p];
        __syncthreads();
        if (t < p) s_x[t] = fma(-s_u[t][p], s_x[p], s_x[t]);
        __syncthreads();
    }
    if (t < nb) x[k + t] = s_x[t];
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

cudaError_t lu_factor(double *A, int64_t lda, int64_t n, int *piv, int *info, void *blas, cudaStream_t st,
                      int64_t *launches) {
    if (!blas || lda > INT32_MAX || n > INT32_MAX) return cudaErrorInvalidValue;
    cublasHandle_t bh = static_cast<cublasHandle_t>(blas);
    if (cublasSetStream(bh, st) != CUBLAS_STATUS_SUCCESS) return cudaErrorUnknown;
    const double minus_one = -1.0, one = 1.0;
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), st);
    for (int64_t k = 0; k < n && e == cudaSuccess; k += kLuNb) {
        const int nb = (int)std::min<int64_t>(kLuNb, n - k);
        for (int s0 = 0; s0 < nb; s0 += kLuSub) {
            const int sb = std::min(kLuSub, nb - s0);
            lu_panel_kernel<<<kPanelCluster, kPanelThreads, 0, st>>>(A, lda, n, k, nb, k + s0, sb, piv, info);
            ++*launches;
            if (s0 + sb < nb && k + s0 + sb < n) {
                const dim3 grid((unsigned)cdiv(n - k - s0 - sb, kUpdThreads),
                                (unsigned)cdiv(std::min<int64_t>(nb, n - k) - s0 - sb, kUpdCols));
                lu_panel_update_kernel<<<grid, kUpdThreads, 0, st>>>(A, lda, n, k, nb, k + s0, sb);
                ++*launches;
            }
        }
        const int64_t rest = n - k - nb;
        if (rest > 0) {
            lu_swap_kernel<<<(unsigned)cdiv(rest, 128), 128, 0, st>>>(A, lda, n, k, nb, k + nb, piv);
            lu_trsm_kernel<<<(unsigned)cdiv(rest, 128), 128, 0, st>>>(A, lda, n, k, nb);
            *launches += 2;  // the GEMM below is cuBLAS's
            e = cudaGetLastError();
            if (e != cudaSuccess) break;
            const int r = (int)rest, ld = (int)lda;
            if (cublasDgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, r, r, nb, &minus_one, A + k * lda + k + nb, ld,
                            A + (k + nb) * lda + k, ld, &one, A + (k + nb) * lda + k + nb, ld) != CUBLAS_STATUS_SUCCESS)
                return cudaErrorUnknown;
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    return e;
}

cudaError_t lu_solve(const double *A, int64_t lda, int64_t n, const int *piv, double *x, cudaStream_t st,
                     int64_t *launches) {
    cudaError_t e = cudaSuccess;
    for (int64_t k = 0; k < n && e == cudaSuccess; k += kLuNb) {
        const int nb = (int)std::min<int64_t>(kLuNb, n - k);
        lu_fwd_diag_kernel<<<1, kLuNb, 0, st>>>(A, lda, k, nb, piv, x);
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
        lu_bwd_diag_kernel<<<1, kLuNb, 0, st>>>(A, lda, k, nb, x);
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
