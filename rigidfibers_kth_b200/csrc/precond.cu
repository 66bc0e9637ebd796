// precond.cu - neighbour-block preconditioners for the right-preconditioned GMRES.
//
// The 3N x 3N diagonal blocks of A are the identity (matrix_assembly.f90:
// 489-492), so plain block-Jacobi is no preconditioning at all, and no
// block-diagonal correction helps either: the lowest eigenvalues of A belong
// to modes localised on two or three close fibers (a pair coupled by a block
// C has eigenvalues 1 +- sigma(C); a block-diagonal P maps them to
// 1/(1 -+ sigma) and keeps their ratio), the highest to modes spread over
// tens of fibers in the dense core.  What does help is coupling a fiber to
// its nearest neighbours:
//
//   z_i = v_i + sum_{m < kp} B_{i,m} v_{j_m},   j_m = the m-th nearest neighbour
//
// with B_{i,m} the coupling blocks of the local inverse:
//
//   RF_PC_CLUSTER  B_{i,m} = [S_i^-1]_{0, m+1}, S_i = A restricted to fiber i
//                  and its kc nearest neighbours (the exact local-cluster
//                  inverse); one CTA per fiber factorises S_i^T in shared
//                  memory (FP32 LU with partial pivoting) and keeps the
//                  first block row.
//   RF_PC_LEARNED  B_{i,m} predicted by a small MLP from the geometry of the
//                  16 nearest neighbours expressed in a frame attached to
//                  fiber i, neighbour m listed first (one evaluation per
//                  pair).  Blocks transform as B(Q config) = Q B(config) Q^T
//                  under rotations Q, and neighbour m's orientation enters
//                  with a canonical sign (the block's odd-order columns
//                  change sign with it), so the network only learns the
//                  rotation- and sign-free part.
//
// The MLP (144 -> 256 -> 256 -> 225, ReLU) is trained by the trainer below
// with hand-written FP32 GEMM kernels (forward and backward) and Adam.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "handle.h"

namespace rf {
namespace {

constexpr int kK = RF_MLP_K;          // neighbours in the features
constexpr int kPair = RF_MLP_PAIRS;   // neighbour blocks per fiber
constexpr int kIn = RF_MLP_IN;        // 144
constexpr int kHid = RF_MLP_HIDDEN;   // 256
constexpr int kOut = RF_MLP_OUT;      // 225
constexpr int kNb = 15;               // block size the MLP is built for (N = 5)

// ------------------------------------------------------------------ k-NN
// One warp per fiber: every lane keeps the K nearest of its sources j = lane,
// lane + 32, ... sorted in registers (unrolled compare-and-swap), then K rounds
// of a warp arg-min over the lane heads merge them.  Order: distance, then the
// lower source index (the order of a sequential scan with strict comparison).
constexpr int kKnnWarps = 4;
__global__ void __launch_bounds__(kKnnWarps * 32) knn_kernel(int M, const double *__restrict__ pos, int K,
                                                             int *__restrict__ knn) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kKnnWarps + (threadIdx.x >> 5);
    if (i >= M) return;  // whole warp
    float bd[kK];
    int bi[kK];
#pragma unroll
    for (int r = 0; r < kK; ++r) {
        bd[r] = 3.4e38f;
        bi[r] = 0x7fffffff;
    }
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int j = lane; j < M; j += 32) {
        if (j == i) continue;
        const float dx = (float)(__ldg(pos + 3 * j) - xi), dy = (float)(__ldg(pos + 3 * j + 1) - yi),
                    dz = (float)(__ldg(pos + 3 * j + 2) - zi);
        float d = dx * dx + dy * dy + dz * dz;
        if (!(d < bd[kK - 1])) continue;
        int jj = j;
#pragma unroll
        for (int r = 0; r < kK; ++r) {
            if (d < bd[r]) {  // this lane's sources arrive in increasing j: ties keep the earlier one
                const float td = bd[r];
                const int ti = bi[r];
                bd[r] = d;
                bi[r] = jj;
                d = td;
                jj = ti;
            }
        }
    }
    for (int r = 0; r < K; ++r) {
        // lexicographic arg-min of (distance, index) over the lane heads
        float md = bd[0];
        int mi = bi[0];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, md, o);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, o);
            if (od < md || (od == md && oi < mi)) {
                md = od;
                mi = oi;
            }
        }
        if (lane == 0) knn[(int64_t)i * K + r] = mi < M ? mi : -1;
        if (bi[0] == mi && bd[0] == md) {  // the winning lane pops its head
#pragma unroll
            for (int q = 0; q < kK - 1; ++q) {
                bd[q] = bd[q + 1];
                bi[q] = bi[q + 1];
            }
            bd[kK - 1] = 3.4e38f;
            bi[kK - 1] = 0x7fffffff;
        }
    }
}

// ------------------------------------------------------------------ cluster inverse rows
// S = A[C, C] with C = {i, knn_0, .., knn_{kc-1}}; solve S^T X = E (E = the
// first nb columns of the identity) by LU with partial pivoting in shared
// memory: X^T is the first block row of S^-1, and its column blocks 1..kp are
// the couplings B_{i,m} (out[i][m], row-major nb x nb; zero for m >= kp).
template <typename T>
__global__ void __launch_bounds__(256) cluster_rows_kernel(int M, int nb, const T *__restrict__ A, int64_t lda,
                                                           int64_t plane, const int *__restrict__ knn, int kstride,
                                                           int kc, int kp, float *__restrict__ out,
                                                           int *__restrict__ singular) {
    extern __shared__ float sm[];
    __shared__ int s_fib[32];
    __shared__ int s_piv;
    __shared__ float s_pval;
    const int i = blockIdx.x;
    const int s = (kc + 1) * nb;
    const int w = s + nb;       // augmented width
    const int ld = w + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid <= kc) s_fib[tid] = tid == 0 ? i : knn[(int64_t)i * kstride + tid - 1];
    __syncthreads();
    // gather S^T: sm[r][c] = S[c][r] = A(row of cluster index c, column of r);
    // consecutive threads read consecutive rows of one column of A
    for (int idx = tid; idx < s * s; idx += nt) {
        const int r = idx / s, c = idx - r * s;
        const int64_t gr = (int64_t)s_fib[c / nb] * nb + c % nb;
        const int64_t gc = (int64_t)s_fib[r / nb] * nb + r % nb;
        sm[r * ld + c] = (float)load_entry<T>(A, gc * lda + gr, plane);
    }
    for (int idx = tid; idx < s * nb; idx += nt) {
        const int r = idx / nb, j = idx - r * nb;
        sm[r * ld + s + j] = (r == j) ? 1.f : 0.f;
    }
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < s; ++k) {
        // pivot: warp 0 finds the largest |S[r][k]|, r >= k
        if (tid < 32) {
            float best = -1.f;
            int br = k;
            for (int r = k + tid; r < s; r += 32) {
                const float v = fabsf(sm[r * ld + k]);
                if (v > best) {
                    best = v;
                    br = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int orow = __shfl_xor_sync(0xffffffffu, br, o);
                if (ob > best || (ob == best && orow < br)) {
                    best = ob;
                    br = orow;
                }
            }
            if (tid == 0) {
                s_piv = br;
                s_pval = best;
            }
        }
        __syncthreads();
        if (!(s_pval > 0.f)) {
            bad = true;
            break;
        }
        const int p = s_piv;
        if (p != k)
            for (int c = k + tid; c < w; c += nt) {
                const float t = sm[k * ld + c];
                sm[k * ld + c] = sm[p * ld + c];
                sm[p * ld + c] = t;
            }
        __syncthreads();
        const float inv = 1.f / sm[k * ld + k];
        for (int r = k + 1 + tid; r < s; r += nt) sm[r * ld + k] *= inv;
        __syncthreads();
        const int rows = s - k - 1, cols = w - k - 1;
        for (int idx = tid; idx < rows * cols; idx += nt) {
            const int rr = idx / cols, cc = idx - rr * cols;
            const int r = k + 1 + rr, c = k + 1 + cc;
            sm[r * ld + c] -= sm[r * ld + k] * sm[k * ld + c];
        }
        __syncthreads();
    }
    float *dst = out + (int64_t)i * kPair * nb * nb;
    if (bad) {
        if (tid == 0) atomicAdd(singular, 1);
        for (int idx = tid; idx < kPair * nb * nb; idx += nt) dst[idx] = 0.f;  // P = I for this fiber
        return;
    }
    // back substitution on the nb right-hand sides, column-oriented: x_k,
    // then remove its contribution from the rows above
    for (int k = s - 1; k >= 0; --k) {
        if (tid < nb) sm[k * ld + s + tid] /= sm[k * ld + k];
        __syncthreads();
        for (int idx = tid; idx < k * nb; idx += nt) {
            const int r = idx / nb, j = idx - r * nb;
            sm[r * ld + s + j] -= sm[r * ld + k] * sm[k * ld + s + j];
        }
        __syncthreads();
    }
    // B_{i,m}[a][b] = (S^-1)[a][(m+1) nb + b] = X[(m+1) nb + b][a]
    for (int idx = tid; idx < kPair * nb * nb; idx += nt) {
        const int m = idx / (nb * nb), e = idx - m * nb * nb;
        const int a = e / nb, b = e - a * nb;
        dst[idx] = m < kp ? sm[((m + 1) * nb + b) * ld + s + a] : 0.f;
    }
}

// ------------------------------------------------------------------ features
// Frame of fiber i: e3 = t_i, e1 = the direction to the nearest neighbour
// with its t_i component removed, e2 = e3 x e1 (rows of E).
__device__ void fiber_frame(const double *__restrict__ pos, const double *__restrict__ ori, int i, int j0,
                            double E[3][3]) {
    const double *xi = pos + 3 * i, *ti = ori + 3 * i;
    const double e3[3] = {ti[0], ti[1], ti[2]};
    const double d1[3] = {pos[3 * j0] - xi[0], pos[3 * j0 + 1] - xi[1], pos[3 * j0 + 2] - xi[2]};
    double dot = d1[0] * e3[0] + d1[1] * e3[1] + d1[2] * e3[2];
    double e1[3] = {d1[0] - dot * e3[0], d1[1] - dot * e3[1], d1[2] - dot * e3[2]};
    double n1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    if (n1 < 1e-9) {  // neighbour on the axis: any perpendicular direction
        const double a[3] = {fabs(e3[0]) < 0.9 ? 1.0 : 0.0, fabs(e3[0]) < 0.9 ? 0.0 : 1.0, 0.0};
        dot = a[0] * e3[0] + a[1] * e3[1];
        e1[0] = a[0] - dot * e3[0];
        e1[1] = a[1] - dot * e3[1];
        e1[2] = -dot * e3[2];
        n1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    }
    for (int a = 0; a < 3; ++a) e1[a] /= n1;
    const double e2[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
    for (int c = 0; c < 3; ++c) {
        E[0][c] = e1[c];
        E[1][c] = e2[c];
        E[2][c] = e3[c];
    }
}

// Features of the pair (fiber i, neighbour m), one thread per pair: nine
// floats per neighbour in fiber i's frame.  Slot 0 is neighbour m: its
// relative centre, its orientation u with the canonical sign (u_z > 0, ties
// broken by u_y then u_x; the sign goes to sign[]) and u squared; slots
// 1..15 are the other neighbours, nearest first: relative centre and the six
// products u_a u_b (the sign of their orientation does not change block m).
__global__ void pair_features_kernel(int M, int kp, const double *__restrict__ pos, const double *__restrict__ ori,
                                     const int *__restrict__ knn, float *__restrict__ feat,
                                     float *__restrict__ sign, float *__restrict__ rot) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)M * kp) return;
    const int i = (int)(t / kp), m = (int)(t - (int64_t)i * kp);
    const int *nb = knn + (int64_t)i * kK;
    double E[3][3];
    fiber_frame(pos, ori, i, nb[0], E);
    if (m == 0)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) rot[(int64_t)i * 9 + r * 3 + c] = (float)E[r][c];
    const double *xi = pos + 3 * i;
    float *f = feat + t * kIn;
    auto local = [&](int j, double dl[3], double ul[3]) {
        const double d[3] = {pos[3 * j] - xi[0], pos[3 * j + 1] - xi[1], pos[3 * j + 2] - xi[2]};
        const double *tj = ori + 3 * j;
        for (int r = 0; r < 3; ++r) {
            dl[r] = E[r][0] * d[0] + E[r][1] * d[1] + E[r][2] * d[2];
            ul[r] = E[r][0] * tj[0] + E[r][1] * tj[1] + E[r][2] * tj[2];
        }
    };
    double dl[3], ul[3];
    local(nb[m], dl, ul);
    const bool pos_sign = ul[2] > 0.0 || (ul[2] == 0.0 && (ul[1] > 0.0 || (ul[1] == 0.0 && ul[0] >= 0.0)));
    const double s = pos_sign ? 1.0 : -1.0;
    sign[t] = (float)s;
    for (int r = 0; r < 3; ++r) {
        f[r] = (float)dl[r];
        f[3 + r] = (float)(s * ul[r]);
        f[6 + r] = (float)(ul[r] * ul[r]);
    }
    int slot = 1;
    for (int n = 0; n < kK; ++n) {
        if (n == m) continue;
        local(nb[n], dl, ul);
        float *g = f + slot * 9;
        g[0] = (float)dl[0];
        g[1] = (float)dl[1];
        g[2] = (float)dl[2];
        g[3] = (float)(ul[0] * ul[0]);
        g[4] = (float)(ul[1] * ul[1]);
        g[5] = (float)(ul[2] * ul[2]);
        g[6] = (float)(ul[0] * ul[1]);
        g[7] = (float)(ul[0] * ul[2]);
        g[8] = (float)(ul[1] * ul[2]);
        ++slot;
    }
}

// local <-> global pair blocks: B = (R_blk^T O R_blk) D (to_global) or
// O = (R_blk B R_blk^T) D (to_local), R_blk = I_5 (x) R of fiber i, D = the
// pair's sign on the columns of odd Legendre order k (lb = k - 1 even).  One
// thread per pair block; the output of pairs m >= kp is zero.
__global__ void pair_frame_kernel(int M, int kp, const float *__restrict__ rot, const float *__restrict__ sign,
                                  const float *__restrict__ in, int64_t in_stride, float *__restrict__ out,
                                  int64_t out_stride, int to_global) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)M * kPair) return;
    const int i = (int)(t / kPair), m = (int)(t - (int64_t)i * kPair);
    const int64_t q = (int64_t)i * kp + m;  // row of the per-pair arrays (features, MLP output)
    float *Y = out + (to_global ? t : q) * out_stride;
    if (m >= kp) {
        if (to_global)
            for (int e = 0; e < kOut; ++e) Y[e] = 0.f;
        return;
    }
    float R[9];
    for (int e = 0; e < 9; ++e) R[e] = rot[(int64_t)i * 9 + e];
    const float s = sign[q];
    const float *X = in + (to_global ? q : t) * in_stride;
    for (int kb = 0; kb < 5; ++kb)
        for (int lb = 0; lb < 5; ++lb) {
            float O[3][3], T[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) O[a][b] = X[(kb * 3 + a) * kNb + lb * 3 + b];
            // to_global: Z = R^T O R ; to_local: Z = R O R^T
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    float acc = 0.f;
                    for (int c = 0; c < 3; ++c) acc += O[a][c] * (to_global ? R[c * 3 + b] : R[b * 3 + c]);
                    T[a][b] = acc;
                }
            const float d = (lb % 2 == 0) ? s : 1.f;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    float acc = 0.f;
                    for (int c = 0; c < 3; ++c) acc += (to_global ? R[c * 3 + a] : R[a * 3 + c]) * T[c][b];
                    Y[(kb * 3 + a) * kNb + lb * 3 + b] = d * acc;
                }
        }
}

// ------------------------------------------------------------------ FP32 GEMM
// C[i][j] = act( alpha * sum_k A(i,k) B(k,j) + bias[j] ) (+ beta C), generic
// strides so one kernel serves X W^T, dY W and dY^T X.  64x64 tiles, 16-deep,
// 256 threads with 4x4 outputs each.
struct GemmArgs {
    int m, n, k;
    const float *A;
    int64_t sai, sak;
    const float *B;
    int64_t sbk, sbj;
    float *C;
    int64_t ldc;
    const float *bias;
    int relu;
    float beta;
};

__global__ void __launch_bounds__(256) gemm_kernel(GemmArgs g) {
    __shared__ float As[16][64 + 4];
    __shared__ float Bs[16][64 + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < g.k; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int kk = t / 64, r = t % 64;
            const int gi = i0 + r, gk = k0 + kk;
            As[kk][r] = (gi < g.m && gk < g.k) ? g.A[gi * g.sai + gk * g.sak] : 0.f;
            const int gj = j0 + r;
            Bs[kk][r] = (gj < g.n && gk < g.k) ? g.B[gk * g.sbk + gj * g.sbj] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = As[kk][ty * 4 + u];
                b[u] = Bs[kk][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i = i0 + ty * 4 + u, j = j0 + tx * 4 + v;
            if (i >= g.m || j >= g.n) continue;
            float val = acc[u][v];
            if (g.bias) val += g.bias[j];
            if (g.relu) val = fmaxf(val, 0.f);
            float *c = g.C + (int64_t)i * g.ldc + j;
            *c = g.beta != 0.f ? g.beta * *c + val : val;
        }
}

cudaError_t gemm(const GemmArgs &g, cudaStream_t st) {
    dim3 grid((g.n + 63) / 64, (g.m + 63) / 64);
    gemm_kernel<<<grid, 256, 0, st>>>(g);
    return cudaGetLastError();
}

// column sums of an m x n row-major matrix (bias gradients)
__global__ void colsum_kernel(int m, int n, const float *__restrict__ X, float *__restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float s = 0.f;
    for (int i = 0; i < m; ++i) s += X[(int64_t)i * n + j];
    out[j] = s;
}

// dY = 2 (Y - T) / count, and per-block partial sums of (Y - T)^2
__global__ void mse_grad_kernel(int64_t cnt, const float *__restrict__ Y, const float *__restrict__ T,
                                float *__restrict__ dY, double *__restrict__ part) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        const float d = Y[e] - T[e];
        dY[e] = 2.f * d / (float)cnt;
        acc += (double)d * d;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void relu_back_kernel(int64_t cnt, const float *__restrict__ H, float *__restrict__ dH) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
        if (H[e] <= 0.f) dH[e] = 0.f;
}

__global__ void adam_kernel(int64_t cnt, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[e];
        const float mi = b1 * m[e] + (1.f - b1) * gi;
        const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        w[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void gather_rows_kernel(int rows, int width, const int *__restrict__ idx, const float *__restrict__ src,
                                   float *__restrict__ dst) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows * width) return;
    const int r = (int)(e / width), c = (int)(e - (int64_t)r * width);
    dst[e] = src[(int64_t)idx[r] * width + c];
}

// parameter offsets inside the packed weight vector
struct MlpLayout {
    int64_t w1 = 0, b1 = w1 + (int64_t)kHid * kIn, w2 = b1 + kHid, b2 = w2 + (int64_t)kHid * kHid, w3 = b2 + kHid,
            b3 = w3 + (int64_t)kOut * kHid, total = b3 + kOut;
};

// Forward pass for `rows` samples: H1, H2, O (row-major)
cudaError_t mlp_forward(const float *W, int rows, const float *X, float *H1, float *H2, float *O, cudaStream_t st) {
    const MlpLayout L;
    GemmArgs g{};
    g.m = rows; g.n = kHid; g.k = kIn;
    g.A = X; g.sai = kIn; g.sak = 1;
    g.B = W + L.w1; g.sbk = 1; g.sbj = kIn;           // B(k,j) = W1[j][k]
    g.C = H1; g.ldc = kHid; g.bias = W + L.b1; g.relu = 1;
    cudaError_t e = gemm(g, st);
    if (e != cudaSuccess) return e;
    g.k = kHid; g.A = H1; g.sai = kHid; g.B = W + L.w2; g.sbj = kHid; g.C = H2; g.bias = W + L.b2;
    e = gemm(g, st);
    if (e != cudaSuccess) return e;
    g.n = kOut; g.A = H2; g.B = W + L.w3; g.sbj = kHid; g.C = O; g.ldc = kOut; g.bias = W + L.b3; g.relu = 0;
    return gemm(g, st);
}

}  // namespace

// ------------------------------------------------------------------ handle side
namespace {
// neighbours found by knn_kernel (stride kK per fiber) and blocks kept per fiber
int knn_count(const rf_handle *h) { return std::min(kK, h->M - 1); }

rf_status ensure_pair_buffers(rf_handle *h) {
    const int M = h->M, nb = 3 * h->N;
    auto ck = [&](cudaError_t e, const char *what) -> rf_status {
        return e == cudaSuccess ? RF_OK : cuda_fail(h, e, what);
    };
    rf_status s;
    if (!h->Pblocks &&
        (s = ck(cudaMalloc(&h->Pblocks, sizeof(float) * (size_t)M * kPair * nb * nb), "alloc blocks")) != RF_OK)
        return s;
    if (!h->knn && (s = ck(cudaMalloc(&h->knn, sizeof(int) * (size_t)M * kK), "alloc knn")) != RF_OK) return s;
    return RF_OK;
}

rf_status ensure_mlp_buffers(rf_handle *h) {
    const size_t rows = (size_t)h->M * kPair;
    auto ck = [&](cudaError_t e, const char *what) -> rf_status {
        return e == cudaSuccess ? RF_OK : cuda_fail(h, e, what);
    };
    rf_status s;
    if (h->feat) return RF_OK;
    // features, then the frames (9 per fiber) and the pair signs (1 per pair)
    if ((s = ck(cudaMalloc(&h->feat, sizeof(float) * (rows * kIn + (size_t)h->M * 9 + rows)), "alloc")) != RF_OK)
        return s;
    if ((s = ck(cudaMalloc(&h->mlp_h1, sizeof(float) * rows * kHid), "alloc")) != RF_OK) return s;
    if ((s = ck(cudaMalloc(&h->mlp_h2, sizeof(float) * rows * kHid), "alloc")) != RF_OK) return s;
    if ((s = ck(cudaMalloc(&h->mlp_out, sizeof(float) * rows * kOut), "alloc")) != RF_OK) return s;
    return RF_OK;
}

float *feat_rot(rf_handle *h) { return h->feat + (size_t)h->M * kPair * kIn; }
float *feat_sign(rf_handle *h) { return feat_rot(h) + (size_t)h->M * 9; }

cudaError_t launch_knn(rf_handle *h) {
    knn_kernel<<<(h->M + kKnnWarps - 1) / kKnnWarps, kKnnWarps * 32, 0, h->stream>>>(h->M, h->X[h->cur], kK, h->knn);
    h->launches++;
    return cudaGetLastError();
}

// pair features (M x kPair rows), the frames and the signs of the current state
cudaError_t launch_pair_features(rf_handle *h) {
    const int64_t rows = (int64_t)h->M * kPair;
    pair_features_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, h->stream>>>(
        h->M, kPair, h->X[h->cur], h->T[h->cur], h->knn, h->feat, feat_sign(h), feat_rot(h));
    h->launches++;
    return cudaGetLastError();
}
}  // namespace

rf_status build_preconditioner(rf_handle *h) {
    const int M = h->M, nb = 3 * h->N;
    cudaStream_t st = h->stream;
    auto ck = [&](cudaError_t e, const char *what) -> rf_status {
        return e == cudaSuccess ? RF_OK : cuda_fail(h, e, what);
    };
    rf_status s;
    if ((s = ensure_pair_buffers(h)) != RF_OK) return s;
    const int K = knn_count(h);
    if ((s = ck(launch_knn(h), "knn")) != RF_OK) return s;
    h->pc_pairs = 0;
    if (h->p.preconditioner == RF_PC_CLUSTER) {
        const int kc = std::max(1, std::min(h->p.cluster_size, K));
        const int kp = std::min(kPair, kc);
        const int sdim = (kc + 1) * nb;
        const size_t smem = sizeof(float) * (size_t)sdim * (sdim + nb + 1);
        if (smem > 227 * 1024)
            return fail(h, RF_ERR_INVALID_ARG, "cluster_size too large for the shared-memory factorisation");
        int *sing = nullptr;
        if ((s = ck(cudaMalloc(&sing, sizeof(int)), "alloc")) != RF_OK) return s;
        cudaMemsetAsync(sing, 0, sizeof(int), st);
        cudaError_t e;
        if (h->A64) {
            e = cudaFuncSetAttribute(cluster_rows_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            if (e == cudaSuccess)
                cluster_rows_kernel<double><<<M, 256, smem, st>>>(M, nb, h->A64, h->lda, 0, h->knn, kK, kc, kp,
                                                                  h->Pblocks, sing);
        } else if (h->A16lo) {
            e = cudaFuncSetAttribute(cluster_rows_kernel<SplitF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            if (e == cudaSuccess)
                cluster_rows_kernel<SplitF32><<<M, 256, smem, st>>>(
                    M, nb, reinterpret_cast<const SplitF32 *>(h->A16), h->lda, h->a_plane, h->knn, kK, kc, kp,
                    h->Pblocks, sing);
        } else {
            e = cudaFuncSetAttribute(cluster_rows_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            if (e == cudaSuccess)
                cluster_rows_kernel<float><<<M, 256, smem, st>>>(M, nb, h->A32, h->lda, 0, h->knn, kK, kc, kp,
                                                                 h->Pblocks, sing);
        }
        h->launches++;
        if (e == cudaSuccess) e = cudaGetLastError();
        cudaFree(sing);
        if ((s = ck(e, "cluster inverse")) != RF_OK) return s;
        h->pc_pairs = kp;
        h->pc_ready = true;
        return RF_OK;
    }
    // learned
    if (!h->mlp_loaded || nb != kNb || K < kK) {
        h->pc_ready = false;  // fallback: no preconditioning (block-Jacobi with identity blocks)
        return RF_OK;
    }
    return apply_mlp(h);
}

rf_status apply_mlp(rf_handle *h) {
    const int M = h->M;
    cudaStream_t st = h->stream;
    auto ck = [&](cudaError_t e, const char *what) -> rf_status {
        return e == cudaSuccess ? RF_OK : cuda_fail(h, e, what);
    };
    rf_status s;
    if ((s = ensure_mlp_buffers(h)) != RF_OK) return s;
    if ((s = ck(launch_pair_features(h), "features")) != RF_OK) return s;
    const int rows = M * kPair;
    // inference on the tensor cores (BF16 operands, FP32 accumulation); the
    // FP32 CUDA-core GEMMs remain for training
    const MlpLayout Lw;
    const int P = mlp_tc_padded_rows();
    __nv_bfloat16 *w1 = h->mlp_wtc, *w2 = w1 + (size_t)P * kIn, *w3 = w2 + (size_t)P * kHid;
    if ((s = ck(mlp_tc_forward(w1, h->mlp_w + Lw.b1, w2, h->mlp_w + Lw.b2, w3, h->mlp_w + Lw.b3, rows, kIn, kHid, kOut,
                               h->feat, reinterpret_cast<__nv_bfloat16 *>(h->mlp_h1),
                               reinterpret_cast<__nv_bfloat16 *>(h->mlp_h2), h->mlp_out, h->mlp_err, st),
                "mlp")) != RF_OK)
        return s;
    pair_frame_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(M, kPair, feat_rot(h), feat_sign(h), h->mlp_out,
                                                                       kOut, h->Pblocks, kOut, 1);
    h->launches += 4;
    if ((s = ck(cudaGetLastError(), "block frame")) != RF_OK) return s;
    h->pc_pairs = kPair;
    h->pc_ready = true;
    return RF_OK;
}

}  // namespace rf

// ------------------------------------------------------------------ C ABI
using namespace rf;

struct rf_trainer {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *W = nullptr, *G = nullptr, *Mom = nullptr, *Var = nullptr;
    float *X = nullptr, *Y = nullptr;      // dataset
    int64_t count = 0, cap = 0;
    float *bx = nullptr, *by = nullptr, *h1 = nullptr, *h2 = nullptr, *o = nullptr, *dO = nullptr, *dh2 = nullptr,
          *dh1 = nullptr;
    int *bidx = nullptr;
    int bcap = 0;
    double *part = nullptr;
    int64_t t = 0;
    std::mt19937_64 rng;
};

extern "C" {

int64_t rf_mlp_num_params(void) { return MlpLayout().total; }

rf_status rf_set_mlp_weights(rf_handle *h, const float *weights, int64_t count) {
    if (!h || !weights || count != MlpLayout().total) return fail(h, RF_ERR_INVALID_ARG, "weights: wrong size");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, RF_ERR_CUDA, "cudaSetDevice");
    if (!h->mlp_w && cudaMalloc(&h->mlp_w, sizeof(float) * count) != cudaSuccess)
        return fail(h, RF_ERR_OOM, "alloc weights");
    if (cudaMemcpy(h->mlp_w, weights, sizeof(float) * count, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(h, RF_ERR_CUDA, "upload weights");
    // BF16 copies of W1, W2, W3 with their rows padded to the tensor-core tile
    const MlpLayout Lw;
    const int P = mlp_tc_padded_rows();
    if (!h->mlp_wtc && (cudaMalloc(&h->mlp_wtc, sizeof(__nv_bfloat16) * (size_t)P * (kIn + 2 * kHid)) != cudaSuccess ||
                        cudaMalloc(&h->mlp_err, sizeof(int)) != cudaSuccess))
        return fail(h, RF_ERR_OOM, "alloc weights");
    __nv_bfloat16 *w1 = h->mlp_wtc, *w2 = w1 + (size_t)P * kIn, *w3 = w2 + (size_t)P * kHid;
    if (mlp_tc_pad_weights(h->mlp_w + Lw.w1, kHid, kIn, w1, h->stream) != cudaSuccess ||
        mlp_tc_pad_weights(h->mlp_w + Lw.w2, kHid, kHid, w2, h->stream) != cudaSuccess ||
        mlp_tc_pad_weights(h->mlp_w + Lw.w3, kOut, kHid, w3, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->mlp_err, 0, sizeof(int), h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return fail(h, RF_ERR_CUDA, "convert weights");
    h->mlp_loaded = true;
    h->pc_ready = false;
    return RF_OK;
}

rf_status rf_compute_features(rf_handle *h, float *features) {
    if (!h || !features) return fail(h, RF_ERR_INVALID_ARG, "null argument");
    if (h->M <= kK) return fail(h, RF_ERR_INVALID_ARG, "features need more than 16 fibers");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, RF_ERR_CUDA, "cudaSetDevice");
    rf_status s;
    if ((s = ensure_pair_buffers(h)) != RF_OK || (s = ensure_mlp_buffers(h)) != RF_OK) return s;
    cudaError_t e = launch_knn(h);
    if (e == cudaSuccess) e = launch_pair_features(h);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(features, h->feat, sizeof(float) * (size_t)h->M * kPair * kIn, cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "features");
    return RF_OK;
}

rf_status rf_compute_cluster_targets(rf_handle *h, float *targets) {
    if (!h || !targets) return fail(h, RF_ERR_INVALID_ARG, "null argument");
    if (!h->assembled) return fail(h, RF_ERR_INVALID_ARG, "cluster targets need an assembled system");
    if (3 * h->N != kNb) return fail(h, RF_ERR_INVALID_ARG, "the learned blocks are built for N = 5");
    if (h->M <= kK) return fail(h, RF_ERR_INVALID_ARG, "targets need more than 16 fibers");
    if (h->p.cluster_size < kPair) return fail(h, RF_ERR_INVALID_ARG, "targets need cluster_size >= 8");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, RF_ERR_CUDA, "cudaSetDevice");
    const int saved = h->p.preconditioner;
    h->p.preconditioner = RF_PC_CLUSTER;
    rf_status s = build_preconditioner(h);   // exact coupling blocks into Pblocks
    h->p.preconditioner = saved;
    if (s != RF_OK) return s;
    // the frames and signs of the same state, then the blocks in that frame
    if ((s = ensure_mlp_buffers(h)) != RF_OK) return s;
    const int64_t rows = (int64_t)h->M * kPair;
    cudaError_t e = launch_pair_features(h);
    if (e == cudaSuccess) {
        pair_frame_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, h->stream>>>(
            h->M, kPair, feat_rot(h), feat_sign(h), h->Pblocks, kOut, h->mlp_out, kOut, 0);
        h->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(targets, h->mlp_out, sizeof(float) * rows * kOut, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "targets");
    if (saved != RF_PC_CLUSTER) h->pc_ready = false;
    return RF_OK;
}

rf_status rf_mlp_predict(int32_t device, const float *weights, const float *features, int64_t count, float *out) {
    if (!weights || !features || !out || count < 1 || count > (1 << 22))
        return fail(nullptr, RF_ERR_INVALID_ARG, "rf_mlp_predict: bad arguments");
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, RF_ERR_NO_DEVICE, "no CUDA device");
    }
    const MlpLayout Lw;
    const int P = mlp_tc_padded_rows();
    float *w = nullptr, *x = nullptr, *o = nullptr;
    __nv_bfloat16 *wt = nullptr, *h1 = nullptr, *h2 = nullptr;
    int *err = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&w, sizeof(float) * Lw.total);
    if (e == cudaSuccess) e = cudaMalloc(&x, sizeof(float) * count * kIn);
    if (e == cudaSuccess) e = cudaMalloc(&o, sizeof(float) * count * kOut);
    if (e == cudaSuccess) e = cudaMalloc(&wt, sizeof(__nv_bfloat16) * (size_t)P * (kIn + 2 * kHid));
    if (e == cudaSuccess) e = cudaMalloc(&h1, sizeof(__nv_bfloat16) * count * kHid);
    if (e == cudaSuccess) e = cudaMalloc(&h2, sizeof(__nv_bfloat16) * count * kHid);
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w, weights, sizeof(float) * Lw.total, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, features, sizeof(float) * count * kIn, cudaMemcpyHostToDevice, st);
    __nv_bfloat16 *w1 = wt, *w2 = w1 + (size_t)P * kIn, *w3 = w2 + (size_t)P * kHid;
    if (e == cudaSuccess) e = mlp_tc_pad_weights(w + Lw.w1, kHid, kIn, w1, st);
    if (e == cudaSuccess) e = mlp_tc_pad_weights(w + Lw.w2, kHid, kHid, w2, st);
    if (e == cudaSuccess) e = mlp_tc_pad_weights(w + Lw.w3, kOut, kHid, w3, st);
    if (e == cudaSuccess)
        e = mlp_tc_forward(w1, w + Lw.b1, w2, w + Lw.b2, w3, w + Lw.b3, (int)count, kIn, kHid, kOut, x, h1, h2, o, err,
                           st);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, o, sizeof(float) * count * kOut, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    void *ptrs[] = {w, x, o, wt, h1, h2, err};
    for (void *p : ptrs) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "rf_mlp_predict");
    if (herr) return fail(nullptr, RF_ERR_DEVICE_TIMEOUT, "rf_mlp_predict: tensor-core wait timed out");
    return RF_OK;
}

rf_status rf_trainer_create(int32_t device, uint64_t seed, rf_trainer **out) {
    if (!out) return fail(nullptr, RF_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, RF_ERR_NO_DEVICE, "no CUDA device");
    }
    rf_trainer *t = new rf_trainer;
    t->device = device;
    t->rng.seed(seed);
    const int64_t P = MlpLayout().total;
    bool ok = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&t->W, sizeof(float) * P) == cudaSuccess && cudaMalloc(&t->G, sizeof(float) * P) == cudaSuccess &&
              cudaMalloc(&t->Mom, sizeof(float) * P) == cudaSuccess && cudaMalloc(&t->Var, sizeof(float) * P) == cudaSuccess &&
              cudaMalloc(&t->part, sizeof(double) * 1024) == cudaSuccess;
    if (!ok) {
        rf_trainer_destroy(t);
        return fail(nullptr, RF_ERR_OOM, "trainer allocation");
    }
    // He-uniform initial weights, small output layer, zero biases
    const MlpLayout L;
    std::vector<float> w(P, 0.f);
    auto fill = [&](int64_t off, int fan_out, int fan_in, float gain) {
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        const float a = gain * std::sqrt(6.f / fan_in);
        for (int64_t e = 0; e < (int64_t)fan_out * fan_in; ++e) w[off + e] = a * u(t->rng);
    };
    fill(L.w1, kHid, kIn, 1.f);
    fill(L.w2, kHid, kHid, 1.f);
    fill(L.w3, kOut, kHid, 0.1f);
    cudaMemcpy(t->W, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice);
    cudaMemset(t->Mom, 0, sizeof(float) * P);
    cudaMemset(t->Var, 0, sizeof(float) * P);
    *out = t;
    return RF_OK;
}

rf_status rf_trainer_destroy(rf_trainer *t) {
    if (!t) return RF_ERR_INVALID_ARG;
    cudaSetDevice(t->device);
    void *ptrs[] = {t->W, t->G, t->Mom, t->Var, t->X, t->Y, t->bx, t->by, t->h1, t->h2, t->o, t->dO, t->dh2, t->dh1,
                    t->bidx, t->part};
    for (void *p : ptrs) cudaFree(p);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
    return RF_OK;
}

rf_status rf_trainer_add_samples(rf_trainer *t, const float *features, const float *targets, int64_t count) {
    if (!t || !features || !targets || count < 1) return fail(nullptr, RF_ERR_INVALID_ARG, "bad samples");
    cudaSetDevice(t->device);
    if (t->count + count > t->cap) {
        int64_t ncap = std::max<int64_t>(t->cap * 2, t->count + count);
        float *nx = nullptr, *ny = nullptr;
        if (cudaMalloc(&nx, sizeof(float) * ncap * kIn) != cudaSuccess ||
            cudaMalloc(&ny, sizeof(float) * ncap * kOut) != cudaSuccess) {
            cudaFree(nx);
            return fail(nullptr, RF_ERR_OOM, "dataset");
        }
        if (t->count) {
            cudaMemcpy(nx, t->X, sizeof(float) * t->count * kIn, cudaMemcpyDeviceToDevice);
            cudaMemcpy(ny, t->Y, sizeof(float) * t->count * kOut, cudaMemcpyDeviceToDevice);
        }
        cudaFree(t->X);
        cudaFree(t->Y);
        t->X = nx;
        t->Y = ny;
        t->cap = ncap;
    }
    if (cudaMemcpy(t->X + t->count * kIn, features, sizeof(float) * count * kIn, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(t->Y + t->count * kOut, targets, sizeof(float) * count * kOut, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(nullptr, RF_ERR_CUDA, "upload samples");
    t->count += count;
    return RF_OK;
}

namespace {
bool ensure_batch(rf_trainer *t, int B) {
    if (B <= t->bcap) return true;
    void *ptrs[] = {t->bx, t->by, t->h1, t->h2, t->o, t->dO, t->dh2, t->dh1, t->bidx};
    for (void *p : ptrs) cudaFree(p);
    bool ok = cudaMalloc(&t->bx, sizeof(float) * B * kIn) == cudaSuccess &&
              cudaMalloc(&t->by, sizeof(float) * B * kOut) == cudaSuccess &&
              cudaMalloc(&t->h1, sizeof(float) * B * kHid) == cudaSuccess &&
              cudaMalloc(&t->h2, sizeof(float) * B * kHid) == cudaSuccess &&
              cudaMalloc(&t->o, sizeof(float) * B * kOut) == cudaSuccess &&
              cudaMalloc(&t->dO, sizeof(float) * B * kOut) == cudaSuccess &&
              cudaMalloc(&t->dh2, sizeof(float) * B * kHid) == cudaSuccess &&
              cudaMalloc(&t->dh1, sizeof(float) * B * kHid) == cudaSuccess &&
              cudaMalloc(&t->bidx, sizeof(int) * B) == cudaSuccess;
    t->bcap = ok ? B : 0;
    return ok;
}

// forward + backward on B samples already in bx/by; gradient into G; returns
// the summed squared error (over B*225 outputs)
cudaError_t forward_backward(rf_trainer *t, int B, double *sse) {
    const MlpLayout L;
    cudaStream_t st = t->stream;
    cudaError_t e = mlp_forward(t->W, B, t->bx, t->h1, t->h2, t->o, st);
    if (e != cudaSuccess) return e;
    const int64_t cnt = (int64_t)B * kOut;
    const int nblk = (int)std::min<int64_t>(1024, (cnt + 255) / 256);
    mse_grad_kernel<<<nblk, 256, 0, st>>>(cnt, t->o, t->by, t->dO, t->part);
    // layer 3: dW3 = dO^T H2, db3 = colsum dO, dH2 = dO W3 (relu mask)
    GemmArgs g{};
    g.m = kOut; g.n = kHid; g.k = B;
    g.A = t->dO; g.sai = 1; g.sak = kOut;           // A(i,k) = dO[k][i]
    g.B = t->h2; g.sbk = kHid; g.sbj = 1;
    g.C = t->G + L.w3; g.ldc = kHid;
    if ((e = gemm(g, st)) != cudaSuccess) return e;
    colsum_kernel<<<(kOut + 255) / 256, 256, 0, st>>>(B, kOut, t->dO, t->G + L.b3);
    g = GemmArgs{};
    g.m = B; g.n = kHid; g.k = kOut;
    g.A = t->dO; g.sai = kOut; g.sak = 1;
    g.B = t->W + L.w3; g.sbk = kHid; g.sbj = 1;     // B(k,j) = W3[k][j]
    g.C = t->dh2; g.ldc = kHid;
    if ((e = gemm(g, st)) != cudaSuccess) return e;
    relu_back_kernel<<<256, 256, 0, st>>>((int64_t)B * kHid, t->h2, t->dh2);
    // layer 2
    g = GemmArgs{};
    g.m = kHid; g.n = kHid; g.k = B;
    g.A = t->dh2; g.sai = 1; g.sak = kHid;
    g.B = t->h1; g.sbk = kHid; g.sbj = 1;
    g.C = t->G + L.w2; g.ldc = kHid;
    if ((e = gemm(g, st)) != cudaSuccess) return e;
    colsum_kernel<<<1, 256, 0, st>>>(B, kHid, t->dh2, t->G + L.b2);
    g = GemmArgs{};
    g.m = B; g.n = kHid; g.k = kHid;
    g.A = t->dh2; g.sai = kHid; g.sak = 1;
    g.B = t->W + L.w2; g.sbk = kHid; g.sbj = 1;
    g.C = t->dh1; g.ldc = kHid;
    if ((e = gemm(g, st)) != cudaSuccess) return e;
    relu_back_kernel<<<256, 256, 0, st>>>((int64_t)B * kHid, t->h1, t->dh1);
    // layer 1
    g = GemmArgs{};
    g.m = kHid; g.n = kIn; g.k = B;
    g.A = t->dh1; g.sai = 1; g.sak = kHid;
    g.B = t->bx; g.sbk = kIn; g.sbj = 1;
    g.C = t->G + L.w1; g.ldc = kIn;
    if ((e = gemm(g, st)) != cudaSuccess) return e;
    colsum_kernel<<<1, 256, 0, st>>>(B, kHid, t->dh1, t->G + L.b1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    std::vector<double> part(nblk);
    e = cudaMemcpyAsync(part.data(), t->part, sizeof(double) * nblk, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    double s = 0.0;
    for (double v : part) s += v;
    *sse = s;
    return e;
}
}  // namespace

rf_status rf_trainer_train(rf_trainer *t, int32_t epochs, int32_t batch, float lr, float *loss) {
    if (!t || epochs < 1 || batch < 1 || t->count < 1) return fail(nullptr, RF_ERR_INVALID_ARG, "bad training call");
    cudaSetDevice(t->device);
    if (!ensure_batch(t, batch)) return fail(nullptr, RF_ERR_OOM, "batch buffers");
    const int64_t P = MlpLayout().total;
    std::vector<int> perm(t->count);
    double last = 0.0;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int64_t i = 0; i < t->count; ++i) perm[i] = (int)i;
        std::shuffle(perm.begin(), perm.end(), t->rng);
        double sse = 0.0;
        for (int64_t b0 = 0; b0 < t->count; b0 += batch) {
            const int B = (int)std::min<int64_t>(batch, t->count - b0);
            cudaMemcpyAsync(t->bidx, perm.data() + b0, sizeof(int) * B, cudaMemcpyHostToDevice, t->stream);
            gather_rows_kernel<<<(unsigned)(((int64_t)B * kIn + 255) / 256), 256, 0, t->stream>>>(B, kIn, t->bidx, t->X,
                                                                                                  t->bx);
            gather_rows_kernel<<<(unsigned)(((int64_t)B * kOut + 255) / 256), 256, 0, t->stream>>>(B, kOut, t->bidx,
                                                                                                   t->Y, t->by);
            double s = 0.0;
            cudaError_t e = forward_backward(t, B, &s);
            if (e != cudaSuccess) return cuda_fail(nullptr, e, "training step");
            sse += s;
            t->t += 1;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)t->t), c2 = 1.f - std::pow(b2, (float)t->t);
            adam_kernel<<<256, 256, 0, t->stream>>>(P, t->W, t->G, t->Mom, t->Var, lr, b1, b2, c1, c2, 1e-8f);
        }
        last = sse / ((double)t->count * kOut);
    }
    if (cudaStreamSynchronize(t->stream) != cudaSuccess) return fail(nullptr, RF_ERR_CUDA, "training");
    if (loss) *loss = (float)last;
    return RF_OK;
}

rf_status rf_trainer_get_weights(rf_trainer *t, float *weights) {
    if (!t || !weights) return fail(nullptr, RF_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(t->device);
    if (cudaMemcpy(weights, t->W, sizeof(float) * MlpLayout().total, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(nullptr, RF_ERR_CUDA, "download weights");
    return RF_OK;
}

rf_status rf_trainer_set_weights(rf_trainer *t, const float *weights) {
    if (!t || !weights) return fail(nullptr, RF_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(t->device);
    if (cudaMemcpy(t->W, weights, sizeof(float) * MlpLayout().total, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(nullptr, RF_ERR_CUDA, "upload weights");
    return RF_OK;
}

rf_status rf_trainer_loss_grad(rf_trainer *t, const float *features, const float *targets, int64_t count, float *loss,
                               float *grad) {
    if (!t || !features || !targets || count < 1 || count > (1 << 20))
        return fail(nullptr, RF_ERR_INVALID_ARG, "bad arguments");
    cudaSetDevice(t->device);
    if (!ensure_batch(t, (int)count)) return fail(nullptr, RF_ERR_OOM, "batch buffers");
    cudaMemcpy(t->bx, features, sizeof(float) * count * kIn, cudaMemcpyHostToDevice);
    cudaMemcpy(t->by, targets, sizeof(float) * count * kOut, cudaMemcpyHostToDevice);
    double sse = 0.0;
    cudaError_t e = forward_backward(t, (int)count, &sse);
    if (e == cudaSuccess && grad)
        e = cudaMemcpy(grad, t->G, sizeof(float) * MlpLayout().total, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "loss/grad");
    if (loss) *loss = (float)(sse / ((double)count * kOut));
    return RF_OK;
}

}  // extern "C"
