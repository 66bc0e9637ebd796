// matfree.cu - matrix-free product y = A x in FP64, the reference's mat_prod
// (fortran/matrix_assembly.f90:159-265): the identity plus, for every ordered
// pair of fibers, the inner integral of the Stokeslet/doublet kernel against
// the source's force expansion f_j(s) = sum_l x_j^l P_l(s) (no external
// force), projected onto P_k over the target's Gauss points and mapped by the
// block formula (k = 1: D1 t (t . IF); k >= 2: gamma_k (IF - E_k t (t . IF))).
// A is never formed: memory O(M), work O(M^2) per product, for systems whose
// matrix would not fit or as an FP64 residual next to a low-precision matrix.
//
// Mapping as the velocity kernel's: a CTA owns TI targets and a chunk of
// sources; thread (ti, q) keeps its target point and sums u_q = sum_j int G f_j
// over the chunk; the projections onto P_1..P_N and the block formula are
// applied once per chunk; per-chunk partials are added in fixed order.
#include "rf_kernels.h"

namespace rf {
namespace {

template <int N, bool NUMERIC, int TI>
__global__ void __launch_bounds__(TI * kMaxLQ) matfree_kernel(MatfreeArgs a) {
    constexpr int NL = N + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LQ = a.LQ;
    const int nthreads = TI * LQ;
    const int tid = threadIdx.x;
    double *s_pv = reinterpret_cast<double *>(smem_raw);  // kMaxLQ
    double *s_wv = s_pv + kMaxLQ;                         // kMaxLQ
    double *s_P = s_wv + kMaxLQ;                          // NL x kMaxLQ
    double *s_u = s_P + NL * kMaxLQ;                      // TI*LQ x 3
    const Tables &tab = *a.tab;
    for (int t = tid; t < LQ; t += nthreads) {
        s_pv[t] = tab.pv[t];
        s_wv[t] = tab.wv[t];
    }
    for (int t = tid; t < NL * LQ; t += nthreads) {
        const int m = t / LQ, q = t % LQ;
        s_P[m * kMaxLQ + q] = tab.P[m][q];
    }
    __syncthreads();
    const int i0 = blockIdx.x * TI;
    const int ti = tid / LQ, q = tid - ti * LQ;
    const int i = i0 + ti;
    const double sq = s_pv[q];
    double xb[3] = {0, 0, 0};
    if (i < a.M) {
        const double *xc = a.pos + 3 * i, *tc = a.ori + 3 * i;
        xb[0] = fadd(xc[0], fmul(sq, tc[0]));
        xb[1] = fadd(xc[1], fmul(sq, tc[1]));
        xb[2] = fadd(xc[2], fmul(sq, tc[2]));
    }
    const double eps2 = tab.eps2;
    double usum[3] = {0, 0, 0};
    const int j0 = blockIdx.y * a.chunk;
    const int j1 = min(a.M, j0 + a.chunk);
    if (i < a.M) {
        for (int j = j0; j < j1; ++j) {
            if (j == i) continue;
            const double xs[3] = {__ldg(a.pos + 3 * j), __ldg(a.pos + 3 * j + 1), __ldg(a.pos + 3 * j + 2)};
            const double ts[3] = {__ldg(a.ori + 3 * j), __ldg(a.ori + 3 * j + 1), __ldg(a.ori + 3 * j + 2)};
            double f[NL][3];
            f[0][0] = f[0][1] = f[0][2] = 0.0;  // the matrix alone: no external force
#pragma unroll
            for (int l = 1; l <= N; ++l)
#pragma unroll
                for (int c = 0; c < 3; ++c) f[l][c] = __ldg(a.x + ((int64_t)j * N + (l - 1)) * 3 + c);
            double u[3] = {0, 0, 0};
            if (!NUMERIC) {
                inner_analytic_force_fp64<N>(fsub(xb[0], xs[0]), fsub(xb[1], xs[1]), fsub(xb[2], xs[2]), ts[0],
                                             ts[1], ts[2], eps2, f, u);
            } else {
                // G_f_GQ (quadrature.f90:166-223): the source force at its own points
                const double e2 = 2.0 * eps2;
                for (int s = 0; s < LQ; ++s) {
                    double fs[3] = {0.0, 0.0, 0.0};
#pragma unroll
                    for (int l = 1; l <= N; ++l) {
                        const double p = s_P[l * kMaxLQ + s];
                        fs[0] += f[l][0] * p;
                        fs[1] += f[l][1] * p;
                        fs[2] += f[l][2] * p;
                    }
                    const double sp = s_pv[s];
                    const double Rx = xb[0] - (xs[0] + ts[0] * sp);
                    const double Ry = xb[1] - (xs[1] + ts[1] * sp);
                    const double Rz = xb[2] - (xs[2] + ts[2] * sp);
                    const double ir = 1.0 / sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                    const double ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
                    const double diag = ir + e2 * ir3, off = ir3 - 3.0 * e2 * ir5;
                    const double rf = (Rx * fs[0] + Ry * fs[1] + Rz * fs[2]) * off;
                    const double w = s_wv[s];
                    u[0] += w * (diag * fs[0] + Rx * rf);
                    u[1] += w * (diag * fs[1] + Ry * rf);
                    u[2] += w * (diag * fs[2] + Rz * rf);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) usum[c] += u[c];
        }
    }
    double *r = s_u + (size_t)tid * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = usum[c];
    __syncthreads();
    // per (target, k): IF = sum_q w_q P_k(s_q) u_q, then the block formula
    for (int t = tid; t < TI * N; t += nthreads) {
        const int gt = t / N, k = t % N + 1;
        const int it = i0 + gt;
        if (it >= a.M) continue;
        double IF[3] = {0.0, 0.0, 0.0};
        for (int qq = 0; qq < LQ; ++qq) {
            const double w = s_wv[qq] * s_P[k * kMaxLQ + qq];
            const double *uq = s_u + ((size_t)gt * LQ + qq) * 3;
            IF[0] += w * uq[0];
            IF[1] += w * uq[1];
            IF[2] += w * uq[2];
        }
        const double *tc = a.ori + 3 * it;
        const double tIF = tc[0] * IF[0] + tc[1] * IF[1] + tc[2] * IF[2];
        double out[3];
        if (k == 1) {
#pragma unroll
            for (int c = 0; c < 3; ++c) out[c] = tab.D1 * tIF * tc[c];
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) out[c] = tab.gamma[k] * (IF[c] - tab.Ek[k] * tIF * tc[c]);
        }
        double *dst = a.part + (int64_t)blockIdx.y * a.n + ((int64_t)it * N + (k - 1)) * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c] = out[c];
    }
}

// y = x + the per-chunk partials, added in chunk order
__global__ void matfree_finish_kernel(int64_t n, int nchunks, const double *part, const double *x, double *y) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    double s = x[r];
    for (int c = 0; c < nchunks; ++c) s += part[(int64_t)c * n + r];
    y[r] = s;
}

template <int N, bool NUMERIC>
cudaError_t launch_matfree_n(const MatfreeArgs &a, int nchunks, cudaStream_t st) {
    constexpr int TI = 8, NL = N + 1;
    const size_t smem = sizeof(double) * (2 * kMaxLQ + NL * kMaxLQ + (size_t)TI * a.LQ * 3);
    auto kern = matfree_kernel<N, NUMERIC, TI>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid((a.M + TI - 1) / TI, nchunks);
    kern<<<grid, TI * a.LQ, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool NUMERIC>
cudaError_t launch_matfree_mode(const MatfreeArgs &a, int nchunks, cudaStream_t st) {
    switch (a.N) {
        case 1: return launch_matfree_n<1, NUMERIC>(a, nchunks, st);
        case 2: return launch_matfree_n<2, NUMERIC>(a, nchunks, st);
        case 3: return launch_matfree_n<3, NUMERIC>(a, nchunks, st);
        case 4: return launch_matfree_n<4, NUMERIC>(a, nchunks, st);
        case 5: return launch_matfree_n<5, NUMERIC>(a, nchunks, st);
        case 6: return launch_matfree_n<6, NUMERIC>(a, nchunks, st);
        case 7: return launch_matfree_n<7, NUMERIC>(a, nchunks, st);
        case 8: return launch_matfree_n<8, NUMERIC>(a, nchunks, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_matfree(const MatfreeArgs &a, bool numeric, int nchunks, const double *x, double *y,
                           cudaStream_t st) {
    cudaError_t e = numeric ? launch_matfree_mode<true>(a, nchunks, st) : launch_matfree_mode<false>(a, nchunks, st);
    if (e != cudaSuccess) return e;
    matfree_finish_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a.n, nchunks, a.part, x, y);
    return cudaGetLastError();
}

}  // namespace rf
