// velocity.cu - K3 velocity recovery and K4 advection.
//
// Reference: fortran/coeffs_and_vels.f90:543-746 (compute_velocities[_an]),
// Int_analytical.f90:772-850, 905-937 (G_compute_GQ_f_kg, TH_f_GQ_kg),
// quadrature.f90:166-259 (G_f_GQ, TH_f_GQ), advect_fibers.f90:498-523;
// src/kernels/update_velocities.cu:101-191, update_fibers*.cu.
//
// Velocity mapping mirrors the assembly: a CTA owns TI targets and a chunk of
// sources; thread (ti, q) keeps its target point and accumulates, over the
// sources of the chunk, IF0 += w_q u_q and IF1 += w_q s_q u_q with
// u_q = int G(xbar_q - x_j - s t_j) f_j(s) ds, f_j = 0.5 F + sum_l a_j^l P_l.
// No synchronisation inside the source loop; the q-reduction happens once per
// chunk through shared memory, partials per chunk are summed in fixed order.
#include "rf_kernels.h"

namespace rf {

template <int N, bool NUMERIC, int TI>
__global__ void __launch_bounds__(TI * kMaxLQ) velocity_kernel(VelArgs a) {
    constexpr int NL = N + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LQ = a.LQ;
    const int nthreads = TI * LQ;
    const int tid = threadIdx.x;
    double *s_pv = reinterpret_cast<double *>(smem_raw);  // kMaxLQ
    double *s_wv = s_pv + kMaxLQ;                         // kMaxLQ
    double *s_wP = s_wv + kMaxLQ;                         // NL x kMaxLQ
    double *s_P = s_wP + NL * kMaxLQ;                     // NL x kMaxLQ
    double *s_red = s_P + NL * kMaxLQ;                    // TI*LQ x 6
    const Tables &tab = *a.tab;
    for (int t = tid; t < LQ; t += nthreads) {
        s_pv[t] = tab.pv[t];
        s_wv[t] = tab.wv[t];
    }
    for (int t = tid; t < NL * LQ; t += nthreads) {
        const int m = t / LQ, q = t % LQ;
        s_wP[m * kMaxLQ + q] = tab.wv[q] * tab.P[m][q];
        s_P[m * kMaxLQ + q] = tab.P[m][q];
    }
    __syncthreads();
    const int i0 = a.t0 + blockIdx.x * TI;   // first target of the tile (global index)
    const int ti = tid / LQ, q = tid - ti * LQ;
    const int i = i0 + ti;
    const double sq = s_pv[q], wq = s_wv[q];
    double xb[3] = {0, 0, 0};
    if (i < a.t1) {
        const double *xc = a.pos + 3 * i, *tc = a.ori + 3 * i;
        xb[0] = fadd(xc[0], fmul(sq, tc[0]));
        xb[1] = fadd(xc[1], fmul(sq, tc[1]));
        xb[2] = fadd(xc[2], fmul(sq, tc[2]));
    }
    const double eps2 = tab.eps2;
    double if0[3] = {0, 0, 0}, if1[3] = {0, 0, 0};
    const int j0 = blockIdx.y * a.chunk;
    const int j1 = min(a.M, j0 + a.chunk);
    if (i < a.t1) {
        for (int j = j0; j < j1; ++j) {
            if (j == i) continue;
            const double xs[3] = {__ldg(a.pos + 3 * j), __ldg(a.pos + 3 * j + 1), __ldg(a.pos + 3 * j + 2)};
            const double ts[3] = {__ldg(a.ori + 3 * j), __ldg(a.ori + 3 * j + 1), __ldg(a.ori + 3 * j + 2)};
            double f[NL][3];
            f[0][0] = tab.half_force[0];
            f[0][1] = tab.half_force[1];
            f[0][2] = tab.half_force[2];
#pragma unroll
            for (int l = 1; l <= N; ++l)
#pragma unroll
                for (int c = 0; c < 3; ++c) f[l][c] = __ldg(a.coeffs + ((int64_t)j * N + (l - 1)) * 3 + c);
            double u[3] = {0, 0, 0};
            if (!NUMERIC) {
                inner_analytic_force_fp64<N>(fsub(xb[0], xs[0]), fsub(xb[1], xs[1]), fsub(xb[2], xs[2]), ts[0],
                                             ts[1], ts[2], eps2, f, u);
            } else {
                const double e2 = 2.0 * eps2;
                for (int s = 0; s < LQ; ++s) {
                    // force on the source fiber at its quadrature point (assemble_forces)
                    double fs[3] = {f[0][0], f[0][1], f[0][2]};
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
            for (int c = 0; c < 3; ++c) {
                if0[c] += wq * u[c];
                if1[c] += wq * u[c] * sq;
            }
        }
    }
    // reduce over the target points of each target
    double *r = s_red + (size_t)tid * 6;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r[c] = if0[c];
        r[3 + c] = if1[c];
    }
    __syncthreads();
    for (int t = tid; t < TI * 6; t += nthreads) {
        const int gt = t / 6, c = t % 6;
        if (i0 + gt >= a.t1) continue;
        double s = 0.0;
        for (int qq = 0; qq < LQ; ++qq) s += s_red[((size_t)gt * LQ + qq) * 6 + c];
        a.part[(int64_t)blockIdx.y * 6 * a.M + (int64_t)(i0 + gt) * 6 + c] = s;
    }
}

template <int N, bool NUMERIC>
static cudaError_t launch_velocity_n(const VelArgs &a, int nchunks, cudaStream_t st) {
    constexpr int TI = 8, NL = N + 1;
    const size_t smem = sizeof(double) * (2 * kMaxLQ + 2 * NL * kMaxLQ + (size_t)TI * a.LQ * 6);
    auto kern = velocity_kernel<N, NUMERIC, TI>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid((a.t1 - a.t0 + TI - 1) / TI, nchunks);
    kern<<<grid, TI * a.LQ, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool NUMERIC>
static cudaError_t launch_velocity_mode(const VelArgs &a, int nchunks, cudaStream_t st) {
    switch (a.N) {
        case 1: return launch_velocity_n<1, NUMERIC>(a, nchunks, st);
        case 2: return launch_velocity_n<2, NUMERIC>(a, nchunks, st);
        case 3: return launch_velocity_n<3, NUMERIC>(a, nchunks, st);
        case 4: return launch_velocity_n<4, NUMERIC>(a, nchunks, st);
        case 5: return launch_velocity_n<5, NUMERIC>(a, nchunks, st);
        case 6: return launch_velocity_n<6, NUMERIC>(a, nchunks, st);
        case 7: return launch_velocity_n<7, NUMERIC>(a, nchunks, st);
        case 8: return launch_velocity_n<8, NUMERIC>(a, nchunks, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_velocity(const VelArgs &a, bool numeric, int nchunks, cudaStream_t st) {
    return numeric ? launch_velocity_mode<true>(a, nchunks, st) : launch_velocity_mode<false>(a, nchunks, st);
}

// Local term and final scaling (coeffs_and_vels.f90:698-705, 723-730).
__global__ void velocity_finish_kernel(int M, int t0, int t1, const double *ori, const Tables *tab,
                                       const double *part, int nchunks, const double *pv_x, const double *pw_x,
                                       double *V, double *W) {
    const int i = t0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t1) return;
    const double d = tab->d, e = tab->e;
    const double *t = ori + 3 * i;
    const double *F = tab->force;
    const double tdf = t[0] * F[0] + t[1] * F[1] + t[2] * F[2];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int c = 0; c < nchunks; ++c)
        for (int k = 0; k < 6; ++k) s[k] += part[(int64_t)c * 6 * M + (int64_t)i * 6 + k];
    if (pv_x) {
        // reuse path: partials already hold scaled l = 0 terms; add the panel products
        for (int a = 0; a < 3; ++a) {
            V[3 * i + a] = 0.5 * ((d + e) * F[a] + (d - e) * tdf * t[a]) / d + s[a] + pv_x[3 * i + a];
            W[3 * i + a] = s[3 + a] + pw_x[3 * i + a];
        }
        return;
    }
    const double tdi = t[0] * s[3] + t[1] * s[4] + t[2] * s[5];
    for (int a = 0; a < 3; ++a) {
        const double loc = 0.5 * ((d + e) * F[a] + (d - e) * tdf * t[a]);
        V[3 * i + a] = (loc + 0.5 * s[a]) / d;
        W[3 * i + a] = 1.5 * (s[3 + a] - tdi * t[a]) / d;
    }
}

cudaError_t launch_velocity_finish(int M, int t0, int t1, const double *ori, const Tables *tab, const double *part,
                                   int nchunks, double *V, double *W, cudaStream_t st) {
    velocity_finish_kernel<<<(t1 - t0 + 127) / 128, 128, 0, st>>>(M, t0, t1, ori, tab, part, nchunks, nullptr,
                                                                   nullptr, V, W);
    return cudaGetLastError();
}

cudaError_t launch_velocity_reuse_finish(int M, const double *ori, const Tables *tab, const double *pv_x,
                                         const double *pw_x, const double *vpart, int nchunks, double *V,
                                         double *W, cudaStream_t st) {
    velocity_finish_kernel<<<(M + 127) / 128, 128, 0, st>>>(M, 0, M, ori, tab, vpart, nchunks, pv_x, pw_x, V, W);
    return cudaGetLastError();
}

// Forward Euler (first step) or the second-order multistep
// x+ = 4/3 x - 1/3 x- + 2/3 dt (2 v - v-), then t <- t/|t|
// (advect_fibers.f90:498-523).
__global__ void advect_kernel(int M, double dt, int first, const double *Xp, const double *Xc,
                              const double *Tp, const double *Tc, const double *Vn, const double *Vo,
                              const double *Wn, const double *Wo, double *Xn, double *Tn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    double tn[3];
    for (int a = 0; a < 3; ++a) {
        const int k = 3 * i + a;
        if (first) {
            Xn[k] = Xc[k] + dt * Vn[k];
            tn[a] = Tc[k] + dt * Wn[k];
        } else {
            Xn[k] = 4.0 / 3.0 * Xc[k] - 1.0 / 3.0 * Xp[k] + 2.0 / 3.0 * dt * (2.0 * Vn[k] - Vo[k]);
            tn[a] = 4.0 / 3.0 * Tc[k] - 1.0 / 3.0 * Tp[k] + 2.0 / 3.0 * dt * (2.0 * Wn[k] - Wo[k]);
        }
    }
    const double tm = sqrt(tn[0] * tn[0] + tn[1] * tn[1] + tn[2] * tn[2]);
    for (int a = 0; a < 3; ++a) Tn[3 * i + a] = tn[a] / tm;
}

cudaError_t launch_advect(int M, double dt, bool first, const double *Xp, const double *Xc, const double *Tp,
                          const double *Tc, const double *Vn, const double *Vo, const double *Wn,
                          const double *Wo, double *Xn, double *Tn, cudaStream_t st) {
    advect_kernel<<<(M + 127) / 128, 128, 0, st>>>(M, dt, first ? 1 : 0, Xp, Xc, Tp, Tc, Vn, Vo, Wn, Wo, Xn, Tn);
    return cudaGetLastError();
}

__global__ void normalize_kernel(int M, double *T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    double *t = T + 3 * i;
    const double tm = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    t[0] /= tm;
    t[1] /= tm;
    t[2] /= tm;
}

cudaError_t launch_normalize(int M, double *T, cudaStream_t st) {
    normalize_kernel<<<(M + 127) / 128, 128, 0, st>>>(M, T);
    return cudaGetLastError();
}

}  // namespace rf
