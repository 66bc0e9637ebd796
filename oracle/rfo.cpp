// rfo.cpp - CPU FP64 oracle (test infrastructure only; see rfo.h).
//
// Plain restatement of the reference Fortran method.  Each routine cites the
// Fortran lines it follows.  Loop order differs from the Fortran in one place:
// the analytic inner integral is evaluated once per (pair, target point) with
// the full expansion length N and feeds every Legendre index l, where the
// Fortran calls it once per l (matrix_assembly.f90:522-542).  The recurrences of
// Int_analytical.f90 produce the same value for index l whatever the upper
// limit (forward recursion stops early, backward recursion always starts at
// index 28), so the arithmetic of every matrix entry is unchanged.

#include "rfo.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kMaxN = 8;
constexpr int kMaxLQ = 3 * 64;

inline void set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

// Model constants, matrix_assembly.f90:450-484 and :582.
struct Consts {
    double c, d, e, D1;
    double lambda[kMaxN + 1];
    double Ek[kMaxN + 1];
    double gamma[kMaxN + 1];
};

Consts make_consts(double eps, int N) {
    Consts k{};
    k.c = std::log(eps * eps * std::exp(1.0));
    k.d = -k.c;
    k.e = 2.0;
    const double cc = 1.0;
    k.D1 = 0.75 / (k.d - 2.0 * cc);
    k.lambda[1] = 2.0;
    for (int i = 2; i <= N; ++i) k.lambda[i] = k.lambda[i - 1] + 2.0 / i;
    for (int i = 1; i <= N; ++i) {
        k.Ek[i] = (k.d - k.e - cc * k.lambda[i]) / 2.0 / (k.d - cc * k.lambda[i]);
        k.gamma[i] = 0.5 * (2.0 * i + 1.0) / (k.d + k.e - cc * k.lambda[i]);
    }
    return k;
}

// Legendre P_m = scale_m * sum_p a_mp s^p, m = 0..8, with the integer
// coefficients and scales of the Fortran combinations (Int_analytical.f90:
// 213-288; compute_LVecs, matrix_assembly.f90:36-56).
const double kLegScale[9] = {1.0, 1.0, 0.5, 0.5, 0.125, 0.125, 0.0625, 0.0625, 1.0 / 128.0};
const double kLegInt[9][9] = {
    {1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 1, 0, 0, 0, 0, 0, 0, 0},
    {-1, 0, 3, 0, 0, 0, 0, 0, 0},
    {0, -3, 0, 5, 0, 0, 0, 0, 0},
    {3, 0, -30, 0, 35, 0, 0, 0, 0},
    {0, 15, 0, -70, 0, 63, 0, 0, 0},
    {-5, 0, 105, 0, -315, 0, 231, 0, 0},
    {0, -35, 0, 315, 0, -693, 0, 429, 0},
    {35, 0, -1260, 0, 6930, 0, -12012, 0, 6435},
};

// Int_analytical.f90:5-293.  Moments I_n = int s^n/R, J_n = int s^n/R^3,
// S_n = int s^n/R^5 over s in [-1,1] with R = |R0 - s pb|, then Legendre
// combinations.  Output L[c][m] for m = 0..N, c = L11,L12,L13,L14,L22,L23,L24.
void analytic_moments(const double *xb, const double *pb, const double *xbar, int N,
                      double L[7][kMaxN + 1]) {
    double I[31] = {0}, J[31] = {0}, S[31] = {0};  // 1-based like the Fortran
    const double clim = 10.0;
    double R0[3] = {xbar[0] - xb[0], xbar[1] - xb[1], xbar[2] - xb[2]};
    const double b = -2.0 * (pb[0] * R0[0] + pb[1] * R0[1] + pb[2] * R0[2]);
    const double c = R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2];
    const double se = 1.0, sb = -1.0;
    const double ue = std::sqrt(1.0 + b + c);
    const double ub = std::sqrt(1.0 - b + c);
    const double te = 1.0 + 0.5 * b;
    const double tb = -1.0 + 0.5 * b;
    const double d = c - 0.25 * b * b;

    I[1] = std::log(std::fabs(2.0 * se + b + 2.0 * ue)) - std::log(std::fabs(2.0 * sb + b + 2.0 * ub));
    I[2] = ue - ub - 1 / 2.0 * b * I[1];
    if (c < clim) {
        double nn = 2.0;
        for (int ii = 3; ii <= N + 3; ++ii) {
            nn = nn + 1.0;
            const double sep = 1.0;                          // se**(ii-2)
            const double sbp = ((ii - 2) % 2 == 0) ? 1.0 : -1.0;  // sb**(ii-2)
            I[ii] = -sep * ue / (1.0 - nn) + sbp * ub / (1.0 - nn)
                    - (0.5 - (nn - 1.0)) * b / (1.0 - nn) * I[ii - 1]
                    + (nn - 2.0) * c / (1.0 - nn) * I[ii - 2];
        }
    } else {
        I[30] = 0.0;
        I[29] = 0.0;
        double nn = 27.0;
        for (int ii = 28; ii >= 3; --ii) {
            const double sbp = (((int)nn + 1) % 2 == 0) ? 1.0 : -1.0;  // sb**(nn+1)
            I[ii] = (nn + 2) / ((nn + 1) * c) *
                    (1.0 * ue / (nn + 2) - sbp * ub / (nn + 2) +
                     (1 - 2 * (nn + 2)) / (2 * (nn + 2)) * b * I[ii + 1] - I[ii + 2]);
            nn = nn - 1.0;
        }
    }
    if (d < 1e-14) {
        J[1] = -1.0 / (2.0 * std::pow(se + b / 2.0, 2.0)) + 1.0 / (2.0 * std::pow(sb + b / 2.0, 2.0));
    } else {
        J[1] = te / (d * ue) - tb / (d * ub);
    }
    J[2] = -1.0 / ue + 1.0 / ub - b / 2.0 * J[1];
    if (c < clim) {
        for (int ii = 3; ii <= N + 3; ++ii) J[ii] = I[ii - 2] - b * J[ii - 1] - c * J[ii - 2];
    } else {
        J[30] = 0;
        J[29] = 0;
        for (int ii = 28; ii >= 3; --ii) J[ii] = 1 / c * (I[ii] - b * J[ii + 1] - J[ii + 2]);
    }
    if (d < 1e-14) {
        S[1] = -4.0 / std::pow(2.0 * se + b, 4.0) + 4.0 / std::pow(2.0 * sb + b, 4.0);
        S[2] = -8.0 / (3.0 * std::pow(2.0 * se + b, 3.0)) + 8.0 / (3.0 * std::pow(2.0 * sb + b, 3.0)) -
               b / 2.0 * S[1];
    } else {
        const double ue3 = std::pow(ue, 3.0), ub3 = std::pow(ub, 3.0);
        S[1] = (2.0 * se + b) / (6.0 * d * ue3) - (2.0 * sb + b) / (6.0 * d * ub3) + 2.0 / (3.0 * d) * J[1];
        S[2] = -(b * se + 2.0 * c) / (6.0 * d * ue3) + (b * sb + 2.0 * c) / (6.0 * d * ub3) -
               b / (3.0 * d) * J[1];
    }
    if (c < clim) {
        for (int ii = 3; ii <= N + 3; ++ii) S[ii] = J[ii - 2] - b * S[ii - 1] - c * S[ii - 2];
    } else {
        S[30] = 0;
        S[29] = 0;
        for (int ii = 28; ii >= 3; --ii) S[ii] = 1 / c * (J[ii] - b * S[ii + 1] - S[ii + 2]);
    }
    // Legendre combinations, highest power first as in the Fortran:
    // L11_m = scale_m * sum_p a_mp I_p (0-based moment p is Fortran index
    // p+1); L13 and L14 shift by one and two powers of s.
    for (int m = 0; m <= N; ++m) {
        double l11 = 0, l12 = 0, l13 = 0, l14 = 0, l22 = 0, l23 = 0, l24 = 0;
        for (int pp = m; pp >= 0; --pp) {
            const double a = kLegInt[m][pp];
            if (a == 0.0) continue;
            l11 += a * I[pp + 1];
            l12 += a * J[pp + 1];
            l13 += a * J[pp + 2];
            l14 += a * J[pp + 3];
            l22 += a * S[pp + 1];
            l23 += a * S[pp + 2];
            l24 += a * S[pp + 3];
        }
        const double sc = kLegScale[m];
        L[0][m] = sc * l11; L[1][m] = sc * l12; L[2][m] = sc * l13; L[3][m] = sc * l14;
        L[4][m] = sc * l22; L[5][m] = sc * l23; L[6][m] = sc * l24;
    }
}

// G tensor from the moments, Int_analytical.f90:735-746 (6 components
// 11,22,33,12,13,23).
inline void g_from_moments(const double *R0, const double *pb, double eps2,
                           double l11, double l12, double l13, double l14,
                           double l22, double l23, double l24, double *G) {
    const int ia[6] = {0, 1, 2, 0, 0, 1};
    const int ib[6] = {0, 1, 2, 1, 2, 2};
    for (int q = 0; q < 6; ++q) {
        const int a = ia[q], bb = ib[q];
        const double id = (a == bb) ? 1.0 : 0.0;
        const double rr = R0[a] * R0[bb];
        const double pr = pb[a] * R0[bb] + R0[a] * pb[bb];
        const double pp = pb[a] * pb[bb];
        G[q] = l11 * id + rr * l12 - pr * l13 + pp * l14 +
               2.0 * eps2 * (id * l12 - 3.0 * rr * l22 + 3.0 * pr * l23 - 3.0 * pp * l24);
    }
}

struct Tables {
    int N, LQ;
    std::vector<double> pv, wv;
    std::vector<double> P;  // P[m*LQ + q], m = 0..N (P_0 = 1)
};

Tables make_tables(int N, int NoQI) {
    Tables t;
    t.N = N;
    t.LQ = 3 * NoQI;
    t.pv.resize(t.LQ);
    t.wv.resize(t.LQ);
    rfo_quadrature(NoQI, t.pv.data(), t.wv.data());
    std::vector<double> L(t.LQ * N);
    rfo_legendre(N, t.LQ, t.pv.data(), L.data());
    t.P.assign((N + 1) * t.LQ, 1.0);
    for (int m = 1; m <= N; ++m)
        for (int q = 0; q < t.LQ; ++q) t.P[m * t.LQ + q] = L[(m - 1) * t.LQ + q];
    return t;
}

// Inner integral over source fiber (xb, pb) at the target point xbar, for all
// Legendre weights l = 0..N: G[l*6 + comp].
// Analytic: Int_analytical.f90:663-767.  Numeric: quadrature.f90:100-164.
void inner_integral(const Tables &t, bool analytic, double eps, const double *xb,
                    const double *pb, const double *xbar, double *G) {
    const int N = t.N;
    const double eps2 = eps * eps;
    if (analytic) {
        double L[7][kMaxN + 1];
        analytic_moments(xb, pb, xbar, N, L);
        const double R0[3] = {xbar[0] - xb[0], xbar[1] - xb[1], xbar[2] - xb[2]};
        for (int l = 0; l <= N; ++l)
            g_from_moments(R0, pb, eps2, L[0][l], L[1][l], L[2][l], L[3][l], L[4][l], L[5][l],
                           L[6][l], G + 6 * l);
    } else {
        const int LQ = t.LQ;
        for (int l = 0; l <= N; ++l)
            for (int q = 0; q < 6; ++q) G[6 * l + q] = 0.0;
        for (int s = 0; s < LQ; ++s) {
            const double Rx = xbar[0] - (xb[0] + pb[0] * t.pv[s]);
            const double Ry = xbar[1] - (xb[1] + pb[1] * t.pv[s]);
            const double Rz = xbar[2] - (xb[2] + pb[2] * t.pv[s]);
            const double Rm = std::sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
            const double R3 = Rm * Rm * Rm, R5 = R3 * Rm * Rm;
            double K[6];
            K[0] = 1.0 / Rm + Rx * Rx / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Rx * Rx / R5);
            K[1] = 1.0 / Rm + Ry * Ry / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Ry * Ry / R5);
            K[2] = 1.0 / Rm + Rz * Rz / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Rz * Rz / R5);
            K[3] = Rx * Ry / R3 - 6.0 * eps2 * Rx * Ry / R5;
            K[4] = Rx * Rz / R3 - 6.0 * eps2 * Rx * Rz / R5;
            K[5] = Ry * Rz / R3 - 6.0 * eps2 * Ry * Rz / R5;
            for (int l = 0; l <= N; ++l) {
                const double wl = t.wv[s] * t.P[l * LQ + s];
                for (int q = 0; q < 6; ++q) G[6 * l + q] += wl * K[q];
            }
        }
    }
}

// Symmetric 3x3 from 6 packed components.
inline double sym(const double *g, int a, int b) {
    static const int idx[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    return g[idx[a][b]];
}

// Assemble the rows of target fiber i into block storage:
// Ablk[(j*3N + col_local) * 3N + row_local] for all sources j (diagonal block
// is the identity), and b rows (3N values).  matrix_assembly.f90:499-626,
// 839-903 (analytic) / 317-400, 678-792 (numeric).
void assemble_target(const rfo_params *p, const Tables &t, const Consts &k, const double *X,
                     const double *T, int i, double *Ablk, double *brow) {
    const int M = p->M, N = p->N, LQ = t.LQ, n3 = 3 * N;
    const double *xc = X + 3 * i, *ta = T + 3 * i;
    std::vector<double> G((size_t)LQ * (N + 1) * 6);
    for (int r = 0; r < n3; ++r) brow[r] = 0.0;
    const double f[3] = {0.5 * p->ext_force[0], 0.5 * p->ext_force[1], 0.5 * p->ext_force[2]};
    for (int j = 0; j < M; ++j) {
        double *blk = Ablk + (size_t)j * n3 * n3;
        if (j == i) {
            for (int cl = 0; cl < n3; ++cl)
                for (int r = 0; r < n3; ++r) blk[cl * n3 + r] = (r == cl) ? 1.0 : 0.0;
            continue;
        }
        const double *xb = X + 3 * j, *tb = T + 3 * j;
        for (int q = 0; q < LQ; ++q) {
            const double xbar[3] = {xc[0] + t.pv[q] * ta[0], xc[1] + t.pv[q] * ta[1],
                                    xc[2] + t.pv[q] * ta[2]};
            inner_integral(t, p->analytic != 0, p->eps, xb, tb, xbar, &G[(size_t)q * (N + 1) * 6]);
        }
        for (int l = 1; l <= N; ++l) {
            for (int kk = 1; kk <= N; ++kk) {
                double th[6] = {0, 0, 0, 0, 0, 0};
                for (int q = 0; q < LQ; ++q) {
                    const double w = t.wv[q] * t.P[kk * LQ + q];
                    const double *g = &G[((size_t)q * (N + 1) + l) * 6];
                    for (int c = 0; c < 6; ++c) th[c] += w * g[c];
                }
                double Q[3];
                for (int bb = 0; bb < 3; ++bb)
                    Q[bb] = sym(th, bb, 0) * ta[0] + sym(th, bb, 1) * ta[1] + sym(th, bb, 2) * ta[2];
                const int rowno = 3 * (kk - 1), col = 3 * (l - 1);
                for (int a = 0; a < 3; ++a)
                    for (int bb = 0; bb < 3; ++bb) {
                        double v;
                        if (kk == 1) v = k.D1 * ta[a] * Q[bb];
                        else v = k.gamma[kk] * (sym(th, a, bb) - k.Ek[kk] * ta[a] * Q[bb]);
                        blk[(col + bb) * n3 + rowno + a] = v;
                    }
            }
        }
        // right-hand side: l = 0 weight contracted with 0.5*ExtForce
        for (int kk = 1; kk <= N; ++kk) {
            double contr[3] = {0, 0, 0};
            for (int q = 0; q < LQ; ++q) {
                const double *g = &G[(size_t)q * (N + 1) * 6];
                const double gf[3] = {sym(g, 0, 0) * f[0] + sym(g, 0, 1) * f[1] + sym(g, 0, 2) * f[2],
                                      sym(g, 1, 0) * f[0] + sym(g, 1, 1) * f[1] + sym(g, 1, 2) * f[2],
                                      sym(g, 2, 0) * f[0] + sym(g, 2, 1) * f[1] + sym(g, 2, 2) * f[2]};
                const double w = t.wv[q] * t.P[kk * LQ + q];
                for (int a = 0; a < 3; ++a) contr[a] += w * gf[a];
            }
            const double tdc = ta[0] * contr[0] + ta[1] * contr[1] + ta[2] * contr[2];
            const int rowno = 3 * (kk - 1);
            for (int a = 0; a < 3; ++a) {
                if (kk == 1) brow[rowno + a] -= k.D1 * tdc * ta[a];
                else brow[rowno + a] -= k.gamma[kk] * (contr[a] - k.Ek[kk] * tdc * ta[a]);
            }
        }
    }
}

// Velocities of target fiber i, coeffs_and_vels.f90:543-746.
void velocity_target(const rfo_params *p, const Tables &t, const Consts &k, const double *X,
                     const double *T, const double *coeffs, int i, double *Vi, double *Wi) {
    const int M = p->M, N = p->N, LQ = t.LQ;
    const double *xc = X + 3 * i, *ta = T + 3 * i;
    const double *F = p->ext_force;
    const double e = k.e, d = k.d;
    const double tdf = ta[0] * F[0] + ta[1] * F[1] + ta[2] * F[2];
    for (int a = 0; a < 3; ++a) {
        Vi[a] = 0.5 * ((d + e) * F[a] + (d - e) * tdf * ta[a]);
        Wi[a] = 0.0;
    }
    std::vector<double> G((size_t)(N + 1) * 6);
    std::vector<double> fx(LQ), fy(LQ), fz(LQ);
    for (int j = 0; j < M; ++j) {
        if (j == i) continue;
        const double *xb = X + 3 * j, *tb = T + 3 * j;
        // force on the source fiber: 0.5*F + sum_l a^l P_l (assemble_forces, :123-157)
        double fl[kMaxN + 1][3];
        for (int a = 0; a < 3; ++a) fl[0][a] = 0.5 * F[a];
        for (int l = 1; l <= N; ++l)
            for (int a = 0; a < 3; ++a) fl[l][a] = coeffs[((size_t)j * N + (l - 1)) * 3 + a];
        if (!p->analytic) {
            for (int s = 0; s < LQ; ++s) {
                fx[s] = fl[0][0]; fy[s] = fl[0][1]; fz[s] = fl[0][2];
                for (int l = 1; l <= N; ++l) {
                    fx[s] += fl[l][0] * t.P[l * LQ + s];
                    fy[s] += fl[l][1] * t.P[l * LQ + s];
                    fz[s] += fl[l][2] * t.P[l * LQ + s];
                }
            }
        }
        double IF0[3] = {0, 0, 0}, IF1[3] = {0, 0, 0};
        for (int q = 0; q < LQ; ++q) {
            const double xbar[3] = {xc[0] + t.pv[q] * ta[0], xc[1] + t.pv[q] * ta[1],
                                    xc[2] + t.pv[q] * ta[2]};
            double u[3] = {0, 0, 0};
            if (p->analytic) {
                // G_compute_GQ_f_kg, Int_analytical.f90:772-850
                inner_integral(t, true, p->eps, xb, tb, xbar, G.data());
                for (int l = 0; l <= N; ++l) {
                    const double *g = &G[6 * l];
                    for (int a = 0; a < 3; ++a)
                        u[a] += sym(g, a, 0) * fl[l][0] + sym(g, a, 1) * fl[l][1] + sym(g, a, 2) * fl[l][2];
                }
            } else {
                // G_f_GQ, quadrature.f90:166-223
                const double eps2 = p->eps * p->eps;
                for (int s = 0; s < LQ; ++s) {
                    const double Rx = xbar[0] - (xb[0] + tb[0] * t.pv[s]);
                    const double Ry = xbar[1] - (xb[1] + tb[1] * t.pv[s]);
                    const double Rz = xbar[2] - (xb[2] + tb[2] * t.pv[s]);
                    const double Rm = std::sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                    const double R3 = Rm * Rm * Rm, R5 = R3 * Rm * Rm;
                    const double K11 = 1.0 / Rm + Rx * Rx / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Rx * Rx / R5);
                    const double K22 = 1.0 / Rm + Ry * Ry / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Ry * Ry / R5);
                    const double K33 = 1.0 / Rm + Rz * Rz / R3 + 2.0 * eps2 * (1.0 / R3 - 3.0 * Rz * Rz / R5);
                    const double K12 = Rx * Ry / R3 - 6.0 * eps2 * Rx * Ry / R5;
                    const double K13 = Rx * Rz / R3 - 6.0 * eps2 * Rx * Rz / R5;
                    const double K23 = Ry * Rz / R3 - 6.0 * eps2 * Ry * Rz / R5;
                    u[0] += t.wv[s] * (K11 * fx[s] + K12 * fy[s] + K13 * fz[s]);
                    u[1] += t.wv[s] * (K12 * fx[s] + K22 * fy[s] + K23 * fz[s]);
                    u[2] += t.wv[s] * (K13 * fx[s] + K23 * fy[s] + K33 * fz[s]);
                }
            }
            // TH_f_GQ(_kg): outer integral with weights 1 (P_0) and s (P_1)
            for (int a = 0; a < 3; ++a) {
                IF0[a] += t.wv[q] * u[a];
                IF1[a] += t.wv[q] * u[a] * t.pv[q];
            }
        }
        const double tdi = ta[0] * IF1[0] + ta[1] * IF1[1] + ta[2] * IF1[2];
        for (int a = 0; a < 3; ++a) {
            Vi[a] += 0.5 * IF0[a];
            Wi[a] += 1.5 * (IF1[a] - tdi * ta[a]);
        }
    }
    for (int a = 0; a < 3; ++a) {
        Vi[a] /= d;
        Wi[a] /= d;
    }
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Random stream of the synthetic layouts: xoshiro256** (Blackman and Vigna)
// whose four state words come from splitmix64 of the seed.  Uniform variates
// take the top 53 bits; normal variates are one Box-Muller value per call.
struct LayoutRng {
    uint64_t w[4];
    explicit LayoutRng(uint64_t seed) {
        uint64_t z = seed;
        for (uint64_t &s : w) {
            z += 0x9e3779b97f4a7c15ull;
            uint64_t v = z;
            v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
            v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
            s = v ^ (v >> 31);
        }
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t bits() {
        const uint64_t out = rotl(w[1] * 5, 7) * 9;
        const uint64_t sh = w[1] << 17;
        w[2] ^= w[0];
        w[3] ^= w[1];
        w[1] ^= w[2];
        w[0] ^= w[3];
        w[2] ^= sh;
        w[3] = rotl(w[3], 45);
        return out;
    }
    double u01() { return (double)(bits() >> 11) * (1.0 / 9007199254740992.0); }
    double gauss() {
        double a = u01();
        while (a <= 0.0) a = u01();
        const double b = u01();
        return std::sqrt(-2.0 * std::log(a)) * std::cos(2.0 * M_PI * b);
    }
};

int assemble_rows_ld(const rfo_params *p, const double *X, const double *T, int i0, int i1, double *Arows,
                     size_t ld, double *brows) {
    // rows of target fibers [i0, i1): Arows[r + col * ld], r = (i - i0) * 3N + row in the block
    if (!p || p->N < 1 || p->N > kMaxN || p->M < 1 || p->NoQI < 1 || 3 * p->NoQI > kMaxLQ) return -1;
    set_threads(p->threads);
    const Tables t = make_tables(p->N, p->NoQI);
    const Consts k = make_consts(p->eps, p->N);
    const int M = p->M, n3 = 3 * p->N;
#pragma omp parallel
    {
        std::vector<double> blk((size_t)M * n3 * n3);
#pragma omp for schedule(dynamic, 1)
        for (int i = i0; i < i1; ++i) {
            double *brow = brows + (size_t)(i - i0) * n3;
            assemble_target(p, t, k, X, T, i, blk.data(), brow);
            for (int j = 0; j < M; ++j)
                for (int cl = 0; cl < n3; ++cl) {
                    const size_t col = (size_t)j * n3 + cl;
                    double *dst = Arows + col * ld + (size_t)(i - i0) * n3;
                    const double *src = &blk[((size_t)j * n3 + cl) * n3];
                    for (int r = 0; r < n3; ++r) dst[r] = src[r];
                }
        }
    }
    return 0;
}

}  // namespace

extern "C" {

void rfo_quadrature(int NoQI, double *pv, double *wv) {
    // quadrature.f90:44-84: 3-point Gauss rule on each of NoQI panels.
    const double pv0[3] = {-std::sqrt(15.0) / 5.0, 0.0, std::sqrt(15.0) / 5.0};
    const double wv0[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    double a = -1.0;
    const double iv = 2.0 / NoQI;
    for (int i = 0; i < NoQI; ++i) {
        for (int k = 0; k < 3; ++k) {
            pv[3 * i + k] = (2.0 * a + iv + pv0[k] * iv) / 2.0;
            wv[3 * i + k] = wv0[k] / NoQI;
        }
        a = a + iv;
    }
}

void rfo_legendre(int N, int LQ, const double *pv, double *L) {
    // matrix_assembly.f90:36-56, explicit polynomials P_1..P_8.
    for (int kk = 1; kk <= N; ++kk)
        for (int q = 0; q < LQ; ++q) {
            const double x = pv[q];
            double v;
            switch (kk) {
                case 1: v = x; break;
                case 2: v = 0.5 * (3.0 * x * x - 1.0); break;
                case 3: v = 0.5 * (5.0 * x * x * x - 3.0 * x); break;
                case 4: v = 0.125 * (35.0 * std::pow(x, 4) - 30.0 * x * x + 3.0); break;
                case 5: v = 0.125 * (63.0 * std::pow(x, 5) - 70.0 * x * x * x + 15.0 * x); break;
                case 6:
                    v = 0.0625 * (231.0 * std::pow(x, 6) - 315.0 * std::pow(x, 4) + 105.0 * x * x - 5.0);
                    break;
                case 7:
                    v = 0.0625 * (429.0 * std::pow(x, 7) - 693.0 * std::pow(x, 5) + 315.0 * x * x * x -
                                  35.0 * x);
                    break;
                default:
                    v = 6435.0 / 128.0 * std::pow(x, 8) - 3003.0 / 32.0 * std::pow(x, 6) +
                        3465.0 / 64.0 * std::pow(x, 4) - 315.0 / 32.0 * x * x + 35.0 / 128.0;
                    break;
            }
            L[(kk - 1) * LQ + q] = v;
        }
}

void rfo_analytic_moments(const double *xb, const double *pb, const double *xbar, int N,
                          double *out) {
    double L[7][kMaxN + 1];
    analytic_moments(xb, pb, xbar, N, L);
    for (int c = 0; c < 7; ++c)
        for (int m = 0; m <= N; ++m) out[c * (N + 1) + m] = L[c][m];
}

int rfo_assemble_rows(const rfo_params *p, const double *X, const double *T, int i0, int i1,
                      double *Arows, double *brows) {
    return assemble_rows_ld(p, X, T, i0, i1, Arows, (size_t)(i1 - i0) * 3 * (p ? p->N : 0), brows);
}

int rfo_assemble_system(const rfo_params *p, const double *X, const double *T, double *A, double *b) {
    return rfo_assemble_rows(p, X, T, 0, p->M, A, b);
}

int rfo_solve_direct(int n, double *A, double *x) {
    // dgesv semantics: Gaussian elimination with partial pivoting (row
    // interchanges), then forward and back substitution.
    std::vector<int> piv(n);
    for (int kcol = 0; kcol < n; ++kcol) {
        int pr = kcol;
        double amax = std::fabs(A[kcol + (size_t)kcol * n]);
        for (int r = kcol + 1; r < n; ++r) {
            const double v = std::fabs(A[r + (size_t)kcol * n]);
            if (v > amax) { amax = v; pr = r; }
        }
        piv[kcol] = pr;
        if (amax == 0.0) return kcol + 1;
        if (pr != kcol) {
            for (int c = 0; c < n; ++c) std::swap(A[kcol + (size_t)c * n], A[pr + (size_t)c * n]);
            std::swap(x[kcol], x[pr]);
        }
        const double inv = 1.0 / A[kcol + (size_t)kcol * n];
        for (int r = kcol + 1; r < n; ++r) A[r + (size_t)kcol * n] *= inv;
#pragma omp parallel for schedule(static)
        for (int c = kcol + 1; c < n; ++c) {
            const double akc = A[kcol + (size_t)c * n];
            if (akc == 0.0) continue;
            double *col = A + (size_t)c * n;
            const double *lc = A + (size_t)kcol * n;
            for (int r = kcol + 1; r < n; ++r) col[r] -= lc[r] * akc;
        }
    }
    for (int c = 0; c < n; ++c) {
        const double xc = x[c];
        if (xc != 0.0)
            for (int r = c + 1; r < n; ++r) x[r] -= A[r + (size_t)c * n] * xc;
    }
    for (int c = n - 1; c >= 0; --c) {
        x[c] /= A[c + (size_t)c * n];
        const double xc = x[c];
        if (xc != 0.0)
            for (int r = 0; r < c; ++r) x[r] -= A[r + (size_t)c * n] * xc;
    }
    return 0;
}

void rfo_matvec_rect(int m, int n, const double *A, long long lda, const double *x, double *y, int threads) {
    // dgemv('N') order: y_i = sum_j A_ij x_j accumulated over j in order.
    set_threads(threads);
    const int RB = 256;
#pragma omp parallel for schedule(static)
    for (int r0 = 0; r0 < m; r0 += RB) {
        const int r1 = std::min(m, r0 + RB);
        double acc[256];
        for (int r = r0; r < r1; ++r) acc[r - r0] = 0.0;
        for (int c = 0; c < n; ++c) {
            const double xc = x[c];
            const double *col = A + (size_t)c * lda;
            for (int r = r0; r < r1; ++r) acc[r - r0] += xc * col[r];
        }
        for (int r = r0; r < r1; ++r) y[r] = acc[r - r0];
    }
}

void rfo_matvec(int n, const double *A, const double *x, double *y, int threads) {
    rfo_matvec_rect(n, n, A, n, x, y, threads);
}

static double dot(int n, const double *a, const double *b) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// Givens rotation construction (LINPACK drotg semantics, blas_rot.f:117-146).
static void rotg(double a, double b, double *c, double *s) {
    const double roe = (std::fabs(a) > std::fabs(b)) ? a : b;
    const double scale = std::fabs(a) + std::fabs(b);
    if (scale == 0.0) { *c = 1.0; *s = 0.0; return; }
    double r = scale * std::sqrt((a / scale) * (a / scale) + (b / scale) * (b / scale));
    r = std::copysign(1.0, roe) * r;
    *c = a / r;
    *s = b / r;
}

static inline void rot(double &x, double &y, double c, double s) {
    const double t = c * x + s * y;
    y = c * y - s * x;
    x = t;
}

int rfo_solve_gmres(int n, const double *A, const double *b, double *x, int m, int max_iters,
                    double tol, int *iters_out, double *be_out, int threads) {
    // Restarted GMRES with the control flow of dGMRES.f:491-1495 as used by
    // coeffs_and_vels.f90:446-500: no preconditioner, modified Gram-Schmidt,
    // initial guess supplied, true residual recomputed at each restart,
    // stop when the Arnoldi estimate and then the true residual satisfy
    // ||r||/||b|| <= tol, or when the iteration budget is spent.
    set_threads(threads);
    std::vector<double> V((size_t)n * m), w(n), r0(n), xcur(n);
    std::vector<double> H((size_t)(m + 1) * (m + 1), 0.0);  // H[row + col*(m+1)], col m = rhs g
    std::vector<double> cs(m), sn(m), y(m);
    auto Hc = [&](int r, int c) -> double & { return H[r + (size_t)c * (m + 1)]; };
    const int iterMax = max_iters > 0 ? max_iters : n;
    const double bn = std::sqrt(dot(n, b, b));
    if (bn == 0.0) {
        for (int i = 0; i < n; ++i) x[i] = 0.0;
        if (iters_out) *iters_out = 0;
        if (be_out) *be_out = 0.0;
        return 0;
    }
    rfo_matvec(n, A, x, r0.data(), threads);
    for (int i = 0; i < n; ++i) r0[i] = b[i] - r0[i];
    double beta = std::sqrt(dot(n, r0.data(), r0.data()));
    if (beta == 0.0) {
        if (iters_out) *iters_out = 0;
        if (be_out) *be_out = 0.0;
        return 0;
    }
    for (int i = 0; i < n; ++i) V[i] = (1.0 / beta) * r0[i];
    int iterOut = 0;
    double bea = 0.0, be = 0.0;
    for (;;) {
        Hc(0, m) = beta;
        for (int j = 1; j <= m; ++j) Hc(j, m) = 0.0;
        int jH;
        for (jH = 0; jH < m; ++jH) {  // 0-based column jH (Fortran jH+1)
            rfo_matvec(n, A, &V[(size_t)jH * n], w.data(), threads);
            for (int j = 0; j <= jH; ++j) Hc(j, jH) = 0.0;
            for (int j = 0; j <= jH; ++j) {
                const double *vj = &V[(size_t)j * n];
                const double h = dot(n, vj, w.data());
                Hc(j, jH) += h;
                for (int i = 0; i < n; ++i) w[i] += -h * vj[i];
            }
            const double hn = std::sqrt(dot(n, w.data(), w.data()));
            Hc(jH + 1, jH) = hn;
            if (jH + 1 < m) {
                double *vn = &V[(size_t)(jH + 1) * n];
                for (int i = 0; i < n; ++i) vn[i] = (1.0 / hn) * w[i];
            }
            for (int j = 0; j < jH; ++j) rot(Hc(j, jH), Hc(j + 1, jH), cs[j], sn[j]);
            rotg(Hc(jH, jH), Hc(jH + 1, jH), &cs[jH], &sn[jH]);
            rot(Hc(jH, m), Hc(jH + 1, m), cs[jH], sn[jH]);
            rot(Hc(jH, jH), Hc(jH + 1, jH), cs[jH], sn[jH]);
            Hc(jH + 1, jH) = 0.0;
            const double dnormres = std::fabs(Hc(jH + 1, m));
            bea = dnormres / bn;
            const int itn = iterOut * m + jH + 1;
            if (bea <= tol || itn >= iterMax) {
                // least squares solve (dtrsv 'U','N'), x_cur = x + V y
                const int k = jH + 1;
                for (int r = 0; r < k; ++r) y[r] = Hc(r, m);
                for (int c = k - 1; c >= 0; --c) {
                    y[c] /= Hc(c, c);
                    for (int r = 0; r < c; ++r) y[r] -= y[c] * Hc(r, c);
                }
                for (int i = 0; i < n; ++i) {
                    double s = 0.0;
                    for (int c = 0; c < k; ++c) s += V[(size_t)c * n + i] * y[c];
                    xcur[i] = x[i] + s;
                }
                rfo_matvec(n, A, xcur.data(), w.data(), threads);
                for (int i = 0; i < n; ++i) w[i] = b[i] - w[i];
                const double trueNormRes = std::sqrt(dot(n, w.data(), w.data()));
                be = trueNormRes / bn;
                if (be <= tol || itn >= iterMax) {
                    for (int i = 0; i < n; ++i) x[i] = xcur[i];
                    if (iters_out) *iters_out = itn;
                    if (be_out) *be_out = be;
                    return be <= tol ? 0 : -4;
                }
            }
        }
        iterOut++;
        if (bea > tol) {
            const int k = m;
            for (int r = 0; r < k; ++r) y[r] = Hc(r, m);
            for (int c = k - 1; c >= 0; --c) {
                y[c] /= Hc(c, c);
                for (int r = 0; r < c; ++r) y[r] -= y[c] * Hc(r, c);
            }
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                for (int c = 0; c < k; ++c) s += V[(size_t)c * n + i] * y[c];
                xcur[i] = x[i] + s;
            }
        }
        for (int i = 0; i < n; ++i) x[i] = xcur[i];
        rfo_matvec(n, A, x, r0.data(), threads);
        for (int i = 0; i < n; ++i) r0[i] = b[i] - r0[i];
        beta = std::sqrt(dot(n, r0.data(), r0.data()));
        for (int i = 0; i < n; ++i) V[i] = (1.0 / beta) * r0[i];
    }
}

int rfo_velocities_rows(const rfo_params *p, const double *X, const double *T, const double *coeffs,
                        int i0, int i1, double *V, double *W) {
    if (!p || p->N < 1 || p->N > kMaxN) return -1;
    set_threads(p->threads);
    const Tables t = make_tables(p->N, p->NoQI);
    const Consts k = make_consts(p->eps, p->N);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = i0; i < i1; ++i)
        velocity_target(p, t, k, X, T, coeffs, i, V + 3 * (i - i0), W + 3 * (i - i0));
    return 0;
}

int rfo_velocities(const rfo_params *p, const double *X, const double *T, const double *coeffs,
                   double *V, double *W) {
    return rfo_velocities_rows(p, X, T, coeffs, 0, p->M, V, W);
}

struct rfo_sim {
    rfo_params p;
    int step = 0;
    // triple buffered state (advect_fibers.f90:239-245), index by role
    std::vector<double> X[3], T[3], V[2], W[2];
    int prev = 0, cur = 1, next = 2, vold = 0, vnew = 1;
    std::vector<double> init_guess, coeffs, b;
    // the step's system matrix (n x n column-major), allocated at the first
    // assembly and kept for the following steps; every entry is rewritten
    std::unique_ptr<double[]> A;
    double assemble_s = 0.0;
    int info = 0, iters = 0;
    double be = 0.0;
    double t4[4] = {0, 0, 0, 0};
};

rfo_sim *rfo_sim_create(const rfo_params *p, const double *X0, const double *T0) {
    if (!p || p->M < 1 || p->N < 1 || p->N > kMaxN) return nullptr;
    rfo_sim *s = new rfo_sim;
    s->p = *p;
    const size_t m3 = 3 * (size_t)p->M, n = m3 * p->N;
    for (int r = 0; r < 3; ++r) { s->X[r].assign(m3, 0.0); s->T[r].assign(m3, 0.0); }
    for (int r = 0; r < 2; ++r) { s->V[r].assign(m3, 0.0); s->W[r].assign(m3, 0.0); }
    std::copy(X0, X0 + m3, s->X[s->cur].begin());
    // normalise the input orientations (advect_fibers.f90:332-340)
    for (int i = 0; i < p->M; ++i) {
        const double *t = T0 + 3 * i;
        const double tm = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        for (int a = 0; a < 3; ++a) s->T[s->cur][3 * i + a] = t[a] / tm;
    }
    s->init_guess.assign(n, 0.0);
    s->coeffs.assign(n, 0.0);
    s->b.assign(n, 0.0);
    return s;
}

void rfo_sim_destroy(rfo_sim *s) { delete s; }

int rfo_sim_assemble_part(rfo_sim *s, int i0, int i1) {
    // Rows of the step's A and b that belong to target fibers [i0, i1)
    // (matrix_assembly.f90:407-629, 796-905 restricted to those targets).
    const rfo_params &p = s->p;
    if (i0 < 0 || i1 > p.M || i0 > i1) return -1;
    const size_t n = 3 * (size_t)p.M * p.N;
    if (!s->A) s->A.reset(new double[n * n]);
    if (i0 == i1) return 0;
    const double t0 = now_s();
    const size_t r0 = (size_t)i0 * 3 * p.N;
    const int rc = assemble_rows_ld(&p, s->X[s->cur].data(), s->T[s->cur].data(), i0, i1, s->A.get() + r0,
                                    n, s->b.data() + r0);
    s->assemble_s += now_s() - t0;
    return rc;
}

int rfo_sim_finish_step(rfo_sim *s) {
    // The rest of the time step on the assembled system: solve, velocities,
    // advection, rotation of the state buffers (advect_fibers.f90:437-593).
    const rfo_params &p = s->p;
    const int M = p.M;
    const size_t m3 = 3 * (size_t)M, n = m3 * p.N;
    if (!s->A) return -1;
    double *A = s->A.get();
    const double *X = s->X[s->cur].data(), *T = s->T[s->cur].data();
    double t1 = now_s();
    // solve (coeffs_and_vels.f90:80-172 direct, 361-532 GMRES with LU fallback)
    if (p.direct) {
        s->coeffs = s->b;
        s->info = rfo_solve_direct((int)n, A, s->coeffs.data());
        s->iters = 0;
        s->be = 0.0;
    } else {
        s->coeffs = s->init_guess;
        s->info = rfo_solve_gmres((int)n, A, s->b.data(), s->coeffs.data(), p.restart, p.max_iters,
                                  p.tol, &s->iters, &s->be, p.threads);
        if (s->info == -4) {
            s->coeffs = s->b;
            rfo_solve_direct((int)n, A, s->coeffs.data());
        }
    }
    s->init_guess = s->coeffs;
    double t2 = now_s();
    // velocities into the "new" slot (advect_fibers.f90:464-477)
    std::swap(s->vold, s->vnew);
    rfo_velocities(&p, X, T, s->coeffs.data(), s->V[s->vnew].data(), s->W[s->vnew].data());
    double t3 = now_s();
    // advection (advect_fibers.f90:498-523)
    double *Xn = s->X[s->next].data(), *Tn = s->T[s->next].data();
    const double *Xc = s->X[s->cur].data(), *Tc = s->T[s->cur].data();
    const double *Xp = s->X[s->prev].data(), *Tp = s->T[s->prev].data();
    const double *Vn = s->V[s->vnew].data(), *Wn = s->W[s->vnew].data();
    const double *Vo = s->V[s->vold].data(), *Wo = s->W[s->vold].data();
    const double dt = p.dt;
    for (size_t i = 0; i < m3; ++i) {
        if (s->step == 0) {
            Xn[i] = Xc[i] + dt * Vn[i];
            Tn[i] = Tc[i] + dt * Wn[i];
        } else {
            Xn[i] = 4.0 / 3.0 * Xc[i] - 1.0 / 3.0 * Xp[i] + 2.0 / 3.0 * dt * (2.0 * Vn[i] - Vo[i]);
            Tn[i] = 4.0 / 3.0 * Tc[i] - 1.0 / 3.0 * Tp[i] + 2.0 / 3.0 * dt * (2.0 * Wn[i] - Wo[i]);
        }
    }
    for (int i = 0; i < M; ++i) {
        const double tm = std::sqrt(Tn[3 * i] * Tn[3 * i] + Tn[3 * i + 1] * Tn[3 * i + 1] +
                                    Tn[3 * i + 2] * Tn[3 * i + 2]);
        for (int a = 0; a < 3; ++a) Tn[3 * i + a] = Tn[3 * i + a] / tm;
    }
    double t4 = now_s();
    // rotate: prev <- cur <- next
    const int oldprev = s->prev;
    s->prev = s->cur;
    s->cur = s->next;
    s->next = oldprev;
    s->step++;
    s->t4[0] = s->assemble_s; s->t4[1] = t2 - t1; s->t4[2] = t3 - t2; s->t4[3] = t4 - t3;
    s->assemble_s = 0.0;
    return s->info == -4 ? 1 : 0;
}

int rfo_sim_step(rfo_sim *s) {
    const int rc = rfo_sim_assemble_part(s, 0, s->p.M);
    if (rc != 0) return rc;
    return rfo_sim_finish_step(s);
}

void rfo_sim_last(const rfo_sim *s, double *b, double *coeffs, double *V, double *W, double *X, double *T) {
    const size_t m3 = 3 * (size_t)s->p.M, n = m3 * s->p.N;
    if (b) std::copy(s->b.begin(), s->b.begin() + n, b);
    if (coeffs) std::copy(s->coeffs.begin(), s->coeffs.begin() + n, coeffs);
    if (V) std::copy(s->V[s->vnew].begin(), s->V[s->vnew].end(), V);
    if (W) std::copy(s->W[s->vnew].begin(), s->W[s->vnew].end(), W);
    if (X) std::copy(s->X[s->cur].begin(), s->X[s->cur].end(), X);
    if (T) std::copy(s->T[s->cur].begin(), s->T[s->cur].end(), T);
}

void rfo_sim_solve_info(const rfo_sim *s, int *info, int *iters, double *be) {
    if (info) *info = s->info;
    if (iters) *iters = s->iters;
    if (be) *be = s->be;
}

void rfo_sim_timings(const rfo_sim *s, double *t4) {
    for (int i = 0; i < 4; ++i) t4[i] = s->t4[i];
}

int rfo_generate_layout(int M, int distribution, double box, double min_dist, unsigned long long seed,
                        double *positions, double *orientations) {
    // Centres: rejection sampling against every accepted centre closer than
    // min_dist, looked up in a grid of cells of side min_dist; uniform in
    // [0, box)^3 (distribution 0) or isotropic normal with deviation box (1).
    // Then every orientation: a normal 3-vector (redrawn if |t|^2 < 1e-12),
    // normalised.  The draws are consumed in that order.
    if (M < 1 || !positions || !orientations || !(box > 0.0) || min_dist < 0.0 ||
        (distribution != 0 && distribution != 1))
        return -1;
    if (distribution == 0) {
        const double r = 0.5 * min_dist;
        if ((double)M * (4.0 / 3.0) * M_PI * std::pow(r, 3.0) > 0.5 * box * box * box) return -1;
    }
    LayoutRng rng(seed);
    const double side = min_dist > 0.0 ? min_dist : 1.0;
    const double lim = min_dist * min_dist;
    std::map<std::array<int, 3>, std::vector<int>> cells;
    const long long budget = (long long)M * 100000;
    long long tries = 0;
    for (int count = 0; count < M;) {
        if (++tries > budget) return -1;
        double c[3];
        for (double &v : c) v = distribution == 0 ? box * rng.u01() : box * rng.gauss();
        const std::array<int, 3> cell = {(int)std::floor(c[0] / side), (int)std::floor(c[1] / side),
                                         (int)std::floor(c[2] / side)};
        bool accept = true;
        if (min_dist > 0.0) {
            for (int a = -1; a <= 1 && accept; ++a)
                for (int bb = -1; bb <= 1 && accept; ++bb)
                    for (int cc = -1; cc <= 1 && accept; ++cc) {
                        const auto it = cells.find({cell[0] + a, cell[1] + bb, cell[2] + cc});
                        if (it == cells.end()) continue;
                        for (const int j : it->second) {
                            const double dx = c[0] - positions[3 * j], dy = c[1] - positions[3 * j + 1],
                                         dz = c[2] - positions[3 * j + 2];
                            if (dx * dx + dy * dy + dz * dz < lim) {
                                accept = false;
                                break;
                            }
                        }
                    }
        }
        if (!accept) continue;
        std::copy(c, c + 3, positions + 3 * count);
        cells[cell].push_back(count);
        ++count;
    }
    for (int i = 0; i < M; ++i) {
        double t[3], q;
        do {
            q = 0.0;
            for (double &v : t) {
                v = rng.gauss();
                q += v * v;
            }
        } while (q < 1e-12);
        q = std::sqrt(q);
        for (int a = 0; a < 3; ++a) orientations[3 * i + a] = t[a] / q;
    }
    return 0;
}

}  // extern "C"
