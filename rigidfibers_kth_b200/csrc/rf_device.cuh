// rf_device.cuh - device-side building blocks shared by the assembly and
// velocity kernels: quadrature tables, the analytic inner integral of
// Int_analytical.f90 and the Stokeslet/doublet tensor.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace rf {

constexpr int kMaxN = 8;
constexpr int kMaxLQ = 48;  // NoQI <= 16

// Per-run tables in device memory, staged to shared memory by each CTA.
struct Tables {
    int N, LQ;
    double pv[kMaxLQ];               // Gauss points on [-1,1]   (quadrature.f90:78-84)
    double wv[kMaxLQ];               // weights (sum 2)
    double P[kMaxN + 1][kMaxLQ];     // P_m(pv[q]), m = 0..N      (matrix_assembly.f90:36-56)
    double eps2;                     // slenderness squared
    double D1;                       // 0.75/(d-2)                 (matrix_assembly.f90:462)
    double Ek[kMaxN + 1];            // E_k                        (:484)
    double gamma[kMaxN + 1];         // gamma_k                    (:582)
    double d;                        // -log(eps^2 e)
    double e;                        // 2
    double half_force[3];            // 0.5 * ExtForce
    double force[3];                 // ExtForce
};

// Legendre P_m = scale_m * sum_p a_mp s^p with the integer coefficients of the
// Fortran combinations (Int_analytical.f90:213-288), highest power first.
__host__ __device__ constexpr double leg_scale(int m) {
    return m <= 1 ? 1.0 : (m <= 3 ? 0.5 : (m <= 5 ? 0.125 : (m <= 7 ? 0.0625 : 1.0 / 128.0)));
}
__host__ __device__ constexpr double leg_coef(int m, int p) {
    // row m, power p
    return m == 0 ? (p == 0 ? 1 : 0)
         : m == 1 ? (p == 1 ? 1 : 0)
         : m == 2 ? (p == 2 ? 3 : p == 0 ? -1 : 0)
         : m == 3 ? (p == 3 ? 5 : p == 1 ? -3 : 0)
         : m == 4 ? (p == 4 ? 35 : p == 2 ? -30 : p == 0 ? 3 : 0)
         : m == 5 ? (p == 5 ? 63 : p == 3 ? -70 : p == 1 ? 15 : 0)
         : m == 6 ? (p == 6 ? 231 : p == 4 ? -315 : p == 2 ? 105 : p == 0 ? -5 : 0)
         : m == 7 ? (p == 7 ? 429 : p == 5 ? -693 : p == 3 ? 315 : p == 1 ? -35 : 0)
         : (p == 8 ? 6435 : p == 6 ? -12012 : p == 4 ? 6930 : p == 2 ? -1260 : p == 0 ? 35 : 0);
}

// Moments I_n = int s^n/R, J_n = int s^n/R^3, S_n = int s^n/R^5 over s in
// [-1,1], R = |R0 - s pb|, n = 0..N+2 (Int_analytical.f90:72-207).
// Forward recursion when c < 10, backward recursion from n = 27 otherwise,
// closed forms for n = 0, 1 with the d < 1e-14 special branch.
// The FP64 instance follows the reference formulas; divisions by loop
// constants are folded into compile-time reciprocals.
// Non-contracted FP64 arithmetic: the reference evaluates the closed forms
// and the forward recursion without fused multiply-adds, and the forward
// recursion amplifies every rounding difference, so these parts follow the
// Fortran operation order exactly.
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return __ddiv_rn(a, b); }

template <int N>
__device__ __forceinline__ void moments_fp64(double b, double c, double *I, double *J, double *S) {
    constexpr int K = N + 3;
    // Int_analytical.f90:96-102
    const double ue = sqrt(fadd(fadd(1.0, b), c));
    const double ub = sqrt(fadd(fsub(1.0, b), c));
    const double te = fadd(1.0, fmul(0.5, b));
    const double tb = fadd(-1.0, fmul(0.5, b));
    const double d = fsub(c, fmul(fmul(0.25, b), b));
    // :113-114
    I[0] = fsub(log(fabs(fadd(fadd(2.0, b), fmul(2.0, ue)))), log(fabs(fadd(fadd(-2.0, b), fmul(2.0, ub)))));
    I[1] = fsub(fsub(ue, ub), fmul(fmul(0.5, b), I[0]));
    // :162-170
    if (d < 1e-14) {
        const double e1 = fadd(1.0, fmul(b, 0.5)), e2 = fadd(-1.0, fmul(b, 0.5));  // b/2 is exact
        J[0] = fadd(fdiv(-1.0, fmul(2.0, fmul(e1, e1))), fdiv(1.0, fmul(2.0, fmul(e2, e2))));
    } else {
        J[0] = fsub(fdiv(te, fmul(d, ue)), fdiv(tb, fmul(d, ub)));
    }
    J[1] = fsub(fadd(fdiv(-1.0, ue), fdiv(1.0, ub)), fmul(fmul(b, 0.5), J[0]));
    // :189-196
    if (d < 1e-14) {
        const double p = fadd(2.0, b), m = fadd(-2.0, b);
        const double p2 = fmul(p, p), m2 = fmul(m, m);
        S[0] = fadd(fdiv(-4.0, fmul(p2, p2)), fdiv(4.0, fmul(m2, m2)));
        S[1] = fsub(fadd(fdiv(-8.0, fmul(3.0, fmul(p2, p))), fdiv(8.0, fmul(3.0, fmul(m2, m)))),
                    fmul(fmul(b, 0.5), S[0]));
    } else {
        const double ue3 = fmul(fmul(ue, ue), ue), ub3 = fmul(fmul(ub, ub), ub);
        const double d6 = fmul(6.0, d);
        S[0] = fadd(fsub(fdiv(fadd(2.0, b), fmul(d6, ue3)), fdiv(fadd(-2.0, b), fmul(d6, ub3))),
                    fmul(fdiv(2.0, fmul(3.0, d)), J[0]));
        S[1] = fsub(fadd(fdiv(-fadd(b, fmul(2.0, c)), fmul(d6, ue3)), fdiv(fadd(-b, fmul(2.0, c)), fmul(d6, ub3))),
                    fmul(fdiv(b, fmul(3.0, d)), J[0]));
    }
    if (c < 10.0) {
        // forward recursion, :123-136, 172-176, 197-200
#pragma unroll
        for (int n = 2; n < K; ++n) {
            const double nn = n + 1.0;                     // Fortran nn
            const double om = 1.0 - nn;
            const double sbp = (n % 2 == 1) ? 1.0 : -1.0;  // sb**(ii-2)
            const double t1 = fdiv(ue, om);
            const double t2 = fdiv(fmul(sbp, ub), om);
            const double t3 = fmul(fdiv(fmul(0.5 - (nn - 1.0), b), om), I[n - 1]);
            const double t4 = fmul(fdiv(fmul(nn - 2.0, c), om), I[n - 2]);
            I[n] = fadd(fsub(fsub(t2, t1), t3), t4);
            J[n] = fsub(fsub(I[n - 2], fmul(b, J[n - 1])), fmul(c, J[n - 2]));
            S[n] = fsub(fsub(J[n - 2], fmul(b, S[n - 1])), fmul(c, S[n - 2]));
        }
    } else {
        // backward recursion from n = 27 (:137-157, 177-183, 201-206); stable, so
        // folded constants and fused arithmetic are used here
        const double ic = 1.0 / c;
        double i1 = 0.0, i2 = 0.0, j1 = 0.0, j2 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int n = 27; n >= 2; --n) {
            const double nn = n;                                       // Fortran nn = ii - 1
            const double a0 = (nn + 2.0) / (nn + 1.0);
            const double r2 = 1.0 / (nn + 2.0);
            const double cb = (1.0 - 2.0 * (nn + 2.0)) / (2.0 * (nn + 2.0));
            const double sbp = ((n + 1) % 2 == 0) ? 1.0 : -1.0;        // (-1)^(nn+1)
            const double in = a0 * ic * (ue * r2 - sbp * ub * r2 + cb * b * i1 - i2);
            const double jn = ic * (in - b * j1 - j2);
            const double sn = ic * (jn - b * s1 - s2);
            if (n < K) { I[n] = in; J[n] = jn; S[n] = sn; }
            i2 = i1; i1 = in; j2 = j1; j1 = jn; s2 = s1; s1 = sn;
        }
    }
}

// First index of the FP32 backward recursion.  Its starting values
// I = J = S = 0 at n + 1, n + 2 are wrong by the true moments there; the error
// reaches n = 0 damped by c^(-n/2) (the recursion's homogeneous solutions grow
// like |lambda|^n, lambda^2 + b lambda + c = 0, |lambda| = sqrt(c) since
// d >= 0) times a polynomial in n that is largest for the S moments of a point
// on the source axis.  From n = 32 that error is below FP32 rounding for every
// c >= 6 and every direction: with sampled b, the Legendre combinations of the
// moments stay within 8e-7 of |X_0| (X = I, J, S) at c = 6, 6.5, 7, 8 on and
// off the axis; from the reference's n = 27 the on-axis S error is 1e-5 at c = 6.
constexpr int kBackTop = 32;

// FP32 moments by the backward recursion alone, run down to n = 0.  The
// three-term relations that the reference uses for n >= 2
// (Int_analytical.f90:137-157, 177-183, 201-206) hold at n = 0 and 1 as well:
// d/ds[s^(n+1) R] = ((n+2) s^(n+2) + (n+3/2) b s^(n+1) + (n+1) c s^n) / R and
// s^n / R = s^n (s^2 + b s + c) / R^3.  The reference's n = 0, 1 closed forms
// (a logarithm of a ratio close to 1, ue - ub - b I_0 / 2, 1/ub - 1/ue and the
// S_0, S_1 differences over d) cancel by a factor that grows like c: a pair
// 100 fiber half-lengths apart loses every FP32 digit in them, and at a point
// near the source axis the 1/d forms cancel too.  The recursion has neither
// cancellation: ue - ub enters only as 2b / (ue + ub), and d not at all.
// Accurate for c >= 6 in every direction (see kBackTop).
template <int N>
__device__ __forceinline__ void moments_backward_fp32(float b, float c, float *I, float *J, float *S) {
    constexpr int K = N + 3;
    const float xe = 1.0f + b + c, xb = 1.0f - b + c;
    const float ue = xe * rsqrtf(xe), ub = xb * rsqrtf(xb);
    const float ic = __fdividef(1.0f, c);
    const float icb = ic * b;
    const float icwp = __fdividef(2.0f * b, ue + ub) * ic;  // (ue - ub) / c
    const float icwm = (ue + ub) * ic;
    const float nic = -ic, nicb = -icb, ic2 = ic * ic;
    // J and S are carried as c J_n and c^2 S_n: their steps become two fused
    // multiply-adds each, c J_n = I_n - (b/c) c J_{n+1} - (1/c) c J_{n+2} and
    // c^2 S_n = c J_n - (b/c) c^2 S_{n+1} - (1/c) c^2 S_{n+2}
    float i1 = 0.f, i2 = 0.f, j1 = 0.f, j2 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
    for (int n = kBackTop; n >= 0; --n) {
        // I_n = (ue - (-1)^(n+1) ub - (n+3/2) b I_{n+1} - (n+2) I_{n+2}) / ((n+1) c)
        const float a0 = (n + 2.0f) / (n + 1.0f);
        const float r2 = 1.0f / (n + 2.0f);
        const float cb = (1.0f - 2.0f * (n + 2.0f)) / (2.0f * (n + 2.0f));
        const float icw = ((n + 1) % 2 == 0) ? icwp : icwm;
        const float in = fmaf((a0 * cb) * icb, i1, fmaf(-a0 * ic, i2, (a0 * r2) * icw));
        const float jn = fmaf(nicb, j1, fmaf(nic, j2, in));
        const float sn = fmaf(nicb, s1, fmaf(nic, s2, jn));
        if (n < K) { I[n] = in; J[n] = jn * ic; S[n] = sn * ic2; }
        i2 = i1; i1 = in; j2 = j1; j1 = jn; s2 = s1; s1 = sn;
    }
}

// The same recursion for two points at once on Blackwell's packed FP32 units
// (__ffma2_rn / __fmul2_rn: one instruction, two FMAs, each rounded exactly as
// fmaf): component .x is one point, .y the other, every operation and its
// order as in moments_backward_fp32, so the moments are bit-identical.
template <int N>
__device__ __forceinline__ void moments_backward_fp32x2(float2 b, float2 c, float2 *I, float2 *J, float2 *S) {
    constexpr int K = N + 3;
    const float xe0 = 1.0f + b.x + c.x, xb0 = 1.0f - b.x + c.x;
    const float xe1 = 1.0f + b.y + c.y, xb1 = 1.0f - b.y + c.y;
    const float ue0 = xe0 * rsqrtf(xe0), ub0 = xb0 * rsqrtf(xb0);
    const float ue1 = xe1 * rsqrtf(xe1), ub1 = xb1 * rsqrtf(xb1);
    const float ic0 = __fdividef(1.0f, c.x), ic1 = __fdividef(1.0f, c.y);
    const float2 ic = make_float2(ic0, ic1);
    const float2 icb = make_float2(ic0 * b.x, ic1 * b.y);
    const float2 icwp = make_float2(__fdividef(2.0f * b.x, ue0 + ub0) * ic0, __fdividef(2.0f * b.y, ue1 + ub1) * ic1);
    const float2 icwm = make_float2((ue0 + ub0) * ic0, (ue1 + ub1) * ic1);
    const float2 nic = make_float2(-ic0, -ic1), nicb = make_float2(-icb.x, -icb.y);
    const float2 ic2 = make_float2(ic0 * ic0, ic1 * ic1);
    const float2 z = make_float2(0.f, 0.f);
    float2 i1 = z, i2 = z, j1 = z, j2 = z, s1 = z, s2 = z;
#pragma unroll
    for (int n = kBackTop; n >= 0; --n) {
        const float a0 = (n + 2.0f) / (n + 1.0f);
        const float r2 = 1.0f / (n + 2.0f);
        const float cb = (1.0f - 2.0f * (n + 2.0f)) / (2.0f * (n + 2.0f));
        const float2 icw = ((n + 1) % 2 == 0) ? icwp : icwm;
        const float2 ca = __fmul2_rn(make_float2(a0 * cb, a0 * cb), icb);
        const float2 cn = __fmul2_rn(make_float2(-a0, -a0), ic);
        const float2 cw = __fmul2_rn(make_float2(a0 * r2, a0 * r2), icw);
        const float2 in = __ffma2_rn(ca, i1, __ffma2_rn(cn, i2, cw));
        const float2 jn = __ffma2_rn(nicb, j1, __ffma2_rn(nic, j2, in));
        const float2 sn = __ffma2_rn(nicb, s1, __ffma2_rn(nic, s2, jn));
        if (n < K) {
            I[n] = in;
            J[n] = __fmul2_rn(jn, ic);
            S[n] = __fmul2_rn(sn, ic2);
        }
        i2 = i1; i1 = in; j2 = j1; j1 = jn; s2 = s1; s1 = sn;
    }
}

// Geometry of one (target point, source fiber) item in FP32 for the moments:
// b = -2 p.R0, c = |R0|^2, and the three quantities that the closed forms
// need near the source and that c and b determine only through cancellation:
// ue^2 = 1 + b + c = |R0 - p|^2, ub^2 = 1 - b + c = |R0 + p|^2 and
// d = c - b^2/4 = |R0 x p|^2 (|p| = 1).  Formed from the vectors they keep
// their relative accuracy when a target point comes within 1e-4 of the
// source fiber (fibers that touch or cross); from b and c they round to zero
// or below, and the closed forms then take the root or logarithm of a
// negative number.
struct Geom32 {
    float b, c, ue2, ub2, d;
    __device__ __forceinline__ Geom32(float r0x, float r0y, float r0z, float px, float py, float pz) {
        b = -2.0f * (px * r0x + py * r0y + pz * r0z);
        c = r0x * r0x + r0y * r0y + r0z * r0z;
        const float ex = r0x - px, ey = r0y - py, ez = r0z - pz;
        const float fx = r0x + px, fy = r0y + py, fz = r0z + pz;
        ue2 = ex * ex + ey * ey + ez * ez;
        ub2 = fx * fx + fy * fy + fz * fz;
        const float cx = fmaf(r0y, pz, -r0z * py), cy = fmaf(r0z, px, -r0x * pz), cz = fmaf(r0x, py, -r0y * px);
        d = cx * cx + cy * cy + cz * cz;
    }
};

// FP32 moments for every point of the plain FP32 method and for the far field
// (c >= near_c >= 10) of the tile mixed-precision kernel.  For c >= 6 the
// backward recursion alone (moments_backward_fp32; it needs only b and c): the
// reference switches at 10 in FP64, but its forward recursion amplifies
// rounding by orders of magnitude as c approaches 10, which FP32 cannot
// absorb, while from 6 on the backward recursion is accurate to FP32 rounding.
// Below 6 (plain FP32 method only) the reference's closed forms and forward
// recursion on ue^2, ub^2 and d formed from the vectors (Geom32), the closed
// forms rewritten without the cancellation te/ue - tb/ub (which loses all FP32
// digits when the target point lies near the source axis):
// te/ue - tb/ub = 2b d / ((te ub + tb ue) ue ub) when te and tb share a sign.
// FAR = true: the caller guarantees c >= 6 (far pairs of the split assembly).
template <int N, bool FAR = false>
__device__ __forceinline__ void moments_fp32(const Geom32 &g, float *I, float *J, float *S) {
    const float b = g.b, c = g.c;
    if (FAR || c >= 6.0f) {
        moments_backward_fp32<N>(b, c, I, J, S);
        return;
    }
    constexpr int K = N + 3;
    const float ue = sqrtf(g.ue2);
    const float ub = sqrtf(g.ub2);
    const float te = 1.0f + 0.5f * b;
    const float tb = -1.0f + 0.5f * b;
    const float d = g.d;
    const float iue = __frcp_rn(ue), iub = __frcp_rn(ub), id = __frcp_rn(d);
    // log((2te + 2ue)/(2tb + 2ub)) with the smaller operand formed stably
    const float ae = (te >= 0.f) ? (te + ue) : d * __frcp_rn(ue - te);
    const float ab = (tb >= 0.f) ? (tb + ub) : d * __frcp_rn(ub - tb);
    I[0] = logf(ae * __frcp_rn(ab));
    I[1] = ue - ub - 0.5f * b * I[0];
    if (d < 1e-6f * c && te * tb > 0.f) {
        // point on the source axis beyond its ends: the d -> 0 limits
        // (Int_analytical.f90:162-164, 189-191).  Within the span (te tb < 0:
        // fibers that touch or cross) the general forms below hold with the
        // accurate d and have no cancellation.
        J[0] = 0.5f * (__frcp_rn(tb * tb) - __frcp_rn(te * te));
        J[1] = -iue + iub - 0.5f * b * J[0];
        const float p = 2.0f + b, m = -2.0f + b;
        const float ip = __frcp_rn(p), im = __frcp_rn(m);
        const float ip2 = ip * ip, im2 = im * im;
        S[0] = 4.0f * (im2 * im2 - ip2 * ip2);
        S[1] = (8.0f / 3.0f) * (im2 * im - ip2 * ip) - 0.5f * b * S[0];
    } else {
        // (te/ue - tb/ub)/d; with te, tb of one sign te/ue - tb/ub = 2b d / ((te ub + tb ue) ue ub)
        if (te * tb > 0.f) J[0] = 2.0f * b * __frcp_rn((te * ub + tb * ue) * ue * ub);
        else J[0] = (te * iue - tb * iub) * id;
        J[1] = -iue + iub - 0.5f * b * J[0];
        const float iue3 = iue * iue * iue, iub3 = iub * iub * iub;
        S[0] = ((2.0f + b) * iue3 - (-2.0f + b) * iub3) * (id * (1.0f / 6.0f)) + (2.0f / 3.0f) * id * J[0];
        S[1] = (-(b + 2.0f * c) * iue3 + (-b + 2.0f * c) * iub3) * (id * (1.0f / 6.0f)) -
               b * (1.0f / 3.0f) * id * J[0];
    }
#pragma unroll
    for (int n = 2; n < K; ++n) {
        const float nn = n + 1.0f;
        const float r = 1.0f / (1.0f - nn);
        const float sbp = (n % 2 == 1) ? 1.0f : -1.0f;
        I[n] = -ue * r + sbp * ub * r - (0.5f - (nn - 1.0f)) * b * r * I[n - 1] + (nn - 2.0f) * c * r * I[n - 2];
        J[n] = I[n - 2] - b * J[n - 1] - c * J[n - 2];
        S[n] = J[n - 2] - b * S[n - 1] - c * S[n - 2];
    }
}

// Outer products of R0 and the source direction pb shared by every Legendre
// weight, packed 11,22,33,12,13,23.
template <typename T>
struct Outer {
    T rr[6], pr[6], pp[6];
    __device__ __forceinline__ Outer(T r0x, T r0y, T r0z, T px, T py, T pz) {
        rr[0] = r0x * r0x; rr[1] = r0y * r0y; rr[2] = r0z * r0z;
        rr[3] = r0x * r0y; rr[4] = r0x * r0z; rr[5] = r0y * r0z;
        pr[0] = (T)2 * px * r0x; pr[1] = (T)2 * py * r0y; pr[2] = (T)2 * pz * r0z;
        pr[3] = px * r0y + r0x * py; pr[4] = px * r0z + r0x * pz; pr[5] = py * r0z + r0y * pz;
        pp[0] = px * px; pp[1] = py * py; pp[2] = pz * pz;
        pp[3] = px * py; pp[4] = px * pz; pp[5] = py * pz;
    }
};

// Legendre-weighted moments for weight m and the tensor G_m (6 packed
// components 11,22,33,12,13,23), Int_analytical.f90:213-288 and 735-746:
// G = L11 I + L12 R0R0 - L13 (pb R0 + R0 pb) + L14 pb pb
//   + 2 eps^2 (L12 I - 3 L22 R0R0 + 3 L23 (pb R0 + R0 pb) - 3 L24 pb pb)
// Each L is scale_m * (sum of integer-weighted moments), highest power first.
template <typename T, int m>
__device__ __forceinline__ void g_coeffs(const T *I, const T *J, const T *S, T eps2, T &cI, T &cRR, T &cPR,
                                         T &cPP) {
    T l11 = 0, l12 = 0, l13 = 0, l14 = 0, l22 = 0, l23 = 0, l24 = 0;
#pragma unroll
    for (int p = m; p >= 0; --p) {
        if (leg_coef(m, p) != 0) {
            const T a = (T)leg_coef(m, p);
            l11 += a * I[p];
            l12 += a * J[p];
            l13 += a * J[p + 1];
            l14 += a * J[p + 2];
            l22 += a * S[p];
            l23 += a * S[p + 1];
            l24 += a * S[p + 2];
        }
    }
    const T sc = (T)leg_scale(m);
    l11 *= sc; l12 *= sc; l13 *= sc; l14 *= sc; l22 *= sc; l23 *= sc; l24 *= sc;
    const T e2 = (T)2 * eps2;
    cI = l11 + e2 * l12;                // identity
    cRR = l12 - (T)3 * e2 * l22;        // R0 R0
    cPR = -l13 + (T)3 * e2 * l23;       // pb R0 + R0 pb
    cPP = l14 - (T)3 * e2 * l24;        // pb pb
}

template <typename T, int m>
__device__ __forceinline__ void g_tensor(const T *I, const T *J, const T *S, const Outer<T> &o, T eps2, T *G) {
    T cI, cRR, cPR, cPP;
    g_coeffs<T, m>(I, J, S, eps2, cI, cRR, cPR, cPP);
#pragma unroll
    for (int c = 0; c < 6; ++c) G[c] = cRR * o.rr[c] + cPR * o.pr[c] + cPP * o.pp[c] + (c < 3 ? cI : (T)0);
}

// Store G_m for m = 0..N straight to shared memory as it is formed:
// dst[(m*6 + c) * ld], converting to double.
template <typename T, int N, int m = 0>
struct GStore {
    __device__ __forceinline__ static void run(const T *I, const T *J, const T *S, const Outer<T> &o, T eps2,
                                               double *dst, int ld) {
        T G[6];
        g_tensor<T, m>(I, J, S, o, eps2, G);
#pragma unroll
        for (int c = 0; c < 6; ++c) dst[(m * 6 + c) * ld] = (double)G[c];
        GStore<T, N, m + 1>::run(I, J, S, o, eps2, dst, ld);
    }
};
template <typename T, int N>
struct GStore<T, N, N + 1> {
    __device__ __forceinline__ static void run(const T *, const T *, const T *, const Outer<T> &, T, double *, int) {}
};

// u = sum_m G_m f_m without forming G_m:
// G f = cI f + R0 (cRR R0.f + cPR pb.f) + pb (cPR R0.f + cPP pb.f)
template <typename T, int N, int m = 0>
struct GForce {
    __device__ __forceinline__ static void run(const T *I, const T *J, const T *S, T r0x, T r0y, T r0z, T px,
                                               T py, T pz, T eps2, const T (*f)[3], T *u) {
        T cI, cRR, cPR, cPP;
        g_coeffs<T, m>(I, J, S, eps2, cI, cRR, cPR, cPP);
        const T rf = r0x * f[m][0] + r0y * f[m][1] + r0z * f[m][2];
        const T pf = px * f[m][0] + py * f[m][1] + pz * f[m][2];
        const T aR = cRR * rf + cPR * pf;
        const T aP = cPR * rf + cPP * pf;
        u[0] += cI * f[m][0] + aR * r0x + aP * px;
        u[1] += cI * f[m][1] + aR * r0y + aP * py;
        u[2] += cI * f[m][2] + aR * r0z + aP * pz;
        GForce<T, N, m + 1>::run(I, J, S, r0x, r0y, r0z, px, py, pz, eps2, f, u);
    }
};
template <typename T, int N>
struct GForce<T, N, N + 1> {
    __device__ __forceinline__ static void run(const T *, const T *, const T *, T, T, T, T, T, T, T,
                                               const T (*)[3], T *) {}
};

// The analytic inner integral for all weights, stored to shared memory.
template <int N>
__device__ __forceinline__ void inner_analytic_store_fp64(double r0x, double r0y, double r0z, double px, double py,
                                                          double pz, double eps2, double *dst, int ld) {
    double I[N + 3], J[N + 3], S[N + 3];
    const double b = fmul(-2.0, fadd(fadd(fmul(px, r0x), fmul(py, r0y)), fmul(pz, r0z)));
    const double c = fadd(fadd(fmul(r0x, r0x), fmul(r0y, r0y)), fmul(r0z, r0z));
    moments_fp64<N>(b, c, I, J, S);
    const Outer<double> o(r0x, r0y, r0z, px, py, pz);
    GStore<double, N>::run(I, J, S, o, eps2, dst, ld);
}

template <int N>
__device__ __forceinline__ void inner_analytic_store_fp32(float r0x, float r0y, float r0z, float px, float py,
                                                          float pz, float eps2, double *dst, int ld) {
    float I[N + 3], J[N + 3], S[N + 3];
    moments_fp32<N>(Geom32(r0x, r0y, r0z, px, py, pz), I, J, S);
    const Outer<float> o(r0x, r0y, r0z, px, py, pz);
    GStore<float, N>::run(I, J, S, o, eps2, dst, ld);
}

// sum_m G_m f_m at one target point (FP64): the velocity integrand
// (G_compute_GQ_f_kg, Int_analytical.f90:772-850)
template <int N>
__device__ __forceinline__ void inner_analytic_force_fp64(double r0x, double r0y, double r0z, double px, double py,
                                                          double pz, double eps2, const double (*f)[3], double *u) {
    double I[N + 3], J[N + 3], S[N + 3];
    const double b = fmul(-2.0, fadd(fadd(fmul(px, r0x), fmul(py, r0y)), fmul(pz, r0z)));
    const double c = fadd(fadd(fmul(r0x, r0x), fmul(r0y, r0y)), fmul(r0z, r0z));
    moments_fp64<N>(b, c, I, J, S);
    GForce<double, N>::run(I, J, S, r0x, r0y, r0z, px, py, pz, eps2, f, u);
}

// Numeric inner integral (quadrature.f90:100-164): 3-point Gauss on each
// panel of the source fiber, kernel
// K = I/R + RR/R^3 + 2 eps^2 (I/R^3 - 3 RR/R^5), weighted by P_m.  The FP64
// instance keeps the reference's operation order (no fused multiply-adds):
// near-touching fibers make K large and the weighted sums cancel.
template <int N>
__device__ __forceinline__ void inner_numeric_fp64(double xbx, double xby, double xbz, const double *xs,
                                                   const double *ts, const double *pv, const double *wP,
                                                   int LQ, double eps2, double (*G)[6]) {
#pragma unroll
    for (int m = 0; m <= N; ++m)
#pragma unroll
        for (int c = 0; c < 6; ++c) G[m][c] = 0.0;
    const double e2 = fmul(2.0, eps2), e6 = fmul(6.0, eps2);
    for (int s = 0; s < LQ; ++s) {
        const double sp = pv[s];
        const double Rx = fsub(xbx, fadd(xs[0], fmul(ts[0], sp)));
        const double Ry = fsub(xby, fadd(xs[1], fmul(ts[1], sp)));
        const double Rz = fsub(xbz, fadd(xs[2], fmul(ts[2], sp)));
        const double Rm = sqrt(fadd(fadd(fmul(Rx, Rx), fmul(Ry, Ry)), fmul(Rz, Rz)));
        const double R3 = fmul(fmul(Rm, Rm), Rm);
        const double R5 = fmul(fmul(R3, Rm), Rm);
        const double iR = fdiv(1.0, Rm), iR3 = fdiv(1.0, R3);
        double K[6];
        K[0] = fadd(fadd(iR, fdiv(fmul(Rx, Rx), R3)), fmul(e2, fsub(iR3, fdiv(fmul(fmul(3.0, Rx), Rx), R5))));
        K[1] = fadd(fadd(iR, fdiv(fmul(Ry, Ry), R3)), fmul(e2, fsub(iR3, fdiv(fmul(fmul(3.0, Ry), Ry), R5))));
        K[2] = fadd(fadd(iR, fdiv(fmul(Rz, Rz), R3)), fmul(e2, fsub(iR3, fdiv(fmul(fmul(3.0, Rz), Rz), R5))));
        K[3] = fsub(fdiv(fmul(Rx, Ry), R3), fdiv(fmul(fmul(e6, Rx), Ry), R5));
        K[4] = fsub(fdiv(fmul(Rx, Rz), R3), fdiv(fmul(fmul(e6, Rx), Rz), R5));
        K[5] = fsub(fdiv(fmul(Ry, Rz), R3), fdiv(fmul(fmul(e6, Ry), Rz), R5));
#pragma unroll
        for (int m = 0; m <= N; ++m) {
            const double w = wP[m * kMaxLQ + s];
#pragma unroll
            for (int c = 0; c < 6; ++c) G[m][c] = fadd(G[m][c], fmul(w, K[c]));
        }
    }
}

template <int N>
__device__ __forceinline__ void inner_numeric_fp32(float xbx, float xby, float xbz, const float *xs,
                                                   const float *ts, const float *pv, const float *wP, int LQ,
                                                   float eps2, float (*G)[6]) {
#pragma unroll
    for (int m = 0; m <= N; ++m)
#pragma unroll
        for (int c = 0; c < 6; ++c) G[m][c] = 0.0f;
    for (int s = 0; s < LQ; ++s) {
        const float sp = pv[s];
        const float Rx = xbx - (xs[0] + ts[0] * sp);
        const float Ry = xby - (xs[1] + ts[1] * sp);
        const float Rz = xbz - (xs[2] + ts[2] * sp);
        const float R2 = Rx * Rx + Ry * Ry + Rz * Rz;
        const float ir = rsqrtf(R2);
        const float ir3 = ir * ir * ir;
        const float ir5 = ir3 * ir * ir;
        const float e2 = 2.0f * eps2;
        const float diag = ir + e2 * ir3;
        const float off = ir3 - 3.0f * e2 * ir5;
        float K[6];
        K[0] = diag + Rx * Rx * off;
        K[1] = diag + Ry * Ry * off;
        K[2] = diag + Rz * Rz * off;
        K[3] = Rx * Ry * off;
        K[4] = Rx * Rz * off;
        K[5] = Ry * Rz * off;
#pragma unroll
        for (int m = 0; m <= N; ++m) {
            const float w = wP[m * kMaxLQ + s];
#pragma unroll
            for (int c = 0; c < 6; ++c) G[m][c] += w * K[c];
        }
    }
}

// D = A B + C for one 8x8x4 FP64 tile (warp-wide; every lane of the warp
// takes part).  Lane l holds A[l/4][l%4], B[l%4][l/4], C/D[l/4][2(l%4)+{0,1}].
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b, double c0, double c1) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};\n"
                 : "=d"(d0), "=d"(d1)
                 : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

__device__ __forceinline__ int sym_index(int a, int b) {
    // packed index of the symmetric 3x3 component (a,b)
    return a == b ? a : (a + b == 1 ? 3 : (a + b == 2 ? 4 : 5));
}

}  // namespace rf
