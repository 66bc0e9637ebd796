// assemble.cu - K1: dense system assembly, one CTA per (target tile, source
// chunk).
//
// Reference: fortran/matrix_assembly.f90:407-629 (matrix, analytic),
// 267-404 (matrix, numeric), 796-905 / 632-794 (right-hand side);
// src/kernels/assemble_system.cu:8-263 (one thread per pair in the CUDA port).
//
// Mapping.  A CTA owns TI = 4 consecutive target fibers and walks a contiguous
// chunk of source fibers.  Thread (ti, q) keeps the target point
// xbar = x_i + s_q t_i in registers; for every source j:
//   P1  evaluates the inner integral over fiber j once for all Legendre
//       weights l = 0..N (6(N+1) tensor values) into shared memory;
//   P2  projects onto the target Legendre polynomials,
//       theta^k_l = sum_q w_q P_k(s_q) G_l(q), as a small FP64 tensor-core
//       product (mma.sync m8n8k4 f64): [k x q] * [q x (target, l, comp)];
//   P3a forms the 3N x 3N block of each (target, k, l) group, the right-hand
//       side (l = 0 against 0.5*ExtForce) and, when asked, the velocity
//       projection panels, staging the block in shared memory;
//   P3b writes the staged 3N columns x TI*3N rows with coalesced stores.
// Per-chunk partial right-hand sides are reduced afterwards in a fixed order
// (deterministic; the reference accumulates with atomicAdd).
#include <algorithm>

#include "rf_kernels.h"

namespace rf {

constexpr int kTI = 4;
#ifndef RF_ASM_MINB96
#define RF_ASM_MINB96 4
#endif
constexpr int kMinBlocks96 = RF_ASM_MINB96;  // resident 96-thread blocks per SM the registers allow

__host__ __device__ constexpr int round_up_int(int v, int m) { return (v + m - 1) / m * m; }

// MAXT: largest block the instance is compiled for (TI*LQ rounded to a warp);
// MINB resident blocks per SM bound the registers per thread.
template <int N, bool NUMERIC, int PMODE, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) assemble_kernel(AsmArgs a) {
    constexpr int TI = kTI;
    constexpr int NL = N + 1;           // weights l = 0..N
    constexpr int NG = NL * 6;          // tensor values per target point
    constexpr int NCOL = TI * NG;       // product columns (target, l, comp)
    constexpr int NTILE = NCOL / 8;
    constexpr int MT = (NL + 7) / 8;    // 8-row tiles over k = 0..N
    constexpr int RT = TI * 3 * N;      // rows of A in the tile
    constexpr int CT = 3 * N;           // columns of A per source
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LQ = a.LQ;
    const int LQP = round_up_int(LQ, 4);   // k-steps of 4
    const int KS = LQP / 4;                // tensor-core k-steps
    const int LDQ = LQP + 2;               // even: 16-byte aligned rows
    const int nwork = TI * LQ;
    const int nthreads = blockDim.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;

    // w_q P_m(q) (16 x kMaxLQ, rows > N zero): the numeric inner integral reads
    // it for every source; the analytic one only loads the tensor-core A
    // operands from it once, so there it lives in the G region (6 KB less
    // shared memory per CTA; the registers still hold the kernel at four CTAs
    // per SM: capped at 128 registers for five it spills and runs 10 % slower)
    constexpr int WP_OWN = NUMERIC || PMODE != kPModeFP64 ? 16 * kMaxLQ : 0;
    double *s_pv = reinterpret_cast<double *>(smem_raw);   // kMaxLQ
    double *s_xt = s_pv + kMaxLQ + WP_OWN;                  // TI x 3
    double *s_tt = s_xt + TI * 3;                           // TI x 3
    double *s_acc = s_tt + TI * 3;                          // TI x NL(k) x 6: sum_j theta^k_0
    double *s_th = s_acc + TI * NL * 6;                     // TI x NL(k) x NG
    // the tensor values of P1/P2 and the staged block of P3 share one region
    double *s_G = s_th + TI * NL * NG;                      // NCOL x LDQ
    double *s_blk = s_G;                                    // CT x RT staged block
    double *s_wP = WP_OWN ? s_pv + kMaxLQ : s_G;
    const int big = max(max(NCOL * LDQ, CT * RT + 2 * CT * TI * 3), 16 * kMaxLQ);
    float *s_pvf = reinterpret_cast<float *>(s_G + big);    // kMaxLQ
    float *s_wPf = s_pvf + kMaxLQ;                          // NL x kMaxLQ

    const Tables &tab = *a.tab;
    for (int t = tid; t < kMaxLQ; t += nthreads) {
        s_pv[t] = t < LQ ? tab.pv[t] : 0.0;
        s_pvf[t] = t < LQ ? (float)tab.pv[t] : 0.f;
    }
    for (int t = tid; t < 16 * kMaxLQ; t += nthreads) {
        const int m = t / kMaxLQ, q = t % kMaxLQ;
        const double w = (m <= N && q < LQ) ? tab.wv[q] * tab.P[m][q] : 0.0;
        s_wP[t] = w;
        if (m < NL) s_wPf[t] = (float)w;
    }
    const int i0 = a.t0 + blockIdx.x * TI;   // first target of the tile (global index)
    for (int t = tid; t < TI * 3; t += nthreads) {
        const int ti = t / 3, c = t % 3;
        const int i = i0 + ti;
        s_xt[t] = (i < a.t1) ? a.pos[3 * i + c] : 0.0;
        s_tt[t] = (i < a.t1) ? a.ori[3 * i + c] : 1.0;
    }
    for (int t = tid; t < TI * NL * 6; t += nthreads) s_acc[t] = 0.0;
    __syncthreads();

    const bool worker = tid < nwork;
    const int ti = worker ? tid / LQ : 0;
    const int q = worker ? tid - ti * LQ : 0;
    const int i = i0 + ti;
    const double sq = s_pv[q];
    // xbar = xc + pv(i)*ta (matrix_assembly.f90:534), not fused
    const double xbx = fadd(s_xt[ti * 3 + 0], fmul(sq, s_tt[ti * 3 + 0]));
    const double xby = fadd(s_xt[ti * 3 + 1], fmul(sq, s_tt[ti * 3 + 1]));
    const double xbz = fadd(s_xt[ti * 3 + 2], fmul(sq, s_tt[ti * 3 + 2]));
    const double eps2 = tab.eps2;
    // G values of point q are stored at position (q%4)*KS + q/4 so that each
    // lane's tensor-core B operands are contiguous
    const int qpos = (q & 3) * KS + (q >> 2);

    // A operands (w_q P_k(q)) of the projection stay in registers
    constexpr int KSMAX = MAXT / (TI * 4);
    double afrag[MT][KSMAX];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int s = 0; s < KSMAX; ++s)
            afrag[mt][s] = s < KS ? s_wP[(mt * 8 + (lane >> 2)) * kMaxLQ + 4 * s + (lane & 3)] : 0.0;
    if (!WP_OWN) __syncthreads();  // s_wP shares the G region the first source overwrites

    const int j0 = blockIdx.y * a.chunk;
    const int j1 = min(a.M, j0 + a.chunk);
    const int64_t row0 = (int64_t)(i0 - a.t0) * 3 * N;   // row of the stored matrix
    const int64_t rows_left = (int64_t)(a.t1 - i0) * 3 * N;
    const int rows_valid = rows_left < (int64_t)RT ? (int)rows_left : RT;

    __shared__ int s_nlist;
    __shared__ short s_list[kTI * kMaxLQ];

    for (int j = j0; j < j1; ++j) {
        // ---------------- P1: inner integral at (target point, source j)
        const double xs0 = __ldg(a.pos + 3 * j), xs1 = __ldg(a.pos + 3 * j + 1), xs2 = __ldg(a.pos + 3 * j + 2);
        const double ts0 = __ldg(a.ori + 3 * j), ts1 = __ldg(a.ori + 3 * j + 1), ts2 = __ldg(a.ori + 3 * j + 2);
        if (PMODE == kPModeFP64) {
            if (worker) {
                double *g = s_G + (size_t)ti * NG * LDQ + qpos;
                if (i < a.t1 && i != j) {
                    const double r0x = fsub(xbx, xs0), r0y = fsub(xby, xs1), r0z = fsub(xbz, xs2);
                    if (NUMERIC) {
                        double G[NL][6];
                        const double xs[3] = {xs0, xs1, xs2}, ts[3] = {ts0, ts1, ts2};
                        inner_numeric_fp64<N>(xbx, xby, xbz, xs, ts, s_pv, s_wP, LQ, eps2, G);
#pragma unroll
                        for (int m = 0; m < NL; ++m)
#pragma unroll
                            for (int c = 0; c < 6; ++c) g[(m * 6 + c) * LDQ] = G[m][c];
                    } else {
                        inner_analytic_store_fp64<N>(r0x, r0y, r0z, ts0, ts1, ts2, eps2, g, LDQ);
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < NG; ++m) g[m * LDQ] = 0.0;
                }
            }
        } else {
            // Mixed precision in two passes: FP32 for the far field, then the
            // points near the source fiber (c < near_c) in FP64, compacted onto
            // consecutive threads so that no warp carries both paths.
            if (tid == 0) s_nlist = 0;
            __syncthreads();
            if (worker) {
                double *g = s_G + (size_t)ti * NG * LDQ + qpos;
                bool need64 = false;
                if (i < a.t1 && i != j) {
                    const double r0x = xbx - xs0, r0y = xby - xs1, r0z = xbz - xs2;
                    const double cq = r0x * r0x + r0y * r0y + r0z * r0z;
                    need64 = cq < a.near_c;
                    if (!need64) {
                        if (NUMERIC) {
                            float G[NL][6];
                            const float xs[3] = {(float)xs0, (float)xs1, (float)xs2};
                            const float ts[3] = {(float)ts0, (float)ts1, (float)ts2};
                            inner_numeric_fp32<N>((float)xbx, (float)xby, (float)xbz, xs, ts, s_pvf, s_wPf, LQ,
                                                  (float)eps2, G);
#pragma unroll
                            for (int m = 0; m < NL; ++m)
#pragma unroll
                                for (int c = 0; c < 6; ++c) g[(m * 6 + c) * LDQ] = (double)G[m][c];
                        } else {
                            inner_analytic_store_fp32<N>((float)r0x, (float)r0y, (float)r0z, (float)ts0, (float)ts1,
                                                         (float)ts2, (float)eps2, g, LDQ);
                        }
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < NG; ++m) g[m * LDQ] = 0.0;
                }
                // warp-aggregated append of the FP64 items
                const unsigned mask = __ballot_sync(__activemask(), need64);
                if (mask) {
                    int base = 0;
                    const int leader = __ffs(mask) - 1;
                    if (lane == leader) base = atomicAdd(&s_nlist, __popc(mask));
                    base = __shfl_sync(__activemask(), base, leader);
                    if (need64) s_list[base + __popc(mask & ((1u << lane) - 1u))] = (short)tid;
                }
            }
            __syncthreads();
            const int nl = s_nlist;
            for (int u = tid; u < nl; u += nthreads) {
                const int item = s_list[u];
                const int ti2 = item / LQ, q2 = item - ti2 * LQ;
                const double sq2 = s_pv[q2];
                const double bx = fadd(s_xt[ti2 * 3 + 0], fmul(sq2, s_tt[ti2 * 3 + 0]));
                const double by = fadd(s_xt[ti2 * 3 + 1], fmul(sq2, s_tt[ti2 * 3 + 1]));
                const double bz = fadd(s_xt[ti2 * 3 + 2], fmul(sq2, s_tt[ti2 * 3 + 2]));
                double *g2 = s_G + (size_t)ti2 * NG * LDQ + (q2 & 3) * KS + (q2 >> 2);
                if (NUMERIC) {
                    double G[NL][6];
                    const double xs[3] = {xs0, xs1, xs2}, ts[3] = {ts0, ts1, ts2};
                    inner_numeric_fp64<N>(bx, by, bz, xs, ts, s_pv, s_wP, LQ, eps2, G);
#pragma unroll
                    for (int m = 0; m < NL; ++m)
#pragma unroll
                        for (int c = 0; c < 6; ++c) g2[(m * 6 + c) * LDQ] = G[m][c];
                } else {
                    inner_analytic_store_fp64<N>(fsub(bx, xs0), fsub(by, xs1), fsub(bz, xs2), ts0, ts1, ts2, eps2, g2,
                                                 LDQ);
                }
            }
        }
        // q padding up to the next multiple of 4 is zero for the tensor-core k-steps
        for (int t = tid; t < NCOL * (LQP - LQ); t += nthreads) {
            const int col = t / (LQP - LQ), qq = LQ + t % (LQP - LQ);
            s_G[(size_t)col * LDQ + (qq & 3) * KS + (qq >> 2)] = 0.0;
        }
        __syncthreads();

        // ---------------- P2: theta[k][col] = sum_q wP[k][q] G[col][q] (FP64 tensor cores)
        for (int t = warp; t < NTILE; t += nwarps) {
            const int col = t * 8 + (lane >> 2);
            const double *bsrc = s_G + (size_t)col * LDQ + (lane & 3) * KS;
            double bfrag[KSMAX];
#pragma unroll
            for (int s = 0; s < KSMAX; ++s) bfrag[s] = s < KS ? bsrc[s] : 0.0;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                double d0 = 0.0, d1 = 0.0;
#pragma unroll
                for (int s = 0; s < KSMAX; ++s)
                    if (s < KS) dmma_8x8x4(d0, d1, afrag[mt][s], bfrag[s], d0, d1);
                // lane holds theta[krow][t*8 + 2*(lane&3) + {0,1}]
                const int krow = mt * 8 + (lane >> 2);
                if (krow < NL) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int cc = t * 8 + 2 * (lane & 3) + h;
                        const int gt = cc / NG, lc = cc - gt * NG;
                        s_th[((size_t)gt * NL + krow) * NG + lc] = h ? d1 : d0;
                    }
                }
            }
        }
        __syncthreads();

        // ---------------- P3a: block entries per (target, k, l) group, staged
        // theta for (target gt, k, l): s_th[(gt*NL + k)*NG + l*6 + c]
        for (int g = tid; g < TI * N * N; g += nthreads) {
            const int l = g / (TI * N) + 1;
            const int r = g - (l - 1) * (TI * N);
            const int gt = r / N, k = r - gt * N + 1;
            const double *tt = s_tt + gt * 3;
            double v[3][3];
            if (i0 + gt == j) {
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb) v[aa][bb] = (k == l && aa == bb) ? 1.0 : 0.0;
            } else {
                const double *th = s_th + ((size_t)gt * NL + k) * NG + l * 6;
                double Q[3];
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
                    Q[bb] = th[sym_index(bb, 0)] * tt[0] + th[sym_index(bb, 1)] * tt[1] + th[sym_index(bb, 2)] * tt[2];
                if (k == 1) {
                    const double D1 = tab.D1;
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 3; ++bb) v[aa][bb] = D1 * tt[aa] * Q[bb];
                } else {
                    const double gk = tab.gamma[k], ek = tab.Ek[k];
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 3; ++bb) v[aa][bb] = gk * (th[sym_index(aa, bb)] - ek * tt[aa] * Q[bb]);
                }
            }
            const int rl = gt * 3 * N + 3 * (k - 1);
            const int cl = 3 * (l - 1);
#pragma unroll
            for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                for (int aa = 0; aa < 3; ++aa) s_blk[(cl + bb) * RT + rl + aa] = v[aa][bb];
        }
        // right-hand side and the l = 0 velocity terms: the external force is the
        // same on every fiber, so theta^k_0 is summed over the sources here and
        // contracted with 0.5*ExtForce once at the end
        for (int t = tid; t < TI * NL * 6; t += nthreads) {
            const int gt = t / (NL * 6);
            const int r = t - gt * (NL * 6);
            if (i0 + gt == j) continue;
            s_acc[t] += s_th[((size_t)gt * NL + r / 6) * NG + r % 6];
        }
        // velocity panels: rows i*3 + aa of PV (P_0) and PW (P_1, projected),
        // per (target, l) group into the staging area after the block
        if (a.PV64 || a.PV32) {
            double *s_pan = s_blk + CT * RT;   // [2][CT][TI*3]
            for (int g = tid; g < TI * N; g += nthreads) {
                const int l = g / TI + 1, gt = g - (l - 1) * TI;
                double pv[3][3], pw[3][3];
                if (i0 + gt != j) {
                    const double *th0 = s_th + ((size_t)gt * NL + 0) * NG + l * 6;
                    const double *th1 = s_th + ((size_t)gt * NL + 1) * NG + l * 6;
                    const double *tt = s_tt + gt * 3;
                    const double sv = 0.5 / tab.d, sw = 1.5 / tab.d;
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb) {
                        const double tdot = tt[0] * th1[sym_index(0, bb)] + tt[1] * th1[sym_index(1, bb)] +
                                            tt[2] * th1[sym_index(2, bb)];
#pragma unroll
                        for (int aa = 0; aa < 3; ++aa) {
                            pv[aa][bb] = sv * th0[sym_index(aa, bb)];
                            pw[aa][bb] = sw * (th1[sym_index(aa, bb)] - tdot * tt[aa]);
                        }
                    }
                } else {
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 3; ++bb) pv[aa][bb] = pw[aa][bb] = 0.0;
                }
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa) {
                        const int cl = 3 * (l - 1) + bb, rl = gt * 3 + aa;
                        s_pan[cl * (TI * 3) + rl] = pv[aa][bb];
                        s_pan[CT * TI * 3 + cl * (TI * 3) + rl] = pw[aa][bb];
                    }
            }
        }
        __syncthreads();

        // ---------------- P3b: coalesced column-major stores of the staged block,
        // two consecutive rows per thread
        {
            const int64_t col0 = (int64_t)j * 3 * N;
            for (int u = tid; u < CT * RT / 2; u += nthreads) {
                const int e = 2 * u;
                const int cl = e / RT;
                const int rl = e - cl * RT;
                if (rl >= rows_valid) continue;
                const double v0 = s_blk[e], v1 = s_blk[e + 1];
                const int64_t idx = (col0 + cl) * a.lda + row0 + rl;
                if (a.A16lo) {  // split FP32 storage: the two 16-bit planes
                    split_store((float)v0, a.A16 + idx, a.A16lo + idx);
                    if (rl + 1 < rows_valid) split_store((float)v1, a.A16 + idx + 1, a.A16lo + idx + 1);
                } else if (rl + 1 < rows_valid) {
                    if (a.A64) *reinterpret_cast<double2 *>(a.A64 + idx) = make_double2(v0, v1);
                    if (a.A32) *reinterpret_cast<float2 *>(a.A32 + idx) = make_float2((float)v0, (float)v1);
                    if (a.A16)
                        *reinterpret_cast<__nv_bfloat162 *>(a.A16 + idx) = __floats2bfloat162_rn((float)v0, (float)v1);
                } else {
                    if (a.A64) a.A64[idx] = v0;
                    if (a.A32) a.A32[idx] = (float)v0;
                    if (a.A16) a.A16[idx] = __float2bfloat16_rn((float)v0);
                }
            }
            if (a.PV64 || a.PV32) {
                constexpr int PRT = TI * 3;
                const double *s_pan = s_blk + CT * RT;
                const int prows = min(PRT, 3 * (a.M - i0));
                const int64_t prow0 = (int64_t)i0 * 3;
                for (int e = tid; e < 2 * CT * PRT; e += nthreads) {
                    const int which = e / (CT * PRT);
                    const int r = e - which * CT * PRT;
                    const int cl = r / PRT, rl = r - cl * PRT;
                    if (rl >= prows) continue;
                    const int64_t idx = (col0 + cl) * a.ldp + prow0 + rl;
                    const double v = s_pan[e];
                    if (a.PV64) (which ? a.PW64 : a.PV64)[idx] = v;
                    if (a.PV32) (which ? a.PW32 : a.PV32)[idx] = (float)v;
                }
            }
        }
        __syncthreads();  // the staged block and the next P1 share shared memory
    }
    // per-chunk partial sums: rhs [chunk][n] and velocity l=0 terms [chunk][6M]
    // from sum_j theta^k_0 (matrix_assembly.f90:874-899)
    for (int t = tid; t < TI * (3 * N + 6); t += nthreads) {
        const int gt = t / (3 * N + 6);
        const int r = t - gt * (3 * N + 6);
        const int ii = i0 + gt;
        if (ii >= a.t1) continue;
        if (r >= 3 * N && !a.vpart) continue;
        const double *tt = s_tt + gt * 3;
        const double *f = tab.half_force;
        const int k = r < 3 * N ? r / 3 + 1 : (r - 3 * N) / 3;
        const int aa = r % 3;
        const double *th = s_acc + (gt * NL + k) * 6;
        double contr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            contr[c] = th[sym_index(c, 0)] * f[0] + th[sym_index(c, 1)] * f[1] + th[sym_index(c, 2)] * f[2];
        const double tdc = tt[0] * contr[0] + tt[1] * contr[1] + tt[2] * contr[2];
        double v;
        if (r < 3 * N) {
            if (k == 1) v = -tab.D1 * tdc * tt[aa];
            else v = -tab.gamma[k] * (contr[aa] - tab.Ek[k] * tdc * tt[aa]);
            a.bpart[(int64_t)blockIdx.y * a.n + (int64_t)(ii - a.t0) * 3 * N + r] = v;
        } else {
            if (k == 0) v = 0.5 / tab.d * contr[aa];
            else v = 1.5 / tab.d * (contr[aa] - tdc * tt[aa]);
            a.vpart[(int64_t)blockIdx.y * 6 * a.M + (int64_t)ii * 6 + (r - 3 * N)] = v;
        }
    }
}

// b[r] = sum_c bpart[c][r] in chunk order
__global__ void reduce_chunks_kernel(const double *part, int nchunks, int64_t stride, int64_t len, double *out) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= len) return;
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += part[c * stride + r];
    out[r] = s;
}

template <int N, bool NUMERIC, int PMODE>
static cudaError_t launch_assemble_n(const AsmArgs &a, int nchunks, cudaStream_t st) {
    constexpr int TI = kTI;
    constexpr int NL = N + 1, NG = NL * 6;
    const int LQ = a.LQ, LDQ = round_up_int(LQ, 4) + 2;
    const size_t big = std::max((size_t)TI * NG * LDQ, (size_t)(3 * N) * (TI * 3 * N) + 2 * (3 * N) * (TI * 3));
    constexpr int WP_OWN = NUMERIC || PMODE != kPModeFP64 ? 16 * kMaxLQ : 0;
    size_t smem = sizeof(double) * (kMaxLQ + WP_OWN + TI * 3 * 2 + TI * NL * 6 + TI * NL * NG +
                                    std::max(big, (size_t)(16 * kMaxLQ)));
    smem += sizeof(float) * (kMaxLQ + NL * kMaxLQ);
    const int threads = round_up_int(TI * LQ, 32);
    auto kern = threads <= 96 ? assemble_kernel<N, NUMERIC, PMODE, 96, kMinBlocks96>
                              : assemble_kernel<N, NUMERIC, PMODE, TI * kMaxLQ, 2>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid((a.t1 - a.t0 + TI - 1) / TI, nchunks);
    kern<<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool NUMERIC, int PMODE>
static cudaError_t launch_assemble_mode(const AsmArgs &a, int nchunks, cudaStream_t st) {
    switch (a.N) {
        case 1: return launch_assemble_n<1, NUMERIC, PMODE>(a, nchunks, st);
        case 2: return launch_assemble_n<2, NUMERIC, PMODE>(a, nchunks, st);
        case 3: return launch_assemble_n<3, NUMERIC, PMODE>(a, nchunks, st);
        case 4: return launch_assemble_n<4, NUMERIC, PMODE>(a, nchunks, st);
        case 5: return launch_assemble_n<5, NUMERIC, PMODE>(a, nchunks, st);
        case 6: return launch_assemble_n<6, NUMERIC, PMODE>(a, nchunks, st);
        case 7: return launch_assemble_n<7, NUMERIC, PMODE>(a, nchunks, st);
        case 8: return launch_assemble_n<8, NUMERIC, PMODE>(a, nchunks, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_assemble(const AsmArgs &a, bool numeric, int pmode, int nchunks, cudaStream_t st) {
    if (pmode == kPModeFP64)
        return numeric ? launch_assemble_mode<true, kPModeFP64>(a, nchunks, st)
                       : launch_assemble_mode<false, kPModeFP64>(a, nchunks, st);
    return numeric ? launch_assemble_mode<true, kPModeMixed>(a, nchunks, st)
                   : launch_assemble_mode<false, kPModeMixed>(a, nchunks, st);
}

cudaError_t launch_reduce_chunks(const double *part, int nchunks, int64_t stride, int64_t len, double *out,
                                 cudaStream_t st) {
    const int bs = 256;
    reduce_chunks_kernel<<<(unsigned)((len + bs - 1) / bs), bs, 0, st>>>(part, nchunks, stride, len, out);
    return cudaGetLastError();
}

}  // namespace rf
