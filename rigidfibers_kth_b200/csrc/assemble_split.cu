// assemble_split.cu - mixed-precision assembly split by pair distance.
//
// Reference: fortran/matrix_assembly.f90:407-629 (matrix, analytic) and
// 796-905 (right-hand side); Int_analytical.f90:72-288 (inner integral).
//
// The mixed path stores A in FP32: as FP32 words (FP32 paths) or as the two
// 16-bit planes of split storage (BF16 path; the high plane is the BF16
// matrix of the inner solves).  A fiber pair (i, j) is "near"
// when one of target i's quadrature points lies within sqrt(near_c) of source
// j's centre (default c < 6: closer, the FP32 backward recursion loses digits;
// the reference itself switches to forward recursion below 10).  Near pairs
// are integrated in FP64, far pairs in FP32, every moment of a far pair by the
// backward recursion run down to n = 0 (moments_backward_fp32: none of the
// reference's n = 0, 1 closed forms, which cancel for distant pairs and close
// to the source axis).  Three kernels:
//   classify_kernel   one warp per target: near-pair bitmap and per-target
//                     lists in ascending source order;
//   far_pairs_kernel  FP32, lane = target fiber, warp-uniform source, eight
//                     warps per CTA stepping through the sources together:
//                     every lane integrates its own pair over the target's
//                     Gauss points with the projection accumulated in
//                     registers, then stages the 3N x 3N block (split into
//                     its two 16-bit planes where stored so) and the
//                     velocity-panel rows in shared memory, and one lane
//                     hands whole column segments to the copy engine;
//   near_pairs_kernel FP64, one warp per near pair: lane = Gauss point, the
//                     projection on the FP64 tensor cores (mma.sync m8n8k4).
// A finish kernel sums the per-chunk right-hand-side partials in a fixed order.
//
// Projection without forming the tensors.  The reference forms, per target
// point q and source weight m, G_m(q) = cI I + cRR R0R0 + cPR (pR0 + R0p)
// + cPP pp and projects theta^k_m = sum_q w_q P_k(s_q) G_m(q).  Here
//   cI  = sc_m sum_p a_mp u_p,        u_p = I_p + 2 eps^2 J_p
//   cRR = sc_m sum_p a_mp v_p,        v_p = J_p - 6 eps^2 S_p
//   cPR = -sc_m sum_p a_mp v_{p+1},   cPP = sc_m sum_p a_mp v_{p+2}
// (a_mp, sc_m the Legendre coefficients of Int_analytical.f90:213-288), and
// R0 = D + s_q t with D = x_i - x_j, t = t_i, so every entry of theta is a
// combination of the scalar projections <u_p>_k, <v_p>_k, <s v_p>_k and
// <s^2 v_p>_k times the seven pair tensors I, DD, Dt+tD, tt, pD+Dp, pt+tp,
// pp.  Bonnet's recursion s P_k = ((k+1) P_{k+1} + k P_{k-1}) / (2k+1) holds
// at every point, so <s f>_k = alpha_k <f>_{k+1} + beta_k <f>_{k-1}: the
// per-point work is 2N+4 scalars projected onto P_0..P_{N+2}, the same sums in
// another order.
#include <algorithm>

#include "rf_kernels.h"

namespace rf {

namespace {

template <int N>
struct SplitDims {
    static constexpr int NL = N + 1;          // u_p and Legendre indices 0..N
    static constexpr int NV = N + 3;          // v_p, p = 0..N+2
    static constexpr int KW = N + 3;          // projection rows k = 0..N+2
    static constexpr int KWP = KW + (KW & 1); // KW rounded up to even: the weight table's row stride
    static constexpr int NC = NL + NV;        // scalars per Gauss point
    static constexpr int RB = 3 * N;          // rows (and columns) of a pair block
    static constexpr int NRHS = 3 * NL;       // theta^k_0 f, k = 0..N
};

// number of projection rows kept for v_p
__host__ __device__ constexpr int vrows(int N, int p) { return p <= N ? N + 3 : (p == N + 1 ? N + 2 : N + 1); }

__host__ __device__ constexpr double bonnet_a(int k) { return (k + 1.0) / (2.0 * k + 1.0); }
__host__ __device__ constexpr double bonnet_b(int k) { return k / (2.0 * k + 1.0); }

// Scalar coefficient sets of source weight m from the projections
// U(p, k) = <u_p>_k and V(p, k) = <v_p>_k.
template <typename T, int N>
struct LegSets {
    T AI[N + 1], R0[N + 3], R1[N + 2], R2[N + 1], C0[N + 2], C1[N + 1], E[N + 1];
};

template <typename T, int N, int m, typename UF, typename VF>
__device__ __forceinline__ void leg_sets(const UF &U, const VF &V, LegSets<T, N> &o) {
    const T sc = (T)leg_scale(m);
#pragma unroll
    for (int k = 0; k <= N; ++k) {
        T s = 0;
#pragma unroll
        for (int p = m; p >= 0; --p)
            if (leg_coef(m, p) != 0) s += (T)leg_coef(m, p) * U(p, k);
        o.AI[k] = sc * s;
    }
#pragma unroll
    for (int k = 0; k <= N + 2; ++k) {
        T s = 0;
#pragma unroll
        for (int p = m; p >= 0; --p)
            if (leg_coef(m, p) != 0) s += (T)leg_coef(m, p) * V(p, k);
        o.R0[k] = sc * s;
    }
#pragma unroll
    for (int k = 0; k <= N + 1; ++k) {
        T s = 0;
#pragma unroll
        for (int p = m; p >= 0; --p)
            if (leg_coef(m, p) != 0) s += (T)leg_coef(m, p) * V(p + 1, k);
        o.C0[k] = -sc * s;
    }
#pragma unroll
    for (int k = 0; k <= N; ++k) {
        T s = 0;
#pragma unroll
        for (int p = m; p >= 0; --p)
            if (leg_coef(m, p) != 0) s += (T)leg_coef(m, p) * V(p + 2, k);
        o.E[k] = sc * s;
    }
#pragma unroll
    for (int k = 0; k <= N + 1; ++k)
        o.R1[k] = (T)bonnet_a(k) * o.R0[k + 1] + (k > 0 ? (T)bonnet_b(k) * o.R0[k > 0 ? k - 1 : 0] : (T)0);
#pragma unroll
    for (int k = 0; k <= N; ++k) {
        o.R2[k] = (T)bonnet_a(k) * o.R1[k + 1] + (k > 0 ? (T)bonnet_b(k) * o.R1[k > 0 ? k - 1 : 0] : (T)0);
        o.C1[k] = (T)bonnet_a(k) * o.C0[k + 1] + (k > 0 ? (T)bonnet_b(k) * o.C0[k > 0 ? k - 1 : 0] : (T)0);
    }
}

// The seven pair tensors, packed 11,22,33,12,13,23 (identity implicit).
template <typename T>
struct PairTensors {
    T DD[6], DT[6], TT[6], PD[6], PT[6], PP[6];
    __device__ __forceinline__ void set(const T *D, const T *t, const T *p) {
        const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const int x = ia[c], y = ib[c];
            DD[c] = D[x] * D[y];
            DT[c] = D[x] * t[y] + t[x] * D[y];
            TT[c] = t[x] * t[y];
            PD[c] = p[x] * D[y] + D[x] * p[y];
            PT[c] = p[x] * t[y] + t[x] * p[y];
            PP[c] = p[x] * p[y];
        }
    }
    // theta for projection row k of the sets
    template <int N>
    __device__ __forceinline__ void theta(const LegSets<T, N> &s, int k, T *th) const {
#pragma unroll
        for (int c = 0; c < 6; ++c)
            th[c] = (c < 3 ? s.AI[k] : (T)0) + s.R0[k] * DD[c] + s.R1[k] * DT[c] + s.R2[k] * TT[c] +
                    s.C0[k] * PD[c] + s.C1[k] * PT[c] + s.E[k] * PP[c];
    }
};

// FP64 moments for the near pairs of the mixed path: the reference formulas
// (Int_analytical.f90:96-207) with ordinary (contracted) arithmetic and the
// loop-constant divisions folded into reciprocals.
template <int N>
__device__ __forceinline__ void moments_near(double b, double c, double *I, double *J, double *S) {
    constexpr int K = N + 3;
    const double xe = 1.0 + b + c, xb = 1.0 - b + c;
    const double iue = rsqrt(xe), iub = rsqrt(xb);
    const double ue = xe * iue, ub = xb * iub;
    const double te = 1.0 + 0.5 * b;
    const double tb = -1.0 + 0.5 * b;
    const double d = c - 0.25 * b * b;
    I[0] = log(fabs((2.0 + b + 2.0 * ue) / (-2.0 + b + 2.0 * ub)));
    I[1] = ue - ub - 0.5 * b * I[0];
    if (d < 1e-14) {
        const double e1 = 1.0 + 0.5 * b, e2 = -1.0 + 0.5 * b;
        J[0] = -0.5 / (e1 * e1) + 0.5 / (e2 * e2);
        J[1] = -iue + iub - 0.5 * b * J[0];
        const double p = 2.0 + b, m = -2.0 + b;
        const double p2 = p * p, m2 = m * m;
        S[0] = -4.0 / (p2 * p2) + 4.0 / (m2 * m2);
        S[1] = -8.0 / (3.0 * p2 * p) + 8.0 / (3.0 * m2 * m) - 0.5 * b * S[0];
    } else {
        const double id = 1.0 / d;
        J[0] = (te * iue - tb * iub) * id;
        J[1] = -iue + iub - 0.5 * b * J[0];
        const double iue3 = iue * iue * iue, iub3 = iub * iub * iub;
        const double id6 = id * (1.0 / 6.0);
        S[0] = ((2.0 + b) * iue3 - (-2.0 + b) * iub3) * id6 + (2.0 / 3.0) * id * J[0];
        S[1] = (-(b + 2.0 * c) * iue3 + (-b + 2.0 * c) * iub3) * id6 - (1.0 / 3.0) * b * id * J[0];
    }
    if (c < 10.0) {
#pragma unroll
        for (int n = 2; n < K; ++n) {
            const double nn = n + 1.0;
            const double r = 1.0 / (1.0 - nn);
            const double sbp = (n % 2 == 1) ? 1.0 : -1.0;
            I[n] = (sbp * r) * ub - r * ue - ((0.5 - (nn - 1.0)) * r) * b * I[n - 1] + ((nn - 2.0) * r) * c * I[n - 2];
            J[n] = I[n - 2] - b * J[n - 1] - c * J[n - 2];
            S[n] = J[n - 2] - b * S[n - 1] - c * S[n - 2];
        }
    } else {
        const double ic = 1.0 / c;
        double i1 = 0.0, i2 = 0.0, j1 = 0.0, j2 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int n = 27; n >= 2; --n) {
            const double nn = n;
            const double a0 = (nn + 2.0) / (nn + 1.0);
            const double r2 = 1.0 / (nn + 2.0);
            const double cb = (1.0 - 2.0 * (nn + 2.0)) / (2.0 * (nn + 2.0));
            const double sbp = ((n + 1) % 2 == 0) ? 1.0 : -1.0;
            const double in = a0 * ic * (ue * r2 - sbp * ub * r2 + cb * b * i1 - i2);
            const double jn = ic * (in - b * j1 - j2);
            const double sn = ic * (jn - b * s1 - s2);
            if (n < K) { I[n] = in; J[n] = jn; S[n] = sn; }
            i2 = i1; i1 = in; j2 = j1; j1 = jn; s2 = s1; s1 = sn;
        }
    }
}

// Near-pair buffer: per pair and source weight m = 1..N a 64-float record
// (16-byte aligned): the block columns 3(m-1)..3(m-1)+2 [col][row] (9N
// floats), then the velocity panel entries [w][col][a] (18 floats).
constexpr int kNearWeight = 64;
constexpr int kNearBlock = 5 * kNearWeight;
static_assert(9 * 5 + 18 <= kNearWeight, "near record");

// ---------------------------------------------------------------- classify
constexpr int kClassifyWarps = 4;

// One warp per target: the near-pair bitmap, the number of near sources before
// each bitmap word, the near sources in ascending order and their count, and
// the target's first slot in the near-pair buffer (claimed with an atomic add;
// slots only place the blocks, they do not change any value).
__global__ void __launch_bounds__(kClassifyWarps * 32) classify_kernel(SplitArgs a) {
    __shared__ double s_pv[kMaxLQ];
    for (int t = threadIdx.x; t < kMaxLQ; t += blockDim.x) s_pv[t] = t < a.LQ ? a.tab->pv[t] : 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = blockIdx.x * kClassifyWarps + warp;
    if (i >= a.M) return;  // whole warp
    const double xi0 = a.pos[3 * i], xi1 = a.pos[3 * i + 1], xi2 = a.pos[3 * i + 2];
    const double ti0 = a.ori[3 * i], ti1 = a.ori[3 * i + 1], ti2 = a.ori[3 * i + 2];
    int count = 0;
    int *list = a.near_list + (int64_t)i * a.M;
    for (int jw = 0; jw < a.words; ++jw) {
        const int j = jw * 32 + lane;
        bool near = false;
        if (j < a.M && j != i) {
            const double D0 = xi0 - a.pos[3 * j], D1 = xi1 - a.pos[3 * j + 1], D2 = xi2 - a.pos[3 * j + 2];
            for (int q = 0; q < a.LQ && !near; ++q) {
                const double s = s_pv[q];
                const double r0 = D0 + s * ti0, r1 = D1 + s * ti1, r2 = D2 + s * ti2;
                const double c = r0 * r0 + r1 * r1 + r2 * r2;
                near = c < a.near_c;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, near);
        if (lane == 0) {
            a.near_bits[(int64_t)i * a.words + jw] = mask;
            a.near_pref[(int64_t)i * a.words + jw] = count;
        }
        if (near) list[count + __popc(mask & ((1u << lane) - 1u))] = j;
        count += __popc(mask);
    }
    if (lane == 0) {
        a.near_cnt[i] = count;
        a.near_off[i] = atomicAdd(a.near_total, count);
    }
}

// ---------------------------------------------------------------- far pairs (FP32)
// One warp per CTA; lane = target fiber, the warp walks a chunk of sources.
// For source weight m the block entries follow from
//   theta = AI I + D X^T + t Y^T + p Z^T,   X = R0 D + R1 t + C0 p,
//   Y = R1 D + R2 t + C1 p,  Z = C0 D + C1 t + E p,
//   Q = theta t = AI t + (D.t) X + (t.t) Y + (p.t) Z,
// the pair tensors of the header expanded.  The m loop runs at run time with
// the Legendre coefficients sc_m a_mp in constant memory, which keeps the
// kernel small enough for the instruction cache.

#define RF_LEG(m, p) ((float)(leg_scale(m) * leg_coef(m, p)))
#define RF_LEG_ROW(m) RF_LEG(m, 0), RF_LEG(m, 1), RF_LEG(m, 2), RF_LEG(m, 3), RF_LEG(m, 4), RF_LEG(m, 5), RF_LEG(m, 6), RF_LEG(m, 7)
__constant__ float c_leg32[8][8] = {{RF_LEG_ROW(0)}, {RF_LEG_ROW(1)}, {RF_LEG_ROW(2)}, {RF_LEG_ROW(3)},
                                    {RF_LEG_ROW(4)}, {RF_LEG_ROW(5)}, {RF_LEG_ROW(6)}, {RF_LEG_ROW(7)}};
#undef RF_LEG_ROW
#undef RF_LEG

#ifndef RF_FAR_MINB
#define RF_FAR_MINB 8
#endif
// Warps per far-pair CTA.  Each warp works on its own 32 targets; the warps
// of a CTA step through the sources together (a barrier before each source's
// post-processing), so the warps sharing a scheduler mostly run the same code
// at the same time and share the instruction cache: the Gauss-point loop and
// the post-processing together exceed it, and warps of separate one-warp CTAs
// drift into different phases.  Measured at M = 4000: assembly 20.35 ms with
// one-warp CTAs, 19.5 ms with barriers before both phases, 19.35 ms with the
// one before the post-processing alone.
#ifndef RF_FAR_WARPS
#define RF_FAR_WARPS 8
#endif

template <int N, bool PANELS>
struct FarSmem {
    static constexpr int GR = 32 * 3 * N;                   // staged rows of one column
    static constexpr int PAN = 2 * 3 * 96;                  // staged panel columns
    static constexpr int STG16 = 3 * GR / 2;                // BF16 copy (split storage: low plane) of the staged columns
    static constexpr size_t kBytes = sizeof(float) * (32 * kNearWeight + 16 + 64 + kMaxLQ +
                                                      kMaxLQ * SplitDims<N>::KWP + 3 * GR + (PANELS ? PAN : 0) +
                                                      STG16);
    static_assert(kBytes % 16 == 0, "each warp's region starts on a 16-byte boundary");
    static size_t bytes() { return kBytes; }
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Bulk asynchronous shared -> global copies (the copy engine streams staged
// columns out while the warp goes on computing).  Addresses and sizes are
// multiples of 16 bytes.
__device__ __forceinline__ void bulk_s2g(void *gdst, const void *ssrc, unsigned bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gdst), "r"(s), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// lanes of a far-pair warp that hand staged column segments to the copy engine
constexpr int kCopyLanes = 12;
// the staged data has been read out: the staging buffers may be rewritten
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the bulk copies
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int N, bool PANELS>
__device__ __forceinline__ void far_store_m(const SplitArgs &a, int m, int j, int i0, int nvalid, const float *stg,
                                            const float *pan, __nv_bfloat16 *stg16, int lane) {
    constexpr int RB = 3 * N, GR = 32 * RB;
    const int64_t row0 = (int64_t)i0 * RB;
    const int nrows = nvalid * RB;
    const int64_t col0 = (int64_t)j * RB + 3 * (m - 1);
    if (nrows == GR) {
        // whole column segments: the 16-bit planes (or the BF16 copy) are
        // staged too, then one lane hands every segment to the copy engine
        // (the matrix: 3 x 32 targets x 3N rows; panels: 2 x 3 x 96 rows),
        // and the warp moves on
        if (a.A16lo) {
            // split FP32 storage: the low plane goes to the BF16 staging, the
            // high plane over the first half of the FP32 staging it is read
            // from (a step's writes reach only entries read by earlier steps
            // or, behind the barrier, by this one).  (u + 0x8000) >> 16 is
            // split_hi(u); the byte permutes pack two 16-bit halves.
            const uint4 *s4 = reinterpret_cast<const uint4 *>(stg);
            uint2 *dh = reinterpret_cast<uint2 *>(const_cast<float *>(stg));
            uint2 *dl = reinterpret_cast<uint2 *>(stg16);
            for (int e0 = 0; e0 < 3 * GR / 4; e0 += 32) {
                const int e = e0 + lane;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (e < 3 * GR / 4) v = s4[e];
                __syncwarp();
                if (e < 3 * GR / 4) {
                    dh[e] = make_uint2(__byte_perm(v.x + 0x8000u, v.y + 0x8000u, 0x7632),
                                       __byte_perm(v.z + 0x8000u, v.w + 0x8000u, 0x7632));
                    dl[e] = make_uint2(__byte_perm(v.x, v.y, 0x5410), __byte_perm(v.z, v.w, 0x5410));
                }
            }
        } else if (a.A16) {
            const float4 *s4 = reinterpret_cast<const float4 *>(stg);
            uint2 *d2 = reinterpret_cast<uint2 *>(stg16);
            for (int e = lane; e < 3 * GR / 4; e += 32) {
                const float4 v = s4[e];
                __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
                uint2 u;
                u.x = *reinterpret_cast<unsigned *>(&lo);
                u.y = *reinterpret_cast<unsigned *>(&hi);
                d2[e] = u;
            }
        }
        fence_async_shared();
        __syncwarp();
        // one segment per lane: lane l copies column bb = l % 3 of kind l / 3
        // (0: the FP32 words or the high plane, 1: the low plane or the BF16
        // copy, 2 and 3: the two panels); each lane commits its own group
        if (lane < kCopyLanes) {
            const int bb = lane % 3, kind = lane / 3;
            const int64_t col = col0 + bb;
            if (kind == 0) {
                if (a.A32)
                    bulk_s2g(a.A32 + col * a.lda + row0, stg + bb * GR, GR * sizeof(float));
                else if (a.A16lo)
                    bulk_s2g(a.A16 + col * a.lda + row0, reinterpret_cast<const unsigned short *>(stg) + bb * GR,
                             GR * sizeof(unsigned short));
            } else if (kind == 1) {
                if (a.A16lo)
                    bulk_s2g(a.A16lo + col * a.lda + row0, reinterpret_cast<const unsigned short *>(stg16) + bb * GR,
                             GR * sizeof(unsigned short));
                else if (a.A16)
                    bulk_s2g(a.A16 + col * a.lda + row0, stg16 + bb * GR, GR * sizeof(__nv_bfloat16));
            } else if (PANELS) {
                const int w = kind - 2;
                bulk_s2g((w ? a.PW32 : a.PV32) + col * a.ldp + (int64_t)i0 * 3, pan + (w * 3 + bb) * 96,
                         96 * sizeof(float));
            }
            bulk_commit();
        }
        return;
    }
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
        const int64_t col = col0 + bb;
        const float *src = stg + bb * GR;
        for (int e = lane; e < nrows; e += 32) {
            const int64_t idx = col * a.lda + row0 + e;
            if (a.A16lo) {
                split_store(src[e], a.A16 + idx, a.A16lo + idx);
            } else {
                if (a.A32) a.A32[idx] = src[e];
                if (a.A16) a.A16[idx] = __float2bfloat16_rn(src[e]);
            }
        }
        if (PANELS) {
            const int prow = 3 * nvalid;
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                float *dst = (w ? a.PW32 : a.PV32) + col * a.ldp + (int64_t)i0 * 3;
                const float *ps = pan + (w * 3 + bb) * 96;
                for (int e = lane; e < prow; e += 32) dst[e] = ps[e];
            }
        }
    }
}

// Coefficient sets of weight m (parity PAR) for rows k = 0..N in registers:
// S[0..6][k] = AI, R0, R1, R2, C0, C1, E.
template <int N, int PAR>
__device__ __forceinline__ void far_sets_reg(int m, const float (&U)[N + 1][N + 1], const float (&V)[N + 3][N + 3],
                                             float (&S)[7][N + 1]) {
    constexpr int NP = (N - PAR) / 2 + 1;
    float cf[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) cf[i] = c_leg32[m][PAR + 2 * i];
    float R0[N + 3], C0[N + 2], R1[N + 2];
#pragma unroll
    for (int k = 0; k < N + 3; ++k) {
        float s1 = 0.f;
#pragma unroll
        for (int i = 0; i < NP; ++i) s1 = fmaf(cf[i], V[PAR + 2 * i][k], s1);
        R0[k] = s1;
    }
#pragma unroll
    for (int k = 0; k < N + 2; ++k) {
        float s1 = 0.f;
#pragma unroll
        for (int i = 0; i < NP; ++i)
            if (k < vrows(N, PAR + 2 * i + 1)) s1 = fmaf(cf[i], V[PAR + 2 * i + 1][k], s1);
        C0[k] = -s1;
    }
#pragma unroll
    for (int k = 0; k < N + 2; ++k)
        R1[k] = (float)bonnet_a(k) * R0[k + 1] + (k > 0 ? (float)bonnet_b(k) * R0[k > 0 ? k - 1 : 0] : 0.f);
#pragma unroll
    for (int k = 0; k <= N; ++k) {
        float ai = 0.f, ee = 0.f;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            ai = fmaf(cf[i], U[PAR + 2 * i][k], ai);
            ee = fmaf(cf[i], V[PAR + 2 * i + 2][k], ee);
        }
        S[0][k] = ai;
        S[1][k] = R0[k];
        S[2][k] = R1[k];
        S[3][k] = (float)bonnet_a(k) * R1[k + 1] + (k > 0 ? (float)bonnet_b(k) * R1[k > 0 ? k - 1 : 0] : 0.f);
        S[4][k] = C0[k];
        S[5][k] = (float)bonnet_a(k) * C0[k + 1] + (k > 0 ? (float)bonnet_b(k) * C0[k > 0 ? k - 1 : 0] : 0.f);
        S[6][k] = ee;
    }
}

// A 3-vector with components 0 and 1 packed for the paired FP32 units.
struct V3p {
    float2 xy;
    float z;
};
__device__ __forceinline__ V3p v3p(const float *v) { return {make_float2(v[0], v[1]), v[2]}; }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
// a A + b B + c C
__device__ __forceinline__ V3p comb3(float a, const V3p &A, float b, const V3p &B, float c, const V3p &C) {
    V3p r;
    r.xy = __ffma2_rn(dup2(c), C.xy, __ffma2_rn(dup2(b), B.xy, __fmul2_rn(dup2(a), A.xy)));
    r.z = fmaf(c, C.z, fmaf(b, B.z, a * A.z));
    return r;
}
// a A + b B + c C + d E
__device__ __forceinline__ V3p comb4(float a, const V3p &A, float b, const V3p &B, float c, const V3p &C, float d,
                                     const V3p &E) {
    V3p r;
    r.xy = __ffma2_rn(dup2(d), E.xy,
                      __ffma2_rn(dup2(c), C.xy, __ffma2_rn(dup2(b), B.xy, __fmul2_rn(dup2(a), A.xy))));
    r.z = fmaf(d, E.z, fmaf(c, C.z, fmaf(b, B.z, a * A.z)));
    return r;
}

// X = R0 D + R1 t + C0 p, Y = R1 D + R2 t + C1 p, Z = C0 D + C1 t + E p for row k
template <int N>
__device__ __forceinline__ void far_xyz_p(const float (&S)[7][N + 1], int k, const V3p &D, const V3p &t,
                                          const V3p &p, V3p &X, V3p &Y, V3p &Z) {
    const float R0 = S[1][k], R1 = S[2][k], R2 = S[3][k], C0 = S[4][k], C1 = S[5][k], E = S[6][k];
    X = comb3(R0, D, R1, t, C0, p);
    Y = comb3(R1, D, R2, t, C1, p);
    Z = comb3(C0, D, C1, t, E, p);
}

// The 3 x 3 entries sc (AI delta_ab + D_a X_b + t_a Y_b + p_a Z_b) at
// dst[b * ld + a]; columns b = 0, 1 as a packed pair.
__device__ __forceinline__ void block3(float *dst, int ld, float sc, float AI, const float *D, const float *t,
                                       const float *p, const V3p &X, const V3p &Y, const V3p &Z) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float2 d0 = make_float2(a == 0 ? AI : 0.f, a == 1 ? AI : 0.f);
        float2 e = __ffma2_rn(dup2(p[a]), Z.xy, __ffma2_rn(dup2(t[a]), Y.xy, __ffma2_rn(dup2(D[a]), X.xy, d0)));
        e = __fmul2_rn(dup2(sc), e);
        dst[a] = e.x;
        dst[ld + a] = e.y;
        dst[2 * ld + a] = sc * fmaf(p[a], Z.z, fmaf(t[a], Y.z, fmaf(D[a], X.z, a == 2 ? AI : 0.f)));
    }
}


template <int N, bool PANELS, bool FAR>
__global__ void __launch_bounds__(32 * RF_FAR_WARPS, RF_FAR_MINB / RF_FAR_WARPS) far_pairs_kernel(SplitArgs a) {
    using SD = SplitDims<N>;
    using SM = FarSmem<N, PANELS>;
    constexpr int NL = SD::NL, NV = SD::NV, KW = SD::KW, NRHS = SD::NRHS, RB = SD::RB, GR = SM::GR;
    extern __shared__ __align__(16) unsigned char smem_all[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *smem_raw = smem_all + (size_t)warp * SM::kBytes;  // this warp's region
    float *s_nb = reinterpret_cast<float *>(smem_raw);               // [near lane][kNearWeight], one weight
    float *s_gk = s_nb + 32 * kNearWeight;                            // gamma_k (0..7), E_k (8..15)
    int *s_nl = reinterpret_cast<int *>(s_gk + 16);                   // near lanes of the source, in order
    int *s_ns = s_nl + 32;                                            // and their buffer slots
    float *s_pv = reinterpret_cast<float *>(s_ns + 32);
    float *s_w = s_pv + kMaxLQ;                                       // [kMaxLQ][KWP]: w_q P_k(s_q), k >= KW zero
    float *s_stg = s_w + kMaxLQ * SD::KWP;                            // [3][GR]
    float *s_pan = s_stg + 3 * GR;                                    // [2][3][96]
    __nv_bfloat16 *s_stg16 = reinterpret_cast<__nv_bfloat16 *>(s_pan + (PANELS ? SM::PAN : 0));  // [3][GR]

    const Tables &tab = *a.tab;
    const int LQ = a.LQ;
    for (int t = lane; t < kMaxLQ; t += 32) s_pv[t] = t < LQ ? (float)tab.pv[t] : 0.f;
    for (int t = lane; t < kMaxLQ * SD::KWP; t += 32) {
        const int q = t / SD::KWP, k = t - q * SD::KWP;
        s_w[t] = (q < LQ && k < KW) ? (float)(tab.wv[q] * tab.P[k][q]) : 0.f;
    }
    if (lane < 8) {
        s_gk[lane] = lane <= N ? (float)tab.gamma[lane] : 0.f;
        s_gk[8 + lane] = lane <= N ? (float)tab.Ek[lane] : 0.f;
    }
    double rhs[NRHS];  // sum over the far sources of theta^k_0 f
#pragma unroll
    for (int r = 0; r < NRHS; ++r) rhs[r] = 0.0;
    __syncwarp();

    const float D1 = (float)tab.D1, sv = (float)(0.5 / tab.d), sw = (float)(1.5 / tab.d);
    const float f[3] = {(float)tab.half_force[0], (float)tab.half_force[1], (float)tab.half_force[2]};
    const float e2 = (float)(2.0 * tab.eps2), e6 = (float)(6.0 * tab.eps2);

    const int i0 = (blockIdx.x * RF_FAR_WARPS + warp) * 32;
    const int i = i0 + lane;
    const bool valid = i < a.M;
    const int nvalid = min(32, a.M - i0);     // <= 0 for a warp past the last target: it only keeps step
    const int ic = valid ? i : min(i0, a.M - 1);
    const double xi0 = a.pos[3 * ic], xi1 = a.pos[3 * ic + 1], xi2 = a.pos[3 * ic + 2];
    const float t[3] = {(float)a.ori[3 * ic], (float)a.ori[3 * ic + 1], (float)a.ori[3 * ic + 2]};
    const float tt = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const int64_t brow = (int64_t)ic * a.words;
    const int slot0 = (valid && a.near_bits) ? a.near_off[ic] : 0;
    const bool merge = a.near_bits != nullptr && a.merge != 0;

    const int j0 = blockIdx.y * a.chunk;
    const int j1 = min(a.M, j0 + a.chunk);
    // the source's centre and direction are loaded one source ahead
    double xj[3] = {0.0, 0.0, 0.0};
    float pj[3] = {0.f, 0.f, 0.f};
    if (j0 < j1) {
        xj[0] = __ldg(a.pos + 3 * j0); xj[1] = __ldg(a.pos + 3 * j0 + 1); xj[2] = __ldg(a.pos + 3 * j0 + 2);
        pj[0] = (float)__ldg(a.ori + 3 * j0); pj[1] = (float)__ldg(a.ori + 3 * j0 + 1); pj[2] = (float)__ldg(a.ori + 3 * j0 + 2);
    }
    // staging offsets of this thread's entries in a near record: block entries
    // e = lane and lane + 32 (e = 3 RB columns-major), panel entry lane < 18
    const int moff0 = (lane / RB) * GR + lane % RB;
    const int moff1 = ((lane + 32) / RB) * GR + (lane + 32) % RB;
    const int poff = 3 * GR + ((lane / 9) * 3 + (lane % 9) / 3) * 96 + (lane % 9) % 3;  // s_pan follows s_stg
    unsigned word = 0u;
    int wpref = 0;
    for (int j = j0; j < j1; ++j) {
        const float D[3] = {(float)(xi0 - xj[0]), (float)(xi1 - xj[1]), (float)(xi2 - xj[2])};
        const float p[3] = {pj[0], pj[1], pj[2]};
        if (j + 1 < j1) {
            xj[0] = __ldg(a.pos + 3 * j + 3); xj[1] = __ldg(a.pos + 3 * j + 4); xj[2] = __ldg(a.pos + 3 * j + 5);
            pj[0] = (float)__ldg(a.ori + 3 * j + 3); pj[1] = (float)__ldg(a.ori + 3 * j + 4); pj[2] = (float)__ldg(a.ori + 3 * j + 5);
        }
        bool near = false;
        int slot = 0;
        if (valid && a.near_bits) {
            if (j == j0 || (j & 31) == 0) {
                word = a.near_bits[brow + (j >> 5)];
                wpref = merge ? a.near_pref[brow + (j >> 5)] : 0;
            }
            near = (word >> (j & 31)) & 1u;
            if (near) slot = slot0 + wpref + __popc(word & ((1u << (j & 31)) - 1u));
        }
        const unsigned nmask = merge ? __ballot_sync(0xffffffffu, near) : 0u;
        const int nnear = __popc(nmask);
        // list the near lanes in order and prefetch their weight-1 records;
        // the Gauss-point loop hides the copy
        if (near && merge) {
            const int r = __popc(nmask & ((1u << lane) - 1u));
            s_nl[r] = lane;
            s_ns[r] = slot;
        }
        __syncwarp();
        for (int u = lane; u < nnear * (kNearWeight / 4); u += 32) {
            const int r = u >> 4, c = u & 15;  // kNearWeight / 4 = 16 chunks per record
            cp_async16(s_nb + r * kNearWeight + 4 * c, a.nearbuf + (int64_t)s_ns[r] * kNearBlock + 4 * c);
        }
        cp_async_commit();
        const bool diag = i == j;
        const bool act = valid && !near && !diag;

        float U[NL][NL], V[NV][KW];
#pragma unroll
        for (int pp = 0; pp < NL; ++pp)
#pragma unroll
            for (int k = 0; k < NL; ++k) U[pp][k] = 0.f;
#pragma unroll
        for (int pp = 0; pp < NV; ++pp)
#pragma unroll
            for (int k = 0; k < KW; ++k) V[pp][k] = 0.f;
        // the Gauss point q's moments, weighted, into the projections
        // Pairs of rows (k, k + 1) go through the packed FP32 units: each half
        // of __ffma2_rn is the fmaf of the scalar form, so the sums are the same.
        auto add_point = [&](int q, const float *I, const float *J, const float *S) {
            constexpr int KWP = SD::KWP;
            const float2 *w2 = reinterpret_cast<const float2 *>(s_w + q * KWP);  // even stride: 8-byte aligned
            float2 wk[KWP / 2];
#pragma unroll
            for (int k = 0; k < KWP / 2; ++k) wk[k] = w2[k];
#pragma unroll
            for (int pp = 0; pp < NL; ++pp) {
                const float u = fmaf(e2, J[pp], I[pp]);
                const float2 u2 = make_float2(u, u);
#pragma unroll
                for (int k = 0; k + 1 < NL; k += 2) {
                    const float2 r = __ffma2_rn(wk[k / 2], u2, make_float2(U[pp][k], U[pp][k + 1]));
                    U[pp][k] = r.x;
                    U[pp][k + 1] = r.y;
                }
                if (NL % 2) U[pp][NL - 1] = fmaf(wk[(NL - 1) / 2].x, u, U[pp][NL - 1]);
            }
#pragma unroll
            for (int pp = 0; pp < NV; ++pp) {
                const float v = fmaf(-e6, S[pp], J[pp]);
                const float2 v2 = make_float2(v, v);
#pragma unroll
                for (int k = 0; k < KW; k += 2) {
                    if (k + 1 < vrows(N, pp)) {
                        const float2 r = __ffma2_rn(wk[k / 2], v2, make_float2(V[pp][k], V[pp][k + 1]));
                        V[pp][k] = r.x;
                        V[pp][k + 1] = r.y;
                    } else if (k < vrows(N, pp)) {
                        V[pp][k] = fmaf(wk[k / 2].x, v, V[pp][k]);
                    }
                }
            }
        };
        if (act) {
            if constexpr (FAR) {
                // every point far (c >= 6): two Gauss points per pass of the
                // packed recursion, added in the order q, q + 1.  Past an odd LQ
                // the partner is the zero padding of s_pv: computed, not added.
                static_assert(kMaxLQ % 2 == 0, "the partner of the last point must lie in s_pv");
                for (int q = 0; q < LQ; q += 2) {
                    const float sa = s_pv[q], sb = s_pv[q + 1];
                    const Geom32 ga(fmaf(sa, t[0], D[0]), fmaf(sa, t[1], D[1]), fmaf(sa, t[2], D[2]), p[0], p[1], p[2]);
                    const Geom32 gb(fmaf(sb, t[0], D[0]), fmaf(sb, t[1], D[1]), fmaf(sb, t[2], D[2]), p[0], p[1], p[2]);
                    float2 I2[KW], J2[KW], S2[KW];
                    moments_backward_fp32x2<N>(make_float2(ga.b, gb.b), make_float2(ga.c, gb.c), I2, J2, S2);
                    float I[KW], J[KW], S[KW];
#pragma unroll
                    for (int k = 0; k < KW; ++k) { I[k] = I2[k].x; J[k] = J2[k].x; S[k] = S2[k].x; }
                    add_point(q, I, J, S);
                    if (q + 1 < LQ) {
#pragma unroll
                        for (int k = 0; k < KW; ++k) { I[k] = I2[k].y; J[k] = J2[k].y; S[k] = S2[k].y; }
                        add_point(q + 1, I, J, S);
                    }
                }
            } else {
                // two Gauss points in flight (two independent recursions): 2 % faster
                // once the warps of a scheduler share the instruction stream
#pragma unroll 2
                for (int q = 0; q < LQ; ++q) {
                    const float sq = s_pv[q];
                    const float r0x = fmaf(sq, t[0], D[0]), r0y = fmaf(sq, t[1], D[1]), r0z = fmaf(sq, t[2], D[2]);
                    float I[KW], J[KW], S[KW];
                    moments_fp32<N, FAR>(Geom32(r0x, r0y, r0z, p[0], p[1], p[2]), I, J, S);
                    add_point(q, I, J, S);
                }
            }
        }
        const float Dt = D[0] * t[0] + D[1] * t[1] + D[2] * t[2];
        const float pt = p[0] * t[0] + p[1] * t[1] + p[2] * t[2];
        cp_async_wait_all();
        __syncthreads();  // the CTA's warps enter each source's post-processing together

        if (act) {
            // right-hand side: theta^k_0 f for weight 0 (near pairs add theirs in the near kernel)
#pragma unroll
            for (int k = 0; k <= N; ++k) {
                float R0[3] = {0.f, 0.f, 0.f}, C0[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    const int kk = k - 1 + o;
                    if (kk >= 0) C0[o] = -V[1][kk];
                }
                const float AI = U[0][k], E = V[2][k];
                const float R0k = V[0][k], R0p = V[0][k + 1], R0pp = V[0][k + 2];
                const float R0m = k > 0 ? V[0][k > 0 ? k - 1 : 0] : 0.f, R0mm = k > 1 ? V[0][k > 1 ? k - 2 : 0] : 0.f;
                const float R1 = (float)bonnet_a(k) * R0p + (float)bonnet_b(k) * R0m;
                const float R1p = (float)bonnet_a(k + 1) * R0pp + (float)bonnet_b(k + 1) * R0k;
                const float R1m = k > 0 ? (float)bonnet_a(k - 1) * R0k + (float)bonnet_b(k - 1) * R0mm : 0.f;
                const float R2 = (float)bonnet_a(k) * R1p + (float)bonnet_b(k) * R1m;
                const float C1 = (float)bonnet_a(k) * C0[2] + (float)bonnet_b(k) * C0[0];
                (void)R0;
                float X[3], Y[3], Z[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    X[c] = R0k * D[c] + R1 * t[c] + C0[1] * p[c];
                    Y[c] = R1 * D[c] + R2 * t[c] + C1 * p[c];
                    Z[c] = C0[1] * D[c] + C1 * t[c] + E * p[c];
                }
                const float Xf = X[0] * f[0] + X[1] * f[1] + X[2] * f[2];
                const float Yf = Y[0] * f[0] + Y[1] * f[1] + Y[2] * f[2];
                const float Zf = Z[0] * f[0] + Z[1] * f[1] + Z[2] * f[2];
#pragma unroll
                for (int c = 0; c < 3; ++c) rhs[3 * k + c] += (double)(AI * f[c] + D[c] * Xf + t[c] * Yf + p[c] * Zf);
            }
        }

        // weights m = 1..N: odd weights first, then even ones (sc_m a_mp vanishes
        // unless p and m have the same parity); the near records of the next
        // weight in this order are prefetched behind the current one
#pragma unroll 1
        for (int it = 0; it < N; ++it) {
            const int m = it < (N + 1) / 2 ? 2 * it + 1 : 2 * (it - (N + 1) / 2) + 2;
            float S[7][N + 1];
            if (m & 1) far_sets_reg<N, 1>(m, U, V, S);
            else far_sets_reg<N, 0>(m, U, V, S);
            // the block entries and panel rows: theta's 3 x 3 blocks with their
            // columns (components of X, Y, Z) paired on the packed FP32 units
            const V3p Dp = v3p(D), tp = v3p(t), pp3 = v3p(p);
            // the copy engine has read the previous weight's staged columns
            // (waited for only here, so that the coefficient sets above
            // overlap the copies)
            if (lane < kCopyLanes) bulk_wait_read();
            __syncwarp();
            // row k = 0: velocity panel P0 only
            if (PANELS) {
                V3p X, Y, Z;
                far_xyz_p<N>(S, 0, Dp, tp, pp3, X, Y, Z);
                block3(s_pan + lane * 3, 96, sv, S[0][0], D, t, p, X, Y, Z);
            }
            // row k = 1: block row D1 t (theta t)^T and velocity panel P1
            {
                V3p X, Y, Z;
                far_xyz_p<N>(S, 1, Dp, tp, pp3, X, Y, Z);
                const float AI = S[0][1];
                const V3p Q = comb4(AI, tp, Dt, X, tt, Y, pt, Z);
                const float Qv[3] = {Q.xy.x, Q.xy.y, Q.z};
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa) s_stg[bb * GR + lane * RB + aa] = D1 * t[aa] * Qv[bb];
                if (PANELS) {
                    V3p YQ;
                    YQ.xy = make_float2(Y.xy.x - Q.xy.x, Y.xy.y - Q.xy.y);
                    YQ.z = Y.z - Q.z;
                    block3(s_pan + 3 * 96 + lane * 3, 96, sw, AI, D, t, p, X, YQ, Z);
                }
            }
            // rows k = 2..N: gamma_k (theta - E_k t (theta t)^T)
#pragma unroll
            for (int k = 2; k <= N; ++k) {
                V3p X, Y, Z;
                far_xyz_p<N>(S, k, Dp, tp, pp3, X, Y, Z);
                const float AI = S[0][k], g = s_gk[k], ek = s_gk[8 + k];
                const V3p Q = comb4(AI, tp, Dt, X, tt, Y, pt, Z);
                V3p W;
                W.xy = __ffma2_rn(dup2(-ek), Q.xy, Y.xy);
                W.z = fmaf(-ek, Q.z, Y.z);
                block3(s_stg + lane * RB + 3 * (k - 1), GR, g, AI, D, t, p, X, W, Z);
            }
            // the diagonal pair (its projections are zero): identity where k = m
            if (diag) {
#pragma unroll
                for (int aa = 0; aa < 3; ++aa) s_stg[aa * GR + lane * RB + 3 * (m - 1) + aa] = 1.f;
            }
            cp_async_wait_all();
            __syncwarp();
            // near pairs: the FP64-integrated columns of weight m replace the
            // staged zeros; entry offsets are fixed per thread
            for (int r = 0; r < nnear; ++r) {
                const int L = s_nl[r];
                const float *src = s_nb + r * kNearWeight;
                if (lane < 3 * RB) s_stg[moff0 + L * RB] = src[lane];
                if (lane < 3 * RB - 32) s_stg[moff1 + L * RB] = src[lane + 32];
                if (PANELS && lane < 18) s_stg[poff + L * 3] = src[3 * RB + lane];
            }
            __syncwarp();
            // the records of the next weight, hidden behind the stores and that weight's work
            if (it + 1 < N) {
                const int mn = it + 1 < (N + 1) / 2 ? 2 * it + 3 : 2 * (it + 1 - (N + 1) / 2) + 2;
                for (int u = lane; u < nnear * (kNearWeight / 4); u += 32) {
                    const int r = u >> 4, c = u & 15;
                    cp_async16(s_nb + r * kNearWeight + 4 * c,
                               a.nearbuf + (int64_t)s_ns[r] * kNearBlock + (mn - 1) * kNearWeight + 4 * c);
                }
                cp_async_commit();
            }
            far_store_m<N, PANELS>(a, m, j, i0, nvalid, s_stg, s_pan, s_stg16, lane);
            __syncwarp();
        }
    }
    if (valid) {
#pragma unroll
        for (int r = 0; r < NRHS; ++r) a.far_contr[((int64_t)blockIdx.y * a.M + i) * NRHS + r] = rhs[r];
    }
    if (lane < kCopyLanes) bulk_wait_all();  // every staged segment written before the CTA's shared memory goes
}

// ---------------------------------------------------------------- near pairs (FP64)
constexpr int kNearWarps = 4;
#ifndef RF_NEAR_MINB
#define RF_NEAR_MINB 4
#endif
constexpr int kXq = 52;  // q stride of X[col][q]: 52 = 4 mod 16 makes the B fragments conflict-free
constexpr int kTmLd = 17;  // row stride of the projections Tm[k][col] (odd: rows fall in different banks)

template <int N>
struct NearSmem {
    static constexpr int X = 16 * kXq;                  // per-point scalars [col][q], cols >= 2N+4 zero
    static constexpr int TM = 8 * kTmLd + (8 * kTmLd) % 2;  // projections [k][col] (even: keeps BLK 16-byte aligned)
    static constexpr int BLK = kNearBlock / 2;          // staged block + panels (floats)
    static constexpr int RHS = 3 * (N + 1) + 1;
    static constexpr int WARP = X + TM + BLK + RHS + ((X + TM + BLK + RHS) & 1);
    static constexpr int TABLES = 8 * kMaxLQ + kMaxLQ + 72 + 32;   // w P, s, Legendre coefficients, row constants
    // every per-warp region and the staged block (read as float4) start on 16 bytes
    static_assert(X % 2 == 0 && (X + TM) % 2 == 0 && WARP % 2 == 0 && TABLES % 2 == 0, "16-byte alignment");
    static size_t bytes() { return sizeof(double) * (TABLES + (size_t)kNearWarps * WARP); }
};

// One CTA per target fiber, warps over its near sources.  Per pair: lane =
// Gauss point for the FP64 moments, the projection on the tensor cores, then
// lane = (source weight m, target row k) for the block entries.  The block
// goes to the near-pair buffer (DIRECT = false; the far kernel merges it into
// its column stores) or straight into A (DIRECT = true, used when the buffer
// could not be grown).
template <int N, bool PANELS, bool DIRECT>
__global__ void __launch_bounds__(kNearWarps * 32, RF_NEAR_MINB) near_pairs_kernel(SplitArgs a) {
    using SD = SplitDims<N>;
    using SM = NearSmem<N>;
    constexpr int NL = SD::NL, NV = SD::NV, RB = SD::RB, NRHS = SD::NRHS;
    constexpr int KSMAX = kMaxLQ / 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *s_wP = reinterpret_cast<double *>(smem_raw);   // [8][kMaxLQ]
    double *s_pv = s_wP + 8 * kMaxLQ;
    double *s_leg = s_pv + kMaxLQ;                          // [8][9]: sc_m a_mp (odd row stride)
    double *s_bon = s_leg + 72;                             // alpha_k, beta_k, gamma_k, E_k (8 each)
    double *base = s_wP + SM::TABLES + (size_t)warp * SM::WARP;
    double *X = base;
    double *Tm = X + SM::X;
    float *blk = reinterpret_cast<float *>(Tm + SM::TM);    // [col][row] RB*RB, then panels [w][col][a]
    double *rhs = Tm + SM::TM + SM::BLK;

    const Tables &tab = *a.tab;
    const int LQ = a.LQ;
    const int KS = (LQ + 3) / 4;
    for (int t = threadIdx.x; t < 8 * kMaxLQ; t += blockDim.x) {
        const int k = t / kMaxLQ, q = t - k * kMaxLQ;
        s_wP[t] = (k < SD::KW && q < LQ) ? tab.wv[q] * tab.P[k][q] : 0.0;
    }
    for (int t = threadIdx.x; t < kMaxLQ; t += blockDim.x) s_pv[t] = t < LQ ? tab.pv[t] : 0.0;
    for (int t = threadIdx.x; t < 72; t += blockDim.x) {
        const int m = t / 9, p = t % 9;
        s_leg[t] = p < 8 ? leg_scale(m) * leg_coef(m, p) : 0.0;
    }
    for (int t = threadIdx.x; t < 8; t += blockDim.x) {
        s_bon[t] = bonnet_a(t);
        s_bon[8 + t] = bonnet_b(t);
        s_bon[16 + t] = t <= N ? tab.gamma[t] : 0.0;
        s_bon[24 + t] = t <= N ? tab.Ek[t] : 0.0;
    }
    for (int t = lane; t < SM::X; t += 32) X[t] = 0.0;
    for (int t = lane; t < NRHS; t += 32) rhs[t] = 0.0;
    for (int t = lane; t < kNearBlock; t += 32) blk[t] = 0.f;
    __syncthreads();

    double afrag[KSMAX];
#pragma unroll
    for (int s = 0; s < KSMAX; ++s) afrag[s] = s_wP[(lane >> 2) * kMaxLQ + 4 * s + (lane & 3)];

    const int i = blockIdx.x;
    const double xi[3] = {a.pos[3 * i], a.pos[3 * i + 1], a.pos[3 * i + 2]};
    const double t[3] = {a.ori[3 * i], a.ori[3 * i + 1], a.ori[3 * i + 2]};
    const double e2 = 2.0 * tab.eps2, e6 = 6.0 * tab.eps2;
    const double D1 = tab.D1, sv = 0.5 / tab.d, sw = 1.5 / tab.d;
    const double *f = tab.half_force;
    const int cnt = a.near_cnt[i];
    const int *list = a.near_list + (int64_t)i * a.M;
    const int slot0 = a.near_off[i];

    for (int sidx = warp; sidx < cnt; sidx += kNearWarps) {
        const int j = list[sidx];
        const double D[3] = {xi[0] - a.pos[3 * j], xi[1] - a.pos[3 * j + 1], xi[2] - a.pos[3 * j + 2]};
        const double p[3] = {a.ori[3 * j], a.ori[3 * j + 1], a.ori[3 * j + 2]};
        // per-point scalars u_p (cols 0..N), v_p (cols N+1..2N+3)
        for (int q = lane; q < LQ; q += 32) {
            const double sq = s_pv[q];
            const double r0x = D[0] + sq * t[0], r0y = D[1] + sq * t[1], r0z = D[2] + sq * t[2];
            const double b = -2.0 * (p[0] * r0x + p[1] * r0y + p[2] * r0z);
            const double c = r0x * r0x + r0y * r0y + r0z * r0z;
            double I[SD::KW], J[SD::KW], S[SD::KW];
            moments_near<N>(b, c, I, J, S);
#pragma unroll
            for (int pp = 0; pp < NL; ++pp) X[pp * kXq + q] = I[pp] + e2 * J[pp];
#pragma unroll
            for (int pp = 0; pp < NV; ++pp) X[(NL + pp) * kXq + q] = J[pp] - e6 * S[pp];
        }
        __syncwarp();
        // projections Tm[k][col] = sum_q w_q P_k(s_q) X[col][q] on the FP64 tensor cores
#pragma unroll
        for (int tile = 0; tile < 2; ++tile) {
            double d0 = 0.0, d1 = 0.0;
#pragma unroll
            for (int s = 0; s < KSMAX; ++s)
                if (s < KS) {
                    const double bf = X[(8 * tile + (lane >> 2)) * kXq + 4 * s + (lane & 3)];
                    dmma_8x8x4(d0, d1, afrag[s], bf, d0, d1);
                }
            Tm[(lane >> 2) * kTmLd + 8 * tile + 2 * (lane & 3)] = d0;
            Tm[(lane >> 2) * kTmLd + 8 * tile + 2 * (lane & 3) + 1] = d1;
        }
        __syncwarp();
        const double Dt = D[0] * t[0] + D[1] * t[1] + D[2] * t[2];
        const double tt = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        const double pt = p[0] * t[0] + p[1] * t[1] + p[2] * t[2];
        // one (weight m, row k) per thread: the N*(N+1) pairs with m >= 1 first,
        // then the N+1 right-hand-side rows of weight 0 (cheaper) in what is left
        for (int u = lane; u < NL * NL; u += 32) {
            const int m = u < N * NL ? u / NL + 1 : 0;
            const int k = u < N * NL ? u - (m - 1) * NL : u - N * NL;
            const double *lg = s_leg + m * 9;
            // coefficient sets of weight m at rows k-2..k+2
            double AI = 0.0, E = 0.0, R0[5] = {0, 0, 0, 0, 0}, C0[3] = {0, 0, 0};
            for (int pp = m; pp >= 0; pp -= 2) {
                const double c = lg[pp];
                AI += c * Tm[k * kTmLd + pp];
                E += c * Tm[k * kTmLd + NL + pp + 2];
#pragma unroll
                for (int o = 0; o < 5; ++o) {
                    const int kk = k - 2 + o;
                    if (kk >= 0) R0[o] += c * Tm[kk * kTmLd + NL + pp];
                }
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    const int kk = k - 1 + o;
                    if (kk >= 0) C0[o] -= c * Tm[kk * kTmLd + NL + pp + 1];
                }
            }
            const double *al = s_bon, *be = s_bon + 8;
            const double R1p = al[k + 1] * R0[4] + be[k + 1] * R0[2];                // R1_{k+1}
            const double R1m = k > 0 ? al[k - 1] * R0[2] + be[k - 1] * R0[0] : 0.0;  // R1_{k-1}
            const double R1 = al[k] * R0[3] + be[k] * R0[1];
            const double R2 = al[k] * R1p + be[k] * R1m;
            const double C1 = al[k] * C0[2] + be[k] * C0[0];
            // theta = AI I + D X^T + t Y^T + p Z^T,  Q = theta t
            double X[3], Y[3], Z[3], Q[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                X[c] = R0[2] * D[c] + R1 * t[c] + C0[1] * p[c];
                Y[c] = R1 * D[c] + R2 * t[c] + C1 * p[c];
                Z[c] = C0[1] * D[c] + C1 * t[c] + E * p[c];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) Q[c] = AI * t[c] + Dt * X[c] + tt * Y[c] + pt * Z[c];
            if (m == 0) {
                const double Xf = X[0] * f[0] + X[1] * f[1] + X[2] * f[2];
                const double Yf = Y[0] * f[0] + Y[1] * f[1] + Y[2] * f[2];
                const double Zf = Z[0] * f[0] + Z[1] * f[1] + Z[2] * f[2];
#pragma unroll
                for (int c = 0; c < 3; ++c) rhs[3 * k + c] += AI * f[c] + D[c] * Xf + t[c] * Yf + p[c] * Zf;
                continue;
            }
            float *rec = blk + (m - 1) * kNearWeight;
            if (k >= 1) {
                // k = 1: D1 t Q^T; k >= 2: gamma_k (theta - E_k t Q^T); one formula
                // g (AI' I + D X'^T + t W^T + p Z'^T) with the row's coefficients
                const bool one = k == 1;
                const double g = one ? D1 : s_bon[16 + k], ek = s_bon[24 + k];
                const double ai = one ? 0.0 : AI;
                double W[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) W[c] = one ? Q[c] : Y[c] - ek * Q[c];
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const double xb = one ? 0.0 : X[bb], zb = one ? 0.0 : Z[bb];
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
                        rec[bb * RB + 3 * (k - 1) + aa] =
                            (float)(g * ((aa == bb ? ai : 0.0) + D[aa] * xb + t[aa] * W[bb] + p[aa] * zb));
                }
            }
            if (PANELS && k <= 1) {
                // P0: sv theta; P1: sw (theta - t Q^T)
                const double sc = k == 0 ? sv : sw, kq = k == 0 ? 0.0 : 1.0;
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
                        rec[3 * RB + k * 9 + bb * 3 + aa] = (float)(
                            sc * ((aa == bb ? AI : 0.0) + D[aa] * X[bb] + t[aa] * (Y[bb] - kq * Q[bb]) + p[aa] * Z[bb]));
            }
        }
        __syncwarp();
        if (!DIRECT) {
            float4 *dst = reinterpret_cast<float4 *>(a.nearbuf + (int64_t)(slot0 + sidx) * kNearBlock);
            const float4 *src = reinterpret_cast<const float4 *>(blk);
            for (int e = lane; e < kNearBlock / 4; e += 32) dst[e] = src[e];
        } else {
            for (int e = lane; e < N * kNearWeight; e += 32) {
                const int mm = e / kNearWeight, r = e - mm * kNearWeight;
                const float v = blk[e];
                if (r < 3 * RB) {
                    const int col = 3 * mm + r / RB, rr = r % RB;
                    const int64_t idx = ((int64_t)j * RB + col) * a.lda + (int64_t)i * RB + rr;
                    if (a.A16lo) {
                        split_store(v, a.A16 + idx, a.A16lo + idx);
                    } else {
                        if (a.A32) a.A32[idx] = v;
                        if (a.A16) a.A16[idx] = __float2bfloat16_rn(v);
                    }
                } else if (PANELS && r < 3 * RB + 18) {
                    const int e2 = r - 3 * RB, w = e2 / 9, rem = e2 - w * 9, bb = rem / 3, aa = rem - bb * 3;
                    (w ? a.PW32 : a.PV32)[((int64_t)j * RB + 3 * mm + bb) * a.ldp + (int64_t)i * 3 + aa] = v;
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int r = threadIdx.x; r < NRHS; r += blockDim.x) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kNearWarps; ++w) s += s_wP[SM::TABLES + (size_t)w * SM::WARP + SM::X + SM::TM + SM::BLK + r];
        a.near_contr[(int64_t)i * NRHS + r] = s;
    }
}

// ---------------------------------------------------------------- finish
// b rows and the l = 0 velocity terms from the summed theta^k_0 f
// (matrix_assembly.f90:874-899; coeffs_and_vels.f90:698-705 for the velocity).
__global__ void split_finish_kernel(SplitArgs a, int nchunks, double *b, double *vpart) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.M) return;
    const int N = a.N, NRHS = 3 * (N + 1);
    const Tables &tab = *a.tab;
    const double *t = a.ori + 3 * i;
    for (int k = 0; k <= N; ++k) {
        double contr[3];
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int ch = 0; ch < nchunks; ++ch) s += a.far_contr[((int64_t)ch * a.M + i) * NRHS + 3 * k + c];
            if (a.near_contr) s += a.near_contr[(int64_t)i * NRHS + 3 * k + c];
            contr[c] = s;
        }
        const double tdc = t[0] * contr[0] + t[1] * contr[1] + t[2] * contr[2];
        for (int aa = 0; aa < 3; ++aa) {
            if (k >= 1) {
                const double v = (k == 1) ? -tab.D1 * tdc * t[aa] : -tab.gamma[k] * (contr[aa] - tab.Ek[k] * tdc * t[aa]);
                b[(int64_t)i * 3 * N + 3 * (k - 1) + aa] = v;
            }
            if (vpart && k == 0) vpart[(int64_t)i * 6 + aa] = 0.5 / tab.d * contr[aa];
            if (vpart && k == 1) vpart[(int64_t)i * 6 + 3 + aa] = 1.5 / tab.d * (contr[aa] - tdc * t[aa]);
        }
    }
}

template <int N, bool PANELS, bool FAR>
cudaError_t launch_far_n(const SplitArgs &a, int far_chunks, cudaStream_t st) {
    const size_t smem = RF_FAR_WARPS * FarSmem<N, PANELS>::bytes();
    auto kern = far_pairs_kernel<N, PANELS, FAR>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const int groups = (a.M + 31) / 32;
    dim3 grid((groups + RF_FAR_WARPS - 1) / RF_FAR_WARPS, far_chunks);
    kern<<<grid, 32 * RF_FAR_WARPS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N, bool PANELS, bool DIRECT>
cudaError_t launch_near_n(const SplitArgs &a, cudaStream_t st) {
    const size_t smem = NearSmem<N>::bytes();
    auto kern = near_pairs_kernel<N, PANELS, DIRECT>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    kern<<<a.M, kNearWarps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

// N <= 5: the near kernel projects onto P_0..P_{N+2} with one 8-row tensor-core tile
bool split_supported(int N, int LQ) { return N >= 1 && N <= 5 && LQ <= kMaxLQ; }

int split_far_chunks(int M, int sm_count) {
    const int groups = (M + 31) / 32;
    const int ctas_x = (groups + RF_FAR_WARPS - 1) / RF_FAR_WARPS;
    // a first guess: about 64 target groups' worth of CTAs per SM
    const int c0 = std::max(1, std::min((sm_count * 64 + groups - 1) / groups, M));
    const int per0 = (M + c0 - 1) / c0;
    // The CTAs (one per SM: registers) run in rounds of sm_count, each CTA
    // taking time in proportion to its sources, so the kernel takes about
    // rounds x sources per CTA: the sources per CTA within a factor 2 of the
    // guess that minimise that product (ties: the larger share, fewer CTAs).
    // At M = 4000 on 148 SMs: 87 sources per CTA, 736 CTAs in 4.97 rounds,
    // instead of 53 sources and 1216 CTAs in 8.2 rounds (17.06 -> 15.92 ms
    // per mixed assembly, the same matrix).
    int best_cost = -1, best_chunks = c0, best_per = per0;
    for (int per = std::max(1, per0 / 2); per <= 2 * per0 && per <= M; ++per) {
        const int chunks = (M + per - 1) / per;
        const int share = (M + chunks - 1) / chunks;
        const int64_t rounds = ((int64_t)ctas_x * chunks + sm_count - 1) / sm_count;
        const int64_t cost = rounds * share;
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && share > best_per)) {
            best_cost = (int)cost;
            best_chunks = chunks;
            best_per = share;
        }
    }
    return std::max(1, std::min(best_chunks, M));
}

cudaError_t launch_split_classify(const SplitArgs &a, cudaStream_t st) {
    cudaError_t err = cudaMemsetAsync(a.near_total, 0, sizeof(int), st);
    if (err != cudaSuccess) return err;
    classify_kernel<<<(a.M + kClassifyWarps - 1) / kClassifyWarps, kClassifyWarps * 32, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_split_far(const SplitArgs &a, int far_chunks, cudaStream_t st) {
    const bool panels = a.PV32 != nullptr;
    // far pairs have c >= near_c >= kSplitMinNearC at every point: the FP32
    // backward recursion alone covers them
    const bool far_only = a.near_bits != nullptr && a.near_c >= kSplitMinNearC;
    switch (a.N) {
#define RF_FAR_CASE(n)                                                                                     \
    case n:                                                                                                \
        if (panels) return far_only ? launch_far_n<n, true, true>(a, far_chunks, st)                       \
                                    : launch_far_n<n, true, false>(a, far_chunks, st);                     \
        return far_only ? launch_far_n<n, false, true>(a, far_chunks, st)                                  \
                        : launch_far_n<n, false, false>(a, far_chunks, st);
        RF_FAR_CASE(1)
        RF_FAR_CASE(2)
        RF_FAR_CASE(3)
        RF_FAR_CASE(4)
        RF_FAR_CASE(5)
#undef RF_FAR_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_split_near(const SplitArgs &a, bool direct, cudaStream_t st) {
    const bool panels = a.PV32 != nullptr;
    switch (a.N) {
#define RF_NEAR_CASE(n)                                                                                    \
    case n:                                                                                                \
        if (panels) return direct ? launch_near_n<n, true, true>(a, st) : launch_near_n<n, true, false>(a, st); \
        return direct ? launch_near_n<n, false, true>(a, st) : launch_near_n<n, false, false>(a, st);
        RF_NEAR_CASE(1)
        RF_NEAR_CASE(2)
        RF_NEAR_CASE(3)
        RF_NEAR_CASE(4)
        RF_NEAR_CASE(5)
#undef RF_NEAR_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_split_finish(const SplitArgs &a, int far_chunks, double *b, double *vpart, cudaStream_t st) {
    split_finish_kernel<<<(a.M + 127) / 128, 128, 0, st>>>(a, far_chunks, b, vpart);
    return cudaGetLastError();
}

}  // namespace rf
