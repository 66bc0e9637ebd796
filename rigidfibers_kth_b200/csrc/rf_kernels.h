// rf_kernels.h - kernel argument blocks and launchers (device side of the
// library).  Host code in api.cpp and gmres.cpp calls only these launchers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "rf_device.cuh"

namespace rf {

constexpr int kPModeFP64 = 0;   // FP64 arithmetic throughout
constexpr int kPModeMixed = 1;  // FP32 far field, FP64 near field, FP32 projections

// Split storage of the FP32 matrix (mixed BF16 path): two 16-bit planes of
// lda x n entries each, the high plane first.  The high plane is the BF16
// matrix of the inner solves: the top 16 bits of each FP32 encoding plus
// bit 15 (round half away from zero on the bit pattern).  The low plane
// (`plane` entries further) holds the bottom 16 bits, from which the FP32
// value is rebuilt exactly: top = high - (low >> 15).  4 bytes per entry
// instead of 6 for separate FP32 and BF16 matrices.
struct SplitF32 {
    unsigned short bits;  // an entry of the high plane
};
__host__ __device__ __forceinline__ unsigned short split_hi(unsigned u) {
    return (unsigned short)((u >> 16) + ((u >> 15) & 1u));
}
__host__ __device__ __forceinline__ unsigned split_join(unsigned hi, unsigned lo) {
    return ((hi - (lo >> 15)) << 16) | lo;
}
__device__ __forceinline__ void split_store(float v, __nv_bfloat16 *hi, unsigned short *lo) {
    const unsigned u = __float_as_uint(v);
    *reinterpret_cast<unsigned short *>(hi) = split_hi(u);
    *lo = (unsigned short)(u & 0xffffu);
}
// one entry of a matrix stored as T (SplitF32: the planes `plane` apart)
template <typename T>
__device__ __forceinline__ double load_entry(const T *A, int64_t idx, int64_t) {
    return (double)A[idx];
}
template <>
__device__ __forceinline__ double load_entry<SplitF32>(const SplitF32 *A, int64_t idx, int64_t plane) {
    const unsigned hi = A[idx].bits, lo = A[idx + plane].bits;
    return (double)__uint_as_float(split_join(hi, lo));
}

// Programmatic dependent launch: a kernel launched by launch_pdl may be
// scheduled while the previous kernel on the stream finishes; it must call
// pdl_wait() before its first global memory access, which returns once that
// kernel has completed and its writes are visible.  Saves the launch gap of
// the short kernels of an inner GMRES step.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

struct AsmArgs {
    int M, N, LQ;
    int t0, t1;                // target fibers [t0, t1) (a row-block shard; 0, M for the whole system)
    int64_t n;                 // rows of the stored matrix: 3*N*(t1 - t0); its row r is the system's row 3*N*t0 + r
    const double *pos, *ori;   // 3M each
    const Tables *tab;         // device tables
    double *A64;               // FP64 matrix or null
    float *A32;                // FP32 matrix or null
    __nv_bfloat16 *A16;        // BF16 matrix (the high plane of split storage) or null
    unsigned short *A16lo;     // split storage: the low plane, or null
    int64_t lda;
    double *bpart;             // [nchunks][n] partial right-hand sides
    double *PV64, *PW64;       // velocity panels (3M x n, ld ldp) or null
    float *PV32, *PW32;
    int64_t ldp;
    double *vpart;             // [nchunks][6M] l = 0 velocity terms (or null)
    int chunk;                 // sources per CTA
    double near_c;             // mixed: c below which the integral stays FP64
};

cudaError_t launch_assemble(const AsmArgs &a, bool numeric, int pmode, int nchunks, cudaStream_t st);

// Mixed-precision assembly split into far pairs (FP32) and near pairs (FP64),
// analytic integration, N <= 5 (assemble_split.cu).
struct SplitArgs {
    int M, N, LQ;
    const double *pos, *ori;
    const Tables *tab;
    float *A32;                // FP32 matrix or null
    __nv_bfloat16 *A16;        // BF16 matrix (the high plane of split storage) or null
    unsigned short *A16lo;     // split storage: the low plane, or null
    int64_t lda;
    float *PV32, *PW32;        // velocity panels or null
    int64_t ldp;
    uint32_t *near_bits;       // [M][words] near-pair bitmap; null: every pair is far
    int words;                 // (M + 31) / 32
    int *near_list;            // [M][M] near sources of each target, ascending
    int *near_cnt;             // [M]
    int *near_pref;            // [M][words] near sources before each bitmap word
    int *near_off;             // [M] first slot of each target in the near-pair buffer
    int *near_total;           // device counter of near pairs (slot allocator)
    float *nearbuf;            // [near pairs][320] FP64-integrated blocks in FP32
    int merge;                 // far kernel copies near blocks from nearbuf
    double *far_contr;         // [far_chunks][M][3(N+1)] partial sums of theta^k_0 f
    double *near_contr;        // [M][3(N+1)] or null
    int chunk;                 // sources per far-pair CTA
    double near_c;             // c below which a pair is near
};
constexpr int kNearBlockFloats = 320;
// Smallest near threshold of the split assembly: from c = 6 on, the FP32
// backward recursion run from n = 32 down to n = 0 (moments_backward_fp32) is
// accurate to FP32 rounding in every direction, on the source axis included.
// (At c = 5 the truncated start already adds errors that lifted a velocity
// error of an M = 8000 trajectory above 1e-6.)
constexpr double kSplitMinNearC = 6.0;
bool split_supported(int N, int LQ);
int split_far_chunks(int M, int sm_count);
cudaError_t launch_split_classify(const SplitArgs &a, cudaStream_t st);
// direct = false: blocks to nearbuf (before the far kernel, which merges them);
// direct = true: blocks straight into A (after the far kernel)
cudaError_t launch_split_near(const SplitArgs &a, bool direct, cudaStream_t st);
cudaError_t launch_split_far(const SplitArgs &a, int far_chunks, cudaStream_t st);
// writes b (n) and, when vpart is not null, the l = 0 velocity terms [6M]
cudaError_t launch_split_finish(const SplitArgs &a, int far_chunks, double *b, double *vpart, cudaStream_t st);
cudaError_t launch_reduce_chunks(const double *part, int nchunks, int64_t stride, int64_t len, double *out,
                                 cudaStream_t st);

// ---- velocities (recompute path) -------------------------------------------
struct VelArgs {
    int M, N, LQ;
    int t0, t1;                // target fibers [t0, t1)
    const double *pos, *ori;
    const double *coeffs;      // n
    const Tables *tab;
    double *part;              // [nchunks][6M]: IF0 (3) and IF1 (3) sums per target
    int chunk;
};
cudaError_t launch_velocity(const VelArgs &a, bool numeric, int nchunks, cudaStream_t st);

// Matrix-free FP64 product y = A x (matfree.cu), the reference's mat_prod.
struct MatfreeArgs {
    int M, N, LQ;
    int64_t n;                 // 3 N M
    const double *pos, *ori;
    const double *x;           // n
    const Tables *tab;
    double *part;              // [nchunks][n] off-diagonal contributions per source chunk
    int chunk;
};
cudaError_t launch_matfree(const MatfreeArgs &a, bool numeric, int nchunks, const double *x, double *y,
                           cudaStream_t st);
// V = (local + 0.5*sum IF0)/d, W = 1.5/d (sum IF1 - (t.sum IF1) t) for targets [t0, t1)
cudaError_t launch_velocity_finish(int M, int t0, int t1, const double *ori, const Tables *tab, const double *part,
                                   int nchunks, double *V, double *W, cudaStream_t st);
// reuse path: V = PV x + v0, W = PW x + w0 (+ local term)
cudaError_t launch_velocity_reuse_finish(int M, const double *ori, const Tables *tab, const double *pv_x,
                                         const double *pw_x, const double *vpart, int nchunks, double *V,
                                         double *W, cudaStream_t st);

// ---- advection ---------------------------------------------------------------
cudaError_t launch_advect(int M, double dt, bool first, const double *Xp, const double *Xc, const double *Tp,
                          const double *Tc, const double *Vn, const double *Vo, const double *Wn,
                          const double *Wo, double *Xn, double *Tn, cudaStream_t st);
cudaError_t launch_normalize(int M, double *T, cudaStream_t st);

// ---- dense matrix-vector products -------------------------------------------
// y[0:m) = A[0:m, 0:k) x, A column-major with leading dimension lda.
// S storage type, X vector type, ACC accumulation type, Y output type.
// mode 0: y = A x;  mode 1: y = r - A x (residual, r given)
// stop (optional, device): when *stop != 0 at launch time every CTA returns at
// once (a product queued ahead for a solve that has finished meanwhile).
// S = SplitF32: A is the high plane, the low plane `plane` entries further.
template <typename S, typename X, typename ACC, typename Y>
cudaError_t launch_gemv(const S *A, int64_t lda, int64_t m, int64_t k, const X *x, Y *y, const Y *r,
                        ACC *work, int64_t work_elems, int sm_count, cudaStream_t st, const int *stop = nullptr,
                        int64_t plane = 0);
int64_t gemv_work_elems(int64_t m, int sm_count, int elem_bytes);

// ---- Krylov vector kernels ----------------------------------------------------
struct RedBuf {                 // deterministic last-block reduction workspace
    double *partials;           // >= max blocks
    unsigned int *counter;      // zero-initialised
    int max_blocks;
};
// w -= hprev * vprev (if vprev); out = dot(v, w)   (modified Gram-Schmidt step)
template <typename T>
cudaError_t launch_mgs_step(int64_t n, T *w, const T *vprev, const double *hprev, const T *v, double *out,
                            const RedBuf &rb, cudaStream_t st);
// w -= hprev * vprev; out = sqrt(dot(w, w))
template <typename T>
cudaError_t launch_mgs_norm(int64_t n, T *w, const T *vprev, const double *hprev, double *out,
                            const RedBuf &rb, cudaStream_t st);
// out = dot(a, b) (double accumulation)
template <typename T>
cudaError_t launch_dot(int64_t n, const T *a, const T *b, double *out, const RedBuf &rb, cudaStream_t st);

// Direct solve (lu.cu): A (n x n, column-major, ld lda) is overwritten by its
// LU factors with partial pivoting, piv[n] the pivot rows (0-based), info the
// first zero pivot (1-based) or 0; lu_solve overwrites x (= b on entry) with
// the solution.  blas: a cuBLAS handle (the trailing updates); launches counts
// the kernels launched.
cudaError_t lu_factor(double *A, int64_t lda, int64_t n, int *piv, int *info, void *blas, cudaStream_t st,
                      int64_t *launches);
cudaError_t lu_solve(const double *A, int64_t lda, int64_t n, const int *piv, double *x, cudaStream_t st,
                     int64_t *launches);
// y = alpha_scale * x where alpha_scale = num/den (den device scalar), i.e. y = x * (num / *den)
template <typename TO, typename TI>
cudaError_t launch_scale(int64_t n, const TI *x, const double *den, double num, TO *y, cudaStream_t st);
// y = alpha * x (alpha host scalar)
template <typename TO, typename TI>
cudaError_t launch_scale_h(int64_t n, const TI *x, double alpha, TO *y, cudaStream_t st);
// xcur = x + V(:, 0:k) y   (V column-major ld n, y device array of k doubles)
template <typename TV>
cudaError_t launch_combine(int64_t n, const double *x, const TV *V, int64_t ldv, const double *y, int k,
                           double *xcur, cudaStream_t st);
// r = b - r
template <typename T>
cudaError_t launch_bmr(int64_t n, const T *b, T *r, cudaStream_t st);
// u = V(:, 0:k) y  (y device array of k doubles)
template <typename T>
cudaError_t launch_vy(int64_t n, const T *V, int64_t ldv, const double *y, int k, T *u, cudaStream_t st);
// out = x + u
template <typename T>
cudaError_t launch_add(int64_t n, const T *x, const T *u, T *out, cudaStream_t st);
// y += alpha * x (alpha host scalar)
cudaError_t launch_axpy_d(int64_t n, double alpha, const double *x, double *y, cudaStream_t st);
// x += scale * d  with d float, scale host
cudaError_t launch_axpy_fd(int64_t n, double alpha, const float *d, double *x, cudaStream_t st);
// convert
template <typename TO, typename TI>
cudaError_t launch_convert(int64_t n, const TI *x, TO *y, cudaStream_t st);
// FP64 copy of rows [row0, row0 + rows) of a column-major matrix (cols columns)
template <typename T>
cudaError_t launch_gather_rows(const T *A, int64_t lda, int64_t row0, int64_t rows, int64_t cols, double *out,
                               cudaStream_t st, int64_t plane = 0);

// ---- neighbour-block preconditioner (FP32 blocks) -----------------------------
// z_i = v_i + omega sum_{m < kp} B[i][m] v_{knn[i][m]}, B[i][m] row-major
// 3N x 3N, pstride blocks per fiber, kstride neighbours per fiber in knn
template <typename T>
cudaError_t launch_pair_apply(int M, int nb, int kp, int pstride, const float *B, const int *knn, int kstride,
                              double omega, const T *v, T *z, cudaStream_t st, const int *stop = nullptr);

// ---- device-controlled Arnoldi steps (arnoldi.cu) -------------------------------
// State of one GMRES(m) solve held on the device: the Hessenberg columns after
// the Givens rotations, the rotations, the rotated right-hand side g, the
// least-squares solution y, the Gram-Schmidt coefficients of the running step.
constexpr int kArnoldiMax = 16;   // longest restart the device-controlled solve takes
struct ArnoldiCtrl {
    double H[kArnoldiMax * kArnoldiMax];   // H[r + c * kArnoldiMax], r <= c (upper triangle after rotation)
    double g[kArnoldiMax + 1];
    double cs[kArnoldiMax], sn[kArnoldiMax];
    double y[kArnoldiMax];
    double h1[kArnoldiMax], h2[kArnoldiMax];   // the two Gram-Schmidt passes of the running step
    double hnext;      // norm of the new basis vector before normalisation
    double bn;         // norm of the solve's right-hand side
    double tol;        // stop when |g_k| / bn <= tol
    double bea;        // the Arnoldi estimate |g_k| / bn after the last step
    int k;             // Arnoldi steps of the current cycle
    int itn;           // steps over all cycles
    int iter_max;      // step budget
    int stop;          // 0 running, 1 estimate <= tol, 2 budget spent, 3 non-finite value
};
// One step's outcome as the host sees it (host-mapped memory written by the device).
struct ArnoldiStat {
    int stop;
    int itn;
    double bea;
};
// Start of a cycle: beta = |r| (r the cycle's residual); g = (beta, 0, ...),
// k = 0, stop = 0 (1 if beta = 0, 3 if not finite), written to *stat
// (host-mapped) too; with first != 0 also bn = beta, itn = 0 and the
// tolerance and budget; then V_0 = r / beta.
template <typename T>
cudaError_t launch_arnoldi_start(int64_t n, const T *r, T *V0, ArnoldiCtrl *c, double tol, int iter_max, int first,
                                 double *part, unsigned int *counter, int max_blocks, ArnoldiStat *stat,
                                 cudaStream_t st);
// Step j after w = A z: two classical Gram-Schmidt passes against V_0..V_j
// (dots; update and dots; update and norm), then the Givens update of column
// j, the stop test, the step's outcome into stat[j] (host-mapped), and
// V_{j+1} = w / |w| unless the solve stopped or j + 1 = m.  Every kernel
// returns at once when the solve has stopped before it.
template <typename T>
cudaError_t launch_arnoldi_orthogonalize(int64_t n, T *w, T *V, int j, int m, ArnoldiCtrl *c, ArnoldiStat *stat,
                                         double *part, unsigned int *counter, int max_blocks, cudaStream_t st);
// End of a cycle: y = H(0:k, 0:k)^-1 g(0:k) and u = V(:, 0:k) y.
template <typename T>
cudaError_t launch_arnoldi_combine(int64_t n, const T *V, ArnoldiCtrl *c, T *u, cudaStream_t st);

}  // namespace rf
