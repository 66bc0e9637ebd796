// handle.h - the rf_handle behind the C ABI (internal).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/rigidfibers.h"
#include "gmres.h"
#include "rf_kernels.h"

struct rf_handle {
    rf_params p{};
    int M = 0, N = 0, LQ = 0;
    int64_t n = 0;        // 3*N*M
    int64_t lda = 0;      // leading dimension of A (multiple of 64 elements)
    int64_t ldp = 0;      // leading dimension of the velocity panels
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t marks[16] = {};

    // state: positions/orientations triple-buffered, velocities double-buffered
    double *X[3] = {nullptr, nullptr, nullptr};
    double *T[3] = {nullptr, nullptr, nullptr};
    int prev = 0, cur = 1, next = 2;
    double *V[2] = {nullptr, nullptr};
    double *W[2] = {nullptr, nullptr};
    int vprev = 0, vcur = 1;
    int vlast = -1;           // slot of the most recent velocities

    // system
    rf::Tables tab_h{};
    rf::Tables *tab = nullptr;
    double *A64 = nullptr;
    double *LU = nullptr;      // direct solver: LU factors of A64 (ld lda), made at the first direct solve
    double *lu_r = nullptr;    // direct solver: residual b - A x for the statistics
    int *lu_piv = nullptr;     // [n] pivot rows
    int *lu_info = nullptr;
    void *blas = nullptr;      // direct solver: cuBLAS handle (cublasHandle_t), made at the first direct solve
    float *A32 = nullptr;
    __nv_bfloat16 *A16 = nullptr;   // BF16 matrix; in split storage also the high plane
    unsigned short *A16lo = nullptr;  // split storage (mixed BF16): the low plane, a_plane entries after A16
    int64_t a_plane = 0;
    double *b = nullptr;       // right-hand side
    double *x = nullptr;       // coefficients (warm start for the next solve)
    double *bpart = nullptr;   // [nchunks][n]
    int asm_chunks = 1, asm_chunk = 1;
    int vel_chunks = 1, vel_chunk = 1;
    double *velpart = nullptr; // [vel_chunks][6M]
    double *mfpart = nullptr;  // [vel_chunks][n] matrix-free product partials, made at its first use
    // velocity panels (reuse mode)
    double *PV64 = nullptr, *PW64 = nullptr;
    float *PV32 = nullptr, *PW32 = nullptr;
    double *vpart = nullptr;   // [asm_chunks][6M]
    int vpart_chunks = 1;      // partial sums held in vpart by the last assembly
    // split mixed-precision assembly
    bool split = false;
    int far_chunks = 1, far_chunk = 1;
    uint32_t *near_bits = nullptr;
    int *near_list = nullptr, *near_cnt = nullptr, *near_pref = nullptr, *near_off = nullptr;
    int *near_total = nullptr;
    float *nearbuf = nullptr;
    int64_t near_cap = 0;      // capacity of nearbuf in pairs
    int64_t near_pairs = 0;    // near pairs of the last assembly
    double *far_contr = nullptr, *near_contr = nullptr;
    double *pvx = nullptr, *pwx = nullptr;
    // matvec workspace
    double *work64 = nullptr;
    float *work32 = nullptr;
    int64_t work_elems = 0;
    // solver
    std::unique_ptr<rf::Gmres<double>> gm64;
    std::unique_ptr<rf::Gmres<float>> gm32;
    double *r64 = nullptr;     // refinement residual
    float *r32 = nullptr;      // scaled residual / rhs in FP32
    float *d32 = nullptr;      // inner correction
    float *x32 = nullptr;      // FP32 iterate (FP32 variant)
    double *dscal = nullptr;   // device scalars (norms)
    double *hscal = nullptr;   // pinned host mirror
    rf::RedBuf rb{};
    // preconditioner
    float *Pblocks = nullptr;  // M x RF_MLP_PAIRS coupling blocks, (3N)^2 row-major each
    bool pc_ready = false;
    int pc_pairs = 0;          // coupling blocks in use per fiber
    int *knn = nullptr;        // M x RF_MLP_K neighbour lists, nearest first
    float *mlp_w = nullptr;    // MLP weights on the device
    __nv_bfloat16 *mlp_wtc = nullptr;  // the three weight matrices in BF16, rows padded to 256 (tensor-core inference)
    int *mlp_err = nullptr;    // set by the tensor-core layers when an MMA wait timed out
    bool mlp_loaded = false;
    float *feat = nullptr;     // (M x RF_MLP_PAIRS) x 144 pair features, M x 9 frames, M x RF_MLP_PAIRS signs
    float *mlp_h1 = nullptr, *mlp_h2 = nullptr, *mlp_out = nullptr;

    // live timing of the inner-solve products (rf_gemv_timer)
    struct GemvTimer {
        bool on = false;
        std::vector<cudaEvent_t> ev;   // start/stop pairs
        int used = 0;
        int64_t count = 0;
        double total_ms = 0.0;
        double bytes = 0.0;
    } gt;

    // row-block shard (shard.cu): target fibers [t0, t1) of M; their rows
    // n_loc = 3 N (t1 - t0) are the rows of the stored matrix (leading
    // dimension lda); everything else is replicated
    int shards = 1, shard = 0;
    int t0 = 0, t1 = 0, tpad = 0;   // tpad: the largest shard's fibers
    int64_t n_loc = 0;
    void *comm = nullptr;           // ncclComm_t of the shards (rf_create_sharded)
    double *shard_send = nullptr;   // 3 N tpad
    double *shard_gather = nullptr; // shards x 3 N tpad

    rf_solve_stats stats{};
    int cold_solves = 0;  // mixed solves left that start from zero (poor warm start seen)
    int warm_wait = 8;    // solves to start from zero after the next poor warm start
    bool x_valid = false; // x holds a solution (solved, or restored by rf_set_history)
    int pc_skips = 0;     // solves left that skip the block preconditioner
    double pc_its[2] = {-1.0, -1.0};  // running mean of solve iterations without / with it (-1: none yet)
    int pc_age = 0;       // preconditioned solves since the last one without it
    bool assembled = false;
    int64_t launches = 0;
    std::string err;
};

namespace rf {
rf_status fail(rf_handle *h, rf_status s, const std::string &msg);
// preconditioner MLP inference on the tensor cores (mlp_tc.cu)
int mlp_tc_padded_rows();
cudaError_t mlp_tc_pad_weights(const float *w, int nout, int K, __nv_bfloat16 *out, cudaStream_t st);
cudaError_t mlp_tc_forward(const __nv_bfloat16 *W1, const float *b1, const __nv_bfloat16 *W2, const float *b2,
                           const __nv_bfloat16 *W3, const float *b3, int rows, int nin, int nhid, int nout,
                           const float *X, __nv_bfloat16 *H1, __nv_bfloat16 *H2, float *O, int *err, cudaStream_t st);
// row-block shards (shard.cu)
void shard_range(int M, int R, int r, int *t0, int *t1);
int shard_pad(int M, int R);
rf_status shard_attach(rf_handle *h, const uint8_t *nccl_id);
void shard_detach(rf_handle *h);
// gathers every shard's segment [unit t0, unit t1) of `full` into `full`;
// send_ready: this shard's segment already in h->shard_send, or null
cudaError_t shard_allgather(rf_handle *h, double *full, int unit, const double *send_ready);
rf_status cuda_fail(rf_handle *h, cudaError_t e, const char *what);
// preconditioner (precond.cu)
rf_status build_preconditioner(rf_handle *h);
rf_status apply_mlp(rf_handle *h);
}  // namespace rf
