// api.cu - the C ABI (include/rigidfibers.h): handle life cycle and the
// reference step API (src/simulation.cu:40-424 of the reference):
// assemble_system -> solve_system -> update_velocities -> update_fibers.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"

namespace {

thread_local std::string g_create_error;

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) return cudaSuccess;
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * count);
}

// y = A x (r null) or y = r - A x over the FP32 matrix of the FP32 and mixed
// paths: its own FP32 storage, or the two 16-bit planes of the mixed BF16 path
template <typename X, typename ACC, typename Y>
cudaError_t fp32_gemv(rf_handle *h, const X *x, Y *y, const Y *r, ACC *work, const int *stop = nullptr) {
    if (h->A16lo)
        return rf::launch_gemv<rf::SplitF32, X, ACC, Y>(reinterpret_cast<const rf::SplitF32 *>(h->A16), h->lda, h->n,
                                                        h->n, x, y, r, work, h->work_elems, h->sm_count, h->stream,
                                                        stop, h->a_plane);
    return rf::launch_gemv<float, X, ACC, Y>(h->A32, h->lda, h->n, h->n, x, y, r, work, h->work_elems, h->sm_count,
                                             h->stream, stop);
}

void free_all(rf_handle *h) {
    rf::shard_detach(h);
    for (int i = 0; i < 3; ++i) {
        cudaFree(h->X[i]);
        cudaFree(h->T[i]);
    }
    for (int i = 0; i < 2; ++i) {
        cudaFree(h->V[i]);
        cudaFree(h->W[i]);
    }
    void *ptrs[] = {h->tab, h->A64, h->LU, h->lu_r, h->lu_piv, h->lu_info, h->mfpart, h->A32, h->A16, h->b, h->x, h->bpart, h->velpart, h->PV64, h->PW64,
                    h->PV32, h->PW32, h->vpart, h->pvx, h->pwx, h->work64, h->work32, h->r64, h->r32,
                    h->d32, h->x32, h->Pblocks, h->knn, h->mlp_w, h->mlp_wtc, h->mlp_err, h->feat, h->mlp_h1, h->mlp_h2, h->mlp_out,
                    h->dscal, h->rb.partials, h->rb.counter, h->near_bits, h->near_list, h->near_cnt,
                    h->far_contr, h->near_contr, h->near_pref, h->near_off, h->near_total, h->nearbuf};
    for (void *p : ptrs) cudaFree(p);
    if (h->blas) cublasDestroy(static_cast<cublasHandle_t>(h->blas));
    h->gm64.reset();
    h->gm32.reset();
    if (h->hscal) cudaFreeHost(h->hscal);
    for (auto &ev : h->marks)
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : h->gt.ev)
        if (ev) cudaEventDestroy(ev);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// Tables of quadrature points, weights, Legendre values and model constants
// (quadrature.f90:44-84, matrix_assembly.f90:36-56 and 450-484).
void make_tables(const rf_params &p, rf::Tables &t) {
    std::memset(&t, 0, sizeof(t));
    const int NoQI = p.num_quadrature_intervals, N = p.num_terms_in_force_expansion;
    t.N = N;
    t.LQ = 3 * NoQI;
    const double pv0[3] = {-std::sqrt(15.0) / 5.0, 0.0, std::sqrt(15.0) / 5.0};
    const double wv0[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    double a = -1.0;
    const double iv = 2.0 / NoQI;
    for (int i = 0; i < NoQI; ++i) {
        for (int k = 0; k < 3; ++k) {
            t.pv[3 * i + k] = (2.0 * a + iv + pv0[k] * iv) / 2.0;
            t.wv[3 * i + k] = wv0[k] / NoQI;
        }
        a = a + iv;
    }
    // Legendre polynomials at the points with the explicit formulas of
    // compute_LVecs (matrix_assembly.f90:36-56); P_0 = 1.  Rows N+1, N+2 (when
    // they fit) serve the split mixed-precision assembly, which projects onto
    // P_0..P_{N+2}.
    const int mmax = std::min(rf::kMaxN, N + 2);
    for (int q = 0; q < t.LQ; ++q) {
        const double x = t.pv[q];
        t.P[0][q] = 1.0;
        for (int m = 1; m <= mmax; ++m) {
            double v;
            switch (m) {
                case 1: v = x; break;
                case 2: v = 0.5 * (3.0 * x * x - 1.0); break;
                case 3: v = 0.5 * (5.0 * x * x * x - 3.0 * x); break;
                case 4: v = 0.125 * (35.0 * std::pow(x, 4) - 30.0 * x * x + 3.0); break;
                case 5: v = 0.125 * (63.0 * std::pow(x, 5) - 70.0 * x * x * x + 15.0 * x); break;
                case 6: v = 0.0625 * (231.0 * std::pow(x, 6) - 315.0 * std::pow(x, 4) + 105.0 * x * x - 5.0); break;
                case 7:
                    v = 0.0625 * (429.0 * std::pow(x, 7) - 693.0 * std::pow(x, 5) + 315.0 * x * x * x - 35.0 * x);
                    break;
                default:
                    v = 6435.0 / 128.0 * std::pow(x, 8) - 3003.0 / 32.0 * std::pow(x, 6) + 3465.0 / 64.0 * std::pow(x, 4) -
                        315.0 / 32.0 * x * x + 35.0 / 128.0;
                    break;
            }
            t.P[m][q] = v;
        }
    }
    const double eps = p.slenderness;
    const double c = std::log(eps * eps * std::exp(1.0));
    t.d = -c;
    t.e = 2.0;
    t.eps2 = eps * eps;
    t.D1 = 0.75 / (t.d - 2.0);
    double lambda[rf::kMaxN + 1] = {0};
    lambda[1] = 2.0;
    for (int k = 2; k <= N; ++k) lambda[k] = lambda[k - 1] + 2.0 / k;
    for (int k = 1; k <= N; ++k) {
        t.Ek[k] = (t.d - t.e - lambda[k]) / 2.0 / (t.d - lambda[k]);
        t.gamma[k] = 0.5 * (2.0 * k + 1.0) / (t.d + t.e - lambda[k]);
    }
    for (int a2 = 0; a2 < 3; ++a2) {
        t.force[a2] = p.external_force[a2];
        t.half_force[a2] = 0.5 * p.external_force[a2];
    }
}

bool finite_all(const double *v, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

#define CK(h, expr, what)                                        \
    do {                                                         \
        cudaError_t e__ = (expr);                                \
        if (e__ != cudaSuccess) return rf::cuda_fail(h, e__, what); \
    } while (0)

bool is_mixed(int prec) { return prec == RF_PREC_MIXED_BF16 || prec == RF_PREC_MIXED_FP32; }

}  // namespace

namespace rf {

rf_status fail(rf_handle *h, rf_status s, const std::string &msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return s;
}

rf_status cuda_fail(rf_handle *h, cudaError_t e, const char *what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    const rf_status s = (e == cudaErrorMemoryAllocation) ? RF_ERR_OOM
                        : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? RF_ERR_NO_DEVICE
                                                                                         : RF_ERR_CUDA;
    cudaGetLastError();  // clear a sticky launch error
    return fail(h, s, msg);
}

}  // namespace rf

namespace {

// Mixed solves that start from zero after a warm start left more than 10 %
// of |b|; the next one tries the warm start again.
constexpr int kWarmRetry = 8;
constexpr int kWarmRetryMax = 64;  // the wait doubles after each poor warm start up to this
// The block preconditioner is kept only while it pays.  The solver keeps a
// running mean of the iterations of its solves with and without it; after a
// solve whose blocks missed a trial (see rf_solve_system), or whose mean is
// above the mean without them, the next kPcRetry assemblies neither build
// nor use them.  While the blocks pay, one solve in kPcExplore runs without
// them to keep that comparison current (the suspension's state drifts).
constexpr int kPcRetry = 8;
// Default damping of the neighbour blocks, z_i = v_i + 0.85 sum_m B_im v_(j_m).
// Single solves of evolved states: on the M = 4000 cloud the learned blocks
// give the same iterations for damping 0.75 .. 1 (20, 20, 18, 17-18 at steps
// 0, 10, 20, 30; 23-25 without); on the uniform M = 8000 box (dt 0.05) 33
// and 45 at steps 10 and 30 against 36 and 70 undamped and 42 and 54
// without; the exact cluster blocks 20 / 18 at 0.7 against 32 / 29
// undamped.  Whole runs: the benchmark's 20 timed steps average 19.25 /
// 19.5 / 19.95 inner iterations at 1 / 0.85 / 0.75, the M = 8000 box's 100
// steps 3.72 steps/s at 0.85 against 3.62 at 0.75.
constexpr double kPcDamping = 0.85;
constexpr int kPcExplore = 32;


// Sum the recorded start/stop pairs of the product timer (waits for them).
cudaError_t gemv_timer_flush(rf_handle *h) {
    auto &g = h->gt;
    if (g.used == 0) return cudaSuccess;
    cudaError_t e = cudaEventSynchronize(g.ev[g.used - 1]);
    for (int i = 0; i + 1 < g.used && e == cudaSuccess; i += 2) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, g.ev[i], g.ev[i + 1]);
        g.total_ms += ms;
        g.count++;
    }
    g.used = 0;
    return e;
}

// Run one inner-solve product, bracketed by events when the timer is on.
template <typename F>
cudaError_t timed_product(rf_handle *h, double bytes, F launch) {
    auto &g = h->gt;
    if (!g.on) return launch();
    if (g.used + 2 > (int)g.ev.size()) {
        cudaError_t e = gemv_timer_flush(h);
        if (e != cudaSuccess) return e;
        while ((int)g.ev.size() < 64) {
            cudaEvent_t ev = nullptr;
            e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return e;
            g.ev.push_back(ev);
        }
    }
    cudaError_t e = cudaEventRecord(g.ev[g.used], h->stream);
    if (e == cudaSuccess) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(g.ev[g.used + 1], h->stream);
    if (e == cudaSuccess) {
        g.used += 2;
        g.bytes = bytes;
    }
    return e;
}

}  // namespace

extern "C" {

void rf_params_default(rf_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->slenderness = 0.01;
    p->timestep = 0.1;
    p->num_fibers = 0;
    p->num_timesteps = 10;
    p->num_terms_in_force_expansion = 5;
    p->num_quadrature_intervals = 8;
    p->use_analytical_integration = 1;
    p->use_direct_solver = 0;
    p->gmres_restart = 10;
    p->gmres_max_iters = 100;
    p->gmres_tol = 1e-5;
    p->external_force[0] = 0.0;
    p->external_force[1] = 0.0;
    p->external_force[2] = -1.0;
    p->precision = RF_PREC_FP64;
    p->preconditioner = RF_PC_NONE;
    p->velocity_mode = RF_VEL_RECOMPUTE;
    p->device = 0;
    p->max_refinements = 30;
    p->cluster_size = 8;
    p->inner_tol = 1e-3;
    p->near_field_c = 6.0;
    p->pc_damping = kPcDamping;
}

const char *rf_status_string(rf_status s) {
    switch (s) {
        case RF_OK: return "ok";
        case RF_ERR_INVALID_ARG: return "invalid argument";
        case RF_ERR_OOM: return "out of device memory";
        case RF_ERR_CUDA: return "CUDA error";
        case RF_ERR_NOT_CONVERGED: return "GMRES did not converge";
        case RF_ERR_DEVICE_TIMEOUT: return "device wait timed out";
        case RF_ERR_NAN: return "non-finite value";
        case RF_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char *rf_last_error(const rf_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

rf_status rf_create(const rf_params *p, const double *positions, const double *orientations, rf_handle **out) {
    if (!out) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    if (!p || !positions || !orientations) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "null argument");
    const int M = p->num_fibers, N = p->num_terms_in_force_expansion, NoQI = p->num_quadrature_intervals;
    if (M < 1) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "num_fibers must be >= 1");
    if (N < 1 || N > rf::kMaxN) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "num_terms_in_force_expansion must be 1..8");
    if (NoQI < 1 || 3 * NoQI > rf::kMaxLQ)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "num_quadrature_intervals must be 1..16");
    if (!(p->slenderness > 0.0 && p->slenderness < 0.5))
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "slenderness must be in (0, 0.5)");
    if (p->precision < RF_PREC_FP64 || p->precision > RF_PREC_MIXED_FP32)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "unknown precision");
    if (p->preconditioner < RF_PC_NONE || p->preconditioner > RF_PC_LEARNED)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "unknown preconditioner");
    if (p->velocity_mode != RF_VEL_RECOMPUTE && p->velocity_mode != RF_VEL_REUSE)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "unknown velocity mode");
    if (!(p->pc_damping >= 0.0 && p->pc_damping <= 2.0))
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "pc_damping must be in [0, 2] (0: the default)");
    if (M < 2 && p->preconditioner != RF_PC_NONE)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "a block preconditioner needs at least two fibers");
    if (p->use_direct_solver && p->precision != RF_PREC_FP64)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "use_direct_solver needs precision RF_PREC_FP64");
    if (p->gmres_restart < 1 || p->gmres_restart > 64 || !(p->gmres_tol > 0.0))
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "gmres_restart must be 1..64 and gmres_tol > 0");
    const int shards = p->shard_count > 1 ? p->shard_count : 1;
    if (shards > 1) {
        if (shards > M || p->shard_index < 0 || p->shard_index >= shards)
            return rf::fail(nullptr, RF_ERR_INVALID_ARG, "need shard_count <= num_fibers and 0 <= shard_index < shard_count");
        if (p->precision != RF_PREC_FP64 || p->use_direct_solver || p->velocity_mode != RF_VEL_RECOMPUTE ||
            p->preconditioner != RF_PC_NONE)
            return rf::fail(nullptr, RF_ERR_INVALID_ARG,
                            "row-block shards take the FP64 GMRES path with recomputed velocities and no block "
                            "preconditioner");
    }
    if (!finite_all(positions, 3 * (size_t)M) || !finite_all(orientations, 3 * (size_t)M))
        return rf::fail(nullptr, RF_ERR_NAN, "non-finite position or orientation");
    for (int i = 0; i < M; ++i) {
        const double *t = orientations + 3 * i;
        if (t[0] * t[0] + t[1] * t[1] + t[2] * t[2] < 1e-24)
            return rf::fail(nullptr, RF_ERR_INVALID_ARG, "zero orientation vector");
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return rf::fail(nullptr, RF_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (p->device < 0 || p->device >= ndev) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "bad device ordinal");

    rf_handle *h = new rf_handle;
    h->p = *p;
    if (h->p.pc_damping == 0.0) h->p.pc_damping = kPcDamping;
    h->M = M;
    h->N = N;
    h->LQ = 3 * NoQI;
    h->n = 3LL * N * M;
    h->shards = shards;
    h->shard = shards > 1 ? p->shard_index : 0;
    rf::shard_range(M, shards, h->shard, &h->t0, &h->t1);
    h->tpad = rf::shard_pad(M, shards);
    h->n_loc = 3LL * N * (h->t1 - h->t0);
    h->lda = round_up(h->n_loc, 64);   // the stored rows: this shard's (all of them unsharded)
    h->ldp = round_up(3LL * M, 64);
    h->device = p->device;
    auto bail = [&](cudaError_t err, const char *what) {
        rf_status s = rf::cuda_fail(nullptr, err, what);
        free_all(h);
        delete h;
        return s;
    };
#define CKC(expr, what)                           \
    do {                                          \
        cudaError_t e__ = (expr);                 \
        if (e__ != cudaSuccess) return bail(e__, what); \
    } while (0)
    CKC(cudaSetDevice(h->device), "cudaSetDevice");
    CKC(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device), "device query");
    CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    CKC(cudaEventCreate(&h->ev0), "event");
    CKC(cudaEventCreate(&h->ev1), "event");
    const size_t m3 = 3 * (size_t)M;
    for (int i = 0; i < 3; ++i) {
        CKC(dalloc(&h->X[i], m3), "alloc state");
        CKC(dalloc(&h->T[i], m3), "alloc state");
        CKC(cudaMemset(h->X[i], 0, m3 * 8), "memset");
        CKC(cudaMemset(h->T[i], 0, m3 * 8), "memset");
    }
    for (int i = 0; i < 2; ++i) {
        CKC(dalloc(&h->V[i], m3), "alloc state");
        CKC(dalloc(&h->W[i], m3), "alloc state");
        CKC(cudaMemset(h->V[i], 0, m3 * 8), "memset");
        CKC(cudaMemset(h->W[i], 0, m3 * 8), "memset");
    }
    make_tables(*p, h->tab_h);
    CKC(dalloc(&h->tab, 1), "alloc tables");
    CKC(cudaMemcpy(h->tab, &h->tab_h, sizeof(rf::Tables), cudaMemcpyHostToDevice), "upload tables");

    const size_t asz = (size_t)h->lda * (size_t)h->n;
    const int prec = p->precision;
    if (prec == RF_PREC_FP64) {
        CKC(dalloc(&h->A64, asz), "alloc A (FP64)");
        CKC(cudaMemset(h->A64, 0, asz * 8), "memset A");
    } else if (prec == RF_PREC_MIXED_BF16) {
        // split FP32 storage: the BF16 high plane (the inner solves' matrix)
        // and the low plane, 4 bytes per entry in all
        CKC(dalloc(&h->A16, 2 * asz), "alloc A (BF16 high and low planes)");
        CKC(cudaMemset(h->A16, 0, asz * 4), "memset A");
        h->A16lo = reinterpret_cast<unsigned short *>(h->A16) + asz;
        h->a_plane = (int64_t)asz;
    } else {
        CKC(dalloc(&h->A32, asz), "alloc A (FP32)");
        CKC(cudaMemset(h->A32, 0, asz * 4), "memset A");
    }
    // assembly chunking (from the whole system's targets also for a
    // row-block shard, so that its right-hand side sums the same source
    // chunks in the same order).  The FP64 assembly runs CTAs of 4 targets,
    // 4 resident per SM, the velocity kernel CTAs of 8 targets, 2 per SM: in
    // both the grid takes about rounds x sources per CTA, rounds =
    // (M / 4) x chunks / (4 SMs' worth of slots).  From a first guess of
    // about 8 CTAs of 8 targets per SM, the sources per CTA (within a factor
    // 4 below, but not below 16, and 2 above) that minimise that product;
    // ties: the larger share.  At M = 4000 on 148 SMs: 13 chunks of 308
    // sources (22 rounds, the last one nearly full) instead of 3 of 1334
    // (6 rounds, the sixth nearly empty).
    const int tiles = (M + 7) / 8;
    const int c0 = std::max(1, std::min(M, (h->sm_count * 8 + tiles - 1) / tiles));
    const int per0 = (M + c0 - 1) / c0;
    const int64_t ctas_x = (M + 3) / 4, slots = 4 * (int64_t)h->sm_count;
    int chunks = c0;
    {
        int64_t best_cost = -1;
        int best_share = per0;
        for (int per = std::max(std::min(per0, 16), per0 / 4); per <= 2 * per0 && per <= M; ++per) {
            const int c = (M + per - 1) / per;
            const int share = (M + c - 1) / c;
            const int64_t cost = ((ctas_x * c + slots - 1) / slots) * share;
            if (best_cost < 0 || cost < best_cost || (cost == best_cost && share > best_share)) {
                best_cost = cost;
                best_share = share;
                chunks = c;
            }
        }
    }
    h->asm_chunk = (M + chunks - 1) / chunks;
    h->asm_chunks = (M + h->asm_chunk - 1) / h->asm_chunk;
    h->vel_chunk = h->asm_chunk;
    h->vel_chunks = h->asm_chunks;
    CKC(dalloc(&h->b, h->n), "alloc b");
    CKC(dalloc(&h->x, h->n), "alloc x");
    CKC(cudaMemset(h->x, 0, h->n * 8), "memset x");
    CKC(cudaMemset(h->b, 0, h->n * 8), "memset b");
    CKC(dalloc(&h->bpart, (size_t)h->asm_chunks * h->n_loc), "alloc rhs partials");
    // the split assembly (FP32 far pairs, FP64 near pairs) for the reduced
    // precisions with analytic integration; near_field_c >= 1e30 asks for FP64
    // integrals everywhere and keeps the tile kernel
    h->split = prec != RF_PREC_FP64 && p->use_analytical_integration != 0 && rf::split_supported(N, h->LQ) &&
               !(prec != RF_PREC_FP32 && p->near_field_c >= 1e30);
    if (h->split) {
        h->far_chunks = rf::split_far_chunks(M, h->sm_count);
        h->far_chunk = (M + h->far_chunks - 1) / h->far_chunks;
        h->far_chunks = (M + h->far_chunk - 1) / h->far_chunk;
        CKC(dalloc(&h->far_contr, (size_t)h->far_chunks * M * 3 * (N + 1)), "alloc rhs partials");
        if (prec != RF_PREC_FP32) {
            const size_t words = (M + 31) / 32;
            CKC(dalloc(&h->near_bits, (size_t)M * words), "alloc near-pair bitmap");
            CKC(dalloc(&h->near_list, (size_t)M * M), "alloc near-pair lists");
            CKC(dalloc(&h->near_cnt, (size_t)M), "alloc near-pair counts");
            CKC(dalloc(&h->near_pref, (size_t)M * words), "alloc near-pair prefix counts");
            CKC(dalloc(&h->near_off, (size_t)M), "alloc near-pair offsets");
            CKC(dalloc(&h->near_total, 1), "alloc near-pair counter");
            CKC(dalloc(&h->near_contr, (size_t)M * 3 * (N + 1)), "alloc rhs partials");
        }
    }
    CKC(dalloc(&h->velpart, (size_t)h->vel_chunks * 6 * M), "alloc velocity partials");
    if (p->velocity_mode == RF_VEL_REUSE) {
        const size_t psz = (size_t)h->ldp * (size_t)h->n;
        if (prec == RF_PREC_FP64) {
            CKC(dalloc(&h->PV64, psz), "alloc velocity panel");
            CKC(dalloc(&h->PW64, psz), "alloc velocity panel");
            CKC(cudaMemset(h->PV64, 0, psz * 8), "memset panel");
            CKC(cudaMemset(h->PW64, 0, psz * 8), "memset panel");
        } else {
            CKC(dalloc(&h->PV32, psz), "alloc velocity panel");
            CKC(dalloc(&h->PW32, psz), "alloc velocity panel");
            CKC(cudaMemset(h->PV32, 0, psz * 4), "memset panel");
            CKC(cudaMemset(h->PW32, 0, psz * 4), "memset panel");
        }
        CKC(dalloc(&h->vpart, (size_t)h->asm_chunks * 6 * M), "alloc velocity partials");
        CKC(dalloc(&h->pvx, m3), "alloc");
        CKC(dalloc(&h->pwx, m3), "alloc");
    }
    // matvec workspace: the largest split buffer over the element sizes in use
    h->work_elems = std::max({rf::gemv_work_elems(h->lda, h->sm_count, 8), rf::gemv_work_elems(h->lda, h->sm_count, 4),
                              rf::gemv_work_elems(h->lda, h->sm_count, 2), rf::gemv_work_elems(h->ldp, h->sm_count, 8),
                              rf::gemv_work_elems(h->ldp, h->sm_count, 4)});
    CKC(dalloc(&h->work64, h->work_elems), "alloc matvec workspace");
    CKC(dalloc(&h->work32, h->work_elems), "alloc matvec workspace");
    CKC(dalloc(&h->dscal, 8), "alloc scalars");
    CKC(cudaMallocHost(&h->hscal, 8 * sizeof(double)), "alloc pinned scalars");
    h->rb.max_blocks = 1024;
    CKC(dalloc(&h->rb.partials, h->rb.max_blocks), "alloc reduction buffer");
    CKC(dalloc(&h->rb.counter, 1), "alloc reduction counter");
    CKC(cudaMemset(h->rb.counter, 0, sizeof(unsigned int)), "memset");
    const int m = p->gmres_restart;
    if (prec == RF_PREC_FP64) {
        h->gm64.reset(new rf::Gmres<double>());
        CKC(h->gm64->init(h->n, m, h->stream), "GMRES workspace");
    } else {
        h->gm32.reset(new rf::Gmres<float>());
        CKC(h->gm32->init(h->n, m, h->stream), "GMRES workspace");
        CKC(dalloc(&h->r64, h->n), "alloc");
        CKC(dalloc(&h->r32, h->n), "alloc");
        CKC(dalloc(&h->d32, h->n), "alloc");
        CKC(dalloc(&h->x32, h->n), "alloc");
    }
#undef CKC
    h->cur = 1;
    h->prev = 0;
    h->next = 2;
    rf_status s = rf_set_state(h, positions, orientations);
    if (s != RF_OK) {
        g_create_error = h->err;
        free_all(h);
        delete h;
        return s;
    }
    *out = h;
    return RF_OK;
}

rf_status rf_create_sharded(const rf_params *p, const double *positions, const double *orientations,
                            const uint8_t *nccl_id, rf_handle **out) {
    if (!out || !p || !nccl_id) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "null argument");
    rf_status s = rf_create(p, positions, orientations, out);
    if (s != RF_OK) return s;
    rf_handle *h = *out;
    h->shards = p->shard_count > 1 ? p->shard_count : 1;   // one shard: a communicator of one rank
    s = rf::shard_attach(h, nccl_id);
    if (s != RF_OK) {
        g_create_error = h->err;
        rf_destroy(h);
        *out = nullptr;
    }
    return s;
}

rf_status rf_destroy(rf_handle *h) {
    if (!h) return RF_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return RF_OK;
}

rf_status rf_set_state(rf_handle *h, const double *positions, const double *orientations) {
    if (!h || !positions || !orientations) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    const size_t m3 = 3 * (size_t)h->M;
    if (!finite_all(positions, m3) || !finite_all(orientations, m3))
        return rf::fail(h, RF_ERR_NAN, "non-finite position or orientation");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    CK(h, cudaMemcpyAsync(h->X[h->cur], positions, m3 * 8, cudaMemcpyHostToDevice, h->stream), "upload positions");
    CK(h, cudaMemcpyAsync(h->T[h->cur], orientations, m3 * 8, cudaMemcpyHostToDevice, h->stream),
       "upload orientations");
    // orientations are normalised as in advect_fibers.f90:332-340
    CK(h, rf::launch_normalize(h->M, h->T[h->cur], h->stream), "normalize");
    h->launches++;
    CK(h, cudaStreamSynchronize(h->stream), "sync");
    h->assembled = false;
    h->pc_ready = false;
    return RF_OK;
}

rf_status rf_assemble_system(rf_handle *h) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    rf::AsmArgs a{};
    a.M = h->M;
    a.N = h->N;
    a.LQ = h->LQ;
    a.t0 = h->t0;
    a.t1 = h->t1;
    a.n = h->n_loc;
    a.pos = h->X[h->cur];
    a.ori = h->T[h->cur];
    a.tab = h->tab;
    a.A64 = h->A64;
    a.A32 = h->A32;
    a.A16lo = h->A16lo;
    a.A16 = h->A16;
    a.lda = h->lda;
    a.bpart = h->bpart;
    a.PV64 = h->PV64;
    a.PW64 = h->PW64;
    a.PV32 = h->PV32;
    a.PW32 = h->PW32;
    a.ldp = h->ldp;
    a.vpart = h->vpart;
    a.chunk = h->asm_chunk;
    const int prec = h->p.precision;
    if (prec == RF_PREC_FP32) {
        a.near_c = 0.0;        // plain FP32 method: every pair in FP32
    } else {
        // FP64 below near_c: at least rf::kSplitMinNearC for the split kernels
        // (their FP32 far field runs the backward recursion, accurate there),
        // at least 10 for the tile kernel (whose FP32 points below 10 would run
        // the forward recursion)
        const double want = h->p.near_field_c > 0.0 ? h->p.near_field_c : rf::kSplitMinNearC;
        a.near_c = std::max(want, h->split ? rf::kSplitMinNearC : 10.0);
    }
    if (h->split) {
        rf::SplitArgs sa{};
        sa.M = h->M;
        sa.N = h->N;
        sa.LQ = h->LQ;
        sa.pos = a.pos;
        sa.ori = a.ori;
        sa.tab = h->tab;
        sa.A32 = h->A32;
        sa.A16lo = h->A16lo;
        sa.A16 = h->A16;
        sa.lda = h->lda;
        sa.PV32 = h->PV32;
        sa.PW32 = h->PW32;
        sa.ldp = h->ldp;
        sa.near_bits = h->near_bits;
        sa.words = (h->M + 31) / 32;
        sa.near_list = h->near_list;
        sa.near_cnt = h->near_cnt;
        sa.near_pref = h->near_pref;
        sa.near_off = h->near_off;
        sa.near_total = h->near_total;
        sa.far_contr = h->far_contr;
        sa.near_contr = h->near_contr;
        sa.chunk = h->far_chunk;
        sa.near_c = a.near_c;
        bool direct = false;
        if (h->near_bits) {
            CK(h, rf::launch_split_classify(sa, h->stream), "near-pair classification");
            // the near-pair count sizes the buffer of FP64-integrated blocks
            int *hcount = reinterpret_cast<int *>(h->hscal + 7);
            CK(h, cudaMemcpyAsync(hcount, h->near_total, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
               "near-pair count");
            CK(h, cudaStreamSynchronize(h->stream), "near-pair count");
            h->near_pairs = *hcount;
            if (h->near_pairs > h->near_cap) {
                // a reallocation of gigabytes costs hundreds of milliseconds and a
                // settling suspension keeps gaining near pairs, so grow to the
                // largest of twice the count, a quarter of all pairs and a quarter
                // of the free device memory (at most all pairs); on failure try
                // the count itself
                cudaFree(h->nearbuf);
                h->nearbuf = nullptr;
                h->near_cap = 0;
                const int64_t all = (int64_t)h->M * (h->M - 1);
                const int64_t rec = (int64_t)sizeof(float) * rf::kNearBlockFloats;
                size_t free_b = 0, total_b = 0;
                if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
                    (void)cudaGetLastError();
                    free_b = 0;
                }
                const int64_t want = std::max<int64_t>({2 * h->near_pairs + 1024, all / 4, (int64_t)(free_b / 4) / rec});
                for (int64_t cap : {std::min<int64_t>(all, want), std::min<int64_t>(all, h->near_pairs)}) {
                    if (cudaMalloc(&h->nearbuf, sizeof(float) * rf::kNearBlockFloats * (size_t)cap) == cudaSuccess) {
                        h->near_cap = cap;
                        break;
                    }
                    (void)cudaGetLastError();  // out of memory
                    h->nearbuf = nullptr;
                }
                // still none: the near kernel writes its blocks into A directly
            }
            direct = h->near_pairs > h->near_cap;
            sa.nearbuf = h->nearbuf;
            sa.merge = direct ? 0 : 1;
            if (!direct) CK(h, rf::launch_split_near(sa, false, h->stream), "near-pair kernel");
        }
        CK(h, rf::launch_split_far(sa, h->far_chunks, h->stream), "far-pair kernel");
        if (h->near_bits && direct) CK(h, rf::launch_split_near(sa, true, h->stream), "near-pair kernel");
        CK(h, rf::launch_split_finish(sa, h->far_chunks, h->b, h->vpart, h->stream), "rhs finish");
        h->vpart_chunks = 1;
        h->launches += h->near_bits ? 4 : 2;
    } else {
        // near_field_c >= 1e30 keeps every integral in FP64 for the mixed paths
        const int pmode = (prec == RF_PREC_FP64 || (prec != RF_PREC_FP32 && a.near_c >= 1e30)) ? rf::kPModeFP64
                                                                                              : rf::kPModeMixed;
        CK(h, rf::launch_assemble(a, h->p.use_analytical_integration == 0, pmode, h->asm_chunks, h->stream),
           "assemble kernel");
        CK(h, rf::launch_reduce_chunks(h->bpart, h->asm_chunks, h->n_loc, h->n_loc, h->b + 3LL * h->N * h->t0,
                                       h->stream),
           "rhs reduction");
        if (h->comm) CK(h, rf::shard_allgather(h, h->b, 3 * h->N, nullptr), "right-hand side exchange");
        h->vpart_chunks = h->asm_chunks;
        h->launches += 2;
    }
    if (h->p.preconditioner != RF_PC_NONE && (h->pc_skips > 0 || h->pc_age >= kPcExplore)) {
        if (h->pc_skips > 0) --h->pc_skips;
        h->pc_ready = false;
    } else if (h->p.preconditioner != RF_PC_NONE) {
        rf_status s = rf::build_preconditioner(h);
        if (s != RF_OK) return s;
    }
    CK(h, cudaStreamSynchronize(h->stream), "assembly");
    if (h->mlp_err && h->pc_ready && h->p.preconditioner == RF_PC_LEARNED) {
        int herr = 0;
        CK(h, cudaMemcpy(&herr, h->mlp_err, sizeof(int), cudaMemcpyDeviceToHost), "preconditioner status");
        if (herr) {
            h->pc_ready = false;
            return rf::fail(h, RF_ERR_DEVICE_TIMEOUT, "tensor-core MLP: an MMA wait timed out");
        }
    }
    h->assembled = true;
    return RF_OK;
}

rf_status rf_gemv_timer(rf_handle *h, int32_t enable, int64_t *count, double *total_ms, double *bytes_per_product) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    CK(h, gemv_timer_flush(h), "product timer");
    if (count) *count = h->gt.count;
    if (total_ms) *total_ms = h->gt.total_ms;
    if (bytes_per_product) *bytes_per_product = h->gt.bytes;
    if (enable) {
        h->gt.count = 0;
        h->gt.total_ms = 0.0;
    }
    h->gt.on = enable != 0;
    return RF_OK;
}

rf_status rf_solve_system(rf_handle *h) {
    if (!h) return RF_ERR_INVALID_ARG;
    if (!h->assembled) return rf::fail(h, RF_ERR_INVALID_ARG, "solve_system before assemble_system");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const int prec = h->p.precision;
    const int m = h->p.gmres_restart;
    const double tol = h->p.gmres_tol;
    const int maxit = h->p.gmres_max_iters;
    cudaStream_t st = h->stream;
    h->stats = rf_solve_stats();
    CK(h, cudaEventRecord(h->ev0, st), "event");
    const bool use_pc = h->p.preconditioner != RF_PC_NONE && h->pc_ready;
    // A preconditioned solve runs in trials of pc_trial Arnoldi steps, each
    // restarted from the current iterate; a trial that has not reduced the
    // residual tenfold ends the preconditioner for the rest of the solve, so
    // a poor block (a network's prediction far off its training data) costs
    // at most a trial and never the tolerance, while a good one on a hard
    // system (slow but steady) is kept.
    const int pc_trial = std::max(3 * m, 30);
    h->stats.preconditioned = use_pc ? 1 : 0;
    const double pc_omega = h->p.pc_damping;
    const int nb = 3 * h->N;
    rf::GmresResult res;
    rf_status status = RF_OK;
    if (prec == RF_PREC_FP64 && h->p.use_direct_solver) {
        // dgesv (coeffs_and_vels.f90:62,158): LU factors of a copy of A (A
        // itself stays available to rf_get_matrix and rf_matvec), then the two
        // triangular solves; the factors' buffer is made at the first call
        const size_t mat = sizeof(double) * (size_t)h->lda * (size_t)h->n;
        if (!h->LU) {
            CK(h, cudaMalloc(&h->LU, mat), "direct solver: LU factors (one more n x n FP64 matrix)");
            CK(h, cudaMalloc(&h->lu_r, sizeof(double) * h->n), "direct solver");
            CK(h, cudaMalloc(&h->lu_piv, sizeof(int) * h->n), "direct solver");
            CK(h, cudaMalloc(&h->lu_info, sizeof(int)), "direct solver");
        }
        if (!h->blas) {
            cublasHandle_t bh = nullptr;
            if (cublasCreate(&bh) != CUBLAS_STATUS_SUCCESS)
                return rf::fail(h, RF_ERR_CUDA, "direct solver: cuBLAS handle could not be created");
            h->blas = bh;
        }
        CK(h, cudaMemcpyAsync(h->LU, h->A64, mat, cudaMemcpyDeviceToDevice, st), "direct solver");
        CK(h, cudaMemcpyAsync(h->x, h->b, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, st), "direct solver");
        CK(h, rf::lu_factor(h->LU, h->lda, h->n, h->lu_piv, h->lu_info, h->blas, st, &h->launches),
           "LU factorisation");
        CK(h, rf::lu_solve(h->LU, h->lda, h->n, h->lu_piv, h->x, st, &h->launches), "LU solve");
        // backward error |b - A x| / |b| for the statistics
        CK(h, (rf::launch_gemv<double, double, double, double>(h->A64, h->lda, h->n, h->n, h->x, h->lu_r, h->b,
                                                                h->work64, h->work_elems, h->sm_count, st)),
           "direct solver residual");
        CK(h, rf::launch_dot<double>(h->n, h->lu_r, h->lu_r, h->dscal, h->rb, st), "direct solver residual");
        CK(h, rf::launch_dot<double>(h->n, h->b, h->b, h->dscal + 1, h->rb, st), "direct solver residual");
        h->launches += 4;
        int *hinfo = reinterpret_cast<int *>(h->hscal + 7);
        CK(h, cudaMemcpyAsync(h->hscal, h->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "direct solver");
        CK(h, cudaMemcpyAsync(hinfo, h->lu_info, sizeof(int), cudaMemcpyDeviceToHost, st), "direct solver");
        CK(h, cudaStreamSynchronize(st), "direct solver");
        const double rr = h->hscal[0], bb = h->hscal[1];
        if (!(std::isfinite(rr) && std::isfinite(bb)) && *hinfo == 0)
            return rf::fail(h, RF_ERR_NAN, "non-finite value in the linear system");
        h->stats.iterations = 0;
        h->stats.matvecs = 1;
        h->stats.residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
        h->stats.converged = *hinfo == 0;
        if (*hinfo != 0) {
            char msg[96];
            std::snprintf(msg, sizeof(msg), "singular matrix: LU pivot %d is zero", *hinfo);
            return rf::fail(h, RF_ERR_NOT_CONVERGED, msg);
        }
    } else if (prec == RF_PREC_FP64) {
        if (h->shards > 1 && !h->comm)
            return rf::fail(h, RF_ERR_INVALID_ARG, "a row-block shard solves with its communicator (rf_create_sharded)");
        rf::Gmres<double>::Op A = [h](const double *in, double *out) {
            h->launches += 2;
            if (h->comm) {
                // this shard's rows, then the row blocks of every shard
                cudaError_t e = timed_product(h, 8.0 * h->lda * h->n, [&] {
                    return rf::launch_gemv<double, double, double, double>(h->A64, h->lda, h->n_loc, h->n, in,
                                                                            h->shard_send, nullptr, h->work64,
                                                                            h->work_elems, h->sm_count, h->stream);
                });
                return e == cudaSuccess ? rf::shard_allgather(h, out, 3 * h->N, h->shard_send) : e;
            }
            return timed_product(h, 8.0 * h->lda * h->n, [&] {
                return rf::launch_gemv<double, double, double, double>(h->A64, h->lda, h->n, h->n, in, out, nullptr,
                                                                       h->work64, h->work_elems, h->sm_count,
                                                                       h->stream);
            });
        };
        rf::Gmres<double>::Op P = [h, nb, pc_omega](const double *in, double *out) {
            return rf::launch_pair_apply<double>(h->M, nb, h->pc_pairs, RF_MLP_PAIRS, h->Pblocks, h->knn, RF_MLP_K, pc_omega, in, out,
                                                  h->stream);
        };
        {
            bool pc_on = use_pc;
            double prev = 1.0;  // residual relative to |b| before this trial
            rf::GmresResult part;
            for (int used = 0;;) {
                const int budget = pc_on ? std::min(maxit - used, pc_trial) : maxit - used;
                CK(h, h->gm64->solve(A, pc_on ? &P : nullptr, h->b, h->x, false, tol, budget, &part), "GMRES");
                used += part.iterations;
                res.iterations += part.iterations;
                res.matvecs += part.matvecs;
                res.launches += part.launches;
                res.info = part.info;
                res.backward_error = part.backward_error;
                if (part.info != rf::kInfoBudget || used >= maxit || part.iterations == 0) break;
                if (pc_on && part.backward_error > 0.1 * prev) {
                    pc_on = false;
                    h->stats.pc_fallback = 1;
                }
                prev = part.backward_error;
            }
        }
        if (res.info == rf::kInfoNaN) return rf::fail(h, RF_ERR_NAN, "non-finite value in the linear system");
        h->launches += res.launches;
        h->stats.iterations = res.iterations;
        h->stats.matvecs = res.matvecs;
        h->stats.residual = res.backward_error;
        h->stats.converged = res.info == 0;
    } else if (prec == RF_PREC_FP32) {
        rf::Gmres<float>::Op A = [h](const float *in, float *out) {
            h->launches += 2;
            return timed_product(h, 4.0 * h->lda * h->n, [&] {
                return fp32_gemv<float, float, float>(h, in, out, nullptr, h->work32);
            });
        };
        rf::Gmres<float>::Op P = [h, nb, pc_omega](const float *in, float *out) {
            return rf::launch_pair_apply<float>(h->M, nb, h->pc_pairs, RF_MLP_PAIRS, h->Pblocks, h->knn, RF_MLP_K, pc_omega, in, out,
                                                 h->stream);
        };
        CK(h, (rf::launch_convert<float, double>(h->n, h->x, h->x32, st)), "convert");
        CK(h, (rf::launch_convert<float, double>(h->n, h->b, h->r32, st)), "convert");
        h->launches += 2;
        {
            bool pc_on = use_pc;
            double prev = 1.0;  // residual relative to |b| before this trial
            rf::GmresResult part;
            for (int used = 0;;) {
                const int budget = pc_on ? std::min(maxit - used, pc_trial) : maxit - used;
                CK(h, h->gm32->solve(A, pc_on ? &P : nullptr, h->r32, h->x32, false, tol, budget, &part), "GMRES");
                used += part.iterations;
                res.iterations += part.iterations;
                res.matvecs += part.matvecs;
                res.launches += part.launches;
                res.info = part.info;
                res.backward_error = part.backward_error;
                if (part.info != rf::kInfoBudget || used >= maxit || part.iterations == 0) break;
                if (pc_on && part.backward_error > 0.1 * prev) {
                    pc_on = false;
                    h->stats.pc_fallback = 1;
                }
                prev = part.backward_error;
            }
        }
        if (res.info == rf::kInfoNaN) return rf::fail(h, RF_ERR_NAN, "non-finite value in the linear system");
        CK(h, (rf::launch_convert<double, float>(h->n, h->x32, h->x, st)), "convert");
        h->launches += res.launches + 1;
        h->stats.iterations = res.iterations;
        h->stats.matvecs = res.matvecs;
        h->stats.residual = res.backward_error;
        h->stats.converged = res.info == 0;
    } else {
        // Mixed precision: inner GMRES on the low-precision matrix (FP32
        // vectors and accumulation, FP64 Hessenberg/Givens), outer iterative
        // refinement with the residual b - A x accumulated in FP64 against
        // the FP32-stored matrix.
        // BF16 while the refinements make progress, then the FP32 A
        bool bf16 = prec == RF_PREC_MIXED_BF16;
        rf::Gmres<float>::Op Alo = [h, &bf16](const float *in, float *out) {
            h->launches += 2;
            return timed_product(h, (bf16 ? 2.0 : 4.0) * h->lda * h->n, [&] {
                if (bf16)
                    return rf::launch_gemv<__nv_bfloat16, float, float, float>(h->A16, h->lda, h->n, h->n, in, out,
                                                                               nullptr, h->work32, h->work_elems,
                                                                               h->sm_count, h->stream);
                return fp32_gemv<float, float, float>(h, in, out, nullptr, h->work32);
            });
        };
        rf::Gmres<float>::Op P = [h, nb, pc_omega](const float *in, float *out) {
            return rf::launch_pair_apply<float>(h->M, nb, h->pc_pairs, RF_MLP_PAIRS, h->Pblocks, h->knn, RF_MLP_K, pc_omega, in, out,
                                                 h->stream);
        };
        // the same operators for the device-controlled inner solve: their
        // kernels return at once once the solve has stopped
        rf::Gmres<float>::StopOp Alo_s = [h, &bf16](const float *in, float *out, const int *stop) {
            h->launches += 2;
            return timed_product(h, (bf16 ? 2.0 : 4.0) * h->lda * h->n, [&] {
                if (bf16)
                    return rf::launch_gemv<__nv_bfloat16, float, float, float>(h->A16, h->lda, h->n, h->n, in, out,
                                                                               nullptr, h->work32, h->work_elems,
                                                                               h->sm_count, h->stream, stop);
                return fp32_gemv<float, float, float>(h, in, out, nullptr, h->work32, stop);
            });
        };
        rf::Gmres<float>::StopOp P_s = [h, nb, pc_omega](const float *in, float *out, const int *stop) {
            return rf::launch_pair_apply<float>(h->M, nb, h->pc_pairs, RF_MLP_PAIRS, h->Pblocks, h->knn, RF_MLP_K, pc_omega, in, out,
                                                 h->stream, stop);
        };
        // a product queued after the inner solve stopped returns at once: not a product to time
        auto drop_skipped = [h] {
            if (h->gt.on && h->gt.used >= 2) h->gt.used -= 2;
        };
        const bool device_control = m <= rf::kArnoldiMax;
        double *dnorm = h->dscal;
        const rf::RedBuf &rb = h->rb;
        auto norm_of = [&](const double *v, double *hv) -> cudaError_t {
            cudaError_t e = rf::launch_dot<double>(h->n, v, v, dnorm, rb, st);
            if (e != cudaSuccess) return e;
            h->launches++;
            e = cudaMemcpyAsync(h->hscal, dnorm, sizeof(double), cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return e;
            e = cudaStreamSynchronize(st);
            *hv = std::sqrt(h->hscal[0]);
            return e;
        };
        auto residual = [&]() -> cudaError_t {  // r64 = b - A32 x (FP64 accumulation)
            h->launches += 2;
            h->stats.matvecs++;
            return fp32_gemv<double, double, double>(h, h->x, h->r64, h->b, h->work64);
        };
        double bn = 0.0, rn = 0.0;
        cudaError_t e = norm_of(h->b, &bn);
        // Start from the previous step's solution only while that pays: on a
        // sedimenting cloud it leaves 40-70 % of |b| (the near-field
        // couplings change too much in one step), less than one inner
        // iteration saves, and checking it costs an FP32-matrix product.
        // After a poor warm start the next kWarmRetry solves start from zero,
        // after a second one twice as many, up to kWarmRetryMax; a handle
        // without a previous solution (none solved or restored yet) starts
        // from zero without the check.
        const bool warm = h->x_valid && h->cold_solves == 0;
        if (warm) {
            if (e == cudaSuccess) e = residual();
            if (e == cudaSuccess) e = norm_of(h->r64, &rn);
            if (e == cudaSuccess && bn > 0.0 && rn > 0.1 * bn) {
                h->cold_solves = h->warm_wait;
                h->warm_wait = std::min(2 * h->warm_wait, kWarmRetryMax);
            } else {
                h->warm_wait = kWarmRetry;
            }
        } else {
            if (h->cold_solves > 0) --h->cold_solves;
            if (e == cudaSuccess) e = cudaMemsetAsync(h->x, 0, sizeof(double) * h->n, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(h->r64, h->b, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, st);
            rn = bn;
        }
        if (e == cudaSuccess && !(std::isfinite(bn) && std::isfinite(rn)))
            return rf::fail(h, RF_ERR_NAN, "non-finite value in the linear system");
        int it = 0, iters = 0;
        bool pc_on = use_pc;
        const int max_ref = h->p.max_refinements > 0 ? h->p.max_refinements : 30;
        const double itol = h->p.inner_tol > 0.0 ? std::min(h->p.inner_tol, 0.5) : 1e-3;
        while (e == cudaSuccess && bn > 0.0 && rn / bn > tol && it < max_ref && iters < maxit * max_ref) {
            // d = argmin |r/rn - A_lo d|, then x += rn * d
            e = rf::launch_scale_h<float, double>(h->n, h->r64, 1.0 / rn, h->r32, st);
            if (e != cudaSuccess) break;
            h->launches++;
            e = cudaMemsetAsync(h->d32, 0, sizeof(float) * h->n, st);
            if (e != cudaSuccess) break;
            // Plan the refinements: the fewest whose inner solves reduce the
            // residual by no more than inner_tol each (the deepest an inner
            // solve goes) reach the tolerance with a factor 2 of margin; this
            // inner solve asks for an equal share of the reduction still
            // needed.  Each refinement costs an FP32-matrix product for its
            // residual, so fewer and deeper inner solves are cheaper.
            const double need = 0.5 * tol * bn / rn;
            const int left = std::max(1, (int)std::ceil(std::log(need) / std::log(itol) - 1e-9));
            const double itol_k = std::min(0.5, std::pow(need, 1.0 / left));
            const int budget = pc_on ? std::min(maxit, pc_trial) : maxit;
            if (device_control)
                e = h->gm32->solve_device(Alo_s, pc_on ? &P_s : nullptr, h->r32, h->d32, itol_k, budget, &res,
                                          drop_skipped);
            else
                e = h->gm32->solve(Alo, pc_on ? &P : nullptr, h->r32, h->d32, true, itol_k, budget, &res, false);
            if (e != cudaSuccess) break;
            if (res.info == rf::kInfoNaN) return rf::fail(h, RF_ERR_NAN, "non-finite value in the linear system");
            // a preconditioned inner solve that spent its trial keeps its partial
            // correction (the residual is recomputed below); without a tenfold
            // reduction (the Arnoldi estimate, relative to the unit right-hand
            // side) the rest of this solve runs without the preconditioner
            const bool pc_failed = pc_on && res.info == rf::kInfoBudget && budget < maxit && res.backward_error > 0.1;
            if (pc_failed) {
                pc_on = false;
                h->stats.pc_fallback = 1;
            }
            h->launches += res.launches;
            iters += res.iterations;
            h->stats.matvecs += res.matvecs;
            e = rf::launch_axpy_fd(h->n, rn, h->d32, h->x, st);
            if (e != cudaSuccess) break;
            h->launches++;
            const double rn_prev = rn;
            e = residual();
            if (e == cudaSuccess) e = norm_of(h->r64, &rn);
            ++it;
            // A refinement reduces the residual by about max(its inner
            // tolerance, |I - A A_lo^-1|); less than half (when it asked for
            // much more) means the stored BF16 matrix is too far from A for
            // this system (its condition times BF16's 2^-9 near 1): the FP32
            // A takes over.
            if (e == cudaSuccess && bf16 && res.info == 0 && rn > std::max(0.5, 4.0 * itol_k) * rn_prev) {
                bf16 = false;
                h->stats.precision_fallback = 1;
            }
        }
        CK(h, e, "mixed-precision solve");
        h->x_valid = true;
        h->stats.iterations = iters;
        h->stats.refinements = it;
        h->stats.residual = bn > 0.0 ? rn / bn : 0.0;
        h->stats.converged = bn == 0.0 || rn / bn <= tol;
    }
    CK(h, cudaEventRecord(h->ev1, st), "event");
    CK(h, cudaEventSynchronize(h->ev1), "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.seconds = ms * 1e-3;
    if (h->p.preconditioner != RF_PC_NONE && h->stats.converged) {
        double &mean = h->pc_its[use_pc ? 1 : 0];
        mean = mean < 0.0 ? h->stats.iterations : 0.5 * (mean + h->stats.iterations);
        if (!use_pc) {
            h->pc_age = 0;
        } else {
            ++h->pc_age;
            if (h->stats.pc_fallback || (h->pc_its[0] >= 0.0 && h->pc_its[1] > 1.05 * h->pc_its[0]))
                h->pc_skips = kPcRetry;
        }
    }
    if (!h->stats.converged) status = rf::fail(h, RF_ERR_NOT_CONVERGED, "GMRES budget spent above tolerance");
    return status;
}

rf_status rf_update_velocities(rf_handle *h) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = h->stream;
    double *V = h->V[h->vcur], *W = h->W[h->vcur];
    if (h->p.velocity_mode == RF_VEL_REUSE) {
        if (!h->assembled) return rf::fail(h, RF_ERR_INVALID_ARG, "reuse velocities need an assembled system");
        const int64_t m3 = 3LL * h->M;
        if (h->PV64) {
            CK(h, (rf::launch_gemv<double, double, double, double>(h->PV64, h->ldp, m3, h->n, h->x, h->pvx, nullptr,
                                                                    h->work64, h->work_elems, h->sm_count, st)),
               "velocity panel");
            CK(h, (rf::launch_gemv<double, double, double, double>(h->PW64, h->ldp, m3, h->n, h->x, h->pwx, nullptr,
                                                                    h->work64, h->work_elems, h->sm_count, st)),
               "velocity panel");
        } else {
            CK(h, (rf::launch_gemv<float, double, double, double>(h->PV32, h->ldp, m3, h->n, h->x, h->pvx, nullptr,
                                                                   h->work64, h->work_elems, h->sm_count, st)),
               "velocity panel");
            CK(h, (rf::launch_gemv<float, double, double, double>(h->PW32, h->ldp, m3, h->n, h->x, h->pwx, nullptr,
                                                                   h->work64, h->work_elems, h->sm_count, st)),
               "velocity panel");
        }
        CK(h, rf::launch_velocity_reuse_finish(h->M, h->T[h->cur], h->tab, h->pvx, h->pwx, h->vpart, h->vpart_chunks,
                                               V, W, st),
           "velocity finish");
        h->launches += 5;
    } else {
        rf::VelArgs a{};
        a.M = h->M;
        a.t0 = h->t0;
        a.t1 = h->t1;
        a.N = h->N;
        a.LQ = h->LQ;
        a.pos = h->X[h->cur];
        a.ori = h->T[h->cur];
        a.coeffs = h->x;
        a.tab = h->tab;
        a.part = h->velpart;
        a.chunk = h->vel_chunk;
        CK(h, rf::launch_velocity(a, h->p.use_analytical_integration == 0, h->vel_chunks, st), "velocity kernel");
        CK(h, rf::launch_velocity_finish(h->M, h->t0, h->t1, h->T[h->cur], h->tab, h->velpart, h->vel_chunks, V, W,
                                         st),
           "velocity finish");
        if (h->comm) {
            CK(h, rf::shard_allgather(h, V, 3, nullptr), "velocity exchange");
            CK(h, rf::shard_allgather(h, W, 3, nullptr), "velocity exchange");
        }
        h->launches += 2;
    }
    CK(h, cudaStreamSynchronize(st), "velocities");
    h->vlast = h->vcur;
    return RF_OK;
}

rf_status rf_update_fibers(rf_handle *h, int first_timestep) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    CK(h, rf::launch_advect(h->M, h->p.timestep, first_timestep != 0, h->X[h->prev], h->X[h->cur], h->T[h->prev],
                            h->T[h->cur], h->V[h->vcur], h->V[h->vprev], h->W[h->vcur], h->W[h->vprev],
                            h->X[h->next], h->T[h->next], h->stream),
       "advect");
    h->launches++;
    CK(h, cudaStreamSynchronize(h->stream), "advect");
    // DoubleSwap of velocities and TripleSwap of state (src/simulation.cu:294-298)
    std::swap(h->vprev, h->vcur);
    const int old_prev = h->prev;
    h->prev = h->cur;
    h->cur = h->next;
    h->next = old_prev;
    h->assembled = false;
    h->pc_ready = false;
    return RF_OK;
}

rf_status rf_step(rf_handle *h, size_t current_timestep) {
    rf_status s = rf_assemble_system(h);
    if (s != RF_OK) return s;
    rf_status solve = rf_solve_system(h);
    if (solve != RF_OK && solve != RF_ERR_NOT_CONVERGED) return solve;
    s = rf_update_velocities(h);
    if (s != RF_OK) return s;
    s = rf_update_fibers(h, current_timestep == 0);
    if (s != RF_OK) return s;
    return solve;
}

rf_status rf_get_state(rf_handle *h, double *positions, double *orientations) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t m3 = 3 * (size_t)h->M;
    if (positions)
        CK(h, cudaMemcpyAsync(positions, h->X[h->cur], m3 * 8, cudaMemcpyDeviceToHost, h->stream), "download");
    if (orientations)
        CK(h, cudaMemcpyAsync(orientations, h->T[h->cur], m3 * 8, cudaMemcpyDeviceToHost, h->stream), "download");
    CK(h, cudaStreamSynchronize(h->stream), "download");
    return RF_OK;
}

rf_status rf_get_velocities(rf_handle *h, double *translational, double *rotational) {
    if (!h) return RF_ERR_INVALID_ARG;
    if (h->vlast < 0) return rf::fail(h, RF_ERR_INVALID_ARG, "no velocities computed yet");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t m3 = 3 * (size_t)h->M;
    if (translational)
        CK(h, cudaMemcpyAsync(translational, h->V[h->vlast], m3 * 8, cudaMemcpyDeviceToHost, h->stream), "download");
    if (rotational)
        CK(h, cudaMemcpyAsync(rotational, h->W[h->vlast], m3 * 8, cudaMemcpyDeviceToHost, h->stream), "download");
    CK(h, cudaStreamSynchronize(h->stream), "download");
    return RF_OK;
}

rf_status rf_get_coeffs(rf_handle *h, double *x) {
    if (!h || !x) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    CK(h, cudaMemcpy(x, h->x, h->n * 8, cudaMemcpyDeviceToHost), "download");
    return RF_OK;
}

rf_status rf_get_rhs(rf_handle *h, double *b) {
    if (!h || !b) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    CK(h, cudaMemcpy(b, h->b, h->n * 8, cudaMemcpyDeviceToHost), "download");
    return RF_OK;
}

rf_status rf_get_matrix(rf_handle *h, double *A) {
    if (!h || !A) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    if (h->shards > 1) return rf::fail(h, RF_ERR_INVALID_ARG, "a row-block shard holds its rows only: rf_get_matrix_rows");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const int64_t n = h->n;
    double *col = nullptr;
    CK(h, cudaMalloc(&col, sizeof(double) * h->lda), "alloc");
    cudaError_t e = cudaSuccess;
    for (int64_t c = 0; c < n && e == cudaSuccess; ++c) {
        if (h->A64) {
            e = cudaMemcpyAsync(A + c * n, h->A64 + c * h->lda, n * 8, cudaMemcpyDeviceToHost, h->stream);
        } else {
            e = h->A16lo ? rf::launch_gather_rows<rf::SplitF32>(reinterpret_cast<const rf::SplitF32 *>(h->A16) +
                                                                    c * h->lda, h->lda, 0, n, 1, col, h->stream,
                                                                h->a_plane)
                         : rf::launch_convert<double, float>(n, h->A32 + c * h->lda, col, h->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(A + c * n, col, n * 8, cudaMemcpyDeviceToHost, h->stream);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(col);
    CK(h, e, "download matrix");
    return RF_OK;
}

rf_status rf_get_matrix_rows(rf_handle *h, int32_t which, int64_t row0, int64_t rows, double *out) {
    if (!h || !out) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    if (which != 0 && which != 1) return rf::fail(h, RF_ERR_INVALID_ARG, "which must be 0 or 1");
    const int64_t first = 3LL * h->N * h->t0;   // the stored rows are the system's rows [first, first + n_loc)
    if (row0 < first || rows < 1 || row0 + rows > first + h->n_loc)
        return rf::fail(h, RF_ERR_INVALID_ARG, "rows out of range (or outside this handle's row-block shard)");
    if (!h->assembled) return rf::fail(h, RF_ERR_INVALID_ARG, "no assembled system");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    row0 -= first;
    double *dev = nullptr;
    const size_t bytes = sizeof(double) * (size_t)rows * (size_t)h->n;
    CK(h, cudaMalloc(&dev, bytes), "row block");
    cudaError_t e;
    if (which == 1 && h->A16)
        e = rf::launch_gather_rows<__nv_bfloat16>(h->A16, h->lda, row0, rows, h->n, dev, h->stream);
    else if (h->A16lo)
        e = rf::launch_gather_rows<rf::SplitF32>(reinterpret_cast<const rf::SplitF32 *>(h->A16), h->lda, row0, rows,
                                                 h->n, dev, h->stream, h->a_plane);
    else if (h->A64)
        e = rf::launch_gather_rows<double>(h->A64, h->lda, row0, rows, h->n, dev, h->stream);
    else
        e = rf::launch_gather_rows<float>(h->A32, h->lda, row0, rows, h->n, dev, h->stream);
    h->launches += 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dev, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dev);
    CK(h, e, "download row block");
    return RF_OK;
}

rf_status rf_matvec(rf_handle *h, const double *x, double *y) {
    if (!h || !x || !y) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    if (h->shards > 1) return rf::fail(h, RF_ERR_INVALID_ARG, "rf_matvec needs the whole system (not a row-block shard)");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    double *dx = nullptr, *dy = nullptr;
    CK(h, cudaMalloc(&dx, h->n * 8), "alloc");
    cudaError_t e = cudaMalloc(&dy, h->n * 8);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, h->n * 8, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        if (h->A64)
            e = rf::launch_gemv<double, double, double, double>(h->A64, h->lda, h->n, h->n, dx, dy, nullptr, h->work64,
                                                                h->work_elems, h->sm_count, h->stream);
        else if (h->A16)
            e = rf::launch_gemv<__nv_bfloat16, double, double, double>(h->A16, h->lda, h->n, h->n, dx, dy, nullptr,
                                                                       h->work64, h->work_elems, h->sm_count,
                                                                       h->stream);
        else
            e = rf::launch_gemv<float, double, double, double>(h->A32, h->lda, h->n, h->n, dx, dy, nullptr, h->work64,
                                                               h->work_elems, h->sm_count, h->stream);
        h->launches += 2;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, h->n * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dx);
    cudaFree(dy);
    CK(h, e, "matvec");
    return RF_OK;
}

rf_status rf_dgesv(int64_t n, const double *A, int64_t lda, const double *b, double *x, int32_t *ipiv,
                   int32_t *info, int32_t device) {
    if (!A || !b || !x || !info) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "rf_dgesv: null pointer");
    if (n < 1 || lda < n || n > INT32_MAX) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "rf_dgesv: need 1 <= n <= lda");
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return rf::fail(nullptr, RF_ERR_NO_DEVICE, "rf_dgesv: no such CUDA device");
    }
    // everything this call makes, released on every return path
    struct Scope {
        int prev;
        cudaStream_t st = nullptr;
        cublasHandle_t blas = nullptr;
        double *dA = nullptr, *dx = nullptr;
        int *dpiv = nullptr, *dinfo = nullptr;
        ~Scope() {
            if (st) cudaStreamSynchronize(st);
            cudaFree(dA);
            cudaFree(dx);
            cudaFree(dpiv);
            cudaFree(dinfo);
            if (blas) cublasDestroy(blas);
            if (st) cudaStreamDestroy(st);
            cudaSetDevice(prev);
        }
    } sc{prev};
    auto cuda = [](cudaError_t e, const char *what) {
        cudaGetLastError();
        return rf::fail(nullptr, e == cudaErrorMemoryAllocation ? RF_ERR_OOM : RF_ERR_CUDA,
                        std::string("rf_dgesv: ") + what + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaStreamCreateWithFlags(&sc.st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda(e, "stream");
    const size_t nn = (size_t)n;
    if ((e = cudaMalloc(&sc.dA, sizeof(double) * nn * nn)) != cudaSuccess) return cuda(e, "device copy of A");
    if ((e = cudaMalloc(&sc.dx, sizeof(double) * nn)) != cudaSuccess ||
        (e = cudaMalloc(&sc.dpiv, sizeof(int) * nn)) != cudaSuccess ||
        (e = cudaMalloc(&sc.dinfo, sizeof(int))) != cudaSuccess)
        return cuda(e, "device buffers");
    if (cublasCreate(&sc.blas) != CUBLAS_STATUS_SUCCESS)
        return rf::fail(nullptr, RF_ERR_CUDA, "rf_dgesv: cuBLAS handle could not be created");
    if ((e = cudaMemcpy2DAsync(sc.dA, sizeof(double) * nn, A, sizeof(double) * (size_t)lda, sizeof(double) * nn, nn,
                               cudaMemcpyHostToDevice, sc.st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(sc.dx, b, sizeof(double) * nn, cudaMemcpyHostToDevice, sc.st)) != cudaSuccess)
        return cuda(e, "upload");
    int64_t launches = 0;
    if ((e = rf::lu_factor(sc.dA, n, n, sc.dpiv, sc.dinfo, sc.blas, sc.st, &launches)) != cudaSuccess)
        return cuda(e, "LU factorisation");
    int hinfo = 0;
    if ((e = cudaMemcpyAsync(&hinfo, sc.dinfo, sizeof(int), cudaMemcpyDeviceToHost, sc.st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(sc.st)) != cudaSuccess)
        return cuda(e, "LU factorisation");
    *info = hinfo;
    if (hinfo == 0) {
        if ((e = rf::lu_solve(sc.dA, n, n, sc.dpiv, sc.dx, sc.st, &launches)) != cudaSuccess)
            return cuda(e, "LU solve");
        if ((e = cudaMemcpyAsync(x, sc.dx, sizeof(double) * nn, cudaMemcpyDeviceToHost, sc.st)) != cudaSuccess)
            return cuda(e, "download");
    }
    if (ipiv) {
        std::vector<int> hp(nn);
        if ((e = cudaMemcpyAsync(hp.data(), sc.dpiv, sizeof(int) * nn, cudaMemcpyDeviceToHost, sc.st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(sc.st)) != cudaSuccess)
            return cuda(e, "download");
        for (size_t i = 0; i < nn; ++i) ipiv[i] = hp[i] + 1;
    }
    if ((e = cudaStreamSynchronize(sc.st)) != cudaSuccess) return cuda(e, "LU solve");
    return RF_OK;
}

rf_status rf_matvec_free(rf_handle *h, const double *x, double *y) {
    if (!h || !x || !y) return rf::fail(h, RF_ERR_INVALID_ARG, "null argument");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (!h->mfpart)
        CK(h, cudaMalloc(&h->mfpart, sizeof(double) * (size_t)h->vel_chunks * h->n), "matrix-free product partials");
    double *dx = nullptr, *dy = nullptr;
    CK(h, cudaMalloc(&dx, h->n * 8), "alloc");
    cudaError_t e = cudaMalloc(&dy, h->n * 8);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, h->n * 8, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        rf::MatfreeArgs a{};
        a.M = h->M;
        a.N = h->N;
        a.LQ = h->LQ;
        a.n = h->n;
        a.pos = h->X[h->cur];
        a.ori = h->T[h->cur];
        a.x = dx;
        a.tab = h->tab;
        a.part = h->mfpart;
        a.chunk = h->vel_chunk;
        e = rf::launch_matfree(a, h->p.use_analytical_integration == 0, h->vel_chunks, dx, dy, h->stream);
        h->launches += 2;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, h->n * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dx);
    cudaFree(dy);
    CK(h, e, "matrix-free product");
    return RF_OK;
}

rf_status rf_get_solve_stats(rf_handle *h, rf_solve_stats *s) {
    if (!h || !s) return RF_ERR_INVALID_ARG;
    *s = h->stats;
    return RF_OK;
}

rf_status rf_get_history(rf_handle *h, double *prev_pos, double *prev_orient, double *prev_vel, double *prev_rot) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t m3 = 3 * (size_t)h->M * 8;
    if (prev_pos) CK(h, cudaMemcpy(prev_pos, h->X[h->prev], m3, cudaMemcpyDeviceToHost), "download");
    if (prev_orient) CK(h, cudaMemcpy(prev_orient, h->T[h->prev], m3, cudaMemcpyDeviceToHost), "download");
    if (prev_vel) CK(h, cudaMemcpy(prev_vel, h->V[h->vprev], m3, cudaMemcpyDeviceToHost), "download");
    if (prev_rot) CK(h, cudaMemcpy(prev_rot, h->W[h->vprev], m3, cudaMemcpyDeviceToHost), "download");
    return RF_OK;
}

rf_status rf_set_history(rf_handle *h, const double *prev_pos, const double *prev_orient, const double *prev_vel,
                         const double *prev_rot, const double *coeffs) {
    if (!h) return RF_ERR_INVALID_ARG;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t m3 = 3 * (size_t)h->M * 8;
    if (prev_pos) CK(h, cudaMemcpy(h->X[h->prev], prev_pos, m3, cudaMemcpyHostToDevice), "upload");
    if (prev_orient) CK(h, cudaMemcpy(h->T[h->prev], prev_orient, m3, cudaMemcpyHostToDevice), "upload");
    if (prev_vel) CK(h, cudaMemcpy(h->V[h->vprev], prev_vel, m3, cudaMemcpyHostToDevice), "upload");
    if (prev_rot) CK(h, cudaMemcpy(h->W[h->vprev], prev_rot, m3, cudaMemcpyHostToDevice), "upload");
    if (coeffs) {
        CK(h, cudaMemcpy(h->x, coeffs, h->n * 8, cudaMemcpyHostToDevice), "upload");
        h->x_valid = true;
    }
    return RF_OK;
}

rf_status rf_timer_mark(rf_handle *h, int32_t slot) {
    if (!h || slot < 0 || slot >= 16) return rf::fail(h, RF_ERR_INVALID_ARG, "timer slot must be 0..15");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (!h->marks[slot]) CK(h, cudaEventCreate(&h->marks[slot]), "event");
    CK(h, cudaEventRecord(h->marks[slot], h->stream), "event record");
    return RF_OK;
}

double rf_timer_elapsed_ms(rf_handle *h, int32_t from, int32_t to) {
    if (!h || from < 0 || from >= 16 || to < 0 || to >= 16 || !h->marks[from] || !h->marks[to]) return -1.0;
    if (cudaSetDevice(h->device) != cudaSuccess) return -1.0;
    if (cudaEventSynchronize(h->marks[to]) != cudaSuccess) return -1.0;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->marks[from], h->marks[to]) != cudaSuccess) return -1.0;
    return ms;
}

rf_status rf_profile_matvec(rf_handle *h, int32_t reps, double *ms_per_product, double *bytes) {
    if (!h || reps < 1 || !ms_per_product) return rf::fail(h, RF_ERR_INVALID_ARG, "bad argument");
    if (h->shards > 1) return rf::fail(h, RF_ERR_INVALID_ARG, "rf_profile_matvec needs the whole system");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const int64_t n = h->n;
    void *xv = nullptr, *yv = nullptr;
    CK(h, cudaMalloc(&xv, n * 8), "alloc");
    cudaError_t e = cudaMalloc(&yv, n * 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(xv, 0, n * 8, h->stream);
    double elem = 8.0;
    if (e == cudaSuccess) e = cudaEventRecord(h->ev0, h->stream);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        if (h->A64) {
            e = rf::launch_gemv<double, double, double, double>(h->A64, h->lda, n, n, (double *)xv, (double *)yv,
                                                                nullptr, h->work64, h->work_elems, h->sm_count,
                                                                h->stream);
            elem = 8.0;
        } else if (h->A16) {
            e = rf::launch_gemv<__nv_bfloat16, float, float, float>(h->A16, h->lda, n, n, (float *)xv, (float *)yv,
                                                                    nullptr, h->work32, h->work_elems, h->sm_count,
                                                                    h->stream);
            elem = 2.0;
        } else {
            e = rf::launch_gemv<float, float, float, float>(h->A32, h->lda, n, n, (float *)xv, (float *)yv, nullptr,
                                                            h->work32, h->work_elems, h->sm_count, h->stream);
            elem = 4.0;
        }
        h->launches += 2;
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->ev1, h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(h->ev1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    cudaFree(xv);
    cudaFree(yv);
    CK(h, e, "profile matvec");
    *ms_per_product = ms / reps;
    if (bytes) *bytes = elem * (double)h->lda * (double)n;
    return RF_OK;
}

int64_t rf_system_size(const rf_handle *h) { return h ? h->n : 0; }
int64_t rf_matrix_ld(const rf_handle *h) { return h ? h->lda : 0; }
void *rf_get_stream(rf_handle *h) { return h ? (void *)h->stream : nullptr; }
int64_t rf_kernel_launches(const rf_handle *h) { return h ? h->launches : 0; }

}  // extern "C"
