/*
 * rigidfibers.h - C ABI of the B200-native rigid-fiber slender-body solver.
 *
 * One handle owns one simulation on one GPU: the fiber state (triple-buffered
 * positions and orientations, double-buffered velocities), the dense system
 * A x = b, the Krylov workspace and the preconditioner.  Every entry point is
 * synchronous at return, takes and returns plain host pointers, and reports a
 * status code; none calls exit().  Handles are independent (one CUDA stream
 * each) and may be used from different host threads; one handle must not be
 * used from two threads at once.
 *
 * Reference interface that each entry point replaces (paths inside
 * ericwolter/rigidfibers_kth):
 *   Simulation(Configuration)          src/simulation.h:39, src/simulation.cu:40-53
 *   Simulation::step(size_t)           src/simulation.h:42, src/simulation.cu:279-301
 *   Simulation::assembleSystem()       src/simulation.h:79, src/simulation.cu:303-322
 *   Simulation::solveSystem()          src/simulation.h:80, src/simulation.cu:324-351
 *   Simulation::updateVelocities()     src/simulation.h:81, src/simulation.cu:353-384
 *   Simulation::updateFibers(bool)     src/simulation.h:82, src/simulation.cu:386-424
 *   FiberParams                        src/common.h:49-68
 *   Parameters::parse*File             src/parameters.cc:24-227
 * and the Fortran boundary solve_coeffs*_ / compute_velocities*
 * (fortran/coeffs_and_vels.f90:10-746) that the same calls cover.
 *
 * Index conventions (identical to the reference):
 *   fiber state      double[3*M], (x,y,z) of fiber 0, then fiber 1, ...
 *   coefficients     n = 3*N*M, index (i*N + k)*3 + d   (fiber i, term k+1, axis d)
 *   system matrix    n x n column-major, A[row + col*n]
 */
#ifndef RIGIDFIBERS_H_
#define RIGIDFIBERS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* every declaration below is exported from librigidfibers.so */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define RF_ABI_VERSION 1

typedef enum rf_status {
    RF_OK = 0,
    RF_ERR_INVALID_ARG = 1,   /* bad size, null pointer, unsupported option */
    RF_ERR_OOM = 2,           /* device allocation failed */
    RF_ERR_CUDA = 3,          /* CUDA runtime error; see rf_last_error() */
    RF_ERR_NOT_CONVERGED = 4, /* GMRES budget spent above tolerance (state still advanced) */
    RF_ERR_DEVICE_TIMEOUT = 5,/* a bounded device wait gave up */
    RF_ERR_NAN = 6,           /* non-finite value in inputs or results */
    RF_ERR_NO_DEVICE = 7      /* no CUDA device / driver */
} rf_status;

/* Storage precision of A and arithmetic of the solve. */
typedef enum rf_precision {
    RF_PREC_FP64 = 0,        /* plain method: FP64 assembly, FP64 A, FP64 GMRES */
    RF_PREC_FP32 = 1,        /* plain method in FP32 (reference "float" build) */
    RF_PREC_MIXED_BF16 = 2,  /* BF16 A for inner GMRES (FP32 accumulate), FP32 A for FP64-residual refinement,
                                held as two 16-bit planes (the BF16 matrix, rounded half away from
                                zero, and the low halves of the FP32 words: 4 bytes per entry);
                                a refinement that reduces the residual by less than half (BF16's
                                2^-9 relative error times the condition of A near 1: fibers that
                                nearly touch) switches the rest of that solve's inner products to
                                the FP32 A (rf_solve_stats.precision_fallback) */
    RF_PREC_MIXED_FP32 = 3   /* FP32 A for inner GMRES and for the FP64-residual refinement */
} rf_precision;

typedef enum rf_preconditioner {
    RF_PC_NONE = 0,          /* block-Jacobi on the fiber's own 15x15 block == identity here */
    RF_PC_CLUSTER = 1,       /* z_i = v_i + sum_m B_im v_(m-th neighbour), B_im the exact coupling blocks
                                of the inverse of the fiber's k-NN cluster submatrix (first block row) */
    RF_PC_LEARNED = 2        /* the same form with B_im predicted by the MLP below; falls back to
                                RF_PC_NONE without weights */
} rf_preconditioner;
/* A preconditioned (inner) GMRES solve runs in trials of max(3 * restart, 30)
 * Arnoldi steps, each restarted from the current iterate; a trial without a
 * tenfold reduction of the residual ends the preconditioner for the rest of
 * that solve, which goes on without it (RF_PC_NONE, block Jacobi), so a poor
 * block never changes the tolerance a solve reaches
 * (rf_solve_stats.pc_fallback records it).  The blocks are kept only while
 * they pay: the handle keeps running means of its solves' iterations with
 * and without them; after a solve that fell back, or while the mean with
 * them is above the one without, the next 8 assemblies neither build nor use
 * them, and while they pay one solve in 32 runs without them to keep the
 * comparison current (rf_solve_stats.preconditioned). */

typedef enum rf_velocity_mode {
    RF_VEL_RECOMPUTE = 0,    /* re-evaluate the pair integrals with the solved forces (reference) */
    RF_VEL_REUSE = 1         /* reuse P0/P1 projections stored during assembly (two GEMVs) */
} rf_velocity_mode;

/* Run parameters.  The first eight fields mirror FiberParams
 * (src/common.h:49-68) and the positional run*.in file
 * (src/parameters.cc:124-180, fortran/advect_fibers.f90:182-222). */
typedef struct rf_params {
    double slenderness;                  /* epsilon (e.g. 0.01) */
    double timestep;                     /* dt (e.g. 0.1) */
    int32_t num_fibers;                  /* M */
    int32_t num_timesteps;               /* informational; rf_step is called by the caller */
    int32_t num_terms_in_force_expansion;/* N, 1..8 */
    int32_t num_quadrature_intervals;    /* NoQI, 1..16; 3 Gauss points each */
    int32_t use_analytical_integration;  /* 1: analytic inner integral, 0: Gauss quadrature */
    int32_t use_direct_solver;           /* 1: dense LU on the device, 0: GMRES */
    int32_t gmres_restart;               /* restart length (run100_iter.in: 10) */
    int32_t gmres_max_iters;             /* iteration budget (100) */
    double gmres_tol;                    /* ||b - A x|| / ||b|| target (1e-5) */
    double external_force[3];            /* per-fiber external force (0, 0, -1) */
    int32_t precision;                   /* rf_precision */
    int32_t preconditioner;              /* rf_preconditioner */
    int32_t velocity_mode;               /* rf_velocity_mode */
    int32_t device;                      /* CUDA device ordinal */
    int32_t max_refinements;             /* mixed precision: outer refinement steps (default 30) */
    int32_t cluster_size;                /* RF_PC_CLUSTER: neighbours per cluster (default 8) */
    double inner_tol;                    /* mixed precision: the deepest reduction one inner GMRES solve
                                            is asked for (default 1e-3); the refinements are planned as the
                                            fewest that reach gmres_tol with inner solves no deeper than
                                            this, each asking for an equal share of what is still needed */
    double near_field_c;                 /* mixed precision: squared distance below which the analytic
                                            integral stays FP64 (default 6: from there on the FP32
                                            backward recursion reaches FP32 accuracy; raised to 10
                                            where the tile kernel runs: numeric integration, N > 5);
                                            >= 1e30 keeps every integral in FP64 */
    int32_t shard_index;                 /* row-block shard of this handle (0 .. shard_count - 1) */
    int32_t shard_count;                 /* row-block shards (GPUs) the system is split over; 0 or 1: the
                                            whole system.  A shard assembles the rows of its target fibers
                                            (rf_shard_range) and keeps all state replicated; FP64,
                                            GMRES, recomputed velocities, no block preconditioner.  Solve and
                                            velocities need the shards' communicator (rf_create_sharded). */
    double pc_damping;                   /* block preconditioners: z_i = v_i + pc_damping sum_m B_im v_(j_m)
                                            (default 0.85; 0 selects the default).  The coupling blocks of
                                            a local cluster inverse overshoot where the couplings are
                                            strong (settled, dense states); damped they help there too */
    int32_t reserved[4];
} rf_params;

/* GMRES / refinement statistics of the last solve. */
typedef struct rf_solve_stats {
    int32_t converged;        /* 1 if ||b-Ax||/||b|| <= tol */
    int32_t iterations;       /* Arnoldi steps (inner steps summed for mixed precision) */
    int32_t matvecs;          /* low- or full-precision matvecs */
    int32_t refinements;      /* outer FP64-residual refinements (mixed precision) */
    double residual;          /* final true ||b-Ax||/||b|| */
    double seconds;           /* device time of the solve */
    int32_t pc_fallback;      /* 1 if the preconditioned solve missed its trial budget and the
                                 solve went on without the preconditioner (see RF_PC_CLUSTER) */
    int32_t precision_fallback; /* 1 if RF_PREC_MIXED_BF16 switched its inner products to the FP32 A */
    int32_t preconditioned;   /* 1 if the solve started with the block preconditioner */
    int32_t reserved;
} rf_solve_stats;

typedef struct rf_handle rf_handle;

/* Fill *p with the reference defaults (run100_iter.in with eps 0.01). */
void rf_params_default(rf_params *p);

/* Simulation(Configuration): allocate device state for p->num_fibers fibers and
 * upload the initial layout.  Orientations are normalised (as the Fortran
 * driver does, advect_fibers.f90:332-340).  One fiber or more; a block
 * preconditioner needs two or more, the direct solver RF_PREC_FP64. */
rf_status rf_create(const rf_params *p, const double *positions, const double *orientations,
                    rf_handle **out);
rf_status rf_destroy(rf_handle *h);

/* ---- Row-block sharding over GPUs (the reference runs on one device; no
 * counterpart there).  The system's rows belong to target fibers: shard r of
 * R assembles the rows of fibers [t0, t1) = [r M / R, (r + 1) M / R)
 * (rf_shard_range) with no communication; state, Krylov vectors and GMRES
 * control are replicated, and each product ends with one NCCL all-gather of
 * the shards' row blocks (the right-hand side and the velocities likewise,
 * once per step).  FP64 GMRES path only.  One process per GPU: rank 0 makes
 * an id with rf_shard_unique_id and sends it to the others by its own means;
 * every rank then calls rf_create_sharded with the same id and
 * p->shard_index = its rank, p->shard_count = the ranks (collective; NCCL is
 * loaded at run time: the file named by RF_NCCL_LIBRARY, else a copy already
 * in the process, else libnccl.so.2; a process that also uses PyTorch loads
 * PyTorch first, so that its NCCL is the one in use).  rf_create with shard_count > 1 makes a shard without
 * a communicator: it assembles and returns its rows (rf_get_matrix_rows; the
 * right-hand side's other rows stay zero) but cannot solve. */
rf_status rf_shard_unique_id(uint8_t *nccl_id /* 128 bytes */);
rf_status rf_shard_range(int32_t M, int32_t shard_count, int32_t shard_index, int32_t *t0, int32_t *t1);
rf_status rf_create_sharded(const rf_params *p, const double *positions, const double *orientations,
                            const uint8_t *nccl_id, rf_handle **out);

/* Simulation::step: assemble, solve, velocities, advect (Euler if
 * current_timestep == 0, else the second-order multistep), then rotate the
 * state buffers. */
rf_status rf_step(rf_handle *h, size_t current_timestep);
/* The four phases of step, callable one by one. */
rf_status rf_assemble_system(rf_handle *h);
rf_status rf_solve_system(rf_handle *h);
rf_status rf_update_velocities(rf_handle *h);
/* Advects the fibers and rotates the triple/double buffers. */
rf_status rf_update_fibers(rf_handle *h, int first_timestep);

/* State access (host buffers of 3*M doubles). */
rf_status rf_get_state(rf_handle *h, double *positions, double *orientations);
rf_status rf_set_state(rf_handle *h, const double *positions, const double *orientations);
rf_status rf_get_velocities(rf_handle *h, double *translational, double *rotational);
/* Coefficient vector (n doubles) and right-hand side (n doubles). */
rf_status rf_get_coeffs(rf_handle *h, double *x);
rf_status rf_get_rhs(rf_handle *h, double *b);
/* Dense matrix, n*n doubles column-major (converted from the stored precision). */
rf_status rf_get_matrix(rf_handle *h, double *A);
/* Rows [row0, row0 + rows) of the stored matrix as FP64, rows x n
 * column-major (leading dimension rows), for checking a sample of a system
 * too large to copy whole (the reference dumps all of A,
 * src/simulation.cu:468-546).  which = 0: the matrix of the FP64 path or of
 * the refinement residual (FP64 or FP32 storage; RF_PREC_MIXED_BF16: the FP32
 * entries rebuilt from its two 16-bit planes); which = 1: the matrix of the
 * inner solve (the BF16 high plane where there is one, else as 0). */
rf_status rf_get_matrix_rows(rf_handle *h, int32_t which, int64_t row0, int64_t rows, double *out);
/* y = A x with the stored matrix (FP64 host vectors of n doubles). */
rf_status rf_matvec(rf_handle *h, const double *x, double *y);
/* y = A x in FP64 without forming A (mat_prod, fortran/matrix_assembly.f90:159-265):
 * the identity plus every pair's inner integral against the source's force
 * expansion from x, projected onto the target's Legendre modes, for the
 * current state and the handle's inner integral (use_analytical_integration;
 * the reference's mat_prod uses the numeric one).  Any precision; memory O(M),
 * work O(M^2) per call.  Host vectors of n doubles. */
rf_status rf_matvec_free(rf_handle *h, const double *x, double *y);
rf_status rf_get_solve_stats(rf_handle *h, rf_solve_stats *s);
/* y = A x in FP64 for callers that cannot allocate device memory: A (n x n
 * column-major, leading dimension lda, lda*n doubles, 16-byte aligned), x and
 * y are the caller's device buffers, and the product's partial sums use a
 * fixed 8 MiB array inside the library.  No counterpart in the reference: it
 * serves hosts whose device memory belongs to their own allocator or pool,
 * and loops that must not stall on cudaMalloc/cudaFree.  Limit: lda <=
 * 1,048,576 (lda even); larger sizes return RF_ERR_INVALID_ARG with the
 * reason in rf_last_error(NULL).  Enqueued on `stream` (cudaStream_t, NULL =
 * default stream) of the current device; y is ready when the stream reaches
 * it.  The first call on a device sets the array up: it looks up the array's
 * device address, and with CUDA's default lazy module loading that is also
 * when the driver loads the library's device code and reserves the 8 MiB on
 * that device (it may synchronise the device); the array then stays until the
 * process exits.  So make the first call on each device before a memory pool
 * claims the device's memory and before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (other streams, other threads)
 * race on it.  Nothing in the array needs to start at zero. */
rf_status rf_matvec_noalloc(const double *A, int64_t lda, int64_t n, const double *x, double *y, void *stream);
/* Dense direct solve of a general system on the device, the LAPACK dgesv
 * call of the reference's direct variant (fortran/coeffs_and_vels.f90:62,158,
 * 333,514: dgesv(n, 1, A, n, ipiv, b, n, info)) without a handle, with the
 * same device LU as use_direct_solver (partial pivoting, first row of largest
 * magnitude).  A: host, n x n column-major with leading dimension lda >= n,
 * left unchanged (the factors stay on the device); x = A^-1 b (host, n; may
 * alias b); ipiv (host, n, or NULL): the pivot rows, 1-based as LAPACK's;
 * *info: 0, or the first zero pivot (1-based; x is then undefined).  Runs on
 * `device`, allocates one n x n FP64 copy of A there and returns when x is
 * on the host; errors are read back with rf_last_error(NULL). */
rf_status rf_dgesv(int64_t n, const double *A, int64_t lda, const double *b, double *x, int32_t *ipiv,
                   int32_t *info, int32_t device);
/* Multistep history for checkpoint/resume: previous positions/orientations
 * and previous velocities (3*M doubles each). */
rf_status rf_get_history(rf_handle *h, double *prev_pos, double *prev_orient, double *prev_vel,
                         double *prev_rot);
rf_status rf_set_history(rf_handle *h, const double *prev_pos, const double *prev_orient,
                         const double *prev_vel, const double *prev_rot, const double *coeffs);

/* Device-time markers on the handle's stream (replaces the cudaEvent timer of
 * src/performance.cc:31-65): record marker slot 0..15; elapsed milliseconds
 * between two recorded slots (waits for the later one).  Returns < 0 on error. */
rf_status rf_timer_mark(rf_handle *h, int32_t slot);
double rf_timer_elapsed_ms(rf_handle *h, int32_t from, int32_t to);
/* Average device time of one matrix-vector product with the stored matrix in
 * the precision the inner GMRES uses (FP64, FP32 or BF16), over reps launches
 * on device-resident vectors; bytes of A streamed per product in *bytes. */
rf_status rf_profile_matvec(rf_handle *h, int32_t reps, double *ms_per_product, double *bytes);
/* Live timing of the inner-solve matrix-vector products (instrumentation; no
 * counterpart in the reference).  enable = 1 resets the counters and brackets
 * every following product of the inner GMRES (mixed and FP32 paths; the FP64
 * GMRES otherwise) with events on the handle's stream; enable = 0 stops.
 * Either way *count, *total_ms and *bytes_per_product report the products
 * timed since the last reset, their summed device time and the bytes of A one
 * product streams.  Pointers may be NULL. */
rf_status rf_gemv_timer(rf_handle *h, int32_t enable, int64_t *count, double *total_ms, double *bytes_per_product);

/* Sizes. */
int64_t rf_system_size(const rf_handle *h);   /* n = 3*N*M */
int64_t rf_matrix_ld(const rf_handle *h);     /* leading dimension of the stored A */
/* CUDA stream (cudaStream_t) the handle launches on; for event timing. */
void *rf_get_stream(rf_handle *h);
/* Number of kernels the handle has launched since creation. */
int64_t rf_kernel_launches(const rf_handle *h);
/* Last error message of the handle (or of the last failed rf_create if h is NULL). */
const char *rf_last_error(const rf_handle *h);
const char *rf_status_string(rf_status s);

/* ---- Seeded synthetic layouts -------------------------------------------
 * Centres by rejection sampling (minimum centre distance min_dist), either
 * uniform in the cube [0, box]^3 (distribution 0) or isotropic Gaussian with
 * standard deviation box (distribution 1); orientations are normalised
 * N(0, I3) samples (uniform on the sphere).  Deterministic in seed.
 * Replaces tools/gen.py of the reference. */
rf_status rf_generate_layout(int32_t M, int32_t distribution, double box, double min_dist,
                             uint64_t seed, double *positions, double *orientations);
/* Minimum distance between the centre-lines (segments of half-length 1) of
 * any two fibers; a geometry diagnostic (the kernels are singular at 0). */
double rf_min_segment_distance(int32_t M, const double *positions, const double *orientations);

/* ---- Learned preconditioner (benchmark addition; no reference counterpart)
 * z_i = v_i + sum_{m < 8} B_im v_(m-th nearest neighbour of i).  The MLP
 * predicts each coupling block B_im (15 x 15) from the features of the pair:
 * the 16 nearest neighbours of fiber i in its own frame (e3 = its
 * orientation, e1 toward the nearest neighbour), 9 floats each, neighbour m
 * first (relative centre, orientation with a canonical sign, orientation
 * squared), then the other 15 nearest first (relative centre and the six
 * products u_a u_b of the orientation), 16 x 9 floats -> 256 -> 256 -> 225,
 * ReLU.  The output is the block in fiber i's frame with the columns of odd
 * Legendre order multiplied by neighbour m's canonical sign.
 * Weights are FP32, layer-major: W1[256x144] b1[256] W2[256x256] b2[256]
 * W3[225x256] b3[225] (row-major, out x in). */
#define RF_MLP_K 16
#define RF_MLP_PAIRS 8
#define RF_MLP_IN (RF_MLP_K * 9)
#define RF_MLP_HIDDEN 256
#define RF_MLP_OUT 225
int64_t rf_mlp_num_params(void);
/* Install weights used by RF_PC_LEARNED. */
rf_status rf_set_mlp_weights(rf_handle *h, const float *weights, int64_t count);
/* Pair features ((M * 8) x 144, fiber-major, neighbour-minor) of the current state. */
rf_status rf_compute_features(rf_handle *h, float *features);
/* Exact coupling blocks of the current assembled system ((M * 8) x 225,
 * row-major 15 x 15, same order as the features), in the frame and sign
 * convention of the MLP output: the training targets.  Needs cluster_size >= 8. */
rf_status rf_compute_cluster_targets(rf_handle *h, float *targets);

/* The network's inference as the preconditioner runs it (tensor cores:
 * tcgen05 MMAs with BF16 operands and FP32 accumulation in tensor memory),
 * on count feature rows (count x 144) with the given weights; out is
 * count x 225.  For checking the inference against the FP32 reference
 * network (no counterpart in the reference). */
rf_status rf_mlp_predict(int32_t device, const float *weights, const float *features, int64_t count, float *out);

/* Stand-alone trainer on the device: owns weights, Adam state and a dataset. */
typedef struct rf_trainer rf_trainer;
rf_status rf_trainer_create(int32_t device, uint64_t seed, rf_trainer **out);
rf_status rf_trainer_destroy(rf_trainer *t);
rf_status rf_trainer_add_samples(rf_trainer *t, const float *features, const float *targets,
                                 int64_t count);
/* Run epochs of minibatch Adam on the MSE loss; returns the mean loss of the
 * last epoch. */
rf_status rf_trainer_train(rf_trainer *t, int32_t epochs, int32_t batch, float lr, float *loss);
rf_status rf_trainer_get_weights(rf_trainer *t, float *weights);
rf_status rf_trainer_set_weights(rf_trainer *t, const float *weights);
/* Forward + backward of one batch with the trainer's weights: loss and
 * gradient (rf_mlp_num_params floats), for gradient checks. */
rf_status rf_trainer_loss_grad(rf_trainer *t, const float *features, const float *targets,
                               int64_t count, float *loss, float *grad);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* RIGIDFIBERS_H_ */
