/*
 * rfo.h - CPU FP64 oracle for the rigid-fiber slender-body step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++17/OpenMP restatement
 * of the reference Fortran program (the fortran/ sources of ericwolter/rigidfibers_kth).
 * It is the checker for the CUDA product path: only tests/, the package's
 * smoke entry and bench.py's CPU-baseline leg may load it.  The product
 * library (librigidfibers.so) never links or calls it.
 *
 * Parity pin: every function is checked against the 48 golden vectors
 * written by the Fortran program (tests/reference/100_{analytic,numeric}_
 * {direct,gmres}/{0,1}_{BVec,XVec,TRANSVel,ROTVel,POS,ORIENT}.ref), stored
 * as tests/golden/golden_m100.npz.
 *
 * Layout conventions follow the Fortran arrays:
 *   X[3*M], T[3*M]       fiber centres / unit orientations, (x,y,z) per fiber
 *   coefficient vector   n = 3*N*M, index (i*N + k)*3 + d  (fiber, Legendre k-1, xyz)
 *   A                    n x n, column-major A[row + col*n]
 */
#ifndef RFO_H_
#define RFO_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int M;              /* number of fibers */
    int N;              /* terms in the force expansion (1..8) */
    int NoQI;           /* quadrature intervals, 3 Gauss points each */
    int analytic;       /* 1: analytic inner integral, 0: Gauss quadrature */
    int direct;         /* 1: LU solve, 0: restarted GMRES */
    int restart;        /* GMRES restart length */
    int max_iters;      /* GMRES iteration budget */
    double tol;         /* GMRES tolerance on ||r||/||b|| */
    double eps;         /* slenderness */
    double dt;          /* time step */
    double ext_force[3];/* external force per fiber (Fortran: (0,0,-1)) */
    int threads;        /* OpenMP threads, <=0: all */
} rfo_params;

/* quadrature.f90:6-96 */
void rfo_quadrature(int NoQI, double *pv, double *wv);
/* matrix_assembly.f90:8-57; L is LQ x N column-major (P_1..P_N) */
void rfo_legendre(int N, int LQ, const double *pv, double *L);
/* Int_analytical.f90:5-293: Legendre moments L11..L24 for m = 0..N.
 * out is 7*(N+1): out[c*(N+1)+m], c = L11,L12,L13,L14,L22,L23,L24. */
void rfo_analytic_moments(const double *xb, const double *pb, const double *xbar,
                          int N, double *out);

/* matrix_assembly.f90:267-629 (A) and 632-905 (b). */
int rfo_assemble_system(const rfo_params *p, const double *X, const double *T,
                        double *A, double *b);
/* dgesv semantics: LU with partial pivoting. A is overwritten. x holds b on input. */
int rfo_solve_direct(int n, double *A, double *x);
/* dGMRES.f semantics (MGS, Givens, true residual at restart, ||r||/||b|| stop).
 * x holds the initial guess on input.  Returns 0 converged, -4 not converged. */
int rfo_solve_gmres(int n, const double *A, const double *b, double *x,
                    int restart, int max_iters, double tol,
                    int *iters, double *backward_error, int threads);
/* y = A x (column-major, dgemv 'N' order) */
void rfo_matvec(int n, const double *A, const double *x, double *y, int threads);
/* y = A x for an m x n column-major A with leading dimension lda */
void rfo_matvec_rect(int m, int n, const double *A, long long lda, const double *x, double *y, int threads);
/* coeffs_and_vels.f90:543-746 */
int rfo_velocities(const rfo_params *p, const double *X, const double *T,
                   const double *coeffs, double *V, double *W);

/* Whole-step driver mirroring advect_fibers.f90:437-593 (with the loop over
 * all requested steps).  Holds the triple-buffered state. */
typedef struct rfo_sim rfo_sim;
rfo_sim *rfo_sim_create(const rfo_params *p, const double *X0, const double *T0);
void rfo_sim_destroy(rfo_sim *s);
/* one time step; step_index 0 is the forward-Euler step */
int rfo_sim_step(rfo_sim *s);
/* The same step in parts, for timing one whole step in bounded pieces:
 * rfo_sim_assemble_part assembles the rows of A and b of target fibers
 * [i0, i1) into the step's system (held by the handle, n x n); once every
 * target's rows are in, rfo_sim_finish_step solves, computes the velocities,
 * advects and rotates the state.  rfo_sim_step = both over all targets. */
int rfo_sim_assemble_part(rfo_sim *s, int i0, int i1);
int rfo_sim_finish_step(rfo_sim *s);
/* outputs of the last step (any pointer may be NULL) */
void rfo_sim_last(const rfo_sim *s, double *b, double *coeffs, double *V, double *W,
                  double *X, double *T);
/* GMRES information of the last step */
void rfo_sim_solve_info(const rfo_sim *s, int *info, int *iters, double *be);
/* seconds spent in assembly / solve / velocity / advection in the last step */
void rfo_sim_timings(const rfo_sim *s, double *t4);

/* Sampled CPU workload used as the timed CPU baseline: assemble the rows of
 * A and b that belong to target fibers [i0, i1) (all sources), in the same
 * arithmetic as rfo_assemble_system.  Arows is (i1-i0)*3N x n column-major
 * with leading dimension (i1-i0)*3N. */
int rfo_assemble_rows(const rfo_params *p, const double *X, const double *T,
                      int i0, int i1, double *Arows, double *brows);
/* velocities of target fibers [i0, i1) only */
int rfo_velocities_rows(const rfo_params *p, const double *X, const double *T,
                        const double *coeffs, int i0, int i1, double *V, double *W);

/* Seeded synthetic layout: the product's generator (rf_generate_layout)
 * restated on the oracle side, so that the CPU baseline builds its input
 * without loading the product library; identical output bit for bit.
 * distribution 0: centres uniform in [0, box)^3; 1: isotropic normal with
 * deviation box; minimum centre distance by rejection; orientations
 * uniform on the sphere.  Returns 0, or -1 for invalid arguments. */
int rfo_generate_layout(int M, int distribution, double box, double min_dist, unsigned long long seed,
                        double *positions, double *orientations);

#ifdef __cplusplus
}
#endif
#endif
