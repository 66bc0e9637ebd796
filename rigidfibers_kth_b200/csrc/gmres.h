// gmres.h - restarted GMRES on the device with the control flow of the
// reference Fortran solver (fortran/dGMRES.f:491-1495 as configured by
// fortran/coeffs_and_vels.f90:446-500): modified Gram-Schmidt, Givens
// rotations on the Hessenberg matrix, the true residual recomputed at each
// restart, and the stopping rule "Arnoldi estimate <= tol, then true
// residual <= tol" on ||b - A x|| / ||b||.  Right preconditioning z = P v is
// optional (the residual keeps its meaning).  Krylov vectors live on the
// device in VT (double or float); the Hessenberg matrix, rotations and the
// least-squares solve are FP64 on the host (a few hundred flops per step);
// solve_device keeps them on the device (arnoldi.cu).
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <vector>

#include "rf_kernels.h"

namespace rf {

constexpr int kInfoBudget = -4;
constexpr int kInfoNaN = -5;

struct GmresResult {
    int info = 0;          // 0 converged, -4 budget spent, -5 non-finite value met
    int iterations = 0;
    int matvecs = 0;
    double backward_error = 0.0;
    int launches = 0;
};

template <typename VT>
class Gmres {
   public:
    using Op = std::function<cudaError_t(const VT *in, VT *out)>;
    // an operator whose kernels return at once when *stop != 0 (stop may be null)
    using StopOp = std::function<cudaError_t(const VT *in, VT *out, const int *stop)>;

    Gmres() = default;
    ~Gmres();
    cudaError_t init(int64_t n, int m, cudaStream_t st);
    // Solve A x = b; x holds the initial guess (device, VT).  If x_is_zero the
    // initial residual is b itself (no matvec, like icntl(6) = 0).  With
    // check_true = false the solve stops on the Arnoldi estimate alone (inner
    // solves of iterative refinement, whose caller recomputes the residual).
    cudaError_t solve(const Op &A, const Op *P, const VT *b, VT *x, bool x_is_zero, double tol, int max_iters,
                      GmresResult *res, bool check_true = true);
    // Inner solve of the refinement, controlled on the device (arnoldi.cu):
    // x = 0 initially, stop on the Arnoldi estimate <= tol or the budget,
    // CGS2 orthogonalisation.  The host queues each step before it learns
    // whether the previous one stopped (the first steps of a cycle also
    // before it learns whether the cycle's start stopped); a step queued
    // after the stop runs as empty launches, and `on_skipped_product` is
    // called once for each such product (the caller's product timer drops
    // it).  Needs m <= kArnoldiMax.
    cudaError_t solve_device(const StopOp &A, const StopOp *P, const VT *b, VT *x, double tol, int max_iters,
                             GmresResult *res, const std::function<void()> &on_skipped_product);
    int restart() const { return m_; }

   private:
    cudaError_t residual(const Op &A, const VT *b, const VT *x, VT *r, GmresResult *res);
    cudaError_t fetch(const double *dev, double *host, int count);
    void lsq(int k, std::vector<double> &y) const;
    cudaError_t update_solution(const Op *P, const VT *x, int k, VT *xcur, GmresResult *res);

    int64_t n_ = 0;
    int m_ = 0;
    cudaStream_t st_ = nullptr;
    VT *V_ = nullptr;      // n x m
    VT *w_ = nullptr;      // n
    VT *z_ = nullptr;      // n (preconditioned vector)
    VT *u_ = nullptr;      // n
    VT *xcur_ = nullptr;   // n
    double *hcol_ = nullptr;   // m+2 device scalars
    double *ydev_ = nullptr;   // m
    double *hpin_ = nullptr;   // pinned host mirror of hcol
    RedBuf rb_{};
    // device-controlled solve
    ArnoldiCtrl *ctrl_ = nullptr;     // device
    ArnoldiStat *hstat_ = nullptr;    // host-mapped, one per step of a cycle, then the cycle start
    ArnoldiStat *dstat_ = nullptr;    // its device address
    double *cpart_ = nullptr;         // kArnoldiMax x max_blocks partial sums
    cudaEvent_t step_ev_[kArnoldiMax] = {};
    std::vector<double> H_;    // (m+1) x (m+1) column-major, column m = rhs g
    std::vector<double> cs_, sn_;
};

extern template class Gmres<double>;
extern template class Gmres<float>;

}  // namespace rf
