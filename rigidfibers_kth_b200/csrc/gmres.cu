// gmres.cu - host driver of the device GMRES (see gmres.h).
#include "gmres.h"

#include <cmath>
#include <cstring>

namespace rf {

namespace {

// LINPACK drotg semantics (fortran/blas_rot.f:117-146)
void rotg(double a, double b, double *c, double *s) {
    const double roe = (std::fabs(a) > std::fabs(b)) ? a : b;
    const double scale = std::fabs(a) + std::fabs(b);
    if (scale == 0.0) {
        *c = 1.0;
        *s = 0.0;
        return;
    }
    double r = scale * std::sqrt((a / scale) * (a / scale) + (b / scale) * (b / scale));
    r = std::copysign(1.0, roe) * r;
    *c = a / r;
    *s = b / r;
}

inline void rot(double &x, double &y, double c, double s) {
    const double t = c * x + s * y;
    y = c * y - s * x;
    x = t;
}

#define RF_TRY(expr)                              \
    do {                                          \
        cudaError_t e__ = (expr);                 \
        if (e__ != cudaSuccess) return e__;       \
    } while (0)

}  // namespace

template <typename VT>
Gmres<VT>::~Gmres() {
    cudaFree(V_);
    cudaFree(w_);
    cudaFree(z_);
    cudaFree(u_);
    cudaFree(xcur_);
    cudaFree(hcol_);
    cudaFree(ydev_);
    cudaFree(rb_.partials);
    cudaFree(rb_.counter);
    if (hpin_) cudaFreeHost(hpin_);
    cudaFree(ctrl_);
    cudaFree(cpart_);
    if (hstat_) cudaFreeHost(hstat_);
    for (cudaEvent_t ev : step_ev_)
        if (ev) cudaEventDestroy(ev);
}

template <typename VT>
cudaError_t Gmres<VT>::init(int64_t n, int m, cudaStream_t st) {
    n_ = n;
    m_ = m;
    st_ = st;
    RF_TRY(cudaMalloc(&V_, sizeof(VT) * n * m));
    RF_TRY(cudaMalloc(&w_, sizeof(VT) * n));
    RF_TRY(cudaMalloc(&z_, sizeof(VT) * n));
    RF_TRY(cudaMalloc(&u_, sizeof(VT) * n));
    RF_TRY(cudaMalloc(&xcur_, sizeof(VT) * n));
    RF_TRY(cudaMalloc(&hcol_, sizeof(double) * (m + 8)));
    RF_TRY(cudaMalloc(&ydev_, sizeof(double) * (m + 8)));
    RF_TRY(cudaMallocHost(&hpin_, sizeof(double) * (m + 8)));
    rb_.max_blocks = 1024;
    RF_TRY(cudaMalloc(&rb_.partials, sizeof(double) * rb_.max_blocks));
    RF_TRY(cudaMalloc(&rb_.counter, sizeof(unsigned int)));
    RF_TRY(cudaMemsetAsync(rb_.counter, 0, sizeof(unsigned int), st));
    H_.assign((size_t)(m + 1) * (m + 1), 0.0);
    cs_.assign(m, 0.0);
    sn_.assign(m, 0.0);
    if (m <= kArnoldiMax) {
        RF_TRY(cudaMalloc(&ctrl_, sizeof(ArnoldiCtrl)));
        RF_TRY(cudaMemsetAsync(ctrl_, 0, sizeof(ArnoldiCtrl), st));
        RF_TRY(cudaMalloc(&cpart_, sizeof(double) * kArnoldiMax * rb_.max_blocks));
        RF_TRY(cudaHostAlloc(&hstat_, sizeof(ArnoldiStat) * (kArnoldiMax + 1), cudaHostAllocMapped));
        std::memset(hstat_, 0, sizeof(ArnoldiStat) * (kArnoldiMax + 1));
        RF_TRY(cudaHostGetDevicePointer((void **)&dstat_, hstat_, 0));
        for (cudaEvent_t &ev : step_ev_) RF_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    return cudaStreamSynchronize(st);
}

template <typename VT>
cudaError_t Gmres<VT>::solve_device(const StopOp &A, const StopOp *P, const VT *b, VT *x, double tol, int max_iters,
                                    GmresResult *res, const std::function<void()> &on_skipped_product) {
    *res = GmresResult();
    const int m = m_;
    if (!ctrl_ || m > kArnoldiMax) return cudaErrorInvalidValue;
    const int iterMax = max_iters > 0 ? max_iters : (int)n_;
    const int *stop = &ctrl_->stop;
    volatile ArnoldiStat *hs = hstat_;
    RF_TRY(cudaMemsetAsync(x, 0, sizeof(VT) * n_, st_));
    RF_TRY(launch_arnoldi_start<VT>(n_, b, V_, ctrl_, tol, iterMax, 1, cpart_, rb_.counter, rb_.max_blocks,
                                    dstat_ + kArnoldiMax, st_));
    res->launches += 3;
    int last_stop = 0;
    for (;;) {
        // The start of a cycle may already stop the solve (zero or non-finite
        // residual).  Its outcome is read after the first step's event: steps
        // queued behind a stopped start return at once and leave their
        // outcome slots untouched.
        bool ahead = false;  // a step was queued after the one that stopped
        int queued = 0;
        int start_stop = -1;  // the start's outcome, once known
        auto read_start = [&] {
            if (start_stop < 0) start_stop = hs[kArnoldiMax].stop;
            return start_stop != 0;
        };
        for (int j = 0; j < m; ++j) {
            const VT *in = V_ + (size_t)j * n_;
            if (P) {
                RF_TRY((*P)(in, z_, stop));
                res->launches++;
                in = z_;
            }
            RF_TRY(A(in, w_, stop));
            res->matvecs++;
            RF_TRY(launch_arnoldi_orthogonalize<VT>(n_, w_, V_, j, m, ctrl_, dstat_, cpart_, rb_.counter,
                                                    rb_.max_blocks, st_));
            res->launches += 4;
            RF_TRY(cudaEventRecord(step_ev_[j], st_));
            ++queued;
            if (j > 0) {
                // step j is queued: now wait for step j - 1 (the GPU is busy with j)
                RF_TRY(cudaEventSynchronize(step_ev_[j - 1]));
                if (read_start()) break;
                last_stop = hs[j - 1].stop;
                res->iterations = hs[j - 1].itn;
                res->backward_error = hs[j - 1].bea;
                if (last_stop) {
                    ahead = true;
                    break;
                }
            }
        }
        if (start_stop <= 0 && !ahead) {
            RF_TRY(cudaEventSynchronize(step_ev_[m - 1]));
            if (!read_start()) {
                last_stop = hs[m - 1].stop;
                res->iterations = hs[m - 1].itn;
                res->backward_error = hs[m - 1].bea;
            }
        }
        if (start_stop > 0) {
            // every step of this cycle returned at once
            for (int q = 0; q < queued; ++q) {
                res->matvecs--;
                if (on_skipped_product) on_skipped_product();
            }
            res->info = start_stop == 3 ? kInfoNaN : 0;
            return cudaSuccess;
        }
        if (ahead) {
            res->matvecs--;  // the queued step's product returned at once
            if (on_skipped_product) on_skipped_product();
        }
        if (last_stop == 3) {
            res->info = kInfoNaN;
            return cudaSuccess;
        }
        // x += P (V y) over the steps of this cycle
        RF_TRY(launch_arnoldi_combine<VT>(n_, V_, ctrl_, u_, st_));
        res->launches += 2;
        const VT *upd = u_;
        if (P) {
            RF_TRY((*P)(u_, z_, nullptr));
            upd = z_;
            res->launches++;
        }
        RF_TRY(launch_add<VT>(n_, x, upd, x, st_));
        res->launches++;
        if (last_stop) {
            res->info = last_stop == 1 ? 0 : kInfoBudget;
            return cudaSuccess;
        }
        // restart from the residual of the updated x
        RF_TRY(A(x, w_, nullptr));
        res->matvecs++;
        RF_TRY(launch_bmr<VT>(n_, b, w_, st_));
        RF_TRY(launch_arnoldi_start<VT>(n_, w_, V_, ctrl_, tol, iterMax, 0, cpart_, rb_.counter, rb_.max_blocks,
                                        dstat_ + kArnoldiMax, st_));
        res->launches += 4;
    }
}

template <typename VT>
cudaError_t Gmres<VT>::fetch(const double *dev, double *host, int count) {
    RF_TRY(cudaMemcpyAsync(hpin_, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, st_));
    RF_TRY(cudaStreamSynchronize(st_));
    for (int i = 0; i < count; ++i) host[i] = hpin_[i];
    return cudaSuccess;
}

// r = b - A x
template <typename VT>
cudaError_t Gmres<VT>::residual(const Op &A, const VT *b, const VT *x, VT *r, GmresResult *res) {
    RF_TRY(A(x, r));
    res->matvecs++;
    RF_TRY(launch_bmr<VT>(n_, b, r, st_));  // r = b - r
    res->launches++;
    return cudaSuccess;
}

template <typename VT>
void Gmres<VT>::lsq(int k, std::vector<double> &y) const {
    // upper-triangular solve H(0:k,0:k) y = g(0:k) (dtrsv 'U','N')
    const int ld = m_ + 1;
    y.assign(k, 0.0);
    for (int r = 0; r < k; ++r) y[r] = H_[r + (size_t)m_ * ld];
    for (int c = k - 1; c >= 0; --c) {
        y[c] /= H_[c + (size_t)c * ld];
        for (int r = 0; r < c; ++r) y[r] -= y[c] * H_[r + (size_t)c * ld];
    }
}

// xcur = x + P (V y)
template <typename VT>
cudaError_t Gmres<VT>::update_solution(const Op *P, const VT *x, int k, VT *xcur, GmresResult *res) {
    std::vector<double> y;
    lsq(k, y);
    for (int i = 0; i < k; ++i) hpin_[i] = y[i];
    RF_TRY(cudaMemcpyAsync(ydev_, hpin_, sizeof(double) * k, cudaMemcpyHostToDevice, st_));
    RF_TRY(cudaStreamSynchronize(st_));  // hpin_ is reused by the next fetch
    RF_TRY(launch_vy<VT>(n_, V_, n_, ydev_, k, u_, st_));  // u = V y
    res->launches++;
    const VT *upd = u_;
    if (P) {
        RF_TRY((*P)(u_, z_));
        upd = z_;
        res->launches++;
    }
    RF_TRY(launch_add<VT>(n_, x, upd, xcur, st_));
    res->launches++;
    return cudaSuccess;
}

template <typename VT>
cudaError_t Gmres<VT>::solve(const Op &A, const Op *P, const VT *b, VT *x, bool x_is_zero, double tol,
                             int max_iters, GmresResult *res, bool check_true) {
    *res = GmresResult();
    const int m = m_;
    const int ld = m + 1;
    const int iterMax = max_iters > 0 ? max_iters : (int)n_;
    auto Hc = [&](int r, int c) -> double & { return H_[r + (size_t)c * ld]; };
    double bn;
    RF_TRY(launch_dot<VT>(n_, b, b, hcol_ + m + 3, rb_, st_));
    res->launches++;
    RF_TRY(fetch(hcol_ + m + 3, &bn, 1));
    bn = std::sqrt(bn);
    if (!std::isfinite(bn)) {
        res->info = kInfoNaN;
        return cudaSuccess;
    }
    if (bn == 0.0) {
        RF_TRY(cudaMemsetAsync(x, 0, sizeof(VT) * n_, st_));
        res->info = 0;
        return cudaSuccess;
    }
    // r0 = b - A x  (w_ holds r0)
    if (x_is_zero) {
        RF_TRY(cudaMemcpyAsync(w_, b, sizeof(VT) * n_, cudaMemcpyDeviceToDevice, st_));
    } else {
        RF_TRY(residual(A, b, x, w_, res));
    }
    double beta;
    RF_TRY(launch_mgs_norm<VT>(n_, w_, nullptr, nullptr, hcol_ + m + 4, rb_, st_));
    res->launches++;
    RF_TRY(fetch(hcol_ + m + 4, &beta, 1));
    if (!std::isfinite(beta)) {
        res->info = kInfoNaN;
        return cudaSuccess;
    }
    if (beta == 0.0) {
        res->info = 0;
        return cudaSuccess;
    }
    RF_TRY((launch_scale<VT, VT>(n_, w_, hcol_ + m + 4, 1.0, V_, st_)));
    res->launches++;
    int iterOut = 0;
    double bea = 0.0, be = 0.0;
    std::vector<double> hh(m + 2);
    for (;;) {
        for (auto &v : H_) v = 0.0;
        Hc(0, m) = beta;
        int jH;
        for (jH = 0; jH < m; ++jH) {
            VT *vj = V_ + (size_t)jH * n_;
            const VT *in = vj;
            if (P) {
                RF_TRY((*P)(vj, z_));
                res->launches++;
                in = z_;
            }
            RF_TRY(A(in, w_));
            res->matvecs++;
            // modified Gram-Schmidt: kernel j applies the update of j-1 and the dot of j
            for (int j = 0; j <= jH; ++j) {
                const VT *vprev = j > 0 ? V_ + (size_t)(j - 1) * n_ : nullptr;
                RF_TRY(launch_mgs_step<VT>(n_, w_, vprev, hcol_ + (j > 0 ? j - 1 : 0), V_ + (size_t)j * n_,
                                           hcol_ + j, rb_, st_));
                res->launches++;
            }
            RF_TRY(launch_mgs_norm<VT>(n_, w_, V_ + (size_t)jH * n_, hcol_ + jH, hcol_ + jH + 1, rb_, st_));
            res->launches++;
            if (jH + 1 < m) {
                RF_TRY((launch_scale<VT, VT>(n_, w_, hcol_ + jH + 1, 1.0, V_ + (size_t)(jH + 1) * n_, st_)));
                res->launches++;
            }
            RF_TRY(fetch(hcol_, hh.data(), jH + 2));
            for (int j = 0; j <= jH + 1; ++j) {
                if (!std::isfinite(hh[j])) {
                    res->info = kInfoNaN;
                    return cudaSuccess;
                }
                Hc(j, jH) = hh[j];
            }
            for (int j = 0; j < jH; ++j) rot(Hc(j, jH), Hc(j + 1, jH), cs_[j], sn_[j]);
            rotg(Hc(jH, jH), Hc(jH + 1, jH), &cs_[jH], &sn_[jH]);
            rot(Hc(jH, m), Hc(jH + 1, m), cs_[jH], sn_[jH]);
            rot(Hc(jH, jH), Hc(jH + 1, jH), cs_[jH], sn_[jH]);
            Hc(jH + 1, jH) = 0.0;
            bea = std::fabs(Hc(jH + 1, m)) / bn;
            const int itn = iterOut * m + jH + 1;
            res->iterations = itn;
            if (bea <= tol || itn >= iterMax) {
                RF_TRY(update_solution(P, x, jH + 1, xcur_, res));
                if (!check_true) {
                    RF_TRY(cudaMemcpyAsync(x, xcur_, sizeof(VT) * n_, cudaMemcpyDeviceToDevice, st_));
                    RF_TRY(cudaStreamSynchronize(st_));
                    res->backward_error = bea;
                    res->info = bea <= tol ? 0 : kInfoBudget;
                    return cudaSuccess;
                }
                RF_TRY(residual(A, b, xcur_, w_, res));
                double tn;
                RF_TRY(launch_dot<VT>(n_, w_, w_, hcol_ + m + 5, rb_, st_));
                res->launches++;
                RF_TRY(fetch(hcol_ + m + 5, &tn, 1));
                be = std::sqrt(tn) / bn;
                if (be <= tol || itn >= iterMax) {
                    RF_TRY(cudaMemcpyAsync(x, xcur_, sizeof(VT) * n_, cudaMemcpyDeviceToDevice, st_));
                    RF_TRY(cudaStreamSynchronize(st_));
                    res->backward_error = be;
                    res->info = be <= tol ? 0 : kInfoBudget;
                    return cudaSuccess;
                }
            }
        }
        iterOut++;
        if (bea > tol) RF_TRY(update_solution(P, x, m, xcur_, res));
        RF_TRY(cudaMemcpyAsync(x, xcur_, sizeof(VT) * n_, cudaMemcpyDeviceToDevice, st_));
        RF_TRY(residual(A, b, x, w_, res));
        RF_TRY(launch_mgs_norm<VT>(n_, w_, nullptr, nullptr, hcol_ + m + 4, rb_, st_));
        res->launches++;
        RF_TRY(fetch(hcol_ + m + 4, &beta, 1));
        RF_TRY((launch_scale<VT, VT>(n_, w_, hcol_ + m + 4, 1.0, V_, st_)));
        res->launches++;
    }
}

template class Gmres<double>;
template class Gmres<float>;

}  // namespace rf
