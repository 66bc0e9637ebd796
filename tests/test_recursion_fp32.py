"""The FP32 far-field moments, checked as an algorithm on the CPU.

The far-pair kernels compute I_n, J_n, S_n (n = 0..N+2) in FP32 by the
backward recursion alone, started at n = 32 and run down to n = 0
(moments_backward_fp32 in rf_device.cuh), with c J and c^2 S carried in the
recursion.  This test restates those operations in numpy float32 (the
kernel's order of operations, without fused multiply-adds) and compares the
Legendre combinations that the block entries use against FP64 Gauss-Legendre
quadrature of the same integrals, for every c >= 6 (the smallest near-pair
threshold the kernels accept) and every direction,
on the source axis included.  It also shows why the reference's n = 0, 1
closed forms are not used in FP32: they cancel for distant pairs.  The GPU
kernels themselves are checked against FP64 in tests/test_gpu_parity.py.
"""
import numpy as np

f32 = np.float32
K = 8  # n = 0..N+2 for N = 5
TOP = 32
XG, WG = np.polynomial.legendre.leggauss(200)
LEG = {0: {0: 1.0}, 1: {1: 1.0}, 2: {2: 1.5, 0: -0.5}, 3: {3: 2.5, 1: -1.5},
       4: {4: 35 / 8, 2: -30 / 8, 0: 3 / 8}, 5: {5: 63 / 8, 3: -70 / 8, 1: 15 / 8}}


def truth(b, c):
    R = np.sqrt(XG * XG + b * XG + c)
    return [np.array([np.sum(WG * XG ** n / R ** k) for n in range(K)]) for k in (1, 3, 5)]


def backward_fp32(b, c):
    b, c, one = f32(b), f32(c), f32(1)
    xe, xb = one + b + c, one - b + c
    ue, ub = xe * (one / np.sqrt(xe)), xb * (one / np.sqrt(xb))
    ic = one / c
    icb = ic * b
    icwp = (f32(2) * b / (ue + ub)) * ic  # (ue - ub) / c without cancellation
    icwm = (ue + ub) * ic
    nic, nicb, ic2 = -ic, -icb, ic * ic
    I, J, S = [0.0] * K, [0.0] * K, [0.0] * K
    i1 = i2 = j1 = j2 = s1 = s2 = f32(0)
    for n in range(TOP, -1, -1):
        a0, r2 = f32((n + 2) / (n + 1)), f32(1 / (n + 2))
        cb = f32((1 - 2 * (n + 2)) / (2 * (n + 2)))
        icw = icwp if (n + 1) % 2 == 0 else icwm
        i_ = (a0 * cb) * icb * i1 + (-a0 * ic) * i2 + (a0 * r2) * icw
        j_ = i_ + nicb * j1 + nic * j2  # c J_n
        s_ = j_ + nicb * s1 + nic * s2  # c^2 S_n
        if n < K:
            I[n], J[n], S[n] = float(i_), float(j_ * ic), float(s_ * ic2)
        i2, i1, j2, j1, s2, s1 = i1, i_, j1, j_, s1, s_
    return [np.array(v) for v in (I, J, S)]


def closed_forms_fp32(b, c):
    """I_0, I_1 of the reference's closed forms (Int_analytical.f90:113-114) in FP32."""
    b, c, one = f32(b), f32(c), f32(1)
    ue, ub = np.sqrt(one + b + c), np.sqrt(one - b + c)
    te, tb = one + f32(0.5) * b, -one + f32(0.5) * b
    d = c - f32(0.25) * b * b
    ae = te + ue if te >= 0 else d / (ue - te)
    ab = tb + ub if tb >= 0 else d / (ub - tb)
    i0 = f32(np.log(f32(ae / ab)))
    return float(i0), float(ue - ub - f32(0.5) * b * i0)


def worst_combination_error(got, want):
    err = 0.0
    for X, Y in zip(got, want):
        for m in range(6):
            lg = sum(a * X[p] for p, a in LEG[m].items())
            lw = sum(a * Y[p] for p, a in LEG[m].items())
            err = max(err, abs(lg - lw) / abs(Y[0]))
    return err


def cases(c):
    for ang in list(np.linspace(0.0, 1.0, 11)) + [1 - 1e-6, 1 - 1e-3]:
        for sign in (1, -1):
            yield sign * 2 * np.sqrt(c) * ang  # b = -2 p.R0, |b| <= 2 sqrt(c)


def test_backward_recursion_fp32_accuracy_for_every_far_point():
    for c in (6.0, 6.5, 8.0, 12.0, 100.0, 1e4, 3e5):
        worst = max(worst_combination_error(backward_fp32(b, c), truth(b, c)) for b in cases(c))
        assert worst <= 1e-6, (c, worst)


def test_reference_closed_forms_cancel_for_distant_pairs_in_fp32():
    c = 1e4
    b = 2 * np.sqrt(c) * 0.5
    I, _, _ = truth(b, c)
    i0, i1 = closed_forms_fp32(b, c)
    # I_1 of a pair 100 half-lengths apart: the closed form keeps no digit
    assert abs(i1 - I[1]) / abs(I[1]) > 1e-2
    got = backward_fp32(b, c)[0]
    assert abs(got[1] - I[1]) / abs(I[1]) <= 1e-5


def test_fp32_geometry_of_touching_fibers_from_the_vectors():
    """A target point 5e-5 from a source fiber's line (fibers that cross,
    as in the uniform layouts): d = c - b^2/4 formed from b and c rounds to
    zero or below in FP32, while |R0 x p|^2 keeps its relative accuracy; the
    same holds for ue^2 = |R0 - p|^2 near the fiber's end (Geom32)."""
    p = np.array([0.6, 0.0, 0.8])
    n = np.array([0.8, 0.0, -0.6])  # unit, perpendicular to p
    for s0, delta in ((0.3, 5e-5), (-0.7, 2e-5), (0.999, 3e-5)):
        R0 = s0 * p + delta * n
        d_true = delta * delta
        r = R0.astype(np.float32)
        pf = p.astype(np.float32)
        b = f32(-2) * f32(np.dot(pf, r))
        c = f32(np.dot(r, r))
        d_from_bc = float(c - f32(0.25) * b * b)
        cr = np.cross(r, pf).astype(np.float32)
        d_vec = float(np.dot(cr, cr))
        assert abs(d_vec - d_true) / d_true < 1e-3
        assert abs(d_from_bc - d_true) / d_true > 1e-2  # cancellation: no digit left
    # ue^2 = 1 + b + c at a point 3e-5 beyond the source's end
    R0 = (1.0 + 3e-5) * p
    r = R0.astype(np.float32)
    ue2_vec = float(np.dot(r - pf, r - pf))
    b = f32(-2) * f32(np.dot(pf, r))
    ue2_bc = float(f32(1) + b + f32(np.dot(r, r)))
    assert abs(ue2_vec - 9e-10) / 9e-10 < 1e-2
    assert abs(ue2_bc - 9e-10) / 9e-10 > 1e-1
