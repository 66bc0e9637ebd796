"""Preconditioners: exact neighbour coupling blocks, the learned MLP, its GPU training.

* the numpy reference MLP (oracle/mlp_ref.py) against finite differences;
* the GPU trainer's loss and gradient against that reference;
* rotation invariance of the pair features and equivariance of the exact
  coupling blocks; their invariance under the sign of a fiber's orientation;
* preconditioned solves reach the same FP64 answer;
* the exact coupling blocks and a trained network cut GMRES iterations
  against the method without them (block-Jacobi = identity blocks).
"""
import numpy as np
import pytest

import rigidfibers_kth_b200 as rf
from oracle import mlp_ref


def _random_weights(rng, scale=0.05):
    n = sum(a * b for a, b in [(256, 144), (256, 1), (256, 256), (256, 1), (225, 256), (225, 1)])
    return (scale * rng.standard_normal(n)).astype(np.float64)


def test_reference_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = _random_weights(rng, 0.1)
    x = rng.standard_normal((5, 144))
    y = rng.standard_normal((5, 225))
    loss, g = mlp_ref.loss_grad(w, x, y)
    for idx in rng.choice(w.size, 40, replace=False):
        e = np.zeros_like(w)
        e[idx] = 1e-6
        fd = (mlp_ref.loss_grad(w + e, x, y)[0] - mlp_ref.loss_grad(w - e, x, y)[0]) / 2e-6
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


@pytest.mark.gpu
def test_trainer_gradient_matches_reference():
    from rigidfibers_kth_b200.learned import Trainer

    rng = np.random.default_rng(1)
    tr = Trainer(seed=3)
    w = tr.weights()
    x = rng.standard_normal((300, 144)).astype(np.float32)
    y = (0.1 * rng.standard_normal((300, 225))).astype(np.float32)
    loss, g = tr.loss_grad(x, y)
    loss_ref, g_ref = mlp_ref.loss_grad(w.astype(np.float64), x, y)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max()
    tr.close()


def _rotation(rng):
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    return q * np.sign(np.linalg.det(q))


@pytest.mark.gpu
def test_features_and_targets_rotate_with_the_configuration():
    rng = np.random.default_rng(2)
    pos, ori = rf.generate_layout(200, "gaussian", 1.2, 0.2, seed=1500)
    Q = _rotation(rng)
    out = []
    for P, T in [(pos, ori), (pos @ Q.T, ori @ Q.T)]:
        with rf.Simulation(rf.Configuration(rf.FiberParams(slenderness=1e-3), P, T)) as sim:
            sim.assemble_system()
            out.append((sim.features(), sim.cluster_targets()))
    (f0, t0), (f1, t1) = out
    assert f0.shape == (200 * 8, 144) and t0.shape == (200 * 8, 225)
    assert np.abs(f0 - f1).max() <= 1e-4 * np.abs(f0).max()
    assert np.abs(t0 - t1).max() <= 1e-3 * np.abs(t0).max()


@pytest.mark.gpu
def test_features_and_targets_ignore_the_sign_of_orientations():
    """A fiber and the same fiber with its orientation reversed are one
    physical object; the coefficients of odd Legendre order change sign with
    the parameterisation.  The neighbours' canonical sign in the features and
    the matching column signs of the targets make both independent of the
    neighbours' orientation signs (the fiber's own sign changes its frame,
    which the network sees)."""
    pos, ori = rf.generate_layout(150, "gaussian", 1.1, 0.2, seed=1505)
    flip = np.ones(150)
    flip[::3] = -1.0
    out = []
    for T in (ori, ori * flip[:, None]):
        with rf.Simulation(rf.Configuration(rf.FiberParams(slenderness=1e-3), pos, T)) as sim:
            sim.assemble_system()
            out.append((sim.features().reshape(150, 8, 144), sim.cluster_targets().reshape(150, 8, 225)))
    (f0, t0), (f1, t1) = out
    keep = flip > 0  # fibers whose own orientation (and frame) is unchanged
    assert np.abs(f0[keep] - f1[keep]).max() <= 1e-5 * np.abs(f0).max()
    assert np.abs(t0[keep] - t1[keep]).max() <= 1e-4 * np.abs(t0).max()


@pytest.mark.gpu
@pytest.mark.parametrize("M", [17, 700])
def test_features_follow_the_nearest_neighbours(M):
    """Slot 0 of pair (i, m) holds neighbour m's centre in fiber i's frame,
    slots 1..15 the other neighbours nearest first: the norms are the 16
    smallest centre distances in that order."""
    pos, ori = rf.generate_layout(M, "gaussian", 1.5 * (M / 200) ** (1 / 3), 0.2, seed=1510 + M)
    with rf.Simulation(rf.Configuration(rf.FiberParams(slenderness=1e-3), pos, ori)) as sim:
        f = sim.features().reshape(M, 8, 16, 9)
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    np.fill_diagonal(d, np.inf)
    want = np.sort(d, axis=1)[:, :16]
    got = np.linalg.norm(f[..., :3], axis=-1)  # (M, 8, 16)
    for m in range(8):
        order = [m] + [n for n in range(16) if n != m]
        assert np.abs(got[:, m] - want[:, order]).max() <= 1e-5 * want.max()
    # slot 0: canonical orientation (u_z >= 0) and its squares
    u = f[:, :, 0, 3:6]
    assert (u[..., 2] >= 0).all()
    assert np.abs(f[:, :, 0, 6:9] - u ** 2).max() <= 1e-6


def _solve(pos, ori, pc, weights=None, prec=rf.PREC_FP64, tol=1e-10, max_iters=600):
    p = rf.FiberParams(slenderness=1e-3, gmres_tol=tol, gmres_max_iters=max_iters, preconditioner=pc, precision=prec,
                       gmres_restart=10)
    with rf.Simulation(rf.Configuration(p, pos, ori)) as sim:
        if weights is not None:
            sim.set_mlp_weights(weights)
        sim.assemble_system()
        st = sim.solve_system()
        if tol > 1e-14:
            assert st == 0
        return sim.coeffs(), sim.solve_stats()


def _residual_after(pos, ori, pc, weights=None, iters=10):
    """Relative residual of GMRES after a fixed budget of iterations."""
    _, s = _solve(pos, ori, pc, weights, tol=1e-15, max_iters=iters)
    return s["residual"]


@pytest.mark.gpu
def test_cluster_preconditioner_same_answer_fewer_iterations():
    pos, ori = rf.generate_layout(800, "gaussian", 3.0 * (800 / 4000) ** (1 / 3), 0.2, seed=1600)
    x0, s0 = _solve(pos, ori, rf.PC_NONE)
    x1, s1 = _solve(pos, ori, rf.PC_CLUSTER)
    assert np.abs(x1 - x0).max() <= 1e-8 * np.abs(x0).max()
    assert s1["iterations"] < s0["iterations"], (s1, s0)
    assert _residual_after(pos, ori, rf.PC_CLUSTER) < _residual_after(pos, ori, rf.PC_NONE)


@pytest.mark.gpu
def test_trainer_learns_the_coupling_blocks():
    """A short training on clouds with seeds disjoint from the evaluation
    cloud: the loss falls, and on the held-out cloud the network's coupling
    blocks are closer to the exact ones than zero blocks (no
    preconditioning) are."""
    from rigidfibers_kth_b200.learned import Trainer, cloud_samples, generate_dataset

    X, Y = generate_dataset(100_000, seed0=7000, m_range=(300, 800))
    tr = Trainer(seed=11)
    tr.add_samples(X, Y)
    first = tr.train(1, batch=512, lr=1e-3)
    for _ in range(9):
        last = tr.train(1, batch=512, lr=1e-3)
    w = tr.weights()
    tr.close()
    assert last < first
    M = 800
    Xh, Yh = cloud_samples(M, 3.0 * (M / 4000) ** (1 / 3), 1601)
    _, _, pred = mlp_ref.forward(w.astype(np.float64), Xh)
    mse_learned = float(np.mean((pred - Yh) ** 2))
    mse_zero = float(np.mean(Yh.astype(np.float64) ** 2))
    assert mse_learned < 0.9 * mse_zero, (mse_learned, mse_zero)


@pytest.mark.gpu
@pytest.mark.parametrize("M", [800, 2000])
def test_shipped_network_cuts_iterations(M):
    """The shipped weights (python -m rigidfibers_kth_b200.train_preconditioner:
    400k pairs from clouds with seeds from 5000) on held-out clouds of the
    benchmark's density: the predicted coupling blocks explain most of the
    exact ones, and the preconditioned FP64 GMRES(10) reaches the same answer
    in fewer iterations than the method without it."""
    import os

    from rigidfibers_kth_b200.learned import cloud_samples

    w = np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy"))
    sigma = 3.0 * (M / 4000) ** (1 / 3)
    Xh, Yh = cloud_samples(M, sigma, 1601 + M)
    _, _, pred = mlp_ref.forward(w.astype(np.float64), Xh)
    mse_learned = float(np.mean((pred - Yh) ** 2))
    mse_zero = float(np.mean(Yh.astype(np.float64) ** 2))
    assert mse_learned < 0.5 * mse_zero, (mse_learned, mse_zero)
    pos, ori = rf.generate_layout(M, "gaussian", sigma, 0.2, seed=1601 + M)
    x0, s0 = _solve(pos, ori, rf.PC_NONE)
    x2, s2 = _solve(pos, ori, rf.PC_LEARNED, weights=w)
    assert np.abs(x2 - x0).max() <= 1e-8 * np.abs(x0).max()
    assert s2["iterations"] < s0["iterations"], (s2, s0)


@pytest.mark.gpu
def test_shipped_weights_load_and_solve():
    import os

    w = np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy"))
    from rigidfibers_kth_b200.learned import num_params

    assert w.shape == (num_params(),) and np.isfinite(w).all()
    pos, ori = rf.generate_layout(600, "gaussian", 3.0 * (600 / 4000) ** (1 / 3), 0.2, seed=1602)
    x0, _ = _solve(pos, ori, rf.PC_NONE)
    xm, _ = _solve(pos, ori, rf.PC_NONE, prec=rf.PREC_MIXED_BF16)
    x1, _ = _solve(pos, ori, rf.PC_LEARNED, weights=w, prec=rf.PREC_MIXED_BF16)
    # same (FP32 far-field) matrix, refined to the same FP64 residual: same answer
    assert np.abs(x1 - xm).max() <= 1e-8 * np.abs(xm).max()
    # against the FP64 method the FP32 far field moves the answer by ~1e-7 of its scale;
    # the velocity bound of the mixed path is 1e-6
    assert np.abs(x1 - x0).max() <= 1e-6 * np.abs(x0).max()


def _bf16(a):
    """Round to BF16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("count", [1, 1000])
def test_tensor_core_inference_matches_bf16_reference(count):
    """The preconditioner's inference (tcgen05 MMAs, BF16 operands, FP32
    accumulation in tensor memory, 128-row tiles; 1000 rows leave a partial
    tile) against numpy with the same roundings: inputs, weights and hidden
    activations rounded to BF16, sums in FP64.  The FP32 sums of the tensor
    cores and the FP64 sums of numpy round a few hidden activations to
    neighbouring BF16 values (2^-8 apart), which moves the outputs by up to
    ~2e-4 of their largest value: bound 1e-3, far below the BF16 effect
    itself (the inference is within 5e-2 of the FP32 network)."""
    import os

    from rigidfibers_kth_b200.learned import predict

    w = np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy")).astype(np.float64)
    pos, ori = rf.generate_layout(200, "gaussian", 1.7, 0.2, seed=1620)
    with rf.Simulation(rf.Configuration(rf.FiberParams(slenderness=1e-3), pos, ori)) as sim:
        X = sim.features()[:count]
    got = predict(w.astype(np.float32), X).astype(np.float64)
    W1, b1, W2, b2, W3, b3 = mlp_ref.unpack(w)
    h1 = _bf16(np.maximum(_bf16(X) @ _bf16(W1).T + b1, 0.0))
    h2 = _bf16(np.maximum(h1 @ _bf16(W2).T + b2, 0.0))
    want = h2 @ _bf16(W3).T + b3
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-3 * scale, np.abs(got - want).max() / scale
    _, _, fp32 = mlp_ref.forward(w, X)
    assert np.abs(got - fp32).max() <= 5e-2 * np.abs(fp32).max()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [rf.PREC_FP64, rf.PREC_MIXED_BF16])
def test_poor_blocks_fall_back_to_no_preconditioner(prec):
    """Weights far off the trained ones (the shipped weights x 50: coupling
    blocks thousands of times too large) make the preconditioned operator so
    ill-conditioned that GMRES stalls; the solve misses its trial budget,
    goes on without the preconditioner from its iterate and still reaches
    the tolerance with the answer of the unpreconditioned method."""
    import os

    w = np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy")) * 50.0
    pos, ori = rf.generate_layout(300, "gaussian", 3.0 * (300 / 4000) ** (1 / 3), 0.2, seed=1603)
    x0, s0 = _solve(pos, ori, rf.PC_NONE, prec=prec)
    x1, s1 = _solve(pos, ori, rf.PC_LEARNED, weights=w, prec=prec)
    assert s1["converged"] and s1["pc_fallback"], s1
    assert not s0["pc_fallback"]
    assert s1["residual"] <= 1e-10
    # both are solutions of the same system to a relative residual of 1e-10
    assert np.abs(x1 - x0).max() <= 1e-8 * np.abs(x0).max()


@pytest.mark.gpu
def test_solver_stops_using_blocks_that_do_not_pay():
    """After a solve whose blocks missed their trial, the next 8 assemblies
    neither build nor use them; then they are tried again.  Every step still
    converges to the tolerance."""
    import os

    w = np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy")) * 50.0
    pos, ori = rf.generate_layout(300, "gaussian", 3.0 * (300 / 4000) ** (1 / 3), 0.2, seed=1604)
    p = rf.FiberParams(slenderness=1e-3, gmres_tol=1e-10, gmres_max_iters=300, preconditioner=rf.PC_LEARNED,
                       precision=rf.PREC_MIXED_BF16, velocity_mode=rf.VEL_REUSE)
    used, fell = [], []
    with rf.Simulation(rf.Configuration(p, pos, ori)) as sim:
        sim.set_mlp_weights(w)
        for t in range(10):
            assert sim.step(t) == 0
            st = sim.solve_stats()
            assert st["converged"] and st["residual"] <= 1e-10
            used.append(st["preconditioned"])
            fell.append(st["pc_fallback"])
    assert used == [True] + [False] * 8 + [True], used
    assert fell[0] and fell[9] and not any(fell[1:9]), fell
