"""Learned neighbour-block preconditioner: data generation and GPU training.

Samples are (features, target) pairs of (fiber, neighbour) couplings: the
geometry of the fiber's 16 nearest neighbours in its own frame, the
neighbour whose block is predicted listed first (144 floats), and the
coupling block of the inverse of the fiber's k-NN cluster submatrix for that
neighbour in the same frame and sign convention (225 floats).  Both come
from the solver itself (rf_compute_features, rf_compute_cluster_targets) on
seeded clouds, 8 pairs per fiber.  The MLP (144 -> 256 -> 256 -> 225, ReLU)
is trained on the GPU by the library's own forward/backward kernels and
Adam (rf_trainer_*).
"""
import ctypes

import numpy as np

from . import _lib as L
from .simulation import Configuration, FiberParams, Simulation, generate_layout

_fp = ctypes.POINTER(ctypes.c_float)


def _f(a):
    return a.ctypes.data_as(_fp)


def num_params():
    return int(L.lib().rf_mlp_num_params())


class Trainer:
    """GPU-resident weights, Adam state and dataset (rf_trainer)."""

    def __init__(self, device=0, seed=0):
        h = ctypes.c_void_p()
        L.check(L.lib().rf_trainer_create(device, seed, ctypes.byref(h)))
        self._h = h

    def add_samples(self, features, targets):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        assert x.shape[0] == y.shape[0] and x.shape[1] == 144 and y.shape[1] == 225
        L.check(L.lib().rf_trainer_add_samples(self._h, _f(x), _f(y), x.shape[0]))

    def train(self, epochs, batch=256, lr=1e-3):
        loss = ctypes.c_float()
        L.check(L.lib().rf_trainer_train(self._h, epochs, batch, lr, ctypes.byref(loss)))
        return loss.value

    def weights(self):
        w = np.zeros(num_params(), dtype=np.float32)
        L.check(L.lib().rf_trainer_get_weights(self._h, _f(w)))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        L.check(L.lib().rf_trainer_set_weights(self._h, _f(w)))

    def loss_grad(self, features, targets):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        loss = ctypes.c_float()
        g = np.zeros(num_params(), dtype=np.float32)
        L.check(L.lib().rf_trainer_loss_grad(self._h, _f(x), _f(y), x.shape[0], ctypes.byref(loss), _f(g)))
        return loss.value, g

    def close(self):
        if getattr(self, "_h", None):
            L.lib().rf_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def predict(weights, features, device=0):
    """The network's output (count x 225) as the preconditioner computes it:
    BF16 tensor-core inference (rf_mlp_predict)."""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32)
    out = np.zeros((x.shape[0], 225), dtype=np.float32)
    L.check(L.lib().rf_mlp_predict(device, _f(w), _f(x), x.shape[0], _f(out)))
    return out


def layout_samples(pos, ori, eps=1e-3, cluster_size=8, device=0):
    """Pair features and exact cluster-inverse coupling blocks of one layout
    ((M * 8) rows each), from its FP64 system."""
    p = FiberParams(slenderness=eps, device=device, cluster_size=cluster_size)
    with Simulation(Configuration(p, pos, ori)) as sim:
        sim.assemble_system()
        y = sim.cluster_targets()
        x = sim.features()
    return x, y


def cloud_samples(M, sigma, seed, eps=1e-3, cluster_size=8, device=0):
    """Pair features and exact cluster-inverse coupling blocks of one seeded
    Gaussian cloud ((M * 8) rows each)."""
    pos, ori = generate_layout(M, "gaussian", sigma, 0.2, seed=seed)
    return layout_samples(pos, ori, eps, cluster_size, device)


def evolve(pos, ori, steps, dt=0.1, eps=1e-3, device=0):
    """The layout after `steps` time steps of the suspension (mixed-precision
    path, no preconditioner): the sedimented states a run goes through."""
    if steps <= 0:
        return pos, ori
    p = FiberParams(slenderness=eps, timestep=dt, gmres_tol=1e-10, gmres_max_iters=300, device=device,
                    precision=L.PREC_MIXED_BF16, velocity_mode=L.VEL_REUSE)
    with Simulation(Configuration(p, pos, ori)) as sim:
        for t in range(steps):
            sim.step(t)
        P, O = sim.state()
    return P.reshape(-1, 3), O.reshape(-1, 3)


def generate_dataset(n_samples, seed0=5000, m_range=(250, 2000), density_sigma4000=3.0, rng_seed=0,
                     kinds=("cloud",), max_steps=0, **kw):
    """n_samples pairs from seeded layouts of M in m_range; seeds start at
    seed0 (disjoint from the evaluation seeds 1000-1999).  Each layout is one
    of `kinds`: "cloud", a Gaussian cloud of the density of the M=4000,
    sigma=3 cloud (sigma scaled by (M/4000)^(1/3), jittered by +-20 %), or
    "box", centres uniform in a cube of 8 fibers per unit volume (the
    uniform configurations' density, jittered by +-30 %); with max_steps > 0
    the layout is first evolved by 0..max_steps time steps (dt 0.1 or 0.05)."""
    rng = np.random.default_rng(rng_seed)
    xs, ys, total, k = [], [], 0, 0
    while total < n_samples:
        M = int(rng.integers(m_range[0], m_range[1] + 1))
        kind = kinds[int(rng.integers(len(kinds)))]
        if kind == "cloud":
            sigma = density_sigma4000 * (M / 4000.0) ** (1 / 3) * float(rng.uniform(0.8, 1.2))
            pos, ori = generate_layout(M, "gaussian", sigma, 0.2, seed=seed0 + k)
        else:
            box = (M / 8.0 * float(rng.uniform(0.7, 1.3))) ** (1 / 3)
            pos, ori = generate_layout(M, "uniform", box, 0.2, seed=seed0 + k)
        steps = int(rng.integers(0, max_steps + 1)) if max_steps > 0 else 0
        dt = 0.1 if rng.uniform() < 0.5 else 0.05
        dev = kw.get("device", 0)
        pos, ori = evolve(pos, ori, steps, dt, kw.get("eps", 1e-3), dev)
        x, y = layout_samples(pos, ori, **kw)
        xs.append(x)
        ys.append(y)
        total += len(x)
        k += 1
    return np.concatenate(xs)[:n_samples], np.concatenate(ys)[:n_samples]


def train_preconditioner(n_samples=200_000, epochs=30, batch=512, lr=1e-3, seed=0, device=0, log=print,
                         kinds=("cloud",), max_steps=0):
    X, Y = generate_dataset(n_samples, device=device, kinds=kinds, max_steps=max_steps)
    tr = Trainer(device=device, seed=seed)
    tr.add_samples(X, Y)
    losses = []
    for e in range(epochs):
        lr_e = lr * (0.5 ** (e // 10))
        losses.append(tr.train(1, batch=batch, lr=lr_e))
        if log:
            log(f"epoch {e + 1}/{epochs} lr {lr_e:.2e} mse {losses[-1]:.4e} (target variance {Y.var():.4e})")
    w = tr.weights()
    tr.close()
    return w, losses, float(Y.var())
