"""rf_matvec_noalloc: the matrix-vector product for callers that cannot allocate.

Some hosts own all device memory through their own allocator or pool, or run
loops that must not stall on cudaMalloc/cudaFree.  They pass their own device
buffers; the product keeps its partial sums in a fixed array inside the
library, whose device address is looked up at the first call on each device.
These tests check it against an FP64 product computed on the host (numpy) and
against the handle's rf_matvec (the existing entry point, which uses a
workspace allocated with the handle), on two calls in a row; with padding rows
(lda > n) that hold NaN, which must not reach y; at the largest leading
dimension the array allows; and that sizes beyond the array are refused.

The file name sorts last so that a run stopping at the first failure has run
every other test first.
"""
import ctypes

import numpy as np
import pytest

import rigidfibers_kth_b200 as rf
from rigidfibers_kth_b200 import _lib as L

REL64 = 1e-10  # the FP64 tolerance of the parity tests (norm-wise relative)


def test_noalloc_refuses_sizes_beyond_its_array():
    """Argument checks run before any device call, so this needs no GPU."""
    lib = L.lib()
    fake = ctypes.c_void_p(1 << 20)  # never dereferenced: the size check fails first
    st = lib.rf_matvec_noalloc(fake, 1_048_578, 1_048_578, fake, fake, None)
    assert st == 1
    assert b"1048576" in lib.rf_last_error(None)
    assert lib.rf_matvec_noalloc(fake, 15, 15, fake, fake, None) == 1  # odd leading dimension
    assert lib.rf_matvec_noalloc(None, 16, 16, fake, fake, None) == 1


def _noalloc(A_dev, lda, n, x, y_dev):
    """One call through the C ABI on the caller's device buffers; returns y."""
    import torch

    lib = L.lib()
    x_dev = torch.from_numpy(np.ascontiguousarray(x)).to("cuda")
    y_dev.fill_(np.nan)  # stale output must not leak through
    torch.cuda.synchronize()
    st = lib.rf_matvec_noalloc(A_dev.data_ptr(), lda, n, x_dev.data_ptr(), y_dev.data_ptr(), None)
    assert st == 0, lib.rf_last_error(None)
    torch.cuda.synchronize()
    return y_dev.cpu().numpy()


def _rel(y, ref):
    return np.abs(y - ref).max() / np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("M", [100, 1000])
def test_noalloc_matches_host_fp64_and_handle_matvec_twice(M):
    import torch

    pos, ori = rf.generate_layout(M, "uniform", 5.0 * (M / 1000) ** (1 / 3), 0.2, seed=2000 + M)
    cfg = rf.Configuration(rf.FiberParams(slenderness=1e-3), pos, ori)
    rng = np.random.default_rng(M)
    with rf.Simulation(cfg) as sim:
        sim.assemble_system()
        A = sim.matrix()                      # n x n column-major
        n = A.shape[0]
        xs = [rng.standard_normal(n), rng.standard_normal(n)]
        handle = [sim.matvec(x) for x in xs]  # existing entry point, handle workspace
    # the caller's own device buffers (allocated by the caller, not the library)
    A_dev = torch.from_numpy(np.asfortranarray(A).ravel(order="F")).to("cuda")
    y_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    for x, ref_handle in zip(xs, handle):
        y = _noalloc(A_dev, n, n, x, y_dev)
        ref = A @ x                           # FP64 on the host
        assert _rel(y, ref) <= REL64, _rel(y, ref)
        assert _rel(y, ref_handle) <= REL64, _rel(y, ref_handle)


@pytest.mark.gpu
def test_noalloc_padding_rows_do_not_reach_y():
    """lda = n + 64: the kernel streams the padding rows too (their partial
    sums land in the array); NaN there must leave y untouched."""
    import torch

    rng = np.random.default_rng(11)
    n = 1500
    lda = n + 64
    A = rng.standard_normal((n, n))
    Apad = np.full((lda, n), np.nan)
    Apad[:n] = A
    A_dev = torch.from_numpy(Apad.ravel(order="F").copy()).to("cuda")
    y_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        x = rng.standard_normal(n)
        y = _noalloc(A_dev, lda, n, x, y_dev)
        assert np.isfinite(y).all()
        assert _rel(y, A @ x) <= REL64


@pytest.mark.gpu
def test_noalloc_at_the_largest_leading_dimension():
    """lda = 1,048,576 (the array's limit: one column split) with n = 128."""
    import torch

    rng = np.random.default_rng(12)
    n, lda = 128, 1 << 20
    A_dev = torch.empty((n, lda), dtype=torch.float64, device="cuda")  # column j = row j of this tensor
    A_dev.normal_(generator=torch.Generator(device="cuda").manual_seed(5))
    A = A_dev[:, :n].T.cpu().numpy()                                   # the n x n matrix the product uses
    y_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        x = rng.standard_normal(n)
        y = _noalloc(A_dev, lda, n, x, y_dev)
        assert _rel(y, A @ x) <= REL64
