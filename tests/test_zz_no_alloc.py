"""rf_matvec_noalloc: the matrix-vector product for callers that cannot allocate.

Some hosts own all device memory through their own allocator or pool, or run
loops that must not stall on cudaMalloc/cudaFree.  They pass their own device
buffers; the product keeps its partial sums in an array the library reserves
when it is loaded.  These tests check it against the handle's rf_matvec (the
existing entry point, which uses a workspace allocated with the handle) on two
calls in a row, and that sizes beyond the array are refused.

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


@pytest.mark.gpu
@pytest.mark.parametrize("M", [100, 1000])
def test_noalloc_matches_handle_matvec_twice(M):
    import torch

    pos, ori = rf.generate_layout(M, "uniform", 5.0 * (M / 1000) ** (1 / 3), 0.2, seed=2000 + M)
    cfg = rf.Configuration(rf.FiberParams(slenderness=1e-3), pos, ori)
    rng = np.random.default_rng(M)
    with rf.Simulation(cfg) as sim:
        sim.assemble_system()
        A = sim.matrix()                      # n x n column-major
        n = A.shape[0]
        xs = [rng.standard_normal(n), rng.standard_normal(n)]
        refs = [sim.matvec(x) for x in xs]    # existing entry point, handle workspace
    # the caller's own device buffers (allocated by the caller, not the library)
    A_dev = torch.from_numpy(np.asfortranarray(A).ravel(order="F")).to("cuda")
    y_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    lib = L.lib()
    for x, ref in zip(xs, refs):
        x_dev = torch.from_numpy(x).to("cuda")
        y_dev.fill_(np.nan)                   # stale output must not leak through
        torch.cuda.synchronize()
        st = lib.rf_matvec_noalloc(A_dev.data_ptr(), n, n, x_dev.data_ptr(), y_dev.data_ptr(), None)
        assert st == 0, lib.rf_last_error(None)
        torch.cuda.synchronize()
        y = y_dev.cpu().numpy()
        err = np.abs(y - ref).max() / np.abs(ref).max()
        assert err <= REL64, err
