"""bench.py's multi-rank plumbing on CPU: two gloo ranks.

`bench.py --gpus N` runs N independent replicas (one process per GPU, launched
by torchrun): every rank times its own steps between barriers and the job
time is the maximum over ranks.  Here two CPU processes stand in for the
GPUs: the same rendezvous (127.0.0.1), the same barrier and max-over-ranks
helpers, on the gloo backend, and the reference arm's rule that only rank 0
works and prints.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_CODE = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup(timeout_s=60)
bench.barrier(world)
worst = bench.max_over_ranks(1.5 + rank, world)
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--M", "20"]
ref = None
if rank != 0:
    ref = bench.run_reference(bench.parse_args())
bench.barrier(world)
import torch.distributed as dist
backend = dist.get_backend()
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "world": world, "max": worst, "backend": backend, "ref": ref}}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_barrier_and_max_over_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("a rank did not finish")
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    for d in outs:
        assert d["world"] == 2 and d["backend"] == "gloo"
        assert d["max"] == 2.5  # the slowest rank's time is the job's time
    assert outs[1]["ref"] is None  # the reference arm runs on rank 0 only


def test_reference_arm_json_line_contract():
    """`bench.py --impl reference` on one process (a small M keeps it short):
    one JSON line with the contract's keys, the CPU baseline describing the
    run, an end-to-end figure without host-device traffic, the same `config`
    as the product arm, and the timed parts adding up to one whole step."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--M", "40",
                        "--steps", "4", "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # K parts of one step: value = 1 step / (K x mean part time)
    assert abs(d["value"] * d["steps"] * d["ms_per_step"] * 1e-3 - 1.0) < 1e-9
    assert d["arm"]["gmres"]["info"] == 0 and d["arm"]["gmres"]["residual"] <= 1e-10
    sys.path.insert(0, ROOT)
    import bench

    assert d["config"] == bench.workload_config(40, 1)


def test_reference_arm_loads_only_the_oracle():
    """The reference arm must not map the product library: its layout comes
    from the oracle's restatement of the generator."""
    code = ("import json, sys; sys.path.insert(0, {root!r}); import bench; "
            "sys.argv = ['bench.py', '--impl', 'reference', '--M', '20', '--steps', '1', '--warmup', '0']; "
            "out = bench.run_reference(bench.parse_args()); maps = open('/proc/self/maps').read(); "
            "print(json.dumps({{'ok': out is not None, 'product': 'librigidfibers' in maps, "
            "'oracle': 'librfo' in maps}}))").format(root=ROOT)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d == {"ok": True, "product": False, "oracle": True}


def test_reference_gpu_arm_parses_the_programs_timers_and_reports_a_missing_build(monkeypatch):
    """`bench.py --impl reference-gpu`: the phase times come from the
    reference program's own "[BENCHMARK]" lines (seconds, last then average);
    without the built program the arm prints its `unavailable` line."""
    import bench

    out = ("     [GPU]      : Assembling system...\n"
           "  [BENCHMARK]   : assemble_system   : 0.00298(0.00298) sec\n"
           "  [BENCHMARK]   : solve_system      : 0.00653(0.00653) sec\n"
           "  [BENCHMARK]   : update_velocities : 0.00735(0.00735) sec\n"
           "  [BENCHMARK]   : update_fibers_firststep : 0.00008(0.00008) sec\n")
    ph = bench._ref_gpu_phases(out)
    assert set(ph) == set(bench.REF_GPU_PHASES)
    assert ph["solve_system"] == 0.00653
    # the parameter file is the positional v1 format of run100_iter.in
    assert len(bench.REF_GPU_PARAMS) == 14 and bench.REF_GPU_PARAMS[3] == "0.01"
    monkeypatch.setattr(bench, "REF_GPU_EXE", os.path.join(ROOT, "oracle", "_ref", "no_such_program"))
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference-gpu", "--steps", "1", "--warmup", "0"])
    d = bench.run_reference_gpu(bench.parse_args())
    assert d["impl"] == "reference-gpu" and "unavailable" in d
