"""The multi-GPU path of bench.py is N independent replicas: its only cross-rank
traffic is a barrier and the max over ranks of the timings.  Exercised here with two
gloo ranks on the CPU (no GPU needed)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import json, os, sys, time
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "pandora-2.0_b200"))
import bench
from pandora.params import workload_params
r = bench.Ranks("gloo", "cpu", timeout_s=60)
r.barrier()
m = r.max(0.25 + r.rank)
p = bench.replica_seeds(workload_params("iso_forced_particles", 16), r.rank)
with open(os.path.join({out!r}, "rank%d.json" % r.rank), "w") as fh:
    json.dump({{"rank": r.rank, "ws": r.ws, "max": m, "seeds": [p.seed_fluid, p.seed_force, p.seed_particles]}}, fh)
r.close()
"""


def _torchrun(nproc, args, port, timeout=240):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(port)] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_two_gloo_ranks_barrier_and_max(tmp_path):
    child = tmp_path / "child.py"
    child.write_text(_CHILD.format(root=ROOT, out=str(tmp_path)))
    r = _torchrun(2, [str(child)], 29611)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in (0, 1)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["ws"] == 2 and x["max"] == 1.25 for x in lines)      # max of 0.25 and 1.25
    assert lines[0]["seeds"] != lines[1]["seeds"]                      # each replica its own member


def test_reference_arm_under_torchrun_prints_on_rank_zero_only():
    """bench.py --impl reference with 2 ranks: rank 0 times the CPU restatement and prints
    one JSON line; the other rank exits 0 without work."""
    r = _torchrun(2, ["bench.py", "--impl", "reference", "--gpus", "2", "--grid", "16", "--particles", "64",
                      "--steps", "1", "--warmup", "0"], 29612)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    # whole RK3 steps, the counts actually run: one warm-up step at least, then the timed one
    assert d["steps"] == 1 and d["warmup"] == 1
    assert d["ms_per_step"] * d["steps"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
