"""CPU: the multi-process path (one process per GPU, each a replica) with two
gloo ranks: barrier, max over ranks, whole-job throughput, and the
reference arm of bench.py under torchrun (rank 0 measures and prints, the
other ranks exit 0 without work)."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RANK = r"""
import sys
sys.path.insert(0, {root!r})
from bluecrunch_b200.replicas import Replicas, job_throughput
reps = Replicas(backend="gloo", timeout_s=60)
assert (reps.world, reps.rank) == (2, {rank})
reps.barrier()
ms = reps.max(10.0 + 5.0 * reps.rank)      # rank 1 is the slow one
assert ms == 15.0, ms
v = job_throughput(100.0, ms, reps.world)  # 2 ranks x 100 units in 15 ms
assert abs(v - 200.0 / 0.015) < 1e-6, v
reps.close()
print("OK", reps.rank)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_max_and_throughput():
    port = str(_free_port())
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=port)
        procs.append(subprocess.Popen([sys.executable, "-c", _RANK.format(root=ROOT, rank=rank)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    for rank, (p, (out, err)) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, err[-2000:]
        assert out.strip().endswith("OK %d" % rank), out


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from bluecrunch_b200.replicas import Replicas
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        reps = Replicas()
        assert (reps.world, reps.rank, reps.dist) == (1, 0, None)
        assert reps.max(3.5) == 3.5
        reps.close()
    finally:
        os.environ.update(env)


def test_reference_arm_under_torchrun_two_ranks():
    port = str(_free_port())
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", port, os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout  # rank 0 alone prints
    ln = lines[0]
    assert ln["impl"] == "reference"
    if "unavailable" not in ln:
        assert ln["n_gpus"] == 2 and ln["value"] > 0 and ln["cpu_baseline"]["kind"] == "reference"


def test_reference_arm_json_contract():
    # the reference arm's line carries the keys the bench contract names
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    ln = lines[0]
    if "unavailable" in ln:
        return
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in ln, k
    assert ln["metric"] == "exact_mul_GBps" and ln["unit"] == "GB/s" and ln["higher_is_better"] is True
    assert ln["e2e"]["h2d_bytes_per_step"] == 0 and ln["e2e"]["d2h_bytes_per_step"] == 0
    assert ln["cpu_baseline"]["value"] == ln["value"] and ln["cpu_baseline"]["cores"] >= 1
    assert "workload" in ln["config"]
