"""bench.py with two processes on CPU (gloo): the multi-GPU path of this build
is replicas only, so N > 1 runs independent builds, rank 0 alone prints one
JSON line, and every rank exits 0.  Exercised through the reference arm
(the CPU oracle), which runs without a GPU."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_reference_arm():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "h2o_ccpvdz", "--steps", "2", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["unit"] == "builds/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
