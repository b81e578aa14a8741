"""bench.py under torchrun with two ranks on the host (gloo, no GPU): the
reference arm runs on rank 0 alone and prints the one JSON line; the other
rank joins the process group and exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

REF_DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.skipif(not os.path.exists(REF_DUMP), reason="oracle/_ref/ref_dump is not built")
def test_reference_arm_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "lj4000",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["n_gpus"] == 2
    assert d["unit"] == "ns/day" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
