"""The bench's N > 1 host path on two CPU ranks (gloo): each rank's timed region is reduced to
the slowest rank, and the whole-job rate counts the units of every rank."""
import json
import os
import re
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_take_the_slowest_time():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.join(ROOT, "tests", "dist_worker.py")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    # Ranks share stdout, so their lines may interleave: take every JSON object.
    lines = [json.loads(x) for x in re.findall(r"\{[^{}]*\}", r.stdout)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    for x in lines:
        assert x["world"] == 2
        assert x["max_seconds"] == 1.5
        assert x["rate"] == 2 * 1000 * 10 / 1.5
