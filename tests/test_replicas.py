"""bench.py with N > 1 ranks (the step does not shard: N independent replicas,
one per GPU).  Its plumbing runs here as two gloo ranks on the CPU: the
barrier and the max over ranks of the timing, and the reference arm, where
rank 0 alone times the reference's CPU step and prints the JSON line while
rank 1 exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch(cmds, timeout=180):
    port = free_port()
    procs = []
    for rank, cmd in enumerate(cmds):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(len(cmds)),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(cmd, cwd=ROOT, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    out = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        out.append((p.returncode, o, e))
    return out


HELPER = """
import sys
sys.path.insert(0, {root!r})
import bench
d = bench.Dist()
d.barrier()
print(repr(d.max(1.5 + d.rank)), d.rank, d.world)
d.close()
"""


def test_dist_barrier_and_max_over_ranks():
    code = HELPER.format(root=ROOT)
    res = launch([[sys.executable, "-c", code]] * 2)
    for rc, o, e in res:
        assert rc == 0, e
    got = sorted(o.split() for _, o, _ in res)
    assert got == [["2.5", "0", "2"], ["2.5", "1", "2"]]


def test_reference_arm_runs_on_rank_0_only():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "dnsref")):
        pytest.skip("reference build absent")
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--workload", "laminar64",
           "--steps", "2", "--warmup", "1"]
    (rc0, o0, e0), (rc1, o1, e1) = launch([cmd, cmd], timeout=300)
    assert rc0 == 0 and rc1 == 0, (e0[-400:], e1[-400:])
    assert o1.strip() == ""
    line = json.loads(o0.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "MLUPS" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
