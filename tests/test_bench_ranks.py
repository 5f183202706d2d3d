"""The multi-process plumbing of bench.py's timing (Ranks, timed_steps), on
CPU with the gloo backend and two ranks: barriers around the timed region,
the timed region's length reduced as the max over ranks, one line from rank
0 only.  The GPU path runs the same functions with NCCL and CUDA events."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, sys, time
sys.path.insert(0, ROOT)
import bench
ranks = bench.Ranks("gloo", device="cpu", timeout_s=60)
delay = 0.01 * (1 + 4 * ranks.rank)          # rank 1 is the slow one
def step():
    time.sleep(delay)
    return ranks.rank
outs, max_ms, local_ms = bench.timed_steps(step, 5, 3, ranks, bench.WallTimer())
line = {"rank": ranks.rank, "outs": outs, "max_ms": max_ms, "local_ms": local_ms, "world": ranks.world}
if ranks.rank == 0:
    print(json.dumps(line), flush=True)
else:
    sys.stderr.write(json.dumps(line) + "\n")
ranks.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_max_over_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        code = RANK_SCRIPT.replace("ROOT", repr(ROOT))
        procs.append(subprocess.Popen([sys.executable, "-c", code], cwd=ROOT, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    r0 = [json.loads(x) for x in outs[0][0].splitlines() if x.strip()]
    assert len(r0) == 1 and outs[1][0].strip() == ""            # rank 1 prints nothing on stdout
    r1 = json.loads(outs[1][1].strip().splitlines()[-1])
    d = r0[0]
    assert d["world"] == 2 and d["outs"] == [0] * 5 and r1["outs"] == [1] * 5
    # the reported time is the slower rank's (5 steps of 50 ms), on both ranks
    assert abs(d["max_ms"] - max(d["local_ms"], r1["local_ms"])) < 1e-6
    assert abs(r1["max_ms"] - d["max_ms"]) < 1e-6
    assert r1["local_ms"] >= 5 * 50 * 0.9 and d["max_ms"] >= r1["local_ms"] - 1e-6
