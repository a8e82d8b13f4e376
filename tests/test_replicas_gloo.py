"""bench.py's multi-process path on CPU: two ranks over gloo (127.0.0.1).

The regular force runs as independent replicas, one per GPU, with no data
exchange; the only collectives are the barrier around the timed region and the
max over ranks of the elapsed time.  Here two CPU ranks check that rendezvous,
the max over ranks and the reference arm's rank gating (rank 0 alone works).
"""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["ROOT"])
import bench

class Args:
    n = 64
    steps = 1
    warmup = 0

world, rank, local, pg = bench.dist_setup(Args())
assert world == 2 and pg is not None
bench.barrier(pg)
slowest = bench.max_over_ranks(pg, 1.0 + rank, local)
called = []
orig = bench.workload
bench.workload = lambda n: called.append(n) or orig(n)
if rank == 1:
    bench.run_reference(Args(), world, rank, local, pg)  # other ranks exit without work
bench.barrier(pg)
print(json.dumps({"rank": rank, "slowest": slowest, "reference_worked": bool(called)}), flush=True)
pg.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_rendezvous_and_max_over_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, ROOT=ROOT, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", SCRIPT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(out.strip().splitlines()[-1])
    import json

    res = sorted((json.loads(o) for o in outs), key=lambda r: r["rank"])
    assert [r["slowest"] for r in res] == [2.0, 2.0]
    assert res[1]["reference_worked"] is False
