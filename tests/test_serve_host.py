"""Host-side pieces of the serving loop and the autotuner, CPU only.

* The request stream (serve.poisson_requests) is seeded and reproducible: its
  arrival rate, model mix and log-uniform particle counts follow the stream's
  parameters.
* A request builds its own cluster from its model and seed (Plummer or King of
  the named W0, Kroupa masses).
* An autotuning table survives its JSON round trip (autotune.save/load).
* Lane requests start in the server's lane order (arrival, or the largest
  first) as lanes free up, never more at once than there are lanes.
"""
import math

import numpy as np

from abyss_b200 import autotune, serve


def test_poisson_stream():
    reqs = serve.poisson_requests(2000.0, 0.5, 256, 2048, seed=5, t_end=0.0625)
    again = serve.poisson_requests(2000.0, 0.5, 256, 2048, seed=5, t_end=0.0625)
    assert [(r.arrival, r.model, r.n, r.seed) for r in reqs] == [(r.arrival, r.model, r.n, r.seed) for r in again]
    # 2000 per second for 0.5 s: 1000 expected, Poisson sd ~32
    assert abs(len(reqs) - 1000) < 5 * math.sqrt(1000)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 0.5
    assert {r.model for r in reqs} == {"plummer", "king3", "king6", "king9"}
    n = np.array([r.n for r in reqs])
    assert n.min() >= 256 and n.max() <= 2048
    # log-uniform: the median sits near the geometric mean of the bounds
    assert abs(math.log(np.median(n)) - 0.5 * (math.log(256) + math.log(2048))) < 0.15
    assert all(r.t_end == 0.0625 and r.k_nb == 24 for r in reqs)


def test_request_builds_its_cluster():
    reqs = serve.poisson_requests(200.0, 0.2, 256, 512, seed=11)
    for r in reqs[:4]:
        c = r.make_cluster()
        assert c.n == r.n and abs(c.m.sum() - 1.0) < 1e-12
        assert c.m.max() > 1.5 * c.m.min()  # Kroupa masses, not equal ones
        c2 = r.make_cluster()
        assert np.array_equal(c.x, c2.x)


def test_tuning_table_round_trip(tmp_path):
    table = [(1, dict(kernel=2, ipt=1), 0.02),
             (1024, dict(kernel=3, mode=2, threads=128, ipt=4, unroll=2, min_blocks=4, j_split=0), 1.3),
             (1 << 20, dict(kernel=3, mode=1, threads=128, ipt=6, unroll=1, min_blocks=3, j_split=0), 1022.0)]
    p = tmp_path / "tuning.json"
    autotune.save(table, p)
    assert autotune.load(p) == table


class _Fut:
    def __init__(self):
        self.finished = False

    def done(self):
        return self.finished

    def result(self):
        return None


class _Pool:
    def submit(self, fn, r):
        return _Fut()


def _lanes(order, sizes, threads):
    srv = serve.Server.__new__(serve.Server)  # the lane queue alone, no GPU
    srv.lane_jobs, srv.done = [], []
    srv.lane_queue = [serve.Request(k, 0.0, "plummer", n, k) for k, n in enumerate(sizes)]
    srv.lane_threads, srv.lane_order, srv.lane_pool = threads, order, _Pool()
    return srv


def test_lane_order():
    """Two lanes, five waiting requests; a lane frees up whenever its oldest job
    finishes.  The start order is the lane order."""
    sizes = [5000, 90000, 7000, 90000, 1200]
    for order, want in (("largest", [90000, 90000, 7000, 5000, 1200]),
                        ("arrival", [5000, 90000, 7000, 90000, 1200])):
        srv = _lanes(order, sizes, 2)
        started = []
        srv._pump_lanes()
        started += [r.rid for r, _ in srv.lane_jobs]
        while srv.lane_jobs:
            assert len(srv.lane_jobs) <= 2
            srv.lane_jobs[0][1].finished = True
            srv._reap_lane()
            started += [r.rid for r, _ in srv.lane_jobs if r.rid not in started]
        assert [sizes[k] for k in started] == want, order
        assert sorted(r.n for r in srv.done) == sorted(sizes)
