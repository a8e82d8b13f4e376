"""Serving loop: admission by device room, continuous batching, completion,
energy, and the same result for a request alone and in a mix."""
import numpy as np
import pytest

from abyss_b200.serve import Request, Server, poisson_requests

pytestmark = pytest.mark.gpu


def test_stream_completes_with_admission_waits():
    reqs = poisson_requests(rate=400.0, duration=0.05, nmin=128, nmax=768, seed=11, t_end=0.03125, k_nb=16)
    assert len(reqs) >= 8
    # room for only ~3 clusters at a time: later requests must wait for retirements
    srv = Server(capacity=2400, max_clusters=16, list_cap=64, host_threads=8)
    for r in reqs:
        srv.submit(r)
    srv.run_until_idle(max_seconds=300)
    done = {r.rid: r for r in srv.done}
    srv.close()
    assert len(done) == len(reqs)
    assert max(r.result["queue_s"] for r in done.values()) > 0.0
    for r in done.values():
        assert r.result["dE_over_E"] < 1e-4, r.result
    print("completed", len(done), "peak active", srv.peak_active, "rounds", srv.rounds)


def test_request_same_alone_and_in_mix():
    mix = poisson_requests(rate=400.0, duration=0.03, nmin=128, nmax=512, seed=12, t_end=0.03125, k_nb=16)
    probe = Request(10_000, 0.0, "king6", 300, 777, t_end=0.03125, k_nb=16)
    srv = Server(capacity=1 << 16, max_clusters=32, list_cap=64, host_threads=8)
    srv.submit(probe)
    for r in mix:
        srv.submit(r)
    srv.run_until_idle(max_seconds=300)
    in_mix = next(r for r in srv.done if r.rid == 10_000).result
    srv.close()
    alone_req = Request(10_000, 0.0, "king6", 300, 777, t_end=0.03125, k_nb=16)
    srv = Server(capacity=1 << 16, max_clusters=32, list_cap=64, host_threads=8)
    srv.submit(alone_req)
    srv.run_until_idle(max_seconds=300)
    alone = srv.done[0].result
    srv.close()
    assert alone["blocks"] == in_mix["blocks"]
    assert np.array_equal(alone["x_final"], in_mix["x_final"])
    assert alone["dE_over_E"] == in_mix["dE_over_E"]


def test_device_irregular_levels_in_serving_give_the_same_results():
    """A stream served with the larger integrations' irregular levels on the GPU
    (several worker threads launching them at once) ends in the same state, bit
    for bit, as the same stream with every integration's levels on its worker
    thread."""
    def run(min_n):
        reqs = poisson_requests(rate=400.0, duration=0.04, nmin=256, nmax=2048, seed=13, t_end=0.03125, k_nb=16)
        srv = Server(capacity=1 << 17, max_clusters=32, list_cap=64, host_threads=8, max_n=2048,
                     device_irregular_min_n=min_n)
        for r in reqs:
            srv.submit(r)
        srv.run_until_idle(max_seconds=300)
        done = {r.rid: r.result for r in srv.done}
        srv.close()
        return done

    host = run(0)
    dev = run(512)
    assert sum(1 for r in dev.values() if r["device_irregular"]) >= 2
    assert sorted(host) == sorted(dev)
    for k in host:
        assert host[k]["blocks"] == dev[k]["blocks"], k
        assert np.array_equal(host[k]["x_final"], dev[k]["x_final"]), k
        assert host[k]["dE_over_E"] == dev[k]["dE_over_E"], k


@pytest.mark.parametrize("device_blocks_min_n", [0, 1])
def test_large_requests_run_whole_on_the_lane(device_blocks_min_n):
    """Requests above the lane size run whole outside the waves (the plain
    single-cluster path on a lane context, device irregular levels; or, with
    device_blocks_min_n, whole blocks on the GPU with the state kept there)
    while the others are served; a lane result equals the same integration run
    directly on the host."""
    from abyss_b200.integrator import ACIntegrator
    from abyss_b200.regforce import RegularForce

    reqs = poisson_requests(rate=400.0, duration=0.04, nmin=256, nmax=3000, seed=14, t_end=0.03125, k_nb=16)
    srv = Server(capacity=1 << 17, max_clusters=32, list_cap=64, host_threads=8, max_n=3000,
                 device_irregular_min_n=1024, lane_min_n=1500, lane_threads=2,
                 device_blocks_min_n=device_blocks_min_n)
    for r in reqs:
        srv.submit(r)
    srv.run_until_idle(max_seconds=300)
    done = {r.rid: r for r in srv.done}
    srv.close()
    assert len(done) == len(reqs)
    lane = [r for r in done.values() if r.result.get("lane")]
    assert lane and len(lane) < len(reqs)
    assert all(bool(r.result["device_blocks"]) == (device_blocks_min_n > 0) for r in lane)
    probe = lane[0]
    c = Request(probe.rid, 0.0, probe.model, probe.n, probe.seed, t_end=probe.t_end, k_nb=probe.k_nb).make_cluster()
    rf = RegularForce(0)
    try:
        ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=1e-8, eta_reg=0.02, eta_irr=0.01, fix_nb=probe.k_nb,
                          nb_max=64, t_end=probe.t_end, threads=1)
        ac.run(1.0)
        assert np.array_equal(ac.state()["x"], probe.result["x_final"])
        ac.close()
    finally:
        rf.close()
