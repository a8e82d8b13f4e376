"""Batched ensemble: many clusters of uneven N and uneven active sets per wave.

* every cluster's rows match the FP64 oracle (lists exact, forces within the
  bar of tests/test_regforce_gpu.py);
* the batched launch, its CUDA-graph replay and the one-cluster-per-launch form
  give bit-identical results, and so does a cluster alone versus in a mix;
* bad waves are refused with a status, and the ensemble stays usable.
"""
import numpy as np
import pytest

import oracle
from abyss_b200 import ic
from abyss_b200.ensemble import BATCHED, GRAPH, PLAIN, Ensemble
from abyss_b200.regforce import RegularForce
from tests.test_regforce_gpu import check

pytestmark = pytest.mark.gpu
EPS2 = 1e-8


@pytest.fixture(scope="module")
def rf():
    r = RegularForce(0)
    yield r
    r.close()


def make_ensemble(rf, k=24, seed=4):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(256), np.log(4096), k)).astype(int)
    clusters = [ic.plummer(int(n), 4000 + i, k_nb=24) for i, n in enumerate(sizes)]
    e = Ensemble(rf, sizes, list_cap=128)
    for i, c in enumerate(clusters):
        a = np.zeros((c.n, 3))
        e.upload_state(i, c.x, c.v, a, a, np.zeros(c.n), c.m, c.r2nb)
    return e, clusters


def random_wave(rng, clusters):
    k = len(clusters)
    chosen = np.sort(rng.choice(k, max(1, k // 2), replace=False))
    targets = []
    for i in chosen:
        n = clusters[i].n
        frac = 2.0 ** -rng.integers(0, 6)
        m = max(1, int(n * frac))
        targets.append(np.sort(rng.choice(n, m, replace=False)).astype(np.int32))
    return chosen, targets


def test_batched_matches_oracle_and_plain(rf):
    e, clusters = make_ensemble(rf)
    rng = np.random.default_rng(9)
    for wave in range(3):
        chosen, targets = random_wave(rng, clusters)
        e.set_wave(chosen, np.zeros(len(chosen)), np.ones(len(chosen)), targets)
        results = {}
        for mode in (BATCHED, GRAPH, PLAIN, GRAPH):
            e.launch(EPS2, mode)
            results[mode] = e.fetch()
        b, g, p = results[BATCHED], results[GRAPH], results[PLAIN]
        for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
            assert np.array_equal(getattr(b, f), getattr(g, f)), f"graph differs in {f}"
            assert np.array_equal(getattr(b, f), getattr(p, f)), f"plain differs in {f}"
        for idx, ci in enumerate(chosen):
            c = clusters[ci]
            r0, r1 = e.row_splits[idx], e.row_splits[idx + 1]
            t = targets[idx]
            ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, EPS2, t, 128)
            sub = type(b)(b.acc_reg[r0:r1], b.jerk_reg[r0:r1], b.acc_irr[r0:r1], b.jerk_irr[r0:r1],
                          b.nnb[r0:r1], b.list[r0:r1])
            check(sub, ref, f"wave{wave}/cluster{ci}", oracle.reg_scale(c.x, c.v, c.m, c.r2nb, EPS2, t))


def test_cluster_result_same_alone_and_in_mix(rf):
    e, clusters = make_ensemble(rf, k=12, seed=5)
    rng = np.random.default_rng(2)
    chosen, targets = random_wave(rng, clusters)
    e.set_wave(chosen, np.zeros(len(chosen)), np.ones(len(chosen)), targets)
    e.launch(EPS2, GRAPH)
    mix = e.fetch()
    for idx, ci in enumerate(chosen):
        c = clusters[ci]
        e.set_wave([ci], [0.0], [1.0], [targets[idx]])
        e.launch(EPS2, BATCHED)
        alone = e.fetch()
        lo = sum(len(t) for t in targets[:idx])
        hi = lo + len(targets[idx])
        # a cluster's chunking depends on its own size only: bit-identical
        for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
            assert np.array_equal(getattr(alone, f), getattr(mix, f)[lo:hi]), f"cluster {ci}: {f}"


def test_bad_waves_are_refused(rf):
    from abyss_b200._lib import AbyssError

    e, clusters = make_ensemble(rf, k=4, seed=6)
    with pytest.raises(AbyssError):
        e.set_wave([0, 0], [0.0, 0.0], [1.0, 1.0], [np.array([1]), np.array([2])])  # repeated cluster
    with pytest.raises(AbyssError):
        e.set_wave([7], [0.0], [1.0], [np.array([1])])  # no such cluster
    with pytest.raises(AbyssError):
        e.set_wave([1], [0.0], [1.0], [np.array([clusters[1].n])])  # index out of range
    e.set_wave([1], [0.0], [1.0], [np.array([0, 1, 2])])
    e.launch(EPS2, BATCHED)
    assert e.fetch().acc_reg.shape == (3, 3)


def test_staged_upload_matches_and_leaves_unlisted_clusters(rf):
    """Staged uploads give the same wave results as per-cluster uploads, and a
    cluster that is not listed keeps its device state even when it lies between
    listed ones (its staging was never written)."""
    e, clusters = make_ensemble(rf, k=6, seed=7)
    rng = np.random.default_rng(3)
    allk = np.arange(len(clusters))
    targets = [np.sort(rng.choice(c.n, max(1, c.n // 3), replace=False)).astype(np.int32) for c in clusters]
    e.set_wave(allk, np.zeros(len(allk)), np.ones(len(allk)), targets)
    e.launch(EPS2, GRAPH)
    want = e.fetch()
    # clusters 0, 2, 4 restaged (same state); 1, 3, 5 keep their device state
    for k in (0, 2, 4):
        st = e.stage(k)
        c = clusters[k]
        st["x"][:] = c.x
        st["v"][:] = c.v
        st["a0"][:] = 0.0
        st["a1"][:] = 0.0
        st["t0"][:] = 0.0
        st["mass"][:] = c.m
        st["r2nb"][:] = c.r2nb
    e.upload_staged([0, 2, 4])
    e.set_wave(allk, np.zeros(len(allk)), np.ones(len(allk)), targets)
    e.launch(EPS2, GRAPH)
    got = e.fetch()
    for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
        assert np.array_equal(getattr(got, f), getattr(want, f)), f
    e.close()


def test_two_waves_in_flight_match_blocking_waves(rf):
    """Two submitted waves (disjoint clusters, staged state) give the same rows
    as the same waves run one at a time with set_wave/launch/fetch."""
    e, clusters = make_ensemble(rf, k=8, seed=11)
    rng = np.random.default_rng(5)
    waves = [np.array([0, 2, 3, 6]), np.array([1, 4, 5, 7])]
    targets = {k: np.sort(rng.choice(c.n, max(1, c.n // 4), replace=False)).astype(np.int32)
               for k, c in enumerate(clusters)}
    want = []
    for w in waves:
        e.set_wave(w, np.zeros(len(w)), np.ones(len(w)), [targets[k] for k in w])
        e.launch(EPS2, GRAPH)
        want.append(e.fetch())
    for k, c in enumerate(clusters):  # the same state, through the staging
        st = e.stage(k)
        st["x"][:] = c.x
        st["v"][:] = c.v
        st["a0"][:] = 0.0
        st["a1"][:] = 0.0
        st["t0"][:] = 0.0
        st["mass"][:] = c.m
        st["r2nb"][:] = c.r2nb
    for rep in range(2):
        tickets = [e.submit(w, np.zeros(len(w)), np.ones(len(w)), [targets[k] for k in w], EPS2, GRAPH)
                   for w in waves]
        got = [e.collect(t) for t in tickets]
        for g, w in zip(got, want):
            for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
                assert np.array_equal(getattr(g, f), getattr(w, f)), (rep, f)
    e.close()


TUNED_SHAPE = dict(kernel=3, mode=2, threads=128, ipt=4, unroll=2, min_blocks=4)
TUNED_CHUNKS = [(1024, 512), (4096, 1024)]


def test_tuned_shape_and_chunks_change_the_plan_not_the_parity(rf):
    """A tuning (launch shape + chunk table by cluster size) changes the work
    list; every cluster's rows still match the oracle, the batched, graph and
    plain forms agree bit for bit, and a cluster alone gives the same rows as
    in the mix (its chunking depends on its own size only)."""
    e, clusters = make_ensemble(rf, k=12, seed=13)
    rng = np.random.default_rng(21)
    chosen, targets = random_wave(rng, clusters)
    e.set_wave(chosen, np.zeros(len(chosen)), np.ones(len(chosen)), targets)
    e.launch(EPS2, GRAPH)
    e.fetch()
    default_shape, default_items = e.shape(), e.last_stats()["items"]
    e.set_tuning(TUNED_SHAPE, TUNED_CHUNKS)
    sh = e.shape()
    assert (sh["threads"], sh["ipt"], sh["unroll"], sh["min_blocks"]) == (128, 4, 2, 4) != (
        default_shape["threads"], default_shape["ipt"], default_shape["unroll"], default_shape["min_blocks"])
    e.set_wave(chosen, np.zeros(len(chosen)), np.ones(len(chosen)), targets)
    res = {}
    for mode in (GRAPH, BATCHED, PLAIN):
        e.launch(EPS2, mode)
        res[mode] = e.fetch()
    assert e.last_stats()["items"] != default_items
    mix = res[GRAPH]
    for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
        assert np.array_equal(getattr(res[BATCHED], f), getattr(mix, f)), f
        assert np.array_equal(getattr(res[PLAIN], f), getattr(mix, f)), f
    for idx, ci in enumerate(chosen):
        c = clusters[ci]
        lo, hi = e.row_splits[idx], e.row_splits[idx + 1]
        t = targets[idx]
        ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, EPS2, t, 128)
        sub = type(mix)(mix.acc_reg[lo:hi], mix.jerk_reg[lo:hi], mix.acc_irr[lo:hi], mix.jerk_irr[lo:hi],
                        mix.nnb[lo:hi], mix.list[lo:hi])
        check(sub, ref, f"tuned/cluster{ci}", oracle.reg_scale(c.x, c.v, c.m, c.r2nb, EPS2, t))
    for idx, ci in enumerate(chosen):
        e.set_wave([ci], [0.0], [1.0], [targets[idx]])
        e.launch(EPS2, GRAPH)
        alone = e.fetch()
        lo, hi = e.row_splits[0], e.row_splits[1]
        lo2 = sum(len(t) for t in targets[:idx])
        for f in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
            assert np.array_equal(getattr(alone, f)[lo:hi], getattr(mix, f)[lo2:lo2 + len(targets[idx])]), (ci, f)
    e.close()


def test_bad_tunings_are_refused(rf):
    from abyss_b200._lib import AbyssError

    e, clusters = make_ensemble(rf, k=4, seed=14)
    for shape, chunks in ((dict(kernel=3, mode=1, threads=128, ipt=2), ()),      # anchor offsets
                          (dict(kernel=2, ipt=4), ()),                           # not a tile kernel
                          (dict(kernel=1, mode=2, threads=32, ipt=1), ()),       # < 128 targets per block
                          (dict(kernel=3, mode=2, threads=96, ipt=2), ()),       # not compiled
                          (None, [(1024, 64)]),                                  # chunk < 128 j
                          (None, [(4096, 512), (1024, 512)])):                   # n_max not rising
        with pytest.raises(AbyssError):
            e.set_tuning(shape, chunks)
    e.set_wave([1], [0.0], [1.0], [np.arange(5, dtype=np.int32)])
    e.launch(EPS2, GRAPH)
    assert e.fetch().acc_reg.shape == (5, 3)
    e.close()


def test_autotuner_picks_a_shape_on_the_ensembles_waves(rf):
    """tune_ensemble times the compiled double-single shapes and chunk lengths
    on the ensemble's own waves, installs the fastest, and the installed shape
    still gives the oracle's lists."""
    from abyss_b200 import autotune

    e, clusters = make_ensemble(rf, k=16, seed=15)
    rng = np.random.default_rng(8)
    waves = [random_wave(rng, clusters) for _ in range(2)]
    res = autotune.tune_ensemble(e, waves, chunks=(512, 2048))
    print("tuned ensemble:", res)
    assert res["ms"] <= res["default_ms"] and res["trials"] > 4
    assert e.shape()["threads"] == res["shape"]["threads"] and e.shape()["ipt"] == res["shape"]["ipt"]
    chosen, targets = waves[0]
    e.set_wave(chosen, np.zeros(len(chosen)), np.ones(len(chosen)), targets)
    e.launch(EPS2, GRAPH)
    got = e.fetch()
    for idx, ci in enumerate(chosen):
        c = clusters[ci]
        lo, hi = e.row_splits[idx], e.row_splits[idx + 1]
        ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, EPS2, targets[idx], 128)
        assert np.array_equal(got.nnb[lo:hi], ref["nnb"])
    e.close()
