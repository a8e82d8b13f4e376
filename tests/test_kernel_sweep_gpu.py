"""GPU parity on the regular-force kernel sweep exactly as bench.py runs it.

Workload: King W0 = 6, N = 2^20 (seed 3), 100 neighbours each, list capacity
256, eps^2 = 1e-8; the j-set is uploaded un-predicted (seeded acceleration,
jerk and last-advance times) and predicted on the device to the block time.
Every active-set size of the sweep -- m = 1, 32, 1024, 32768 and m = N --
runs with the library's default plan (no tuning argument), the plan the
benchmark times.  The oracle (FP64, the reference's CPU rule of
src_mpi/Particle/ComputeAcceleration.cpp:235-299) predicts the same j-set on
the CPU (bit-identical to the device predictor) and checks:

  * m <= 1024: every row;
  * m = 32768 and m = N: 512 random rows plus every row of the i-blocks whose
    anchor offsets are least accurate.  In anchor mode (the default for
    m >= 16384) targets are ordered along a Hilbert curve and a block's FP32
    offsets are taken relative to the centre of its bounding box, so their
    error grows with the block's spread -- the largest distance of a block's
    target from that anchor -- relative to the targets' neighbour radius; the
    blocks with the largest spread / R_nb and the largest spread are checked
    whole.

Bar: the one of tests/test_regforce_gpu.py (lists and counts bit-exact; per
row |da| <= 1e-6 |a| + 1e-7 A, jerk 1e-5 / 1e-6; norm-wise 1e-6 / 1e-5;
irregular part 1e-12).  The number of rows that needed the summation-floor
term is printed for each case.
"""
import numpy as np
import pytest

import oracle
from abyss_b200 import workloads
from abyss_b200.regforce import RegularForce
from tests.helpers import check_force

pytestmark = pytest.mark.gpu

LIST_CAP = 256
EPS2 = 1e-8
N = 1 << 20


@pytest.fixture(scope="module")
def sweep():
    st = workloads.kernel_sweep_state(N)
    c = st.cluster
    rf = RegularForce(0)
    rf.upload_state(c.x, c.v, st.a0, st.a1, st.t0, c.m, c.r2nb)
    rf.predict(st.new_time, st.time_scale)
    px, pv = oracle.predict(c.x, c.v, st.a0, st.a1, st.t0, st.new_time, st.time_scale)
    yield rf, c, px, pv
    rf.close()


def widest_blocks(order_rows, targets, px, r2nb, per_block, k):
    """Indices (into the target rows) of the k i-blocks with the largest
    spread / R_nb and of the block with the largest spread."""
    slots = targets[order_rows]
    nb = (len(slots) + per_block - 1) // per_block
    rel = np.zeros(nb)
    spread = np.zeros(nb)
    for b in range(nb):
        s = slots[b * per_block:(b + 1) * per_block]
        lo, hi = px[s].min(axis=0), px[s].max(axis=0)
        d = np.abs(px[s] - (lo + 0.5 * (hi - lo))).max(axis=1)
        spread[b] = d.max()
        rel[b] = (d.max() / np.sqrt(r2nb[s])).max()
    pick = list(np.argsort(rel)[-k:]) + [int(np.argmax(spread))]
    rows = np.unique(np.concatenate([order_rows[b * per_block:(b + 1) * per_block] for b in pick]))
    return rows, float(spread.max()), float(rel.max())


def run_case(rf, c, px, pv, targets, sample_all):
    m = len(targets)
    rf.set_targets(targets)
    rf.launch(EPS2, LIST_CAP)
    res = rf.fetch(LIST_CAP)
    assert res.overflow_rows == 0
    plan = res.plan
    if sample_all:
        rows = np.arange(m)
        note = "all rows"
    else:
        per_block = plan["threads"] * plan["ipt"] if plan["kernel"] in (1, 3) else m
        order = rf.last_order()
        assert np.array_equal(np.sort(order), np.arange(m)), "processing order is not a permutation"
        wide, sp, rel = widest_blocks(order, targets, px, c.r2nb, per_block, 2)
        rand = np.random.default_rng(m).choice(m, 512, replace=False)
        rows = np.unique(np.concatenate([wide, rand]))
        note = f"{len(rows)} rows (widest blocks: spread {sp:.3g}, spread/R_nb {rel:.3g})"
    t = targets[rows]
    ref = oracle.reg_force(px, pv, c.m, c.r2nb, EPS2, t, LIST_CAP)
    scale = oracle.reg_scale(px, pv, c.m, c.r2nb, EPS2, t)
    sub = type(res)(res.acc_reg[rows], res.jerk_reg[rows], res.acc_irr[rows], res.jerk_irr[rows],
                    res.nnb[rows], res.list[rows], plan=plan)
    stats = check_force(sub, ref, f"king{N}/m={m} {note}", scale)
    return plan, stats


@pytest.mark.parametrize("m", list(workloads.SWEEP_SIZES))
def test_sweep_sizes_default_plan(sweep, m):
    rf, c, px, pv = sweep
    targets = workloads.sweep_targets(N)[m]
    plan, _ = run_case(rf, c, px, pv, targets, sample_all=m <= 1024)
    if m >= 16384:
        assert plan["kernel"] == 3 and plan["mode"] == 1, plan  # the anchor plan is the one checked


def test_full_block_default_plan(sweep):
    """m = N: the benchmark's timed step (default anchor plan, 128 x 6)."""
    rf, c, px, pv = sweep
    plan, stats = run_case(rf, c, px, pv, np.arange(N, dtype=np.int32), sample_all=False)
    assert plan["kernel"] == 3 and plan["mode"] == 1, plan
    assert stats["rows"] >= 512


def test_anchor_order_is_the_hilbert_order(sweep):
    """The device's processing order for anchor offsets is the stable sort of
    the targets' Hilbert keys on a 1024^3 grid over their FP32 bounding box,
    restated here on the CPU with the kernel's FP32 quantisation."""
    from tests.test_curve_key import numpy_hilbert

    rf, c, px, pv = sweep
    targets = workloads.sweep_targets(N)[32768]
    rf.set_targets(targets)
    rf.launch(EPS2, LIST_CAP)
    rf.fetch(LIST_CAP)
    order = rf.last_order()
    p = px[targets].astype(np.float32)
    lo, hi = p.min(axis=0), p.max(axis=0)
    sc = np.float32(1023.0) / (hi - lo)
    q = np.clip((p - lo) * sc, np.float32(0.0), np.float32(1023.0)).astype(np.int64)
    want = np.argsort(numpy_hilbert(q), kind="stable")
    assert np.array_equal(order, want)
