"""GPU parity of the regular-force path against the CPU oracle, through the C ABI.

Bar (written here, checked below):
  * neighbour lists and counts: bit-exact against the FP64 oracle
    (rule r2 < R_nb^2, self excluded, ascending index);
  * regular acceleration, per target i:  |da_i| <= 1e-6 |a_i| + 1e-7 A_i,
    where A_i = sum_j |m_j r_ij^-3 x_ij| over the regular j.  The first term is
    the 1e-6 relative tolerance; the second is the rounding floor of any FP32
    pair sum (about 2 FP32 ulps of the summed magnitudes) and only matters for
    targets whose terms cancel (A_i >> |a_i|);
  * regular jerk, the same with 1e-5 and 1e-6;
  * norm-wise over all targets of a call: ||da|| / ||a|| <= 1e-6 (acc) and
    <= 1e-5 (jerk);
  * irregular part (FP64 on the device): <= 1e-12 relative.
"""
import numpy as np
import pytest

import oracle
from abyss_b200 import ic
from abyss_b200.regforce import RegularForce
from tests.helpers import ACC_TOL, IRR_TOL, JERK_TOL, check_force, golden, lists_equal, row_rel_err

pytestmark = pytest.mark.gpu

TILE_DS = dict(kernel=1, mode=2)
TILE_ANCHOR = dict(kernel=1, mode=1)
JMAJOR = dict(kernel=2)
PACKED = dict(kernel=3, mode=2)
SPLIT = dict(kernel=4)
SPLIT_PACKED = dict(kernel=5)
SHAPES = [
    ("packed-ds-128x2", dict(kernel=3, mode=2, threads=128, ipt=2)),
    ("packed-ds-256x4", dict(kernel=3, mode=2, threads=256, ipt=4)),
    ("packed-ds-128x4-u2", dict(kernel=3, mode=2, threads=128, ipt=4, unroll=2, min_blocks=4)),
    ("packed-ds-128x3", dict(kernel=3, mode=2, threads=128, ipt=3)),
    ("packed-ds-128x8", dict(kernel=3, mode=2, threads=128, ipt=8)),
    ("packed-anchor-128x2", dict(kernel=3, mode=1, threads=128, ipt=2)),
    ("tile-ds-32x1", dict(kernel=1, mode=2, threads=32, ipt=1)),
    ("tile-ds-64x1", dict(kernel=1, mode=2, threads=64, ipt=1)),
    ("tile-ds-128x1", dict(kernel=1, mode=2, threads=128, ipt=1)),
    ("tile-ds-128x2", dict(kernel=1, mode=2, threads=128, ipt=2)),
    ("tile-ds-256x2", dict(kernel=1, mode=2, threads=256, ipt=2)),
    ("tile-anchor-128x1", dict(kernel=1, mode=1, threads=128, ipt=1)),
    ("jmajor-1", dict(kernel=2, ipt=1)),
    ("jmajor-8", dict(kernel=2, ipt=8)),
    ("split-ds-128x1", dict(kernel=4, ipt=1)),
    ("split-ds-128x2", dict(kernel=4, ipt=2)),
    ("split-ds-128x1-u2", dict(kernel=4, ipt=1, unroll=2)),
    ("split-ds-128x2-u2", dict(kernel=4, ipt=2, unroll=2)),
    ("split-packed-128x1", dict(kernel=5, ipt=1)),
    ("split-packed-128x2", dict(kernel=5, ipt=2)),
    ("split-packed-128x2-u2", dict(kernel=5, ipt=2, unroll=2)),
]


@pytest.fixture(scope="module")
def rf():
    r = RegularForce(0)
    yield r
    r.close()


def check(res, ref, tag, scale, acc_tol=ACC_TOL, jerk_tol=JERK_TOL):
    """Lists exact; forces within the bar in the module docstring.  `scale` is
    (A, J): per-target sums of the magnitudes of the regular acc / jerk terms."""
    return check_force(res, ref, tag, scale, acc_tol, jerk_tol)


@pytest.mark.parametrize("name", ["ref_plummer1024_s1.npz", "ref_king2048_s3.npz"])
@pytest.mark.parametrize("tag,tuning", SHAPES)
def test_golden_reference_outputs(rf, name, tag, tuning):
    """The reference's own CPU outputs (golden vectors, eps = 0)."""
    g = golden(name)
    rf.send_to_device(g["m"], g["px"], g["pv"], g["r2nb"])
    res = rf.calculate_acceleration(g["targets"], eps2=0.0, list_cap=512, tuning=tuning)
    ref = dict(nnb=g["out_nnb"], list=g["out_list"], acc_reg=g["out_a_reg"][:, :, 0],
               jerk_reg=g["out_a_reg"][:, :, 1], acc_irr=g["out_a_irr"][:, :, 0],
               jerk_irr=g["out_a_irr"][:, :, 1])
    check(res, ref, f"{name}/{tag}", oracle.reg_scale(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, g["targets"]))


@pytest.mark.parametrize("name", ["ref_plummer1024_s1.npz", "ref_king2048_s3.npz"])
def test_device_predictor_bit_exact(rf, name):
    g = golden(name)
    rf.upload_state(g["x"], g["v"], g["a_tot"][:, :, 0], g["a_tot"][:, :, 1], g["t0"], g["m"], g["r2nb"])
    rf.predict(float(g["new_time"]), float(g["time_scale"]))
    px, pv, vm = rf.read_predicted()
    assert np.array_equal(px, g["px"])
    assert np.array_equal(pv, g["pv"])
    assert np.array_equal(vm[:, 3], g["m"].astype(np.float32))
    # and the force through the device-predicted j-set equals the golden output lists
    res = rf.calculate_acceleration(g["targets"], eps2=0.0, list_cap=512)
    assert lists_equal(res.nnb, res.list, g["out_nnb"], g["out_list"])


@pytest.mark.parametrize("tag,tuning", SHAPES)
def test_softened_plummer_vs_oracle(rf, tag, tuning):
    c = ic.plummer(3000, 21, k_nb=40)
    t = np.sort(np.random.default_rng(1).choice(c.n, 1111, replace=False)).astype(np.int32)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    res = rf.calculate_acceleration(t, eps2=1e-8, list_cap=256, tuning=tuning)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 1e-8, t, 256)
    check(res, ref, f"plummer3000-eps/{tag}", oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 1e-8, t))


@pytest.mark.parametrize("m", [1, 2, 3, 31, 33, 64, 65, 257, 4095, 4096, 10000])
def test_active_block_sizes_auto(rf, m):
    c = ic.king(12000, 3, 6.0, k_nb=60)
    t = np.sort(np.random.default_rng(m).choice(c.n, m, replace=False)).astype(np.int32)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    res = rf.calculate_acceleration(t, eps2=1e-8, list_cap=256)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 1e-8, t, 256)
    check(res, ref, f"king12000/m={m}", oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 1e-8, t))


@pytest.mark.parametrize("split", [1, 2, 3, 7, 40])
def test_forced_j_splits(rf, split):
    c = ic.plummer(5001, 5, k_nb=50)
    t = np.arange(0, c.n, 3, dtype=np.int32)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 0.0, t, 256)
    scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 0.0, t)
    for tu in (dict(kernel=1, mode=2, j_split=split), dict(kernel=1, mode=1, j_split=split),
               dict(kernel=2, ipt=8, j_split=split), dict(kernel=3, mode=2, j_split=split),
               dict(kernel=4, ipt=2, j_split=split), dict(kernel=5, ipt=1, j_split=split)):
        res = rf.calculate_acceleration(t, eps2=0.0, list_cap=256, tuning=tu)
        check(res, ref, f"split{split}/{tu}", scale)


def test_unsorted_and_repeated_targets(rf):
    c = ic.plummer(2000, 8, k_nb=30)
    rng = np.random.default_rng(3)
    t = rng.integers(0, c.n, 900).astype(np.int32)  # unsorted, with repeats
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 0.0, t, 256)
    scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 0.0, t)
    for tu in (TILE_DS, TILE_ANCHOR, JMAJOR, PACKED, SPLIT, SPLIT_PACKED):
        res = rf.calculate_acceleration(t, 0.0, 256, tu)
        check(res, ref, f"unsorted/{tu}", scale)


def test_no_neighbours_and_all_neighbours(rf):
    c = ic.plummer(700, 4, k_nb=10)
    t = np.arange(c.n, dtype=np.int32)
    # R_nb = 0: every j is regular
    r0 = np.zeros(c.n)
    rf.send_to_device(c.m, c.x, c.v, r0)
    ref = oracle.reg_force(c.x, c.v, c.m, r0, 1e-8, t, 64)
    scale = oracle.reg_scale(c.x, c.v, c.m, r0, 1e-8, t)
    # (anchor offsets are left out: with R_nb = 0 the closest pairs enter the
    # regular sum, and anchor offsets of a spread-out block of targets are only
    # accurate for pairs wider than the block; the library picks anchor mode only
    # for large active sets ordered along a Hilbert curve)
    for tu in (TILE_DS, JMAJOR, PACKED, SPLIT, SPLIT_PACKED):
        res = rf.calculate_acceleration(t, 1e-8, 64, tu)
        assert res.nnb.sum() == 0
        check(res, ref, f"R=0/{tu}", scale)
    # R_nb huge: every j is a neighbour, lists overflow a small cap with exact counts
    big = np.full(c.n, 1e6)
    rf.send_to_device(c.m, c.x, c.v, big)
    ref = oracle.reg_force(c.x, c.v, c.m, big, 1e-8, t, 100)
    for tu in (TILE_DS, TILE_ANCHOR, JMAJOR, PACKED, SPLIT, SPLIT_PACKED):
        res = rf.calculate_acceleration(t, 1e-8, 100, tu)
        assert res.overflow_rows == c.n
        assert np.all(res.nnb == c.n - 1)
        assert np.array_equal(res.list, ref["list"])
        assert np.abs(res.acc_reg).max() == 0.0 and np.abs(res.jerk_reg).max() == 0.0
        # the irregular part of an overflowed row sums all its neighbours, not the first list_cap
        assert row_rel_err(res.acc_irr, ref["acc_irr"]).max() <= IRR_TOL, tu
        assert row_rel_err(res.jerk_irr, ref["jerk_irr"]).max() <= IRR_TOL, tu


@pytest.mark.parametrize("m", [1, 37, 250])
def test_overflow_with_few_rows(rf, m):
    """Launches of at most 2 x 148 rows finalize a row per block and re-list an
    overflowed row inside that block: the same truncated ascending list and full
    irregular sums as the warp-per-row path."""
    c = ic.plummer(700, 4, k_nb=10)
    t = np.sort(np.random.default_rng(m).choice(c.n, m, replace=False)).astype(np.int32)
    big = np.full(c.n, 1e6)
    rf.send_to_device(c.m, c.x, c.v, big)
    ref = oracle.reg_force(c.x, c.v, c.m, big, 1e-8, t, 100)
    for tu in (TILE_DS, JMAJOR, PACKED, SPLIT, SPLIT_PACKED):
        res = rf.calculate_acceleration(t, 1e-8, 100, tu)
        assert res.overflow_rows == m, tu
        assert np.all(res.nnb == c.n - 1), tu
        assert np.array_equal(res.list, ref["list"]), tu
        assert np.abs(res.acc_reg).max() == 0.0 and np.abs(res.jerk_reg).max() == 0.0
        assert row_rel_err(res.acc_irr, ref["acc_irr"]).max() <= IRR_TOL, tu
        assert row_rel_err(res.jerk_irr, ref["jerk_irr"]).max() <= IRR_TOL, tu


@pytest.mark.parametrize("n", [2, 3, 5, 127, 129, 255, 257])
def test_tiny_and_ragged_jsets(rf, n):
    c = ic.plummer(n, 100 + n, k_nb=min(4, n - 1) + 0.5)
    t = np.arange(n, dtype=np.int32)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 0.0, t, 32)
    scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 0.0, t)
    for tu in (TILE_DS, TILE_ANCHOR, JMAJOR, PACKED, SPLIT, SPLIT_PACKED):
        res = rf.calculate_acceleration(t, 0.0, 32, tu)
        check(res, ref, f"n={n}/{tu}", scale)


def test_bad_arguments_are_reported_not_trapped(rf):
    from abyss_b200._lib import AbyssError

    c = ic.plummer(100, 1, k_nb=5)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    with pytest.raises(AbyssError):
        rf.calculate_acceleration(np.array([0, 100], np.int32))  # index out of range
    with pytest.raises(AbyssError):
        rf.calculate_acceleration(np.array([], np.int32))
    with pytest.raises(AbyssError):
        rf.calculate_acceleration(np.array([1], np.int32), eps2=-1.0)
    with pytest.raises(AbyssError):
        rf.calculate_acceleration(np.array([1], np.int32), tuning=dict(kernel=1, threads=96))
    # the context is still usable
    res = rf.calculate_acceleration(np.array([1, 2], np.int32), list_cap=16)
    assert res.acc_reg.shape == (2, 3)


@pytest.mark.parametrize("kernel,threads,ipt", [(1, 128, 2), (1, 128, 4), (1, 256, 2), (3, 128, 2),
                                                (3, 128, 3), (3, 128, 4), (3, 256, 2), (3, 256, 4),
                                                (3, 128, 6), (3, 128, 8)])
def test_anchor_mode_on_dense_active_set(rf, kernel, threads, ipt):
    """Anchor offsets are accurate when a block's targets are spatially compact,
    which the library arranges by ordering large active sets along a Hilbert
    curve (blocks anchored at the centre of their bounding box)."""
    c = ic.king(65536, 17, 6.0, k_nb=80)
    t = np.arange(c.n, dtype=np.int32)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    res = rf.calculate_acceleration(t, eps2=1e-8, list_cap=256,
                                    tuning=dict(kernel=kernel, mode=1, threads=threads, ipt=ipt))
    sample = np.random.default_rng(4).choice(c.n, 2048, replace=False)
    ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, 1e-8, t[sample], 256)
    scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, 1e-8, t[sample])
    sub = type(res)(res.acc_reg[sample], res.jerk_reg[sample], res.acc_irr[sample],
                    res.jerk_irr[sample], res.nnb[sample], res.list[sample], plan=res.plan)
    check(sub, ref, f"king65536-anchor-k{kernel}-{threads}x{ipt}", scale)
    assert np.all(res.nnb == 80)


def test_blocking_wait_policy_gives_the_same_results():
    """abyss_set_wait changes how the host waits, not what is computed: with a
    spin of 0 or 50 us before the blocking wait, every output is identical to
    the default wait's; a negative spin restores the default."""
    c = ic.king(4000, 9, 6.0, k_nb=40)
    t = np.arange(0, c.n, 2, dtype=np.int32)
    r = RegularForce(0)
    try:
        r.send_to_device(c.m, c.x, c.v, c.r2nb)
        want = r.calculate_acceleration(t, eps2=1e-8, list_cap=256)
        for spin in (0, 50, -1):
            r.set_wait(spin)
            r.send_to_device(c.m, c.x, c.v, c.r2nb)
            got = r.calculate_acceleration(t, eps2=1e-8, list_cap=256)
            for k in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr", "nnb", "list"):
                assert np.array_equal(getattr(got, k), getattr(want, k)), (spin, k)
            assert r.energy(c.x, c.v, c.m, 1e-8) == r.energy(c.x, c.v, c.m, 1e-8)
    finally:
        r.close()


def test_whole_launch_timing(rf):
    """abyss_set_profiling(2): one interval around the whole launch, reported as
    the force time with the other two zero; per-phase timing sums to about it."""
    c = ic.plummer(4096, 9, k_nb=40)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    t = np.arange(0, c.n, 2, dtype=np.int32)
    rf.set_targets(t)
    rf.set_profiling("whole")
    rf.launch(0.0, 256)
    whole = rf.last_timing()
    assert whole["order_ms"] == 0.0 and whole["finalize_ms"] == 0.0 and whole["force_ms"] > 0.0
    rf.set_profiling(True)
    rf.launch(0.0, 256)
    parts = rf.last_timing()
    assert parts["force_ms"] > 0.0 and parts["finalize_ms"] > 0.0
    rf.set_profiling(False)
