"""The host integrator's irregular step and level rules (include/abyss_host.h)
against the reference's own outputs, CPU only.

Golden vectors from the reference's CPU code (tests/golden/make_golden.py):
* computeAccelerationIrr then calculateTimeStepIrr (the IrrForce task,
  WorkerRoutines.cpp:46-64) for every particle with neighbours, and a few
  without, of the two regular-step states: the new velocity, a_irr, a_tot and
  irregular level are bit-exact.  The new position differs by exactly the
  corrector's a3 dt^5/120 term: the reference reads an uninitialised dt5
  (ComputeAcceleration.cpp:162), which the compiled reference treats as zero,
  and the integrator uses dt^4 * dt.
* calculateTimeStepIrr, calculateTimeStepReg, initializeTimeStep and
  updateRadius on seeded block states that reach each branch: bit-exact
  levels, blocks and steps.  (The
  regular rule's clamp at the end of the run is not reached from states on the
  block grid: a level only rises where the current block is aligned to it.)
With the reference tree built (oracle/_ref), a fresh seeded state is checked
against the reference library directly as well.
"""
import ctypes as C

import numpy as np
import pytest

from abyss_b200 import _lib
from abyss_b200._lib import ptr, _ip
from tests.helpers import golden

CASES = ["ref_plummer1024_s1", "ref_king2048_s3"]


def _c(a, dt=None):
    return np.ascontiguousarray(a, dt)


def host_irregular(st, idx, eps2=0.0):
    """abyss_host_irregular_steps over the listed particles of a state dict."""
    L = _lib.lib()
    n = st["x"].shape[0]
    idx = _c(idx, np.int32)
    k = idx.shape[0]
    pos = np.zeros((k, 3))
    vel = np.zeros((k, 3))
    a_irr = np.zeros((k, 3, 4))
    a_tot = np.zeros((k, 3, 4))
    nb = _c(st["nb"], np.int32)
    rc = L.abyss_host_irregular_steps(n, ptr(_c(st["x"])), ptr(_c(st["v"])), ptr(_c(st["m"])),
                                      ptr(_c(st["a_tot"])), ptr(_c(st["a_reg"])), ptr(_c(st["a_irr"])),
                                      ptr(_c(st["t_reg"])), ptr(_c(st["t_irr"])), ptr(_c(st["dt_irr"])),
                                      ptr(_c(st["nnb"], np.int32), _ip), ptr(nb, _ip), nb.shape[1], eps2,
                                      float(st["time_scale"]), k, ptr(idx, _ip), ptr(pos), ptr(vel),
                                      ptr(a_irr), ptr(a_tot))
    assert rc == 0
    return pos, vel, a_irr, a_tot


def host_level_irr(scale, time_block, eta, has_nb, a_tot, a_irr, new_cur, cur_reg, tb_reg, lv_reg, lv_irr,
                   dt_irr, tb_irr):
    L = _lib.lib()
    lv = C.c_int(int(lv_irr))
    dt = C.c_double(float(dt_irr))
    tb = C.c_ulonglong(int(tb_irr))
    rc = L.abyss_host_time_level_irr(float(scale), int(time_block), float(eta), int(has_nb),
                                     ptr(_c(a_tot, np.float64)), ptr(_c(a_irr, np.float64)), int(new_cur),
                                     int(cur_reg), int(tb_reg), int(lv_reg), C.byref(lv), C.byref(dt), C.byref(tb))
    return rc, lv.value, dt.value, tb.value


def _pos_matches_without_a3_term(pos, ref_pos, a3, dt):
    """ours = ref + a3 dt^5/120, up to the rounding of the two sums."""
    term = a3 * dt ** 5 / 120.0
    slack = 4 * np.spacing(np.abs(ref_pos)) + 4 * np.spacing(np.abs(term))
    return np.all(np.abs((pos - ref_pos) - term) <= slack)


@pytest.mark.parametrize("name", CASES)
def test_irregular_step_bit_exact(name):
    base = golden(name + ".npz")
    g = golden(name + "_irr.npz")
    idx = g["idx"]
    pos, vel, a_irr, a_tot = host_irregular(base, idx)
    assert np.array_equal(vel, g["out_newvel"])
    assert np.array_equal(a_irr, g["out_a_irr"])
    assert np.array_equal(a_tot, g["out_a_tot"])
    has = base["nnb"][idx] > 0
    assert has.sum() > 0 and (~has).sum() > 0
    # no neighbours: nothing moves, as in the reference
    assert np.array_equal(pos[~has], g["out_newpos"][~has])
    dt = base["dt_irr"][idx][has] * float(base["time_scale"])
    assert _pos_matches_without_a3_term(pos[has], g["out_newpos"][has], a_irr[has][:, :, 3], dt[:, None])


@pytest.mark.parametrize("name", CASES)
def test_irregular_level_after_the_step_bit_exact(name):
    base = golden(name + ".npz")
    g = golden(name + "_irr.npz")
    tblock = int(g["time_block"])
    step = 2.0 ** tblock
    eta = float(golden("ref_levels.npz")["eta"])
    for r, i in enumerate(g["idx"]):
        cur_irr = int(round(base["t_irr"][i] / step))
        tb = int(round(base["dt_irr"][i] / step))
        rc, lv, dt, tbo = host_level_irr(float(base["time_scale"]), tblock, eta, base["nnb"][i] > 0,
                                         g["out_a_tot"][r], g["out_a_irr"][r], cur_irr + tb, 0,
                                         int(round(base["dt_reg"][i] / step)), int(round(np.log2(base["dt_reg"][i]))),
                                         int(round(np.log2(base["dt_irr"][i]))), base["dt_irr"][i], tb)
        assert rc == 0
        assert (lv, dt, tbo) == (g["out_lv_irr"][r], g["out_dt_irr"][r], g["out_tb_irr"][r]), r


def test_irregular_level_rules_bit_exact():
    g = golden("ref_levels.npz")
    tblock, eta = int(g["time_block"]), float(g["eta"])
    k = g["irr_scale"].shape[0]
    outcomes = set()
    for q in range(k):
        rc, lv, dt, tb = host_level_irr(g["irr_scale"][q], tblock, eta, g["irr_has_nb"][q], g["irr_a_tot"][q],
                                        g["irr_a_irr"][q], g["irr_new_cur_irr"][q], g["irr_cur_reg"][q],
                                        g["irr_tb_reg"][q], g["irr_lv_reg"][q], g["irr_lv_irr"][q],
                                        g["irr_dt_irr"][q], g["irr_tb_irr"][q])
        assert rc == 0
        assert (lv, dt, tb) == (g["irr_out_lv_irr"][q], g["irr_out_dt_irr"][q], g["irr_out_tb_irr"][q]), q
        outcomes.add(int(lv) - int(g["irr_lv_irr"][q]))
    # up one, kept, down one and two
    assert {1, 0, -1, -2} <= outcomes


def test_regular_level_rules_bit_exact():
    L = _lib.lib()
    g = golden("ref_levels.npz")
    tblock, eta, bmax = int(g["time_block"]), float(g["eta"]), int(g["block_max"])
    k = g["reg_scale"].shape[0]
    moves = set()
    for q in range(k):
        lv = C.c_int(int(g["reg_lv_reg"][q]))
        dt = C.c_double(float(g["reg_dt_reg"][q]))
        tb = C.c_ulonglong(int(g["reg_tb_reg"][q]))
        lvi = C.c_int(int(g["reg_lv_irr"][q]))
        rc = L.abyss_host_time_level_reg(float(g["reg_scale"][q]), tblock, bmax, eta, int(g["reg_has_nb"][q]),
                                         ptr(_c(g["reg_a_reg"][q])), float(g["reg_t_reg"][q]),
                                         int(g["reg_cur_reg"][q]), C.byref(lv), C.byref(dt), C.byref(tb),
                                         C.byref(lvi))
        assert rc == 0
        got = (lv.value, dt.value, tb.value, lvi.value)
        want = (g["reg_out_lv_reg"][q], g["reg_out_dt_reg"][q], g["reg_out_tb_reg"][q], g["reg_out_lv_irr"][q])
        assert got == want, (q, got, want)
        moves.add(min(lv.value - int(g["reg_lv_reg"][q]), 2))
    # kept, one down, two down, one up, several up at once
    assert {-2, -1, 0, 1, 2} <= moves


def test_update_radius_bit_exact():
    L = _lib.lib()
    g = golden("ref_levels.npz")
    fix, nbmax = int(g["rad_fix"]), int(g["rad_nb_max"])
    for c, r2, want in zip(g["rad_counts"], g["rad_r2_in"], g["rad_r2_out"]):
        assert L.abyss_host_update_radius(float(r2), int(c), fix, nbmax) == want, c


def test_irregular_steps_rejects_bad_lists():
    base = golden("ref_plummer1024_s1.npz")
    st = {k: np.array(base[k]) for k in base.files}
    i = int(np.flatnonzero(st["nnb"] > 0)[0])
    st["nb"][i, 0] = i  # a particle in its own list
    L = _lib.lib()
    n = st["x"].shape[0]
    out = np.zeros(12)
    idx = np.array([i], np.int32)
    rc = L.abyss_host_irregular_steps(n, ptr(_c(st["x"])), ptr(_c(st["v"])), ptr(_c(st["m"])),
                                      ptr(_c(st["a_tot"])), ptr(_c(st["a_reg"])), ptr(_c(st["a_irr"])),
                                      ptr(_c(st["t_reg"])), ptr(_c(st["t_irr"])), ptr(_c(st["dt_irr"])),
                                      ptr(_c(st["nnb"]), _ip), ptr(_c(st["nb"]), _ip), st["nb"].shape[1], 0.0,
                                      float(st["time_scale"]), 1, ptr(idx, _ip), ptr(out), ptr(out), ptr(out),
                                      ptr(out))
    assert rc == _lib.ABYSS_ERR_ARG


def test_irregular_step_against_the_reference_library():
    """A fresh state (other seed, other lags) through the reference library
    itself, when it has been built here."""
    import oracle

    if not oracle.ref_available():
        pytest.skip("reference library not built")
    from oracle import _p

    L = oracle.ref()
    base = golden("ref_king2048_s3.npz")
    st = {k: np.array(base[k]) for k in base.files}
    n = st["x"].shape[0]
    rng = np.random.default_rng(123)
    st["dt_irr"] = rng.choice([2.0 ** -10, 2.0 ** -9, 2.0 ** -8], size=n)
    st["t_irr"] = np.where(st["nnb"] > 0, 2.0 ** -7 - rng.choice([0.0, 2.0 ** -8, 2.0 ** -7], size=n), 0.0)
    L.ref_alloc(n)
    scale = float(st["time_scale"])
    L.ref_set_globals(scale, -30, 1 << 30)
    nb = _c(st["nb"], np.int32)
    for i in range(n):
        L.ref_set_particle(i, _p(_c(st["x"][i])), _p(_c(st["v"][i])), float(st["m"][i]), float(st["r2nb"][i]),
                           _p(_c(st["a_tot"][i])), _p(_c(st["a_reg"][i])), _p(_c(st["a_irr"][i])),
                           float(st["t_reg"][i]), float(st["t_irr"][i]), float(st["dt_reg"][i]),
                           float(st["dt_irr"][i]), int(st["nnb"][i]), _p(nb[i], _ip))
    idx = np.flatnonzero(st["nnb"] > 0)[::3].astype(np.int32)
    pos, vel, a_irr, a_tot = host_irregular(st, idx)
    cap = 2000
    for r, i in enumerate(idx):
        one = np.array([i], np.int32)
        L.ref_compute_irr(1, _p(one, _ip), 1)
        x = np.zeros(3); v = np.zeros(3); at = np.zeros(12); ar = np.zeros(12); ai = np.zeros(12)
        npos = np.zeros(3); nvel = np.zeros(3); r2 = np.zeros(1)
        c1 = np.zeros(1, np.int32); c2 = np.zeros(1, np.int32); lst = np.zeros(cap, np.int32)
        L.ref_get_particle(int(i), _p(x), _p(v), _p(at), _p(ar), _p(ai), _p(npos), _p(nvel), _p(r2),
                           _p(c1, _ip), _p(lst, _ip), _p(c2, _ip), _p(lst, _ip), cap)
        assert np.array_equal(vel[r], nvel), r
        assert np.array_equal(a_irr[r].reshape(12), ai), r
        assert np.array_equal(a_tot[r].reshape(12), at), r
        dt = st["dt_irr"][i] * scale
        assert _pos_matches_without_a3_term(pos[r], npos, a_irr[r][:, 3], dt), r
        # restore the particle for the next one's neighbour prediction
        L.ref_set_particle(int(i), _p(_c(st["x"][i])), _p(_c(st["v"][i])), float(st["m"][i]), float(st["r2nb"][i]),
                           _p(_c(st["a_tot"][i])), _p(_c(st["a_reg"][i])), _p(_c(st["a_irr"][i])),
                           float(st["t_reg"][i]), float(st["t_irr"][i]), float(st["dt_reg"][i]),
                           float(st["dt_irr"][i]), int(st["nnb"][i]), _p(nb[i], _ip))


def test_initial_time_steps_bit_exact():
    L = _lib.lib()
    g = golden("ref_levels.npz")
    tblock, eta, bmax = int(g["time_block"]), float(g["eta"]), int(g["block_max"])
    capped = 0
    for q in range(g["init_scale"].shape[0]):
        lv_reg, lv_irr = C.c_int(), C.c_int()
        dt_reg, dt_irr = C.c_double(), C.c_double()
        tb_reg, tb_irr = C.c_ulonglong(), C.c_ulonglong()
        L.abyss_host_initial_time_steps(float(g["init_scale"][q]), tblock, bmax, eta, eta, int(g["init_has_nb"][q]),
                                        ptr(_c(g["init_a_tot"][q])), ptr(_c(g["init_a_reg"][q])),
                                        ptr(_c(g["init_a_irr"][q])), C.byref(lv_reg), C.byref(dt_reg),
                                        C.byref(tb_reg), C.byref(lv_irr), C.byref(dt_irr), C.byref(tb_irr))
        got = (lv_reg.value, dt_reg.value, tb_reg.value, lv_irr.value, dt_irr.value, tb_irr.value)
        want = tuple(g["init_out_" + c][q] for c in ("lv_reg", "dt_reg", "tb_reg", "lv_irr", "dt_irr", "tb_irr"))
        assert got == want, (q, got, want)
        capped += dt_reg.value == 1.0
    assert capped > 0  # steps above the run's length are capped at 1
