"""Whole regular blocks on the GPU with the state kept there
(include/abyss_irr.h abyss_ac_set_device_resident) against the host integrator.

The same integration is run twice, block by block: on the host (host irregular
levels, host corrector and time steps, the GPU for the regular force only) and
with every part of the block on the device.  Every few blocks both are
checkpointed (abyss_ac_save, which reads the device state back) and the
particle sections of the two files -- every field of every particle:
positions, velocities, the three derivative sets, radii, times, steps, levels
and neighbour lists -- must be equal byte for byte; block times, step counts
and level counts must agree, and no level decision may have been borderline
(within 1e-12 of a power-of-two boundary, where the device's log and the
host's could differ).  One case runs with nb_max close to the neighbour
target so that lists overflow and radii are shrunk and the force re-run.

Switching the mode off and on again mid-run, and the last block's record
(abyss_ac_last_regular) against the FP64 oracle, are checked too.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from abyss_b200 import _lib, ic
from abyss_b200.integrator import ACIntegrator
from abyss_b200.regforce import RegularForce
from tests.helpers import first_list_mismatch

pytestmark = pytest.mark.gpu

EPS2 = 1e-8
# checkpoint header: magic, version, Star::a_tot size, n, parameters, scale,
# time_block, block_max, time_step, next_reg_block, done, statistics
HEADER = 8 + 4 + 4 + 4 + C.sizeof(_lib.ACParams) + 8 + 4 + 8 + 8 + 8 + 4 + C.sizeof(_lib.ACStats)


def _particles(ac, path):
    ac.save(str(path))
    return open(path, "rb").read()[HEADER:]


def _pair(c, fix_nb, t_end, nb_max=None):
    rfs = [RegularForce(0), RegularForce(0)]
    acs = [ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS2, eta_reg=0.02, eta_irr=0.01, fix_nb=fix_nb,
                        nb_max=nb_max, t_end=t_end) for rf in rfs]
    return rfs, acs


def _close(rfs, acs):
    for a in acs:
        a.close()
    for rf in rfs:
        rf.close()


def _cluster(model, n, fix_nb):
    if model == "plummer":
        return ic.plummer(n, 1, k_nb=fix_nb)
    return ic.king(n, 7, 6.0, masses="kroupa", k_nb=fix_nb)


@pytest.mark.parametrize("model,n,fix_nb,nb_max,blocks", [("plummer", 1024, 32, None, 150),
                                                         ("plummer", 8192, 48, None, 40),
                                                         ("king_kroupa", 16384, 64, None, 25),
                                                         ("king_kroupa", 4096, 32, 36, 40)])
def test_device_blocks_equal_host_blocks(model, n, fix_nb, nb_max, blocks, tmp_path):
    c = _cluster(model, n, fix_nb)
    rfs, acs = _pair(c, fix_nb, 10.0 if n <= 1024 else 2.0, nb_max)
    try:
        acs[1].set_device_resident(True)
        for b in range(blocks):
            d0 = acs[0].advance_block()
            d1 = acs[1].advance_block()
            assert d0 == d1 and acs[0].time == acs[1].time, f"block {b}"
            if b % 10 == 9 or d0:
                assert _particles(acs[0], tmp_path / "h.ckpt") == _particles(acs[1], tmp_path / "d.ckpt"), \
                    f"block {b}: states differ"
            if d0:
                break
        assert _particles(acs[0], tmp_path / "h.ckpt") == _particles(acs[1], tmp_path / "d.ckpt")
        s0, s1 = acs[0].stats(), acs[1].stats()
        res = acs[1].device_resident_info()
        irr = acs[1].device_irregular_info()
        print(f"{model} n={n} nb_max={acs[0].nb_max}: {s0['blocks']} blocks to t = {acs[0].time:.4g}, "
              f"{s0['irr_steps']} irregular steps, radius retries {s0['radius_retries']}; host regular corrector "
              f"{s0['sec_reg_host']:.3f} s, device {s1['sec_reg_host']:.3f} s; irregular host {s0['sec_irr']:.3f} s, "
              f"device {s1['sec_irr']:.3f} s; state copies {res['sec_sync']:.3f} s")
        for k in ("blocks", "reg_steps", "irr_steps", "irr_levels", "radius_retries"):
            assert s0[k] == s1[k], k
        assert res["on"] and res["borderline"] == 0 and irr["borderline"] == 0
        if nb_max is not None:
            assert s0["radius_retries"] > 0, "the overflow case did not overflow"
    finally:
        _close(rfs, acs)


def test_switching_device_blocks_off_and_on(tmp_path):
    """Device blocks, host blocks, device blocks again: the same state as a run
    on the host throughout (the state goes down at each switch off and up at
    each switch on)."""
    c = ic.plummer(2048, 3, k_nb=32)
    rfs, acs = _pair(c, 32, 10.0)
    try:
        for phase, on in enumerate((True, False, True, False)):
            acs[1].set_device_resident(on)
            for _ in range(12):
                acs[0].advance_block()
                acs[1].advance_block()
            assert _particles(acs[0], tmp_path / "h.ckpt") == _particles(acs[1], tmp_path / "d.ckpt"), \
                f"phase {phase}"
    finally:
        _close(rfs, acs)


def test_device_block_record_matches_oracle():
    """abyss_ac_last_regular after device blocks: the block's targets, radii and
    predicted j-set, and its lists (bit-exact) and forces against the oracle."""
    c = ic.plummer(1024, 1, k_nb=32)
    rf = RegularForce(0)
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS2, eta_reg=0.02, eta_irr=0.01, fix_nb=32, t_end=10.0)
    try:
        ac.set_device_resident(True)
        worst = 0.0
        for b in range(40):
            ac.advance_block()
            last = ac.last_regular()
            t = last["targets"]
            assert np.all(np.diff(t) > 0), "targets not ascending"
            ref = oracle.reg_force(last["px"], last["pv"], c.m, last["r2nb"], EPS2, t, ac.nb_max)
            mm = first_list_mismatch(last["nnb"], last["list"], ref["nnb"], ref["list"])
            assert mm is None, f"block {b}: list mismatch {mm}"
            sa, _ = oracle.reg_scale(last["px"], last["pv"], c.m, last["r2nb"], EPS2, t)
            na = np.linalg.norm(ref["acc_reg"], axis=1)
            da = np.linalg.norm(last["acc_reg"] - ref["acc_reg"], axis=1)
            worst = max(worst, (da / (1e-6 * na + 1e-7 * sa)).max())
        assert worst <= 1.0
    finally:
        ac.close()
        rf.close()


def test_split_blocks_refused_while_resident():
    c = ic.plummer(256, 4, k_nb=16)
    rf = RegularForce(0)
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS2, fix_nb=16, t_end=1.0)
    try:
        ac.set_device_resident(True)
        ac.advance_block()
        m = C.c_int(0)
        t = C.c_double(0.0)
        s = C.c_double(0.0)
        d = C.c_int(0)
        rc = ac._L.abyss_ac_begin_block(ac._h, C.byref(m), C.byref(t), C.byref(s), C.byref(d))
        assert rc == _lib.ABYSS_ERR_STATE
        ac.set_device_resident(False)
        ac.advance_block()
    finally:
        ac.close()
        rf.close()


def test_pooled_engine_reused_for_a_smaller_cluster(tmp_path):
    """Device blocks of an N = 1024 integration on the engine an N = 2048 one
    has just returned to the pool (its arrays reused, cleared): the same state
    as the host integration, byte for byte."""
    big = ic.plummer(2048, 5, k_nb=32)
    rf = RegularForce(0)
    ac = ACIntegrator(rf, big.x, big.v, big.m, big.r2nb, eps2=EPS2, fix_nb=32, t_end=10.0)
    try:
        ac.set_device_resident(True)
        for _ in range(15):
            ac.advance_block()
    finally:
        ac.close()
        rf.close()
    c = ic.plummer(1024, 6, k_nb=32)
    rfs, acs = _pair(c, 32, 10.0)
    try:
        acs[1].set_device_resident(True)
        for _ in range(30):
            acs[0].advance_block()
            acs[1].advance_block()
        assert _particles(acs[0], tmp_path / "h.ckpt") == _particles(acs[1], tmp_path / "d.ckpt")
    finally:
        _close(rfs, acs)
