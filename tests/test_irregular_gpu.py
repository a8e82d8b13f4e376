"""Irregular steps on the GPU (include/abyss_irr.h) against the reference and
the host integrator.

* Single steps, abyss_device_irregular_steps, on the two golden regular-step
  states (the reference's own computeAccelerationIrr + calculateTimeStepIrr
  outputs, tests/golden/*_irr.npz): new velocity, a_irr, a_tot and the new
  level, step and block count bit-exact against the reference; the new
  position bit-exact against the host integrator's step
  (abyss_host_irregular_steps), which differs from the reference's by exactly
  the a3 dt^5/120 term the reference drops (it reads an uninitialised dt5,
  ComputeAcceleration.cpp:162).
* Whole integrations with the level loop on the device: the same state, bit
  for bit, as the same integration with the host's irregular levels, block
  after block, and the same step and level counts; level decisions near a
  power-of-two boundary (where the device's and host's log could differ) are
  counted and must not occur in these runs.
"""
import ctypes as C

import numpy as np
import pytest

from abyss_b200 import _lib, ic
from abyss_b200._lib import _ip, ptr
from abyss_b200.integrator import ACIntegrator
from abyss_b200.regforce import RegularForce
from tests.helpers import golden
from tests.test_host_irregular import CASES, host_irregular

pytestmark = pytest.mark.gpu

_ull = C.POINTER(C.c_ulonglong)


def _c(a, dt=None):
    return np.ascontiguousarray(a, dt)


def device_irregular(st, idx, time_block, eta, lv_reg, cur_reg, tb_reg, eps2=0.0):
    L = _lib.lib()
    n = st["x"].shape[0]
    idx = _c(idx, np.int32)
    k = idx.shape[0]
    out = dict(pos=np.zeros((k, 3)), vel=np.zeros((k, 3)), a_irr=np.zeros((k, 3, 4)), a_tot=np.zeros((k, 3, 4)),
               lv=np.zeros(k, np.int32), dt=np.zeros(k), tb=np.zeros(k, np.uint64))
    nb = _c(st["nb"], np.int32)
    lv_reg = _c(lv_reg, np.int32)
    cur_reg = _c(cur_reg, np.uint64)
    tb_reg = _c(tb_reg, np.uint64)
    rc = L.abyss_device_irregular_steps(
        0, n, ptr(_c(st["x"])), ptr(_c(st["v"])), ptr(_c(st["m"])), ptr(_c(st["a_tot"])), ptr(_c(st["a_reg"])),
        ptr(_c(st["a_irr"])), ptr(_c(st["t_reg"])), ptr(_c(st["t_irr"])), ptr(_c(st["dt_irr"])),
        ptr(_c(st["nnb"], np.int32), _ip), ptr(nb, _ip), nb.shape[1], eps2, float(st["time_scale"]), int(time_block),
        float(eta), ptr(lv_reg, _ip), cur_reg.ctypes.data_as(_ull), tb_reg.ctypes.data_as(_ull), k, ptr(idx, _ip),
        ptr(out["pos"]), ptr(out["vel"]), ptr(out["a_irr"]), ptr(out["a_tot"]), ptr(out["lv"], _ip), ptr(out["dt"]),
        out["tb"].ctypes.data_as(_ull))
    assert rc == 0, rc
    return out


@pytest.mark.parametrize("name", CASES)
def test_device_steps_against_reference_and_host(name):
    base = golden(name + ".npz")
    g = golden(name + "_irr.npz")
    idx = g["idx"]
    tblock = int(g["time_block"])
    step = 2.0 ** tblock
    eta = float(golden("ref_levels.npz")["eta"])
    n = base["x"].shape[0]
    lv_reg = np.round(np.log2(base["dt_reg"])).astype(np.int32)
    tb_reg = np.round(base["dt_reg"] / step).astype(np.uint64)
    dev = device_irregular(base, idx, tblock, eta, lv_reg, np.zeros(n, np.uint64), tb_reg)
    # the reference's own outputs
    assert np.array_equal(dev["vel"], g["out_newvel"])
    assert np.array_equal(dev["a_irr"], g["out_a_irr"])
    assert np.array_equal(dev["a_tot"], g["out_a_tot"])
    assert np.array_equal(dev["lv"], g["out_lv_irr"])
    assert np.array_equal(dev["dt"], g["out_dt_irr"])
    assert np.array_equal(dev["tb"], g["out_tb_irr"].astype(np.uint64))
    # the host integrator's step, position included
    pos, vel, a_irr, a_tot = host_irregular(base, idx)
    assert np.array_equal(dev["pos"], pos)
    assert np.array_equal(dev["vel"], vel)
    assert np.array_equal(dev["a_irr"], a_irr)
    assert np.array_equal(dev["a_tot"], a_tot)


def _pair(c, fix_nb, t_end, eps2=1e-8, threads=0):
    rfs = [RegularForce(0), RegularForce(0)]
    acs = [ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=eps2, eta_reg=0.02, eta_irr=0.01, fix_nb=fix_nb,
                        t_end=t_end, threads=threads) for rf in rfs]
    acs[1].set_device_irregular(True)
    return rfs, acs


def _same(a, b):
    sa, sb = a.state(), b.state()
    return all(np.array_equal(sa[k], sb[k]) for k in ("x", "v", "nnb", "r2nb"))


@pytest.mark.parametrize("model,n,fix_nb,blocks", [("plummer", 1024, 32, 120), ("plummer", 8192, 48, 40),
                                                  ("king_kroupa", 16384, 64, 25)])
def test_device_levels_equal_host_levels(model, n, fix_nb, blocks):
    if model == "plummer":
        c = ic.plummer(n, 1, k_nb=fix_nb)
    else:
        c = ic.king(n, 7, 6.0, masses="kroupa", k_nb=fix_nb)
    rfs, acs = _pair(c, fix_nb, 10.0 if n <= 1024 else 2.0)
    try:
        for b in range(blocks):
            d0 = acs[0].advance_block()
            d1 = acs[1].advance_block()
            assert d0 == d1
            if b % 5 == 4 or d0:
                assert _same(acs[0], acs[1]), f"block {b}: states differ"
            if d0:
                break
        s0, s1 = acs[0].stats(), acs[1].stats()
        info = acs[1].device_irregular_info()
        print(f"{model} n={n}: {s0['blocks']} blocks, {s0['irr_steps']} irregular steps in {s0['irr_levels']} "
              f"levels; host irregular {s0['sec_irr']:.3f} s, device {s1['sec_irr']:.3f} s "
              f"(copies {info['sec_copy']:.3f} s); borderline level decisions {info['borderline']}; "
              f"cycles per level {({k: v // max(s1['irr_levels'], 1) for k, v in info['cycles'].items()})}")
        assert _same(acs[0], acs[1])
        for k in ("blocks", "reg_steps", "irr_steps", "irr_levels"):
            assert s0[k] == s1[k], k
        assert info["on"] and info["borderline"] == 0
    finally:
        for a in acs:
            a.close()
        for rf in rfs:
            rf.close()


def test_switching_between_host_and_device_levels():
    """Host levels, then device levels, then host again: the same state as a
    run on the host throughout (the device copy is refreshed on each switch)."""
    c = ic.plummer(2048, 3, k_nb=32)
    rfs, acs = _pair(c, 32, 10.0)
    try:
        acs[1].set_device_irregular(False)
        for phase, dev in enumerate((False, True, False, True)):
            acs[1].set_device_irregular(dev)
            for _ in range(10):
                acs[0].advance_block()
                acs[1].advance_block()
            assert _same(acs[0], acs[1]), f"phase {phase}"
    finally:
        for a in acs:
            a.close()
        for rf in rfs:
            rf.close()
