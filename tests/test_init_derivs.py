"""Initialisation pass of the acceleration's second and third derivatives
(CalculateAcceleration23, src_mpi/Particle/Initialize.cpp:102-185).

* CPU: the FP64 oracle restatement equals the reference's own function, bit for
  bit, at eps = 0.  The reference's particle loop runs j < LastParticleIndex =
  n - 1, so it never visits the last particle; the comparison gives the oracle
  the first n - 1 particles as its j-set.
* GPU: abyss_init_derivs23 equals the oracle bit for bit, with and without
  softening (one target per thread, j ascending, round-to-nearest FP64).
"""

import numpy as np
import pytest

import oracle
from abyss_b200 import ic


def _state(n, seed):
    c = ic.plummer(n, seed, k_nb=24)
    rng = np.random.default_rng(seed)
    a0 = rng.normal(size=(n, 3))
    a1 = rng.normal(size=(n, 3))
    return c, a0, a1


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU library not built")
def test_oracle_matches_reference_function():
    n = 600
    c, a0, a1 = _state(n, 21)
    L = oracle.ref()
    L.ref_alloc(n)
    L.ref_set_globals(1.0, -30, 1 << 30)
    a_tot = np.zeros((n, 3, 4))
    a_tot[:, :, 0] = a0
    a_tot[:, :, 1] = a1
    a_tot = np.ascontiguousarray(a_tot.reshape(n, 12))
    z = np.zeros(n)
    dt = np.full(n, 2.0 ** -10)
    L.ref_set_all(n, oracle._p(np.ascontiguousarray(c.x)), oracle._p(np.ascontiguousarray(c.v)),
                  oracle._p(c.m), oracle._p(c.r2nb), oracle._p(a_tot), oracle._p(z), oracle._p(z), oracle._p(dt))
    targets = np.arange(0, n - 1, 7, dtype=np.int32)
    got = {k: np.zeros((targets.size, 3)) for k in ("reg2", "reg3", "irr2", "irr3")}
    buf = {k: np.zeros(12) for k in ("tot", "reg", "irr")}
    xv = [np.zeros(3) for _ in range(4)]
    r2 = np.zeros(1)
    ints = [np.zeros(1, np.int32) for _ in range(2)]
    lists = [np.zeros(8, np.int32) for _ in range(2)]
    for k, i in enumerate(targets):
        L.ref_init_acc23(int(i))
        L.ref_get_particle(int(i), oracle._p(xv[0]), oracle._p(xv[1]), oracle._p(buf["tot"]),
                           oracle._p(buf["reg"]), oracle._p(buf["irr"]), oracle._p(xv[2]), oracle._p(xv[3]),
                           oracle._p(r2), oracle._p(ints[0], oracle._ip), oracle._p(lists[0], oracle._ip),
                           oracle._p(ints[1], oracle._ip), oracle._p(lists[1], oracle._ip), 8)
        reg = buf["reg"].reshape(3, 4)
        irr = buf["irr"].reshape(3, 4)
        got["reg2"][k], got["reg3"][k] = reg[:, 2], reg[:, 3]
        got["irr2"][k], got["irr3"][k] = irr[:, 2], irr[:, 3]
    L.ref_free()
    m = n - 1  # the reference's j-set
    want = oracle.init_derivs23(c.x[:m], c.v[:m], c.m[:m], c.r2nb[:m], a0[:m], a1[:m], 0.0, targets)
    for key in got:
        assert np.array_equal(got[key], want[key]), key
    assert np.abs(want["irr2"]).sum() > 0 and np.abs(want["reg2"]).sum() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("eps2", [0.0, 1e-8])
def test_device_matches_oracle(eps2):
    from abyss_b200 import _lib
    from abyss_b200.regforce import RegularForce

    n = 3000
    c, a0, a1 = _state(n, 22)
    rf = RegularForce(0)
    try:
        out = rf.init_derivs23(c.x, c.v, c.m, c.r2nb, a0, a1, eps2)
    finally:
        rf.close()
    want = oracle.init_derivs23(c.x, c.v, c.m, c.r2nb, a0, a1, eps2, np.arange(n, dtype=np.int32))
    for key in want:
        assert np.array_equal(out[key], want[key]), key
