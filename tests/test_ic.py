"""The seeded initial conditions behind every workload (abyss_b200/ic.py), CPU only.

* Plummer (Aarseth-Henon-Wielen) and King W0 = 6: total mass 1, centre of mass
  and of momentum at the origin, total energy -1/4 (N-body units) within the
  sampling noise, virial ratio 1/2; the same arrays for the same seed.
* Plummer radii stay inside the 10 a truncation.
* The neighbour radii put exactly k neighbours inside R_nb for every particle
  (the default, midway between the k-th and (k+1)-th neighbour distances).
* Kroupa (2001): masses inside [0.08, 100] Msun, and the share below the 0.5 Msun
  break is the IMF's integral share.
"""
import math

import numpy as np
import pytest

from abyss_b200 import ic


def _energy(c):
    d = c.x[:, None, :] - c.x[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    np.fill_diagonal(r, np.inf)
    pot = -0.5 * (c.m[:, None] * c.m[None, :] / r).sum()
    kin = 0.5 * (c.m * (c.v * c.v).sum(1)).sum()
    return kin, pot


def _neighbour_counts(c):
    d = c.x[:, None, :] - c.x[None, :, :]
    r2 = (d * d).sum(-1)
    np.fill_diagonal(r2, np.inf)
    return (r2 < c.r2nb[:, None]).sum(1)


@pytest.mark.parametrize("make", [lambda: ic.plummer(2048, 7, k_nb=24),
                                  lambda: ic.plummer(2048, 8, masses="kroupa", k_nb=24),
                                  lambda: ic.king(2048, 9, 6.0, k_nb=24)])
def test_model_normalisation_and_neighbours(make):
    c = make()
    assert c.n == 2048 and c.x.shape == (2048, 3) and c.v.shape == (2048, 3)
    assert abs(c.m.sum() - 1.0) < 1e-12
    assert np.abs((c.m[:, None] * c.x).sum(0)).max() < 1e-12
    assert np.abs((c.m[:, None] * c.v).sum(0)).max() < 1e-12
    kin, pot = _energy(c)
    # N-body units: E = -1/4 and 2T + W = 0, up to the noise of 2048 samples
    assert abs((kin + pot) + 0.25) < 0.025, kin + pot
    assert abs(2 * kin / -pot - 1.0) < 0.1, 2 * kin / -pot
    assert np.all(_neighbour_counts(c) == 24)
    again = make()
    for a, b in ((c.x, again.x), (c.v, again.v), (c.m, again.m), (c.r2nb, again.r2nb)):
        assert np.array_equal(a, b)


def test_plummer_truncation():
    c = ic.plummer(4096, 3, k_nb=8)
    a = 3.0 * math.pi / 16.0  # the Plummer scale length in N-body units
    r = np.sqrt((c.x * c.x).sum(1))
    # radii were drawn inside 10 a; centring on the sample's centre of mass
    # moves them by far less than 1 %
    assert r.max() <= 10.0 * a * 1.01
    assert r.max() > 5.0 * a  # the tail is sampled at all


def test_kroupa_masses():
    rng = np.random.default_rng(5)
    m = ic.kroupa_masses(200000, rng)
    assert m.min() >= 0.08 and m.max() <= 100.0
    a1, a2, lo, brk, hi = 1.3, 2.3, 0.08, 0.5, 100.0
    k2 = brk ** (a2 - a1)
    w1 = (brk ** (1 - a1) - lo ** (1 - a1)) / (1 - a1)
    w2 = k2 * (hi ** (1 - a2) - brk ** (1 - a2)) / (1 - a2)
    share = (m < brk).mean()
    assert abs(share - w1 / (w1 + w2)) < 0.005, share
