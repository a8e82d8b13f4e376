"""The host Ahmad-Cohen integrator with the GPU regular force.

* Every regular block of a Plummer run (the N = 1024 configuration's cluster,
  eps = 1e-4, ~32 neighbours, eta_reg = 0.02, eta_irr = 0.01) is re-done by the
  FP64 oracle on the same predicted j-set: lists bit-exact, forces within the
  per-target bound of tests/test_regforce_gpu.py (|da| <= 1e-6 |a| + 1e-7 A).
* Energy drift of short complete runs stays small.
"""
import numpy as np
import pytest

import oracle
from abyss_b200 import ic
from abyss_b200.integrator import ACIntegrator
from abyss_b200.regforce import RegularForce
from tests.helpers import first_list_mismatch

pytestmark = pytest.mark.gpu

EPS2 = 1e-4 ** 2


@pytest.fixture(scope="module")
def rf():
    r = RegularForce(0)
    yield r
    r.close()


def test_every_regular_block_matches_oracle(rf):
    c = ic.plummer(1024, 1, k_nb=32)
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS2, eta_reg=0.02, eta_irr=0.01, fix_nb=32,
                      t_end=10.0)
    blocks = 0
    worst_a = worst_j = 0.0
    while blocks < 150:
        done = ac.advance_block()
        blocks += 1
        last = ac.last_regular()
        ref = oracle.reg_force(last["px"], last["pv"], c.m, last["r2nb"], EPS2, last["targets"], ac.nb_max)
        mm = first_list_mismatch(last["nnb"], last["list"], ref["nnb"], ref["list"])
        assert mm is None, f"block {blocks}: list mismatch {mm}"
        sa, sj = oracle.reg_scale(last["px"], last["pv"], c.m, last["r2nb"], EPS2, last["targets"])
        na = np.linalg.norm(ref["acc_reg"], axis=1)
        nj = np.linalg.norm(ref["jerk_reg"], axis=1)
        da = np.linalg.norm(last["acc_reg"] - ref["acc_reg"], axis=1)
        dj = np.linalg.norm(last["jerk_reg"] - ref["jerk_reg"], axis=1)
        worst_a = max(worst_a, (da / (1e-6 * na + 1e-7 * sa)).max())
        worst_j = max(worst_j, (dj / (1e-5 * nj + 1e-6 * sj)).max())
        if done:
            break
    print(f"{blocks} blocks to code time {ac.time:.4g}: worst acc {worst_a:.2e} jerk {worst_j:.2e}; "
          f"stats {ac.stats()}")
    assert worst_a <= 1.0 and worst_j <= 1.0  # in units of the per-target bound


def test_short_run_energy_conservation(rf):
    c = ic.plummer(1024, 1, k_nb=32)
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS2, eta_reg=0.02, eta_irr=0.01, fix_nb=32,
                      t_end=0.25)
    e0 = ac.energy()
    ac.run(1.0)
    e1 = ac.energy()
    de = abs((e1 - e0) / e0)
    print(f"N=1024 to t=0.25: E0={e0:.8f} E1={e1:.8f} |dE/E|={de:.2e} stats {ac.stats()}")
    assert abs(e0 + 0.25) < 0.02
    assert de < 1e-5


def test_integrator_rejects_bad_parameters(rf):
    from abyss_b200._lib import AbyssError

    c = ic.plummer(64, 2, k_nb=8)
    with pytest.raises(AbyssError):
        ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, fix_nb=8, nb_max=4)
    with pytest.raises(AbyssError):
        ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eta_reg=-1.0)
