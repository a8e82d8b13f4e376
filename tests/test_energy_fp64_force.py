"""Configuration 1 finished on the CPU with the FP64 oracle as the regular force.

Starts from tests/golden/ac_plummer1024_b200.ckpt (configuration 1 -- Plummer
N = 1024, eps = 1e-4, ~32 neighbours, eta_reg = 0.02, eta_irr = 0.01, t_end =
10 -- after 200 of its regular blocks, written on a GPU), loaded without a GPU
context, and runs the remaining blocks with the host integrator, each block's
regular force taken from the FP64 oracle.  |dE/E| between the initial
conditions and the end (all particles synchronised there) is pinned: with an
FP64 force the run still drifts by 6.39e-6, so the FP32 device force is not
what sets configuration 1's drift (close encounters are).
"""
import numpy as np

import oracle
from abyss_b200 import ic
from abyss_b200.integrator import ACIntegrator
from tests.test_host_checkpoint import CKPT, _load, run_blocks_with_oracle


def test_configuration1_drift_with_fp64_force():
    c = ic.plummer(1024, 1, masses="equal", k_nb=32)
    e0 = oracle.energy(c.x, c.v, c.m, 1e-8)
    ac = _load(4)
    assert isinstance(ac, ACIntegrator) and CKPT
    try:
        blocks = run_blocks_with_oracle(ac, 1 << 30)
        mass = ac.block_state()["mass"]
        st = ac.state()
    finally:
        ac.close()
    assert np.array_equal(mass, c.m)
    de = abs((oracle.energy(st["x"], st["v"], mass, 1e-8) - e0) / e0)
    print(f"{blocks} blocks with the FP64 oracle force: |dE/E| = {de:.4e}")
    assert blocks == 1346
    assert 6.38e-6 < de < 6.40e-6
