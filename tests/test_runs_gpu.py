"""Configuration 1 integrated to its end on the GPU, with regular blocks
re-checked against the FP64 oracle.

Plummer N = 1024 (seed 1, equal masses), eps = 1e-4, ~32 neighbours, eta_reg =
0.02, eta_irr = 0.01, to t = 10 (abyss_b200.runs "c1").  Every 5th regular
block is recomputed by the oracle on the same predicted j-set: lists and
counts identical, and per-target force errors within the bound of
tests/test_regforce_gpu.py (|da| <= 1e-6 |a| + 1e-7 A; jerk 1e-5 and 1e-6;
A the sum of the term magnitudes).  The run's |dE/E| is printed.
"""
import numpy as np
import pytest

import oracle
from abyss_b200 import runs

pytestmark = pytest.mark.gpu


def block_checker(every: int, sample_targets: int = 256):
    checks = dict(blocks_checked=0, list_mismatches=0, worst_acc=0.0, worst_jerk=0.0)

    def on_block(ac, c, blocks):
        if blocks % every:
            return
        last = ac.last_regular()
        t = last["targets"]
        rows = np.arange(len(t))
        if len(t) > sample_targets:
            rows = np.sort(np.random.default_rng(len(t)).choice(len(t), sample_targets, replace=False))
        eps2 = runs.EPS * runs.EPS
        ref = oracle.reg_force(last["px"], last["pv"], c.m, last["r2nb"], eps2, t[rows], ac.nb_max)
        sa, sj = oracle.reg_scale(last["px"], last["pv"], c.m, last["r2nb"], eps2, t[rows])
        for k, r in enumerate(rows):
            n = int(ref["nnb"][k])
            if int(last["nnb"][r]) != n or not np.array_equal(last["list"][r, :n], ref["list"][k, :n]):
                checks["list_mismatches"] += 1
        da = np.linalg.norm(last["acc_reg"][rows] - ref["acc_reg"], axis=1)
        dj = np.linalg.norm(last["jerk_reg"][rows] - ref["jerk_reg"], axis=1)
        na = np.linalg.norm(ref["acc_reg"], axis=1)
        nj = np.linalg.norm(ref["jerk_reg"], axis=1)
        checks["worst_acc"] = max(checks["worst_acc"], float((da / (1e-6 * na + 1e-7 * sa)).max()))
        checks["worst_jerk"] = max(checks["worst_jerk"], float((dj / (1e-5 * nj + 1e-6 * sj)).max()))
        checks["blocks_checked"] += 1

    return on_block, checks


def test_configuration1_to_the_end_every_5th_block_against_oracle():
    on_block, checks = block_checker(5)
    out = runs.run("c1", on_block=on_block)
    print(f"c1: {out['stats']['blocks']} blocks, |dE/E| = {out['dE_over_E']:.3e}, oracle checks {checks}")
    assert out["code_time"] >= 1.0
    assert checks["blocks_checked"] >= 100
    assert checks["list_mismatches"] == 0
    assert checks["worst_acc"] <= 1.0 and checks["worst_jerk"] <= 1.0
