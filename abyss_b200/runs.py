"""Integration runs of the single-cluster configurations with energy diagnostics.

  c1: Plummer N = 1024 (seed 1, equal masses, radii <= 10 a), eps = 1e-4,
      ~32 neighbours, eta_reg = 0.02, eta_irr = 0.01, integrated to t = 10.
  c2: Plummer N = 65536 (seed 2), Kroupa IMF 0.08-100 Msun rescaled to total
      mass 1, eps = 1e-4, ~64 neighbours, integrated to t = 2.

Each run reports |dE/E| between t = 0 and the end (all particles synchronised
there), the step counts and where the time went.  ``--check-every k`` re-does
every k-th regular block with the FP64 oracle on the same predicted j-set
(lists exact; worst per-target force error in units of the test bound); that
check needs the oracle under oracle/ and is a test of the run, not part of it.

    python -m abyss_b200.runs c1 [--check-every 1]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import ic
from .integrator import ACIntegrator
from .regforce import RegularForce

CONFIGS = {
    "c1": dict(n=1024, seed=1, masses="equal", k_nb=32, t_end=10.0),
    "c2": dict(n=65536, seed=2, masses="kroupa", k_nb=64, t_end=2.0),
}
EPS = 1e-4


def run(name: str, check_every: int = 0, sample_targets: int = 256, threads: int = 0, t_stop: float = 1.0):
    cfg = CONFIGS[name]
    c = ic.plummer(cfg["n"], cfg["seed"], masses=cfg["masses"], k_nb=cfg["k_nb"])
    rf = RegularForce(0)
    t0 = time.perf_counter()
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS * EPS, eta_reg=0.02, eta_irr=0.01,
                      fix_nb=cfg["k_nb"], t_end=cfg["t_end"], threads=threads)
    e0 = ac.energy()
    checks = dict(blocks_checked=0, list_mismatches=0, worst_acc=0.0, worst_jerk=0.0)
    blocks = 0
    done = False
    while not done and ac.time < t_stop:
        done = ac.advance_block()
        blocks += 1
        if check_every and blocks % check_every == 0:
            _check(ac, c, checks, sample_targets)
    wall = time.perf_counter() - t0
    e1 = ac.energy()
    out = dict(config=name, n=c.n, t_end=cfg["t_end"], code_time=ac.time, e0=e0, e1=e1,
               dE_over_E=abs((e1 - e0) / e0), wall_s=wall, stats=ac.stats())
    if check_every:
        out["oracle_checks"] = checks
    ac.close()
    rf.close()
    return out


def _check(ac, c, checks, sample_targets):
    import oracle  # the checker, only when a check is asked for

    last = ac.last_regular()
    t = last["targets"]
    rows = np.arange(len(t))
    if len(t) > sample_targets:
        rows = np.sort(np.random.default_rng(len(t)).choice(len(t), sample_targets, replace=False))
    ref = oracle.reg_force(last["px"], last["pv"], c.m, last["r2nb"], EPS * EPS, t[rows], ac.nb_max)
    sa, sj = oracle.reg_scale(last["px"], last["pv"], c.m, last["r2nb"], EPS * EPS, t[rows])
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--check-every", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--t-stop", type=float, default=1.0, help="stop at this code time (1 = t_end)")
    args = ap.parse_args()
    print(json.dumps(run(args.config, args.check_every, threads=args.threads, t_stop=args.t_stop)))


if __name__ == "__main__":
    main()
