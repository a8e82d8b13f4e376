"""The single-cluster integrations of abyss_b200.runs with their regular blocks
re-checked against the FP64 oracle (needs a CUDA GPU).

    python tests/check_runs.py c1 --check-every 5

Every k-th regular block is recomputed by the oracle on the same predicted
j-set: the lists must be identical, and the worst per-target force error is
reported in units of the test bound (|da| <= 1e-6 |a| + 1e-7 A for the
acceleration, 1e-5 and 1e-6 for the jerk, A the sum of the term magnitudes).
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from abyss_b200 import runs  # noqa: E402


def block_checker(every: int, sample_targets: int = 256):
    checks = dict(blocks_checked=0, list_mismatches=0, worst_acc=0.0, worst_jerk=0.0)

    def on_block(ac, c, blocks):
        if every <= 0 or blocks % every:
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(runs.CONFIGS))
    ap.add_argument("--check-every", type=int, default=5)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--t-stop", type=float, default=1.0)
    args = ap.parse_args()
    on_block, checks = block_checker(args.check_every)
    out = runs.run(args.config, threads=args.threads, t_stop=args.t_stop, on_block=on_block)
    out["oracle_checks"] = checks
    print(json.dumps(out))


if __name__ == "__main__":
    main()
