"""One regular-force call on a seeded Plummer sphere, for profiling a launch.

    python -m abyss_b200.profile_case N M [TUNING_JSON]

builds an N-particle Plummer sphere (seed 3, 100 neighbours per particle),
uploads it, and computes the regular force of M evenly spaced targets with
list capacity 256 and eps2 = 1e-8.  TUNING_JSON (default '{}', the built-in
launch plan) is an abyss_tuning as a JSON object, for example
'{"kernel": 3, "mode": 1, "threads": 256, "ipt": 4}'.  The chosen launch plan
and the mean neighbour count are printed, so a profiler capture of the force
kernel can be tied to its shape.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import ic
from .regforce import RegularForce


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("n", type=int)
    ap.add_argument("m", type=int)
    ap.add_argument("tuning", nargs="?", default="{}")
    ap.add_argument("--repeat", type=int, default=1)
    args = ap.parse_args()
    c = ic.plummer(args.n, 3, k_nb=100)
    rf = RegularForce(0)
    rf.send_to_device(c.m, c.x, c.v, c.r2nb)
    t = np.arange(0, args.n, max(1, args.n // args.m), dtype=np.int32)[: args.m]
    tu = json.loads(args.tuning)
    for _ in range(args.repeat):
        res = rf.calculate_acceleration(t, eps2=1e-8, list_cap=256, tuning=tu)
    print("plan", res.plan, "nnb", float(res.nnb.mean()))
    rf.close()


if __name__ == "__main__":
    main()
