"""Writes tests/golden/ac_plummer1024_b200.ckpt (needs a CUDA GPU and the built
library): configuration 1's Plummer sphere (N = 1024, seed 1, equal masses,
~32 neighbours, eps = 1e-4, eta_reg = 0.02, eta_irr = 0.01, t_end = 10) after
200 regular blocks, as a binary checkpoint (include/abyss_io.h).

    python tests/golden/make_ac_checkpoint.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from abyss_b200 import ic  # noqa: E402
from abyss_b200.integrator import ACIntegrator  # noqa: E402
from abyss_b200.regforce import RegularForce  # noqa: E402


def main():
    rf = RegularForce(0)
    c = ic.plummer(1024, 1, masses="equal", k_nb=32)
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=1e-8, eta_reg=0.02, eta_irr=0.01, fix_nb=32, t_end=10.0,
                      threads=16)
    for _ in range(200):
        ac.advance_block()
    ac.save(os.path.join(HERE, "ac_plummer1024_b200.ckpt"))
    ac.close()
    rf.close()


if __name__ == "__main__":
    main()
