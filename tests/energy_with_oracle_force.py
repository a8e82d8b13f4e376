"""Configuration 1 finished with the FP64 oracle as the regular force, on the CPU.

    python tests/energy_with_oracle_force.py

Starts from tests/golden/ac_plummer1024_b200.ckpt (configuration 1 after 200
of its regular blocks, written on a GPU) loaded without a GPU context, runs the
remaining blocks with the host integrator, taking each block's regular force
from the FP64 oracle, and prints |dE/E| between the initial conditions and the
end (all particles synchronised there).  Set beside the GPU runs, it shows how
much of configuration 1's energy drift the FP32 regular force is responsible
for.
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from abyss_b200 import ic  # noqa: E402
from abyss_b200.integrator import ACIntegrator  # noqa: E402
from tests.test_host_checkpoint import CKPT, run_blocks_with_oracle  # noqa: E402


def main(threads: int = 8):
    c = ic.plummer(1024, 1, masses="equal", k_nb=32)
    e0 = oracle.energy(c.x, c.v, c.m, 1e-8)
    ac = ACIntegrator.load(None, CKPT, threads=threads)
    t0 = time.perf_counter()
    blocks = run_blocks_with_oracle(ac, 1 << 30)
    mass = ac.block_state()["mass"]
    st = ac.state()
    ac.close()
    e1 = oracle.energy(st["x"], st["v"], mass, 1e-8)
    print(f"{blocks} blocks with the FP64 oracle force: |dE/E| = {abs((e1 - e0) / e0):.3e} "
          f"({time.perf_counter() - t0:.1f} s)")


if __name__ == "__main__":
    main()
