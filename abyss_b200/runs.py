"""Integration runs of the single-cluster configurations with energy diagnostics.

  c1: Plummer N = 1024 (seed 1, equal masses, radii <= 10 a), eps = 1e-4,
      ~32 neighbours, eta_reg = 0.02, eta_irr = 0.01, integrated to t = 10.
  c2: Plummer N = 65536 (seed 2), Kroupa IMF 0.08-100 Msun rescaled to total
      mass 1, eps = 1e-4, ~64 neighbours, integrated to t = 2.

Each run reports |dE/E| between t = 0 and the end (all particles synchronised
there), the step counts and where the time went.  The irregular levels run on
the host threads, or with ``device_irregular`` on the GPU; with ``device_blocks`` whole blocks run on the GPU
with the state kept there (the same results either way).  ``on_block`` is called after
every regular block with (integration, initial conditions, block count); the
test suite uses it to re-check blocks against the FP64 oracle
(tests/test_runs_gpu.py).

    python -m abyss_b200.runs c1
"""
from __future__ import annotations

import argparse
import json
import time

from . import ic
from .integrator import ACIntegrator
from .regforce import RegularForce

CONFIGS = {
    "c1": dict(n=1024, seed=1, masses="equal", k_nb=32, t_end=10.0),
    "c2": dict(n=65536, seed=2, masses="kroupa", k_nb=64, t_end=2.0),
}
EPS = 1e-4


def run(name: str, threads: int = 0, t_stop: float = 1.0, on_block=None, device_irregular: bool = False,
        device_blocks: bool = False):
    cfg = CONFIGS[name]
    c = ic.plummer(cfg["n"], cfg["seed"], masses=cfg["masses"], k_nb=cfg["k_nb"])
    rf = RegularForce(0)
    t0 = time.perf_counter()
    ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=EPS * EPS, eta_reg=0.02, eta_irr=0.01,
                      fix_nb=cfg["k_nb"], t_end=cfg["t_end"], threads=threads)
    if device_irregular:
        ac.set_device_irregular(True)
    if device_blocks:
        ac.set_device_resident(True)
    e0 = ac.energy()
    blocks = 0
    done = False
    while not done and ac.time < t_stop:
        done = ac.advance_block()
        blocks += 1
        if on_block is not None:
            on_block(ac, c, blocks)
    wall = time.perf_counter() - t0
    e1 = ac.energy()
    out = dict(config=name, n=c.n, t_end=cfg["t_end"], code_time=ac.time, e0=e0, e1=e1,
               dE_over_E=abs((e1 - e0) / e0), wall_s=wall, stats=ac.stats(),
               irregular="device" if device_irregular or device_blocks else "host",
               blocks_on="device" if device_blocks else "host", host_timers=ac.host_timers())
    if device_irregular or device_blocks:
        out["device_irregular"] = ac.device_irregular_info()
    if device_blocks:
        out["device_blocks"] = ac.device_resident_info()
    ac.close()
    rf.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--t-stop", type=float, default=1.0, help="stop at this code time (1 = t_end)")
    ap.add_argument("--device-irregular", action="store_true", help="irregular levels on the GPU")
    ap.add_argument("--device-blocks", action="store_true", help="whole blocks on the GPU, state kept there")
    args = ap.parse_args()
    print(json.dumps(run(args.config, threads=args.threads, t_stop=args.t_stop,
                         device_irregular=args.device_irregular, device_blocks=args.device_blocks)))


if __name__ == "__main__":
    main()
