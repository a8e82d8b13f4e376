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
import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from abyss_b200 import _lib, ic  # noqa: E402

CKPT = os.path.join(HERE, "golden", "ac_plummer1024_b200.ckpt")


def main(threads: int = 8):
    L = _lib.lib()
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    c = ic.plummer(1024, 1, masses="equal", k_nb=32)
    e0 = oracle.energy(c.x, c.v, c.m, 1e-8)
    h = C.c_void_p()
    assert L.abyss_ac_load(None, CKPT.encode(), threads, C.byref(h)) == 0
    n = C.c_int(0)
    prm = _lib.ACParams()
    assert L.abyss_ac_info(h, C.byref(n), C.byref(prm)) == 0
    n, cap = int(n.value), int(prm.nb_max)
    blocks, t0 = 0, time.perf_counter()
    mass = None
    while True:
        m, done = C.c_int(0), C.c_int(0)
        new_time, scale = C.c_double(0.0), C.c_double(0.0)
        assert L.abyss_ac_begin_block(h, C.byref(m), C.byref(new_time), C.byref(scale), C.byref(done)) == 0
        if done.value or m.value == 0:
            break
        targets = np.zeros(m.value, np.int32)
        assert L.abyss_ac_block_targets(h, targets.ctypes.data_as(ip)) == 0
        st = {k: np.zeros((n, 3)) for k in ("x", "v", "a0", "a1")}
        st.update({k: np.zeros(n) for k in ("t0", "m", "r2")})
        assert L.abyss_ac_block_state(h, *[st[k].ctypes.data_as(dp) for k in ("x", "v", "a0", "a1", "t0", "m",
                                                                              "r2")]) == 0
        mass = st["m"]
        px, pv = oracle.predict(st["x"], st["v"], st["a0"], st["a1"], st["t0"], new_time.value, scale.value)
        ref = oracle.reg_force(px, pv, st["m"], st["r2"], prm.eps2, targets, cap)
        res = [np.ascontiguousarray(ref[k]) for k in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr")]
        nnb = np.ascontiguousarray(ref["nnb"], np.int32)
        lst = np.ascontiguousarray(ref["list"], np.int32)
        assert L.abyss_ac_end_block(h, *[r.ctypes.data_as(dp) for r in res], nnb.ctypes.data_as(ip),
                                    lst.ctypes.data_as(ip), cap, C.byref(done)) == 0
        blocks += 1
        if done.value:
            break
    x, v = np.zeros((n, 3)), np.zeros((n, 3))
    assert L.abyss_ac_get_state(h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None, None) == 0
    L.abyss_ac_destroy(h)
    e1 = oracle.energy(x, v, mass, 1e-8)
    print(f"{blocks} blocks with the FP64 oracle force: |dE/E| = {abs((e1 - e0) / e0):.3e} "
          f"({time.perf_counter() - t0:.1f} s)")


if __name__ == "__main__":
    main()
