"""The host integrator's irregular steps, on the CPU, from a checkpoint.

tests/golden/ac_plummer1024_b200.ckpt holds configuration 1 (Plummer N = 1024,
seed 1) after 200 regular blocks, written on a GPU by
tests/golden/make_ac_checkpoint.py.  Loaded without a GPU context
(include/abyss_io.h: ctx = NULL serves host-side calls only), the integration
runs the irregular levels up to its next regular block
(abyss_ac_begin_block), and then whole regular blocks whose forces come from
the FP64 oracle.  The resulting positions and velocities:
  * are the same, bit for bit, for 1 and 4 host threads (a level's particles
    are computed from the pre-level state and committed one by one);
  * match the digest recorded when the fixture was made, which pins the host's
    irregular step (prediction, the vectorised neighbour terms, the corrector,
    the time-step rules, the level order) against any change of its results.
Calls that need the GPU fail with ABYSS_ERR_ARG instead of touching a device.
"""
import ctypes as C
import hashlib
import os

import numpy as np
import pytest

from abyss_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
CKPT = os.path.join(HERE, "golden", "ac_plummer1024_b200.ckpt")
# sha256 of x then v (float64, [1024][3] each) after abyss_ac_begin_block
STATE_DIGEST = "386e0cf5ccd5fe789ef67b0a5698b29b73fec2f20df81498168b89cb6dbaa162"
# the same after 30 regular blocks driven by the FP64 oracle's regular force
BLOCKS30_DIGEST = "de20b636a5ada0dc9cf4010882b1765f04feddbe321631f5507bbf20c8217a22"
dp = C.POINTER(C.c_double)


def _begin_block(L, threads):
    h = C.c_void_p()
    assert L.abyss_ac_load(None, CKPT.encode(), threads, C.byref(h)) == 0
    try:
        m, done = C.c_int(0), C.c_int(0)
        new_time, scale = C.c_double(0.0), C.c_double(0.0)
        assert L.abyss_ac_begin_block(h, C.byref(m), C.byref(new_time), C.byref(scale), C.byref(done)) == 0
        x = np.zeros((1024, 3))
        v = np.zeros((1024, 3))
        assert L.abyss_ac_get_state(h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None, None) == 0
        e = C.c_double(0.0)
        gpu_rc = L.abyss_ac_energy(h, C.byref(e))
        return m.value, new_time.value, x, v, gpu_rc
    finally:
        L.abyss_ac_destroy(h)


def test_irregular_levels_from_checkpoint_on_cpu():
    try:
        L = _lib.lib()
    except (RuntimeError, OSError) as exc:
        pytest.skip(f"library not built: {exc}")
    runs = [_begin_block(L, t) for t in (1, 4)]
    (m1, t1, x1, v1, rc1), (m4, t4, x4, v4, rc4) = runs
    assert m1 == m4 and m1 > 0 and t1 == t4
    assert np.array_equal(x1, x4) and np.array_equal(v1, v4)
    assert hashlib.sha256(x1.tobytes() + v1.tobytes()).hexdigest() == STATE_DIGEST
    assert rc1 == _lib.ABYSS_ERR_ARG and rc4 == _lib.ABYSS_ERR_ARG


def _run_blocks_with_oracle(L, threads, blocks):
    """The split-block form of the integration (abyss_ac_begin_block /
    abyss_ac_end_block), its regular forces from the FP64 oracle on the CPU."""
    import oracle

    h = C.c_void_p()
    assert L.abyss_ac_load(None, CKPT.encode(), threads, C.byref(h)) == 0
    try:
        n = C.c_int(0)
        prm = _lib.ACParams()
        assert L.abyss_ac_info(h, C.byref(n), C.byref(prm)) == 0
        n, cap = int(n.value), int(prm.nb_max)
        ip = C.POINTER(C.c_int)
        done_blocks = 0
        for _ in range(blocks):
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
            px, pv = oracle.predict(st["x"], st["v"], st["a0"], st["a1"], st["t0"], new_time.value, scale.value)
            ref = oracle.reg_force(px, pv, st["m"], st["r2"], prm.eps2, targets, cap)
            res = [np.ascontiguousarray(ref[k]) for k in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr")]
            nnb = np.ascontiguousarray(ref["nnb"], np.int32)
            lst = np.ascontiguousarray(ref["list"], np.int32)
            rc = L.abyss_ac_end_block(h, *[r.ctypes.data_as(dp) for r in res], nnb.ctypes.data_as(ip),
                                      lst.ctypes.data_as(ip), cap, C.byref(done))
            assert rc == 0, rc
            done_blocks += 1
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        assert L.abyss_ac_get_state(h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None, None) == 0
        return done_blocks, x, v
    finally:
        L.abyss_ac_destroy(h)


def test_regular_blocks_with_the_oracle_force_on_cpu():
    """Thirty regular blocks of configuration 1 from the checkpoint: the host
    integrator's whole step (irregular levels, regular corrector, neighbour
    changes, time steps, radius updates) driven by the FP64 oracle force.  The
    result is independent of the thread count and matches a recorded digest of
    the final state."""
    try:
        L = _lib.lib()
    except (RuntimeError, OSError) as exc:
        pytest.skip(f"library not built: {exc}")
    b1, x1, v1 = _run_blocks_with_oracle(L, 1, 30)
    b4, x4, v4 = _run_blocks_with_oracle(L, 4, 30)
    assert b1 == b4 == 30
    assert np.array_equal(x1, x4) and np.array_equal(v1, v4)
    assert hashlib.sha256(x1.tobytes() + v1.tobytes()).hexdigest() == BLOCKS30_DIGEST
