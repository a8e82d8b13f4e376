"""The CPU oracle (oracle/abyss_oracle.c) pinned against the golden vectors that
tests/golden/make_golden.py produced by running the reference's own CPU code.

Bit-exact: the restatement keeps the reference's FP64 operation order."""
import numpy as np
import pytest

import oracle
from tests.helpers import golden, lists_equal

CASES = ["ref_plummer1024_s1.npz", "ref_king2048_s3.npz"]


@pytest.mark.parametrize("name", CASES)
def test_predictor_bit_exact(name):
    g = golden(name)
    px, pv = oracle.predict(g["x"], g["v"], np.ascontiguousarray(g["a_tot"][:, :, 0]),
                            np.ascontiguousarray(g["a_tot"][:, :, 1]), g["t0"], float(g["new_time"]),
                            float(g["time_scale"]))
    assert np.array_equal(px, g["px"])
    assert np.array_equal(pv, g["pv"])
    # The reference's CUDA_REAL = float predictor (UpdateParticle.cpp:30-31) casts
    # only the inner bracket to float before the last multiply-add:
    # x_p = float(float((a1 dt/3 + a0) dt/2 + v) * dt + x).
    dt = ((float(g["new_time"]) - g["t0"]) * float(g["time_scale"]))[:, None]
    a0, a1 = g["a_tot"][:, :, 0], g["a_tot"][:, :, 1]
    inner = ((a1 * dt / 3 + a0) * dt / 2 + g["v"]).astype(np.float32).astype(np.float64)
    p32 = np.where(dt == 0, g["x"], inner * dt + g["x"]).astype(np.float32)
    innv = (a1 * dt / 2 + a0).astype(np.float32).astype(np.float64)
    v32 = np.where(dt == 0, g["v"], innv * dt + g["v"]).astype(np.float32)
    assert np.array_equal(p32, g["px32"])
    assert np.array_equal(v32, g["pv32"])


@pytest.mark.parametrize("name", CASES)
def test_regular_force_bit_exact(name):
    g = golden(name)
    r = oracle.reg_force(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, g["targets"], 2000, nthreads=4)
    assert np.array_equal(r["acc_reg"], g["out_a_reg"][:, :, 0])
    assert np.array_equal(r["jerk_reg"], g["out_a_reg"][:, :, 1])
    assert np.array_equal(r["acc_irr"], g["out_a_irr"][:, :, 0])
    assert np.array_equal(r["jerk_irr"], g["out_a_irr"][:, :, 1])
    assert lists_equal(r["nnb"], r["list"], g["out_nnb"], g["out_list"])
    # lists: ascending, no self
    for k, t in enumerate(g["targets"]):
        lst = r["list"][k, : r["nnb"][k]]
        assert np.all(np.diff(lst) > 0)
        assert t not in lst


def test_range_sums_add_up():
    g = golden("ref_plummer1024_s1.npz")
    t = g["targets"][:64]
    full = oracle.reg_force(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t, 2000, nthreads=2)
    a1, j1, n1 = oracle.reg_force_range(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t, 0, 500)
    a2, j2, n2 = oracle.reg_force_range(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t, 500, 1024)
    np.testing.assert_allclose(a1 + a2, full["acc_reg"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(j1 + j2, full["jerk_reg"], rtol=1e-12, atol=1e-14)
    assert np.array_equal(n1 + n2, full["nnb"])


def test_softening_changes_force_not_lists():
    g = golden("ref_plummer1024_s1.npz")
    t = g["targets"][:128]
    r0 = oracle.reg_force(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t, 2000)
    r1 = oracle.reg_force(g["px"], g["pv"], g["m"], g["r2nb"], 1e-4, t, 2000)
    assert lists_equal(r0["nnb"], r0["list"], r1["nnb"], r1["list"])
    assert not np.array_equal(r0["acc_reg"], r1["acc_reg"])


def test_overflow_counts_exact():
    g = golden("ref_king2048_s3.npz")
    t = g["targets"][:32]
    r = oracle.reg_force(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t, 16)
    assert r["overflow"] == int((g["out_nnb"][:32] > 16).sum())
    assert np.array_equal(r["nnb"], g["out_nnb"][:32])
    for k in range(32):
        assert np.array_equal(r["list"][k], g["out_list"][k, :16])


def test_timestep_rules_bit_exact():
    g = golden("ref_timesteps.npz")
    L = oracle.lib()
    eta = float(g["eta"])
    for i in range(g["f"].shape[0]):
        v = np.ascontiguousarray(g["v"][i])
        f = np.ascontiguousarray(g["f"][i])
        df = np.ascontiguousarray(g["df"][i])
        assert L.oracle_time_step_reg(oracle._p(v), oracle._p(df), eta) == g["reg"][i]
        assert L.oracle_time_step_irr(oracle._p(f), oracle._p(df), eta) == g["irr"][i]
    import ctypes as C

    for i in range(g["dts"].shape[0]):
        lv = np.zeros(1, np.int32)
        bl = np.zeros(1, np.uint64)
        st = np.zeros(1)
        L.oracle_block_time_step(float(g["dts"][i]), float(g["time_scale"]), int(g["time_block"]),
                                 oracle._p(lv, oracle._ip), bl.ctypes.data_as(C.POINTER(C.c_ulonglong)),
                                 oracle._p(st))
        assert lv[0] == g["level"][i] and bl[0] == g["block"][i] and st[0] == g["step"][i]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU library not built here")
def test_restatement_matches_reference_eps0_fresh_case():
    """Beyond the stored vectors: a fresh seeded case through both codes."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np\n"
        "from tests.golden.make_golden import make_case\n"
        "from abyss_b200 import ic\n"
        "import oracle\n"
        "c = ic.plummer(512, 99, k_nb=20, exact_k=True)\n"
        "g = make_case(c, 4.0, 5)\n"
        "r = oracle.reg_force(g['px'], g['pv'], g['m'], g['r2nb'], 0.0, g['targets'], 2000)\n"
        "ok = np.array_equal(r['acc_reg'], g['out_a_reg'][:, :, 0]) and "
        "np.array_equal(r['jerk_irr'], g['out_a_irr'][:, :, 1]) and np.array_equal(r['nnb'], g['out_nnb'])\n"
        "print('OK' if ok else 'MISMATCH')\n" % here
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=here)
    assert "OK" in out.stdout, out.stdout + out.stderr
