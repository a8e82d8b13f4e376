"""The host integrator's per-particle rules (include/abyss_host.h) against the
reference's own outputs (golden vectors).  CPU only."""
import ctypes as C

import numpy as np
import pytest

from abyss_b200 import _lib
from abyss_b200._lib import ptr, _ip
from tests.helpers import golden

CASES = ["ref_plummer1024_s1.npz", "ref_king2048_s3.npz"]


@pytest.mark.parametrize("name", CASES)
def test_host_predictor_bit_exact(name):
    L = _lib.lib()
    g = golden(name)
    scale = float(g["time_scale"])
    for j in range(0, g["x"].shape[0], 7):
        pos = np.zeros(3)
        vel = np.zeros(3)
        a0 = np.ascontiguousarray(g["a_tot"][j, :, 0])
        a1 = np.ascontiguousarray(g["a_tot"][j, :, 1])
        L.abyss_host_predict(ptr(np.ascontiguousarray(g["x"][j])), ptr(np.ascontiguousarray(g["v"][j])),
                             ptr(a0), ptr(a1), float(g["new_time"]) - float(g["t0"][j]), scale,
                             ptr(pos), ptr(vel))
        assert np.array_equal(pos, g["px"][j]) and np.array_equal(vel, g["pv"][j])


def test_host_time_steps_bit_exact():
    L = _lib.lib()
    g = golden("ref_timesteps.npz")
    eta = float(g["eta"])
    for i in range(g["f"].shape[0]):
        f = np.ascontiguousarray(g["f"][i])
        df = np.ascontiguousarray(g["df"][i])
        assert L.abyss_host_time_step_reg(ptr(df), eta) == g["reg"][i]
        assert L.abyss_host_time_step_irr(ptr(f), ptr(df), eta) == g["irr"][i]
    for i in range(g["dts"].shape[0]):
        lv = np.zeros(1, np.int32)
        bl = np.zeros(1, np.uint64)
        st = np.zeros(1)
        L.abyss_host_block_time_step(float(g["dts"][i]), float(g["time_scale"]), int(g["time_block"]),
                                     ptr(lv, _ip), bl.ctypes.data_as(C.POINTER(C.c_ulonglong)), ptr(st))
        assert (lv[0], bl[0], st[0]) == (g["level"][i], g["block"][i], g["step"][i])


@pytest.mark.parametrize("name", CASES)
def test_host_regular_corrector_bit_exact(name):
    """updateRegularParticleCuda: fed the reference's new list, regular force and the
    FP64 irregular part, the host corrector reproduces the reference's new position,
    velocity and derivatives bit for bit."""
    L = _lib.lib()
    g = golden(name)
    n = g["x"].shape[0]
    a_tot = np.ascontiguousarray(g["a_tot"].reshape(n, 12))
    for k, i in enumerate(g["targets"][:200]):
        old = np.ascontiguousarray(g["nb"][i, : g["nnb"][i]], np.int32)
        new = np.ascontiguousarray(g["out_list"][k, : g["out_nnb"][k]], np.int32)
        acc = np.ascontiguousarray(g["out_a_reg"][k, :, 0])
        jerk = np.ascontiguousarray(g["out_a_reg"][k, :, 1])
        airr = np.ascontiguousarray(g["out_a_irr"][k, :, 0])
        jirr = np.ascontiguousarray(g["out_a_irr"][k, :, 1])
        npos = np.zeros(3)
        nvel = np.zeros(3)
        areg = np.zeros(12)
        atot = np.zeros(12)
        rc = L.abyss_host_regular_correct(n, ptr(g["x"]), ptr(g["v"]), ptr(a_tot), ptr(g["t0"]), ptr(g["m"]),
                                          0.0, float(g["new_time"]), float(g["time_scale"]), int(i),
                                          float(g["dt_reg"][i]), ptr(np.ascontiguousarray(g["a_reg"][i])),
                                          old.shape[0], ptr(old, _ip), new.shape[0], ptr(new, _ip),
                                          ptr(acc), ptr(jerk), ptr(airr), ptr(jirr), ptr(npos), ptr(nvel),
                                          ptr(areg), ptr(atot))
        assert rc == 0
        assert np.array_equal(npos, g["cuda_newpos"][k]), (k, npos, g["cuda_newpos"][k])
        assert np.array_equal(nvel, g["cuda_newvel"][k])
        assert np.array_equal(areg.reshape(3, 4), g["cuda_a_reg"][k])
        assert np.array_equal(atot.reshape(3, 4)[:, :2], g["cuda_a_tot"][k][:, :2])
