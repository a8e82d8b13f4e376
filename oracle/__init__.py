"""Test infrastructure only: ctypes bindings to the CPU checkers.

* ``liboracle.so`` -- the plain-C FP64 restatement (oracle/abyss_oracle.c).
* ``_ref/libabyss_ref.so`` -- the reference's own CPU physics compiled from its
  sources by oracle/Makefile (present only where it has been built).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the product (abyss_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


def _p(a, t=_dp):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)


def build(quiet: bool = True) -> None:
    """Build liboracle.so (and _ref when the reference tree is present)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.oracle_predict.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp]
        L.oracle_reg_force.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_int, _ip, C.c_int,
                                       _dp, _dp, _dp, _dp, _ip, _ip, C.c_int]
        L.oracle_reg_force.restype = C.c_int
        L.oracle_reg_force_range.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_int, _ip,
                                             C.c_int, C.c_int, _dp, _dp, _ip, C.c_int]
        L.oracle_hermite_correct.argtypes = [_dp] * 7 + [C.c_double] + [_dp] * 4
        L.oracle_time_step_reg.argtypes = [_dp, _dp, C.c_double]
        L.oracle_time_step_reg.restype = C.c_double
        L.oracle_time_step_irr.argtypes = [_dp, _dp, C.c_double]
        L.oracle_time_step_irr.restype = C.c_double
        L.oracle_block_time_step.argtypes = [C.c_double, C.c_double, C.c_int, _ip,
                                             C.POINTER(C.c_ulonglong), _dp]
        L.oracle_energy.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, C.c_int]
        L.oracle_reg_scale.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_int, _ip, _dp, _dp,
                                       C.c_int]
        L.oracle_energy.restype = C.c_double
        L.oracle_init_derivs23.argtypes = [C.c_int] + [_dp] * 6 + [C.c_double, C.c_int, _ip] + [_dp] * 4 + [C.c_int]
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libabyss_ref.so"))


def ref():
    """The reference's own CPU physics (oracle/_ref/libabyss_ref.so)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libabyss_ref.so")
        L = C.CDLL(path)
        L.ref_alloc.argtypes = [C.c_int]
        L.ref_set_globals.argtypes = [C.c_double, C.c_int, C.c_ulonglong]
        L.ref_set_particle.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, _dp, _dp, _dp,
                                       C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _ip]
        L.ref_set_all.argtypes = [C.c_int] + [_dp] * 8
        L.ref_set_blocks.argtypes = [C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong,
                                     C.c_ulonglong, C.c_int, C.c_int, C.c_ulonglong]
        L.ref_get_blocks.argtypes = [C.c_int, C.POINTER(C.c_ulonglong), _ip, _dp]
        L.ref_get_particle.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                       _ip, _ip, C.c_int]
        L.ref_compute_reg.argtypes = [C.c_int, _ip, C.c_int]
        L.ref_compute_irr.argtypes = [C.c_int, _ip, C.c_int]
        L.ref_compute_reg_isolated.argtypes = [C.c_int, _ip, _dp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_int]
        L.ref_update_reg_cuda.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp]
        L.ref_update_reg_cuda_isolated.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_predict.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.ref_predict_f32.argtypes = [C.c_int, C.c_double, _fp, _fp]
        for name in ("ref_update_particle", "ref_update_radius", "ref_time_step_reg",
                     "ref_time_step_irr", "ref_initialize_time_step", "ref_init_acc01",
                     "ref_init_acc23"):
            getattr(L, name).argtypes = [C.c_int]
        L.ref_new_time_step_reg.argtypes = [_dp, _dp]
        L.ref_new_time_step_reg.restype = C.c_double
        L.ref_new_time_step_irr.argtypes = [_dp, _dp]
        L.ref_new_time_step_irr.restype = C.c_double
        L.ref_block_time_step.argtypes = [C.c_double, _ip, C.POINTER(C.c_ulonglong), _dp]
        L.ref_eta.restype = C.c_double
        L.ref_particle_from_row.argtypes = [_dp, _dp, _dp, _dp]
        _REF = L
    return _REF


# ---------------------------------------------------------------- numpy helpers

def predict(x, v, a0, a1, t0, new_time, time_scale):
    n = x.shape[0]
    px = np.empty_like(x)
    pv = np.empty_like(v)
    lib().oracle_predict(n, _p(x), _p(v), _p(a0), _p(a1), _p(t0), new_time, time_scale,
                         _p(px), _p(pv))
    return px, pv


def reg_force(px, pv, m, r2nb, eps2, targets, cap, nthreads=0, with_irr=True):
    """FP64 oracle regular force.  Returns dict of arrays (per target)."""
    px = np.ascontiguousarray(px, np.float64)
    pv = np.ascontiguousarray(pv, np.float64)
    m = np.ascontiguousarray(m, np.float64)
    r2nb = np.ascontiguousarray(r2nb, np.float64)
    t = np.ascontiguousarray(targets, np.int32)
    nt = t.shape[0]
    out = {k: np.zeros((nt, 3)) for k in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr")}
    nnb = np.zeros(nt, np.int32)
    lst = np.full((nt, cap), -1, np.int32)
    ov = lib().oracle_reg_force(px.shape[0], _p(px), _p(pv), _p(m), _p(r2nb), eps2, nt, _p(t, _ip),
                                cap, _p(out["acc_reg"]), _p(out["jerk_reg"]),
                                _p(out["acc_irr"]) if with_irr else _p(None),
                                _p(out["jerk_irr"]) if with_irr else _p(None),
                                _p(nnb, _ip), _p(lst, _ip), nthreads)
    out["nnb"] = nnb
    out["list"] = lst
    out["overflow"] = ov
    return out


def reg_force_range(px, pv, m, r2nb, eps2, targets, j0, j1, nthreads=0):
    t = np.ascontiguousarray(targets, np.int32)
    nt = t.shape[0]
    acc = np.zeros((nt, 3))
    jerk = np.zeros((nt, 3))
    nnb = np.zeros(nt, np.int32)
    lib().oracle_reg_force_range(px.shape[0], _p(px), _p(pv), _p(m), _p(r2nb), eps2, nt, _p(t, _ip),
                                 j0, j1, _p(acc), _p(jerk), _p(nnb, _ip), nthreads)
    return acc, jerk, nnb


def reg_scale(px, pv, m, r2nb, eps2, targets, nthreads=0):
    """Per-target sums of |regular acc term| and |regular jerk term|."""
    t = np.ascontiguousarray(targets, np.int32)
    a = np.zeros(t.shape[0])
    j = np.zeros(t.shape[0])
    lib().oracle_reg_scale(px.shape[0], _p(np.ascontiguousarray(px)), _p(np.ascontiguousarray(pv)),
                           _p(np.ascontiguousarray(m)), _p(np.ascontiguousarray(r2nb)), eps2, t.shape[0],
                           _p(t, _ip), _p(a), _p(j), nthreads)
    return a, j


def hermite_correct(pos, vel, a_reg_old, a_new, adot_new, a_tmp, adot_tmp, dt):
    npos = np.zeros(3)
    nvel = np.zeros(3)
    a2 = np.zeros(3)
    a3 = np.zeros(3)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (pos, vel, a_reg_old, a_new, adot_new,
                                                           a_tmp, adot_tmp)]
    lib().oracle_hermite_correct(*[_p(a) for a in arrs], dt, _p(npos), _p(nvel), _p(a2), _p(a3))
    return npos, nvel, a2, a3


def energy(x, v, m, eps2, nthreads=0):
    return lib().oracle_energy(x.shape[0], _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(v)),
                               _p(np.ascontiguousarray(m)), eps2, nthreads)


def init_derivs23(x, v, m, r2nb, a0, a1, eps2, targets, nthreads=0):
    """Second and third acceleration derivatives, split (CalculateAcceleration23)."""
    f = lambda a: np.ascontiguousarray(a, np.float64)
    x, v, m, r2nb, a0, a1 = map(f, (x, v, m, r2nb, a0, a1))
    t = np.ascontiguousarray(targets, np.int32)
    out = [np.zeros((t.shape[0], 3)) for _ in range(4)]
    lib().oracle_init_derivs23(x.shape[0], _p(x), _p(v), _p(m), _p(r2nb), _p(a0), _p(a1), eps2, t.shape[0],
                               _p(t, _ip), *[_p(o) for o in out], nthreads)
    return dict(reg2=out[0], reg3=out[1], irr2=out[2], irr3=out[3])
