"""Python handle on the host Ahmad-Cohen integrator (include/abyss_ac.h).

The integration itself -- block timesteps, irregular steps, Hermite corrector --
is C++ in libabyss_reg.so; every regular block calls the GPU regular force.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import ACParams, ACStats, ptr, _ip
from .regforce import RegularForce


class ACIntegrator:
    """Integrate one cluster with the Ahmad-Cohen scheme to code time 1 (= t_end)."""

    def __init__(self, rf: RegularForce, x, v, m, r2nb, *, eps2: float = 1e-8, eta_reg: float = 0.02,
                 eta_irr: float = 0.01, fix_nb: int = 32, nb_max: int | None = None, t_end: float = 1.0,
                 threads: int = 0):
        self._L = _lib.lib()
        self.rf = rf
        self.n = int(np.asarray(m).shape[0])
        self.nb_max = int(nb_max if nb_max is not None else 10 * fix_nb)
        self.params = ACParams(float(eps2), float(eta_reg), float(eta_irr), int(fix_nb), self.nb_max,
                               float(t_end), int(threads))
        self.m = np.ascontiguousarray(m, np.float64)
        xs = np.ascontiguousarray(x, np.float64).reshape(self.n, 3)
        vs = np.ascontiguousarray(v, np.float64).reshape(self.n, 3)
        rs = np.ascontiguousarray(r2nb, np.float64)
        h = C.c_void_p()
        rc = self._L.abyss_ac_create(rf._h, C.byref(self.params), self.n, ptr(xs), ptr(vs), ptr(self.m),
                                     ptr(rs), C.byref(h))
        if rc != 0:
            raise _lib.AbyssError(rc, "abyss_ac_create failed: " + rf._L.abyss_last_error(rf._h).decode())
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise _lib.AbyssError(rc, self._L.abyss_ac_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.abyss_ac_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance_block(self) -> bool:
        done = C.c_int(0)
        self._check(self._L.abyss_ac_advance_block(self._h, C.byref(done)))
        return bool(done.value)

    def run(self, t_code: float = 1.0):
        self._check(self._L.abyss_ac_run(self._h, float(t_code)))

    @property
    def time(self) -> float:
        return float(self._L.abyss_ac_time(self._h))

    def state(self):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        nnb = np.zeros(self.n, np.int32)
        r2 = np.zeros(self.n)
        self._check(self._L.abyss_ac_get_state(self._h, ptr(x), ptr(v), ptr(nnb, _ip), ptr(r2)))
        return dict(x=x, v=v, nnb=nnb, r2nb=r2)

    def energy(self) -> float:
        e = C.c_double(0.0)
        self._check(self._L.abyss_ac_energy(self._h, C.byref(e)))
        return float(e.value)

    def stats(self) -> dict:
        st = ACStats()
        self._check(self._L.abyss_ac_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def last_regular(self) -> dict:
        """The last regular-force call: targets, predicted j-set, radii and GPU results."""
        m = C.c_int(0)
        self._check(self._L.abyss_ac_last_regular(self._h, C.byref(m), None, None, None, None, None, None,
                                                  None, None, 0))
        k = int(m.value)
        t = np.zeros(k, np.int32)
        px = np.zeros((self.n, 3))
        pv = np.zeros((self.n, 3))
        r2 = np.zeros(self.n)
        acc = np.zeros((k, 3))
        jerk = np.zeros((k, 3))
        nnb = np.zeros(k, np.int32)
        lst = np.zeros((k, self.nb_max), np.int32)
        self._check(self._L.abyss_ac_last_regular(self._h, C.byref(m), ptr(t, _ip), ptr(px), ptr(pv), ptr(r2),
                                                  ptr(acc), ptr(jerk), ptr(nnb, _ip), ptr(lst, _ip),
                                                  self.nb_max))
        return dict(targets=t, px=px, pv=pv, r2nb=r2, acc_reg=acc, jerk_reg=jerk, nnb=nnb, list=lst)
