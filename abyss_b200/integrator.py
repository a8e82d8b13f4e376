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

    @classmethod
    def load(cls, rf: RegularForce | None, path: str, threads: int = 0) -> "ACIntegrator":
        """An integration restored from a checkpoint written by save() (include/abyss_io.h).
        With rf None it serves host-side calls only (state, save, the split
        form's begin_block/block_state/end_block); the others raise AbyssError."""
        self = cls.__new__(cls)
        self._L = _lib.lib()
        self.rf = rf
        h = C.c_void_p()
        rc = self._L.abyss_ac_load(rf._h if rf is not None else None, str(path).encode(), int(threads), C.byref(h))
        if rc != 0:
            raise _lib.AbyssError(rc, f"abyss_ac_load failed for {path}")
        self._h = h
        n = C.c_int(0)
        self.params = ACParams()
        self._check(self._L.abyss_ac_info(self._h, C.byref(n), C.byref(self.params)))
        self.n = int(n.value)
        self.nb_max = int(self.params.nb_max)
        self.m = None
        return self

    def save(self, path: str):
        """Checkpoint between regular blocks (include/abyss_io.h abyss_ac_save)."""
        self._check(self._L.abyss_ac_save(self._h, str(path).encode()))

    def write_snapshot(self, path: str, output_time: float = 0.0, output_time_step: float = 0.0):
        """The state as a snapshot in the reference's text format."""
        self._check(self._L.abyss_ac_write_snapshot(self._h, str(path).encode(), float(output_time),
                                                    float(output_time_step)))

    def last_error(self) -> str:
        return self._L.abyss_ac_last_error(self._h).decode()

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

    # ---- split form: the regular force of the block comes from elsewhere
    def begin_block(self):
        """Irregular levels up to the next regular block; returns (targets, new_time,
        time_scale) or None when the run is done."""
        m = C.c_int(0)
        nt = C.c_double(0.0)
        sc = C.c_double(1.0)
        done = C.c_int(0)
        self._check(self._L.abyss_ac_begin_block(self._h, C.byref(m), C.byref(nt), C.byref(sc), C.byref(done)))
        if done.value or m.value == 0:
            return None
        t = np.zeros(m.value, np.int32)
        self._check(self._L.abyss_ac_block_targets(self._h, ptr(t, _ip)))
        return t, float(nt.value), float(sc.value)

    def block_state(self):
        n = self.n
        arrs = dict(x=np.zeros((n, 3)), v=np.zeros((n, 3)), a0=np.zeros((n, 3)), a1=np.zeros((n, 3)),
                    t0=np.zeros(n), mass=np.zeros(n), r2nb=np.zeros(n))
        self._check(self._L.abyss_ac_block_state(self._h, *[ptr(arrs[k]) for k in
                                                             ("x", "v", "a0", "a1", "t0", "mass", "r2nb")]))
        return arrs

    def end_block(self, acc, jerk, acc_irr, jerk_irr, nnb, lst) -> str:
        """Commit the block; returns 'ok', 'done' or 'redo' (a list overflowed: the
        radii were shrunk, fetch block_state again and recompute)."""
        a = [np.ascontiguousarray(x, np.float64) for x in (acc, jerk, acc_irr, jerk_irr)]
        nb = np.ascontiguousarray(nnb, np.int32)
        ls = np.ascontiguousarray(lst, np.int32)
        done = C.c_int(0)
        rc = self._L.abyss_ac_end_block(self._h, *[ptr(x) for x in a], ptr(nb, _ip), ptr(ls, _ip),
                                        int(ls.shape[1]), C.byref(done))
        if rc == _lib.ABYSS_WARN_OVERFLOW:
            return "redo"
        self._check(rc)
        return "done" if done.value else "ok"

    def host_timers(self) -> dict:
        t = np.zeros(2)
        self._check(self._L.abyss_ac_host_timers(self._h, ptr(t)))
        return {"sec_jset": float(t[0]), "sec_sched": float(t[1])}

    def set_device_irregular(self, on: bool = True):
        """Run the irregular levels on the GPU (include/abyss_irr.h); the
        results are the same as on the host threads."""
        self._check(self._L.abyss_ac_set_device_irregular(self._h, 1 if on else 0))

    def device_irregular_info(self) -> dict:
        on = C.c_int(0)
        border = C.c_longlong(0)
        sec = C.c_double(0.0)
        cyc = (C.c_longlong * 6)()
        self._check(self._L.abyss_ac_device_irregular_info(self._h, C.byref(on), C.byref(border), C.byref(sec), cyc))
        parts = ("member_list", "unused", "steps", "barrier_after_steps", "commit", "barrier_after_commit")
        return {"on": bool(on.value), "borderline": int(border.value), "sec_copy": float(sec.value),
                "cycles": dict(zip(parts, [int(c) for c in cyc]))}

    def set_device_resident(self, on: bool = True):
        """Run whole blocks on the GPU with the state kept there
        (include/abyss_irr.h); the results are the same as on the host."""
        self._check(self._L.abyss_ac_set_device_resident(self._h, 1 if on else 0))

    def device_resident_info(self) -> dict:
        on = C.c_int(0)
        border = C.c_longlong(0)
        sec = C.c_double(0.0)
        self._check(self._L.abyss_ac_device_resident_info(self._h, C.byref(on), C.byref(border), C.byref(sec)))
        return {"on": bool(on.value), "borderline": int(border.value), "sec_sync": float(sec.value)}

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
