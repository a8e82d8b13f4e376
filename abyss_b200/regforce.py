"""Host-side mirror of the reference's GPU regular-force interface.

``RegularForce`` wraps one library context (include/abyss_reg.h).  Its calls
map onto the reference's C ABI (src_mpi/cuda/cuda_functions.h:3-10):

=================================  ============================================
reference                          here
=================================  ============================================
InitializeDevice / OpenDevice      ``RegularForce(device)``
SendToDevice(NNB, m, x, v, r2, .)  ``send_to_device(m, x, v, r2)`` (predicted j-set)
                                   or ``upload_state(...)`` + ``predict(t, scale)``
CalculateAccelerationOnDevice      ``calculate_acceleration(targets, ...)``
CloseDevice                        ``close()``
=================================  ============================================

Results are the reference's outputs -- regular acceleration and jerk
(neighbours excluded), neighbour counts and ascending lists -- plus the
irregular part over the new list in FP64 (the reference recomputes it on the
host, src_mpi/Particle/ComputeAcceleration.cpp:537-566).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import Tuning, ptr, _ip, _fp


@dataclass
class ForceResult:
    acc_reg: np.ndarray
    jerk_reg: np.ndarray
    acc_irr: np.ndarray
    jerk_irr: np.ndarray
    nnb: np.ndarray
    list: np.ndarray
    overflow_rows: int = 0
    plan: dict = field(default_factory=dict)

    def neighbours(self, r: int) -> np.ndarray:
        k = min(int(self.nnb[r]), self.list.shape[1])
        return self.list[r, :k]


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class RegularForce:
    """One CUDA context of the regular-force library on one device."""

    def __init__(self, device: int = 0):
        self._L = _lib.lib()
        h = C.c_void_p()
        rc = self._L.abyss_create(device, C.byref(h))
        if rc != 0:
            raise _lib.AbyssError(rc, "abyss_create failed (no usable CUDA device?)")
        self._h = h
        self.n = 0

    # ------------------------------------------------------------ plumbing
    def _check(self, rc: int, allow_overflow: bool = False) -> int:
        if rc < 0 or (rc > 0 and not allow_overflow):
            raise _lib.AbyssError(rc, self._L.abyss_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.abyss_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self._L.abyss_stream(self._h) or 0)

    def synchronize(self):
        self._check(self._L.abyss_synchronize(self._h))

    def set_wait(self, spin_us: int):
        """How this context's calls wait for the GPU: spin_us < 0 keeps the
        stream synchronisation (the default); spin_us >= 0 polls that long,
        then sleeps in a blocking wait (include/abyss_reg.h abyss_set_wait)."""
        self._check(self._L.abyss_set_wait(self._h, int(spin_us)))

    def reserve(self, n: int, m: int, list_cap: int):
        self._check(self._L.abyss_reserve(self._h, n, m, list_cap))

    # ------------------------------------------------------------ j-set
    def upload_state(self, x, v, a0, a1, t0, mass, r2nb):
        n = int(np.asarray(mass).shape[0])
        arrs = [_f64(x, (n, 3)), _f64(v, (n, 3)), _f64(a0, (n, 3)), _f64(a1, (n, 3)), _f64(t0),
                _f64(mass), _f64(r2nb)]
        self._check(self._L.abyss_upload_state(self._h, n, *[ptr(a) for a in arrs]))
        self._keep = arrs  # host copies stay alive until the async copies finish
        self.synchronize()
        self.n = n

    def predict(self, new_time: float, time_scale: float = 1.0):
        self._check(self._L.abyss_predict(self._h, float(new_time), float(time_scale)))

    def send_to_device(self, mass, px, pv, r2nb):
        """SendToDevice: upload an already predicted j-set."""
        n = int(np.asarray(mass).shape[0])
        arrs = [_f64(px, (n, 3)), _f64(pv, (n, 3)), _f64(mass), _f64(r2nb)]
        self._check(self._L.abyss_upload_predicted(self._h, n, *[ptr(a) for a in arrs]))
        self._keep = arrs
        self.synchronize()
        self.n = n

    def read_predicted(self):
        px = np.zeros((self.n, 3))
        pv = np.zeros((self.n, 3))
        vm = np.zeros((self.n, 4), np.float32)
        self._check(self._L.abyss_read_predicted(self._h, ptr(px), ptr(pv), ptr(vm, _fp)))
        return px, pv, vm

    # ------------------------------------------------------------ force
    def set_targets(self, targets):
        t = np.ascontiguousarray(targets, dtype=np.int32)
        self._check(self._L.abyss_set_targets(self._h, int(t.shape[0]), ptr(t, _ip)))
        self._targets = t
        self.m = int(t.shape[0])

    def launch(self, eps2: float = 0.0, list_cap: int = 256, tuning: dict | None = None):
        tu = Tuning(**tuning) if tuning else None
        self._check(self._L.abyss_launch(self._h, float(eps2), int(list_cap),
                                         C.byref(tu) if tu is not None else None))

    def fetch(self, list_cap: int) -> ForceResult:
        m = self.m
        out = ForceResult(np.zeros((m, 3)), np.zeros((m, 3)), np.zeros((m, 3)), np.zeros((m, 3)),
                          np.zeros(m, np.int32), np.zeros((m, list_cap), np.int32))
        ovf = C.c_int(0)
        self._check(self._L.abyss_fetch(self._h, ptr(out.acc_reg), ptr(out.jerk_reg), ptr(out.acc_irr),
                                        ptr(out.jerk_irr), ptr(out.nnb, _ip), ptr(out.list, _ip),
                                        C.byref(ovf)), allow_overflow=True)
        out.overflow_rows = int(ovf.value)
        out.plan = self.last_plan()
        return out

    def calculate_acceleration(self, targets, eps2: float = 0.0, list_cap: int = 256,
                               tuning: dict | None = None) -> ForceResult:
        """CalculateAccelerationOnDevice for the given active indices."""
        self.set_targets(targets)
        self.launch(eps2, list_cap, tuning)
        return self.fetch(list_cap)

    def last_plan(self) -> dict:
        t = Tuning()
        s = C.c_int(0)
        self._check(self._L.abyss_last_plan(self._h, C.byref(t), C.byref(s)))
        d = t.as_dict()
        d["n_chunks"] = int(s.value)
        return d

    def last_order(self) -> np.ndarray:
        """Target rows in the order the last launch processed them; consecutive
        runs of threads x ipt rows share an i-block (and, in anchor mode, the
        anchor position of the run's first row)."""
        rows = np.zeros(self.m, np.int32)
        self._check(self._L.abyss_last_order(self._h, ptr(rows, _ip)))
        return rows

    def set_profiling(self, on):
        """True: time each phase of later launches; "whole": the whole launch
        with two events (no events between phases); False: off."""
        self._check(self._L.abyss_set_profiling(self._h, 2 if on == "whole" else 1 if on else 0))

    def last_timing(self):
        ms = np.zeros(3, np.float32)
        self._check(self._L.abyss_last_timing(self._h, ptr(ms, _fp)))
        return {"order_ms": float(ms[0]), "force_ms": float(ms[1]), "finalize_ms": float(ms[2])}

    def set_tuning_table(self, entries):
        """entries: list of (m_max, tuning dict) in increasing m_max."""
        k = len(entries)
        mm = np.array([e[0] for e in entries], np.int32)
        arr = (Tuning * max(k, 1))()
        for i, (_, d) in enumerate(entries):
            arr[i] = Tuning(**d)
        self._check(self._L.abyss_set_tuning_table(self._h, k, ptr(mm, _ip), arr))

    def init_derivs23(self, x, v, mass, r2nb, a0, a1, eps2: float = 0.0) -> dict:
        """Second and third acceleration derivatives at a common time, split into
        regular and irregular parts (include/abyss_reg.h abyss_init_derivs23)."""
        n = int(np.asarray(mass).shape[0])
        ins = [_f64(x, (n, 3)), _f64(v, (n, 3)), _f64(mass), _f64(r2nb), _f64(a0, (n, 3)), _f64(a1, (n, 3))]
        out = {k: np.zeros((n, 3)) for k in ("reg2", "reg3", "irr2", "irr3")}
        self._check(self._L.abyss_init_derivs23(self._h, n, *[ptr(a) for a in ins], float(eps2),
                                                *[ptr(out[k]) for k in ("reg2", "reg3", "irr2", "irr3")]))
        return out

    def energy(self, x, v, mass, eps2: float = 0.0) -> float:
        n = int(np.asarray(mass).shape[0])
        e = C.c_double(0.0)
        xs, vs, ms = _f64(x, (n, 3)), _f64(v, (n, 3)), _f64(mass)
        self._check(self._L.abyss_energy(self._h, n, ptr(xs), ptr(vs), ptr(ms), float(eps2), C.byref(e)))
        return float(e.value)
