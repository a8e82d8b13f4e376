"""Batched regular force over many clusters (include/abyss_ens.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Tuning, ptr, _ip, _fp, _dp, _vp
from .regforce import ForceResult, RegularForce, _f64

BATCHED, GRAPH, PLAIN = 0, 1, 2


def _bind(L):
    if getattr(L, "_ens_bound", False):
        return
    L.abyss_ens_create.argtypes = [_vp, C.c_int, _ip, C.c_int, C.POINTER(_vp)]
    L.abyss_ens_destroy.argtypes = [_vp]
    L.abyss_ens_device_bytes.argtypes = [_vp]
    L.abyss_ens_device_bytes.restype = C.c_longlong
    L.abyss_ens_upload_state.argtypes = [_vp, C.c_int] + [_dp] * 7
    L.abyss_ens_set_wave.argtypes = [_vp, C.c_int, _ip, _dp, _dp, _ip, _ip]
    L.abyss_ens_launch.argtypes = [_vp, C.c_double, C.c_int, C.POINTER(Tuning)]
    L.abyss_ens_fetch.argtypes = [_vp, _dp, _dp, _dp, _dp, _ip, _ip, _ip]
    L.abyss_ens_last_ms.argtypes = [_vp, _fp]
    L.abyss_ens_last_stats.argtypes = [_vp, _ip, _ip, _ip]
    L.abyss_ens_create_arena.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]
    L.abyss_ens_attach.argtypes = [_vp, C.c_int, _ip]
    L.abyss_ens_detach.argtypes = [_vp, C.c_int]
    L.abyss_ens_free_particles.argtypes = [_vp]
    L.abyss_ens_stage_reserve.argtypes = [_vp]
    L.abyss_ens_stage.argtypes = [_vp, C.c_int] + [C.POINTER(_dp)] * 7
    L.abyss_ens_upload_staged.argtypes = [_vp, C.c_int, _ip]
    L.abyss_ens_list_cap.argtypes = [_vp]
    L.abyss_ens_set_chunk.argtypes = [_vp, C.c_int]
    L.abyss_ens_set_tuning.argtypes = [_vp, C.POINTER(Tuning), C.c_int, _ip, _ip]
    L.abyss_ens_get_shape.argtypes = [_vp, C.POINTER(Tuning)]
    L.abyss_ens_submit.argtypes = [_vp, C.c_int, _ip, _dp, _dp, _ip, _ip, C.c_double, C.c_int, _ip]
    L.abyss_ens_ready.argtypes = [_vp, C.c_int]
    L.abyss_ens_collect.argtypes = [_vp, C.c_int] + [C.POINTER(_dp)] * 4 + [C.POINTER(_ip)] * 2 + [_ip, _fp]
    L._ens_bound = True


class Ensemble:
    """K clusters resident on one GPU; regular force for waves of (cluster, targets)."""

    def __init__(self, rf: RegularForce, sizes=None, list_cap: int = 256, capacity: int = 0,
                 max_clusters: int = 0):
        """Fixed clusters of the given sizes, or (sizes=None) an empty arena with room
        for `capacity` particles in at most `max_clusters` clusters."""
        self._L = _lib.lib()
        _bind(self._L)
        self.rf = rf
        self.cap = int(list_cap)
        h = C.c_void_p()
        if sizes is not None:
            self.sizes = np.ascontiguousarray(sizes, np.int32)
            rc = self._L.abyss_ens_create(rf._h, int(self.sizes.shape[0]), ptr(self.sizes, _ip), self.cap,
                                          C.byref(h))
        else:
            self.sizes = np.zeros(int(max_clusters), np.int32)
            rc = self._L.abyss_ens_create_arena(rf._h, int(capacity), int(max_clusters), self.cap, C.byref(h))
        if rc != 0:
            raise _lib.AbyssError(rc, "abyss_ens_create failed")
        self._h = h
        self.rows = 0

    def attach(self, n: int):
        """Place a cluster of n particles; returns its id, or None when it does not fit."""
        k = C.c_int(-1)
        rc = self._L.abyss_ens_attach(self._h, int(n), C.byref(k))
        if rc == _lib.ABYSS_ERR_OOM:
            return None
        self._check(rc)
        self.sizes[k.value] = n
        return int(k.value)

    def detach(self, k: int):
        self._check(self._L.abyss_ens_detach(self._h, int(k)))
        self.sizes[k] = 0

    @property
    def free_particles(self) -> int:
        return int(self._L.abyss_ens_free_particles(self._h))

    def _check(self, rc, allow_overflow=False):
        if rc < 0 or (rc > 0 and not allow_overflow):
            raise _lib.AbyssError(rc, "ensemble call failed")
        return rc

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.abyss_ens_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(self._L.abyss_ens_device_bytes(self._h))

    def upload_state(self, k, x, v, a0, a1, t0, mass, r2nb):
        n = int(self.sizes[k])
        arrs = [_f64(x, (n, 3)), _f64(v, (n, 3)), _f64(a0, (n, 3)), _f64(a1, (n, 3)), _f64(t0), _f64(mass),
                _f64(r2nb)]
        self._check(self._L.abyss_ens_upload_state(self._h, int(k), *[ptr(a) for a in arrs]))

    def stage(self, k: int) -> dict:
        """Cluster k's seven state arrays in the ensemble's pinned staging, as
        writable numpy views (x, v, a0, a1 [n][3]; t0, mass, r2nb [n])."""
        self._check(self._L.abyss_ens_stage_reserve(self._h))
        n = int(self.sizes[k])
        ptrs = [_dp() for _ in range(7)]
        self._check(self._L.abyss_ens_stage(self._h, int(k), *[C.byref(p) for p in ptrs]))
        shapes = [(n, 3)] * 4 + [(n,)] * 3
        names = ("x", "v", "a0", "a1", "t0", "mass", "r2nb")
        return {nm: np.ctypeslib.as_array(p, shape=sh) for nm, p, sh in zip(names, ptrs, shapes)}

    def submit(self, clusters, new_time, time_scale, targets, eps2: float = 0.0, mode: int = GRAPH) -> int:
        """Launch a wave of staged clusters without waiting (at most two in flight);
        returns its ticket for collect()."""
        cl = np.ascontiguousarray(clusters, np.int32)
        nt = np.ascontiguousarray(new_time, np.float64)
        sc = np.ascontiguousarray(time_scale, np.float64)
        mp = np.array([len(t) for t in targets], np.int32)
        tg = np.ascontiguousarray(np.concatenate([np.asarray(t, np.int32) for t in targets]), np.int32)
        ticket = C.c_int(-1)
        self._check(self._L.abyss_ens_submit(self._h, int(cl.shape[0]), ptr(cl, _ip), ptr(nt), ptr(sc),
                                              ptr(mp, _ip), ptr(tg, _ip), float(eps2), int(mode),
                                              C.byref(ticket)))
        return int(ticket.value)

    def collect(self, ticket: int) -> ForceResult:
        """Wait for a submitted wave; its rows, copied out of the pinned staging."""
        p = [_dp() for _ in range(4)]
        q = [_ip() for _ in range(2)]
        rows = C.c_int(0)
        ms = np.zeros(1, np.float32)
        rc = self._L.abyss_ens_collect(self._h, int(ticket), *[C.byref(x) for x in p], *[C.byref(x) for x in q],
                                       C.byref(rows), ptr(ms, _fp))
        self._check(rc, allow_overflow=True)
        m = int(rows.value)
        arr = [np.ctypeslib.as_array(x, shape=(m, 3)).copy() for x in p]
        nnb = np.ctypeslib.as_array(q[0], shape=(m,)).copy()
        lst = np.ctypeslib.as_array(q[1], shape=(m, self.cap)).copy()
        return ForceResult(arr[0], arr[1], arr[2], arr[3], nnb, lst)

    def set_chunk(self, j_per_chunk: int):
        """j per chunk of a cluster's work items (its chunk count depends on its size only)."""
        self._check(self._L.abyss_ens_set_chunk(self._h, int(j_per_chunk)))

    def set_tuning(self, shape: dict | None = None, chunks=()):
        """Launch shape of the force kernel (a tile shape with double-single
        offsets, as autotune.tune_ensemble picks it; None keeps it) and the
        j-chunk length by cluster size: `chunks` is [(n_max, j_per_chunk)] in
        rising n_max, the first entry with n_k <= n_max applies (include/abyss_ens.h
        abyss_ens_set_tuning).  Applies from the next wave."""
        tu = Tuning(**shape) if shape else None
        nm = np.array([c[0] for c in chunks], np.int32)
        jc = np.array([c[1] for c in chunks], np.int32)
        self._check(self._L.abyss_ens_set_tuning(self._h, C.byref(tu) if tu is not None else None, len(chunks),
                                                 ptr(nm, _ip), ptr(jc, _ip)))

    def shape(self) -> dict:
        t = Tuning()
        self._check(self._L.abyss_ens_get_shape(self._h, C.byref(t)))
        return t.as_dict()

    def upload_staged(self, clusters):
        cl = np.ascontiguousarray(clusters, np.int32)
        self._check(self._L.abyss_ens_upload_staged(self._h, int(cl.shape[0]), ptr(cl, _ip)))

    def set_wave(self, clusters, new_time, time_scale, targets):
        """targets: list of cluster-local index arrays, one per listed cluster."""
        cl = np.ascontiguousarray(clusters, np.int32)
        nt = np.ascontiguousarray(new_time, np.float64)
        sc = np.ascontiguousarray(time_scale, np.float64)
        mp = np.array([len(t) for t in targets], np.int32)
        tg = np.ascontiguousarray(np.concatenate([np.asarray(t, np.int32) for t in targets]), np.int32)
        self._check(self._L.abyss_ens_set_wave(self._h, int(cl.shape[0]), ptr(cl, _ip), ptr(nt), ptr(sc),
                                               ptr(mp, _ip), ptr(tg, _ip)))
        self.rows = int(mp.sum())
        self.row_splits = np.concatenate([[0], np.cumsum(mp)])

    def launch(self, eps2: float = 0.0, mode: int = BATCHED, tuning: dict | None = None):
        tu = Tuning(**tuning) if tuning else None
        self._check(self._L.abyss_ens_launch(self._h, float(eps2), int(mode),
                                             C.byref(tu) if tu is not None else None))

    def fetch(self) -> ForceResult:
        m = self.rows
        out = ForceResult(np.zeros((m, 3)), np.zeros((m, 3)), np.zeros((m, 3)), np.zeros((m, 3)),
                          np.zeros(m, np.int32), np.zeros((m, self.cap), np.int32))
        ovf = C.c_int(0)
        self._check(self._L.abyss_ens_fetch(self._h, ptr(out.acc_reg), ptr(out.jerk_reg), ptr(out.acc_irr),
                                            ptr(out.jerk_irr), ptr(out.nnb, _ip), ptr(out.list, _ip),
                                            C.byref(ovf)), allow_overflow=True)
        out.overflow_rows = int(ovf.value)
        return out

    def last_ms(self) -> float:
        ms = np.zeros(1, np.float32)
        self._check(self._L.abyss_ens_last_ms(self._h, ptr(ms, _fp)))
        return float(ms[0])

    def last_stats(self) -> dict:
        r, i, l = C.c_int(0), C.c_int(0), C.c_int(0)
        self._check(self._L.abyss_ens_last_stats(self._h, C.byref(r), C.byref(i), C.byref(l)))
        return {"rows": r.value, "items": i.value, "launches": l.value}
