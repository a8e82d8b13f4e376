"""Synthetic initial conditions in N-body units (G = M = 1).

The reference reads particle tables from text files (src_mpi/ReadWrite.cpp:20-107)
and ships no initial conditions, so the workloads here are generated from the
published methods, seeded:

* Plummer sphere -- Aarseth, Henon & Wielen (1974, A&A 37, 183): radii from the
  inverted cumulative mass, speeds by von Neumann rejection on
  g(q) = q^2 (1 - q^2)^{7/2}; scaled to E = -1/4 with the standard 3 pi / 16 factor.
* King (1966, AJ 71, 64) model of central potential W0: the dimensionless Poisson
  equation is integrated to the tidal radius, radii are drawn from the tabulated
  cumulative mass and speeds by rejection from the lowered Maxwellian
  f(v) ~ v^2 (exp(W - v^2/2) - 1); scaled to M = 1, E = -1/4 (virial estimate).
* Kroupa (2001, MNRAS 322, 231) IMF: dN/dm ~ m^-1.3 on [0.08, 0.5) and m^-2.3 on
  [0.5, 100] Msun, sampled segment-wise by inverse CDF and rescaled to sum 1.

Each generator also returns a per-particle squared neighbour radius R_nb^2 for a
target neighbour count k: by default the midpoint of the squared k-th and
(k+1)-th neighbour distances (scipy cKDTree), so every particle starts with
exactly k neighbours; with ``exact_k=False`` it comes from the model's local
number density (N n(r) 4/3 pi R^3 = k), which is only right on average.
"""
from __future__ import annotations

import functools
import math
import threading
from dataclasses import dataclass

import numpy as np


@dataclass
class Cluster:
    """Particle set: x, v are (N, 3) float64; m and r2nb are (N,) float64."""

    x: np.ndarray
    v: np.ndarray
    m: np.ndarray
    r2nb: np.ndarray
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.m.shape[0])


def _isotropic(rng: np.random.Generator, r: np.ndarray) -> np.ndarray:
    n = r.shape[0]
    cost = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sint = np.sqrt(1.0 - cost * cost)
    return np.stack([r * sint * np.cos(phi), r * sint * np.sin(phi), r * cost], axis=1)


def kroupa_masses(n: int, rng: np.random.Generator, mmin: float = 0.08,
                  mbreak: float = 0.5, mmax: float = 100.0) -> np.ndarray:
    """Kroupa (2001) two-segment IMF in Msun (not normalised)."""
    a1, a2 = 1.3, 2.3
    # continuity at mbreak: k1 m^-a1 = k2 m^-a2 -> k2 = k1 mbreak^(a2 - a1)
    k1 = 1.0
    k2 = k1 * mbreak ** (a2 - a1)

    def seg_int(k, a, lo, hi):
        return k * (hi ** (1 - a) - lo ** (1 - a)) / (1 - a)

    w1 = seg_int(k1, a1, mmin, mbreak)
    w2 = seg_int(k2, a2, mbreak, mmax)
    u = rng.uniform(0.0, 1.0, n)
    pick1 = rng.uniform(0.0, 1.0, n) < w1 / (w1 + w2)

    def inv(a, lo, hi, uu):
        e = 1.0 - a
        return (lo ** e + uu * (hi ** e - lo ** e)) ** (1.0 / e)

    m = np.where(pick1, inv(a1, mmin, mbreak, u), inv(a2, mbreak, mmax, u))
    return m


def _r2_from_density(r: np.ndarray, dens: np.ndarray, k: float) -> np.ndarray:
    """R^2 such that n(r) * 4/3 pi R^3 = k, with n the number density."""
    dens = np.maximum(dens, 1e-300)
    rad = (3.0 * k / (4.0 * math.pi * dens)) ** (1.0 / 3.0)
    return rad * rad


def _r2_exact_k(x: np.ndarray, k: int) -> np.ndarray:
    from scipy.spatial import cKDTree

    tree = cKDTree(x)
    k = min(k, x.shape[0] - 2)
    # all host cores for large clusters; one for small ones, which callers build
    # many at a time on their own threads
    d, _ = tree.query(x, k=k + 2, workers=-1 if x.shape[0] >= 65536 else 1)
    # self is d[:, 0]; place R between the k-th and (k+1)-th neighbour
    lo = d[:, k] ** 2
    hi = d[:, k + 1] ** 2
    return 0.5 * (lo + hi)


def plummer(n: int, seed: int, rmax_a: float = 10.0, masses: str = "equal",
            k_nb: float = 32.0, exact_k: bool = True) -> Cluster:
    """Plummer sphere, Aarseth-Henon-Wielen sampling, radii truncated at rmax_a * a."""
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    filled = 0
    while filled < n:
        want = n - filled
        x1 = rng.uniform(1e-12, 1.0, 2 * want + 16)
        rr = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
        rr = rr[rr <= rmax_a][:want]
        r[filled:filled + rr.shape[0]] = rr
        filled += rr.shape[0]
    pos = _isotropic(rng, r)
    q = np.empty(n)
    filled = 0
    while filled < n:
        want = n - filled
        qq = rng.uniform(0.0, 1.0, 4 * want + 16)
        yy = rng.uniform(0.0, 0.1, qq.shape[0])
        ok = qq[yy < qq * qq * (1.0 - qq * qq) ** 3.5][:want]
        q[filled:filled + ok.shape[0]] = ok
        filled += ok.shape[0]
    vesc = math.sqrt(2.0) * (1.0 + r * r) ** (-0.25)
    vel = _isotropic(rng, q * vesc)
    if masses == "equal":
        m = np.full(n, 1.0 / n)
    elif masses == "kroupa":
        m = kroupa_masses(n, rng)
        m = m / m.sum()
    else:
        raise ValueError(f"unknown mass spectrum {masses!r}")
    # Plummer model units (G = M = a = 1) -> N-body units (E = -1/4)
    sx = 3.0 * math.pi / 16.0
    sv = 1.0 / math.sqrt(sx)
    pos *= sx
    vel *= sv
    pos -= (m[:, None] * pos).sum(0) / m.sum()
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    if exact_k:
        r2nb = _r2_exact_k(pos, int(k_nb))
    else:
        rr = np.sqrt((pos * pos).sum(1)) / sx
        dens = n * 3.0 / (4.0 * math.pi) * (1.0 + rr * rr) ** (-2.5) / sx ** 3
        r2nb = _r2_from_density(rr * sx, dens, k_nb)
    return Cluster(pos, vel, m, r2nb, name=f"plummer_n{n}_s{seed}")


_KING_LOCK = threading.Lock()


def _king_profile(w0: float):
    """King's profile for W0, computed once per W0 and shared (read-only arrays).
    The lock makes concurrent first requests for one W0 wait for a single
    computation instead of each repeating it."""
    with _KING_LOCK:
        return _king_profile_solve(float(w0))


@functools.lru_cache(maxsize=16)
def _king_profile_solve(w0: float, npts: int = 4000):
    """Integrate King's equation in units r0 = sigma = G = 1 (rho0 = 9 / 4 pi).

    Returns radius grid, W(r), cumulative mass M(r), density rho(r), tidal radius.
    """
    def rho_of(w):
        w = np.maximum(w, 0.0)
        sw = np.sqrt(w)
        from scipy.special import erf

        return np.exp(w) * erf(sw) - np.sqrt(4.0 * w / math.pi) * (1.0 + 2.0 * w / 3.0)

    rho_c = rho_of(np.array([w0]))[0]
    rho0 = 9.0 / (4.0 * math.pi)

    def deriv(r, y):
        w, dw = y
        rho = rho0 * rho_of(np.array([w]))[0] / rho_c
        d2 = -4.0 * math.pi * rho - (2.0 / r) * dw if r > 0 else -4.0 * math.pi * rho / 3.0
        return np.array([dw, d2])

    # RK4 with a fixed small step until W crosses zero
    h = 1e-3
    r = 1e-6
    y = np.array([w0, 0.0])
    rs, ws = [0.0], [w0]
    while y[0] > 0.0 and r < 1e4:
        k1 = deriv(r, y)
        k2 = deriv(r + h / 2, y + h / 2 * k1)
        k3 = deriv(r + h / 2, y + h / 2 * k2)
        k4 = deriv(r + h, y + h * k3)
        ynew = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        if ynew[0] <= 0.0:
            frac = y[0] / (y[0] - ynew[0])
            r = r + frac * h
            rs.append(r)
            ws.append(0.0)
            y = ynew
            break
        r += h
        y = ynew
        rs.append(r)
        ws.append(y[0])
        if r > 0.5:
            h = min(0.02, h * 1.002)
    rs = np.array(rs)
    ws = np.maximum(np.array(ws), 0.0)
    rho = rho0 * rho_of(ws) / rho_c
    # cumulative mass by trapezoid on 4 pi r^2 rho
    shell = 4.0 * math.pi * rs * rs * rho
    mass = np.concatenate([[0.0], np.cumsum(0.5 * (shell[1:] + shell[:-1]) * np.diff(rs))])
    for a in (rs, ws, mass, rho):
        a.setflags(write=False)
    return rs, ws, mass, rho, float(rs[-1])


def king(n: int, seed: int, w0: float = 6.0, masses: str = "equal",
         k_nb: float = 100.0, exact_k: bool = True) -> Cluster:
    """King (1966) model with central dimensionless potential w0."""
    rng = np.random.default_rng(seed)
    rs, ws, mcum, rho, rt = _king_profile(w0)
    mtot = mcum[-1]
    u = rng.uniform(0.0, mtot, n)
    r = np.interp(u, mcum, rs)
    w = np.interp(r, rs, ws)
    pos = _isotropic(rng, r)
    # speeds: f(v) ~ v^2 (exp(w - v^2/2) - 1), v < sqrt(2 w)
    speed = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        wt = w[todo]
        vmax = np.sqrt(2.0 * wt)
        v = rng.uniform(0.0, 1.0, todo.size) * vmax
        f = v * v * (np.exp(wt - 0.5 * v * v) - 1.0)
        # bound on f over [0, vmax]: at most vmax^2 (exp(w) - 1)
        fmax = vmax * vmax * (np.exp(wt) - 1.0) + 1e-300
        ok = rng.uniform(0.0, 1.0, todo.size) * fmax < f
        speed[todo[ok]] = v[ok]
        todo = todo[~ok]
    vel = _isotropic(rng, speed)
    if masses == "equal":
        m = np.full(n, 1.0 / n)
    elif masses == "kroupa":
        m = kroupa_masses(n, rng)
        m = m / m.sum()
    else:
        raise ValueError(f"unknown mass spectrum {masses!r}")
    # model units (G = 1, total mass mtot) -> N-body units via the virial estimate
    kin_model = 0.5 * mtot * float(np.mean(speed * speed))
    mu = 1.0 / mtot
    lam = 4.0 * kin_model * mu * mu  # E_model = -K; E_new = E_model mu^2 / lam = -1/4
    lv = math.sqrt(mu / lam)
    pos *= lam
    vel *= lv
    pos -= (m[:, None] * pos).sum(0) / m.sum()
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    if exact_k:
        r2nb = _r2_exact_k(pos, int(k_nb))
    else:
        dens_model = np.interp(r, rs, rho) / mtot * n  # number density in model units
        r2nb = _r2_from_density(r * lam, dens_model / lam ** 3, k_nb)
    return Cluster(pos, vel, m, r2nb, name=f"king{w0:g}_n{n}_s{seed}")


def read_reference(path: str, k_nb: float = 32.0) -> Cluster:
    """A cluster from an input file in the reference's text format (x y z in kpc,
    vx vy vz in km/s, mass in 1e9 Msun per line; include/abyss_io.h), in code
    units, with neighbour radii for k_nb neighbours."""
    import ctypes as C

    from . import _lib

    L = _lib.lib()
    n = C.c_int(0)
    rc = L.abyss_read_reference_ic(str(path).encode(), C.byref(n), None, None, None)
    if rc != 0:
        raise _lib.AbyssError(rc, f"cannot read {path}")
    x = np.zeros((n.value, 3))
    v = np.zeros((n.value, 3))
    m = np.zeros(n.value)
    dp = C.POINTER(C.c_double)
    rc = L.abyss_read_reference_ic(str(path).encode(), C.byref(n), x.ctypes.data_as(dp), v.ctypes.data_as(dp),
                                   m.ctypes.data_as(dp))
    if rc != 0:
        raise _lib.AbyssError(rc, f"cannot read {path}")
    return Cluster(x, v, m, _r2_exact_k(x, int(k_nb)), name=f"reference_ic_{n.value}")
