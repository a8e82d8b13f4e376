"""Seeded synthetic workloads of the benchmark configurations.

* ``kernel_sweep``: King W0 = 6, N = 2^20 (seed 3), 100 neighbours, equal masses.
* ``kernel_sweep_state``: that cluster as an un-predicted j-set (seeded
  acceleration, jerk and last-advance times), so that the device prediction
  to the block time does its arithmetic; ``sweep_targets`` the sweep's active
  sets.
* ``ensemble``: K Plummer clusters, N log-uniform in [256, 16384] (seed 4,
  cluster k seeded 4000 + k), equal masses, 24 neighbours.
* ``ensemble_waves``: uneven regular blocks: each wave takes every cluster with
  an active fraction 2^-L, L uniform in {0..levels}, mimicking the spread of
  block-timestep levels.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import ic


def kernel_sweep(n: int = 1 << 20):
    return ic.king(n, 3, 6.0, k_nb=100)


@dataclass
class SweepState:
    """Un-predicted FP64 j-set of the kernel sweep (arrays as for
    ``RegularForce.upload_state``) and the block time it is predicted to."""

    cluster: ic.Cluster
    a0: np.ndarray
    a1: np.ndarray
    t0: np.ndarray
    new_time: float
    time_scale: float = 1.0


def kernel_sweep_state(n: int = 1 << 20, seed: int = 103) -> SweepState:
    """The kernel-sweep cluster with seeded second-order prediction inputs:
    |a| ~ 1 and |da/dt| ~ 4 per component (normal), each particle last advanced
    2^-k before the block time, k uniform in {12..16}, so that predicted
    positions move by at most a few 1e-4 and the neighbour counts stay near 100."""
    c = kernel_sweep(n)
    rng = np.random.default_rng(seed)
    a0 = rng.normal(0.0, 1.0, (n, 3))
    a1 = rng.normal(0.0, 4.0, (n, 3))
    new_time = 0.125
    t0 = new_time - np.ldexp(1.0, -rng.integers(12, 17, n))
    return SweepState(c, a0, a1, t0, new_time)


SWEEP_SIZES = (1, 32, 1024, 32768)


def sweep_targets(n: int, sizes=SWEEP_SIZES, seed: int = 0) -> dict:
    """Sorted active sets of the sweep sizes, drawn in order from one seeded generator."""
    rng = np.random.default_rng(seed)
    return {mm: np.sort(rng.choice(n, mm, replace=False)).astype(np.int32) for mm in sizes}


def ensemble(k: int = 512, nmin: int = 256, nmax: int = 16384, seed: int = 4, k_nb: int = 24):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), k)).astype(int)
    clusters = [ic.plummer(int(n), 4000 + i, k_nb=k_nb) for i, n in enumerate(sizes)]
    return clusters


def ensemble_waves(clusters, n_waves: int, seed: int = 5, levels: int = 8, frac_clusters: float = 1.0):
    rng = np.random.default_rng(seed)
    k = len(clusters)
    waves = []
    for _ in range(n_waves):
        nk = max(1, int(round(frac_clusters * k)))
        chosen = np.sort(rng.choice(k, nk, replace=False))
        targets = []
        for i in chosen:
            n = clusters[i].n
            m = max(1, int(n * 2.0 ** -rng.integers(0, levels + 1)))
            targets.append(np.sort(rng.choice(n, m, replace=False)).astype(np.int32))
        waves.append((chosen, targets))
    return waves
