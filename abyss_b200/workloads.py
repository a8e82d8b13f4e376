"""Seeded synthetic workloads of the benchmark configurations.

* ``kernel_sweep``: King W0 = 6, N = 2^20 (seed 3), 100 neighbours, equal masses.
* ``ensemble``: K Plummer clusters, N log-uniform in [256, 16384] (seed 4,
  cluster k seeded 4000 + k), equal masses, 24 neighbours.
* ``ensemble_waves``: uneven regular blocks: each wave takes every cluster with
  an active fraction 2^-L, L uniform in {0..levels}, mimicking the spread of
  block-timestep levels.
"""
from __future__ import annotations

import numpy as np

from . import ic


def kernel_sweep(n: int = 1 << 20):
    return ic.king(n, 3, 6.0, k_nb=100)


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
