"""Autotuner of the regular-force launch shape.

Single cluster (``tune``): for each active-set size bucket it times every compiled tile-kernel shape
(abyss_tile_variants: threads, targets per thread, anchor or double-single
offsets, packed FP32x2 or scalar arithmetic, j unroll, register cap) and the
j-major kernel, over a few j-split choices, on the caller's own j-set, and keeps
the fastest shape whose offsets are accurate at that size (anchor offsets only
from `anchor_min` targets up).  The result is a table of (m_max, shape) entries;
``install`` hands it to the library (abyss_set_tuning_table), ``save``/``load``
keep it as JSON.

Batched ensemble (``tune_ensemble``): on the ensemble's own waves (its
clusters and their uneven active sets, in the CUDA-graph form) it times every
compiled double-single tile shape with at least 128 targets per block, keeps
the fastest, then picks the j-chunk length of each cluster-size bucket in turn
(``Ensemble.set_tuning``).  The chunk length trades work-list parallelism
against the FP64 chunk partials that the finalize pass sums.

    python -m abyss_b200.autotune --n 1048576 --out tuning.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np

from . import _lib
from .regforce import RegularForce

BUCKETS = (1, 8, 64, 1024, 16384, 131072, 1 << 20)


def variants():
    L = _lib.lib()
    out = []
    for i in range(L.abyss_tile_variants()):
        sh = np.zeros(6, np.int32)
        L.abyss_tile_variant(i, sh.ctypes.data_as(C.POINTER(C.c_int)))
        nt, ipt, anchor, pack, unr, minb = (int(x) for x in sh)
        out.append(dict(kernel=3 if pack else 1, mode=1 if anchor else 2, threads=nt, ipt=ipt, unroll=unr,
                        min_blocks=minb))
    return out


def _time(rf: RegularForce, tuning, reps=2, list_cap=256, eps2=1e-8):
    rf.launch(eps2, list_cap, tuning)
    rf.synchronize()
    best = float("inf")
    for _ in range(reps):
        rf.launch(eps2, list_cap, tuning)
        t = rf.last_timing()
        best = min(best, t["order_ms"] + t["force_ms"] + t["finalize_ms"])
    return best


def tune(rf: RegularForce, n: int, buckets=BUCKETS, anchor_min: int = 16384, seed: int = 0,
         splits=(0, 2, 4), verbose=False):
    """rf must hold a predicted j-set of n particles.  Returns [(m_max, shape, ms)]."""
    rf.set_profiling("whole")
    rng = np.random.default_rng(seed)
    table = []
    shapes = variants()
    for m in buckets:
        if m > n:
            break
        t = np.sort(rng.choice(n, m, replace=False)).astype(np.int32) if m < n else np.arange(n, dtype=np.int32)
        rf.set_targets(t)
        cands = []
        if m <= 64:
            cands += [dict(kernel=2, ipt=i) for i in (1, 2, 4, 8) if i <= max(1, m)]
        if 16 <= m <= 256:  # warps sharing targets, scalar and packed
            cands += [dict(kernel=k, ipt=i, j_split=s) for k in (4, 5) for i in (1, 2) for s in (0, 1024, 2048)]
        for sh in shapes:
            if sh["mode"] == 1 and m < anchor_min:
                continue
            if m < sh["threads"] * sh["ipt"] // 4:
                continue  # mostly idle lanes
            for s in splits:
                cands.append(dict(sh, j_split=s))
        best = None
        for c in cands:
            try:
                ms = _time(rf, c)
            except _lib.AbyssError:
                continue
            if verbose:
                print(m, c, round(ms, 4))
            if best is None or ms < best[1]:
                best = (c, ms)
        if best is not None:
            table.append((int(m), best[0], best[1]))
    return table


ENS_CHUNKS = (512, 1024, 2048, 4096, 8192)
ENS_BUCKETS = (1024, 4096, 16384)


def _ensemble_ms(ens, waves, eps2: float = 1e-8, reps: int = 1) -> float:
    """GPU milliseconds of all waves in the graph form (after one warm launch each)."""
    from .ensemble import GRAPH

    total = 0.0
    for ks, ts in waves:
        ens.set_wave(ks, np.zeros(len(ks)), np.ones(len(ks)), ts)
        ens.launch(eps2, GRAPH)
        ens.last_ms()  # waits for the wave; its rows are not needed here
        best = float("inf")
        for _ in range(reps):
            ens.launch(eps2, GRAPH)
            best = min(best, ens.last_ms())
        total += best
    return total


def tune_ensemble(ens, waves, chunks=ENS_CHUNKS, buckets=ENS_BUCKETS, verbose=False):
    """Launch shape and per-size chunk table for an Ensemble whose clusters
    are uploaded, timed on `waves` [(clusters, targets)].  Installs the winner
    and returns {"shape", "chunks", "ms", "default_ms", "trials"}."""
    default_shape = ens.shape()
    ens.set_tuning(None, ())
    default_ms = _ensemble_ms(ens, waves)
    trials = []
    shapes = [sh for sh in variants() if sh["mode"] == 2 and sh["threads"] * sh["ipt"] >= 128]
    best_shape, best_ms = default_shape, default_ms
    for sh in shapes:
        try:
            ens.set_tuning(sh, ())
            ms = _ensemble_ms(ens, waves)
        except _lib.AbyssError:
            continue
        trials.append(("shape", sh, ms))
        if verbose:
            print("shape", sh, round(ms, 3))
        if ms < best_ms:
            best_shape, best_ms = sh, ms
    # chunk length per cluster-size bucket, one bucket at a time
    table = [[b, 2048] for b in buckets]
    for q in range(len(table)):
        keep = table[q][1]
        for cj in chunks:
            table[q][1] = cj
            ens.set_tuning(best_shape, [tuple(e) for e in table])
            ms = _ensemble_ms(ens, waves)
            trials.append(("chunk", (table[q][0], cj), ms))
            if verbose:
                print("chunk", table[q][0], cj, round(ms, 3))
            if ms < best_ms:
                best_ms, keep = ms, cj
        table[q][1] = keep
    chunks_out = [tuple(e) for e in table]
    ens.set_tuning(best_shape, chunks_out)
    return {"shape": {k: best_shape[k] for k in ("kernel", "mode", "threads", "ipt", "unroll", "min_blocks")},
            "chunks": chunks_out, "ms": best_ms, "default_ms": default_ms, "trials": len(trials)}


def install(rf: RegularForce, table):
    entries = []
    for i, (m, sh, _) in enumerate(table):
        m_max = 2 ** 31 - 1 if i == len(table) - 1 else int(m)
        entries.append((m_max, sh))
    rf.set_tuning_table(entries)


def save(table, path):
    with open(path, "w") as f:
        json.dump([{"m": m, "shape": sh, "ms": ms} for m, sh, ms in table], f, indent=1)


def load(path):
    with open(path) as f:
        return [(d["m"], d["shape"], d["ms"]) for d in json.load(f)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--out", default="tuning.json")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    from . import workloads

    c = workloads.kernel_sweep(args.n)
    rf = RegularForce(0)
    z = np.zeros((c.n, 3))
    rf.upload_state(c.x, c.v, z, z, np.zeros(c.n), c.m, c.r2nb)
    rf.predict(0.0, 1.0)
    table = tune(rf, c.n, verbose=args.verbose)
    save(table, args.out)
    for m, sh, ms in table:
        print(m, sh, f"{ms:.3f} ms", f"{m * c.n / ms / 1e6:.1f} Gpairs/s")


if __name__ == "__main__":
    main()
