"""Batched-ensemble throughput (the many-cluster configuration).

Regular blocks of K clusters of uneven N with uneven active sets, run as
  graph    one captured CUDA graph per wave (predict, one persistent force
           launch over the whole work list, finalize)
  batched  the same three launches without the graph
  plain    the same kernels, one cluster per launch
on the same GPU, same inputs.  Reported: cluster blocks per second (a cluster
block is one regular-force evaluation of one cluster's active set), pairs per
second and the ratio of each form to plain; with ``tune``, the graph form again
with the shape and chunk table that autotune.tune_ensemble picks on these waves.

    python -m abyss_b200.bench_ensemble [--clusters 512] [--waves 6]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads
from .ensemble import BATCHED, GRAPH, PLAIN, Ensemble
from .regforce import RegularForce

EPS2 = 1e-8
LIST_CAP = 128


def measure(rf: RegularForce, clusters, waves, warmup: int = 1, tune: bool = False):
    sizes = [c.n for c in clusters]
    ens = Ensemble(rf, sizes, list_cap=LIST_CAP)
    for i, c in enumerate(clusters):
        a = np.zeros((c.n, 3))
        ens.upload_state(i, c.x, c.v, a, a, np.zeros(c.n), c.m, c.r2nb)
    out = {"clusters": len(clusters), "particles": int(sum(sizes)), "waves": len(waves),
           "device_bytes": ens.device_bytes}
    blocks = sum(len(w[0]) for w in waves)
    pairs = float(sum(len(t) * clusters[k].n for (ks, ts) in waves for k, t in zip(ks, ts)))
    out["cluster_blocks"] = blocks
    out["pairs"] = pairs
    for name, mode in (("graph", GRAPH), ("batched", BATCHED), ("plain", PLAIN)):
        gpu_ms = 0.0
        wall = 0.0
        launches = 0
        for wi, (ks, ts) in enumerate(waves):
            ens.set_wave(ks, np.zeros(len(ks)), np.ones(len(ks)), ts)
            for _ in range(warmup if wi == 0 else 0):
                ens.launch(EPS2, mode)
                ens.fetch()
            t0 = time.perf_counter()
            ens.launch(EPS2, mode)
            ens.fetch()
            wall += time.perf_counter() - t0
            gpu_ms += ens.last_ms()
            launches += ens.last_stats()["launches"]
        out[name] = {"gpu_ms": gpu_ms, "wall_s": wall, "cluster_blocks_per_s": blocks / (gpu_ms / 1e3),
                     "gpairs_s": pairs / (gpu_ms / 1e3) / 1e9, "kernel_launches": launches}
    out["graph_vs_plain"] = out["graph"]["cluster_blocks_per_s"] / out["plain"]["cluster_blocks_per_s"]
    out["batched_vs_plain"] = out["batched"]["cluster_blocks_per_s"] / out["plain"]["cluster_blocks_per_s"]
    if tune:
        # the autotuner's shape and chunk table, picked on these waves (its own
        # timing runs are not counted), then the graph form measured again
        from . import autotune

        t0 = time.perf_counter()
        res = autotune.tune_ensemble(ens, waves)
        out["tuning"] = {"shape": res["shape"], "chunks": res["chunks"], "trials": res["trials"],
                         "tuning_s": time.perf_counter() - t0}
        gpu_ms = 0.0
        for wi, (ks, ts) in enumerate(waves):
            ens.set_wave(ks, np.zeros(len(ks)), np.ones(len(ks)), ts)
            for _ in range(warmup if wi == 0 else 0):
                ens.launch(EPS2, GRAPH)
                ens.fetch()
            ens.launch(EPS2, GRAPH)
            ens.fetch()
            gpu_ms += ens.last_ms()
        out["graph_tuned"] = {"gpu_ms": gpu_ms, "cluster_blocks_per_s": blocks / (gpu_ms / 1e3),
                              "gpairs_s": pairs / (gpu_ms / 1e3) / 1e9}
        out["graph_tuned_vs_plain"] = out["graph_tuned"]["cluster_blocks_per_s"] / out["plain"]["cluster_blocks_per_s"]
    ens.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=512)
    ap.add_argument("--waves", type=int, default=6)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--tune", action="store_true")
    args = ap.parse_args()
    clusters = workloads.ensemble(k=args.clusters)
    waves = workloads.ensemble_waves(clusters, args.waves)
    rf = RegularForce(args.device)
    res = measure(rf, clusters, waves, tune=args.tune)
    print(json.dumps(res))
    rf.close()


if __name__ == "__main__":
    main()
