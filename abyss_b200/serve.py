"""Serving loop: many cluster integrations on one GPU with continuous batching.

A request asks for one cluster (Plummer, or King of a given W0; N particles;
Kroupa IMF) to be integrated with the Ahmad-Cohen scheme to code time 1.
The server keeps every admitted cluster's state resident in one ensemble arena
on the GPU and runs rounds:

  1. admit   waiting requests while the arena has a free slot and a contiguous
             particle range for them (admission by device-memory footprint;
             a request that does not fit waits, the loop never allocates);
  2. begin   every active integration runs its irregular levels up to its next
             regular block (host threads, in parallel);
  3. wave    the regular forces of all open blocks -- each cluster at its own
             time, with its own active set -- run as ONE replayed CUDA graph
             (prediction, one persistent force launch, finalize);
  4. end     every integration applies its corrector (host threads);
  5. retire  finished integrations report energy drift, free their range.

Requests arriving while others are on the GPU join the next round: their work
shares the device with the ones already running (continuous batching).  A
cluster's regular forces do not depend on what else is in a wave (its j-chunking
depends on its own size only), so its integration is the same alone and in any
mix, bit for bit.
"""
from __future__ import annotations

import argparse
import json
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .ensemble import GRAPH, Ensemble
from .integrator import ACIntegrator
from .regforce import RegularForce


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the server started
    model: str              # "plummer" or "king3", "king6", "king9"
    n: int
    seed: int
    t_end: float = 1.0
    k_nb: int = 24
    # runtime
    slot: int = -1
    ac: ACIntegrator | None = None
    admitted: float = -1.0
    finished: float = -1.0
    e0: float = 0.0
    e1: float = 0.0
    blocks: int = 0
    pending: tuple | None = None   # open block: (targets, new_time, time_scale)
    result: dict = field(default_factory=dict)

    def make_cluster(self):
        if self.model == "plummer":
            return ic.plummer(self.n, self.seed, masses="kroupa", k_nb=self.k_nb)
        return ic.king(self.n, self.seed, float(self.model[4:]), masses="kroupa", k_nb=self.k_nb)


class Server:
    def __init__(self, device: int = 0, capacity: int = 1 << 21, max_clusters: int = 512, list_cap: int = 128,
                 eps2: float = 1e-8, eta_reg: float = 0.02, eta_irr: float = 0.01, host_threads: int = 16):
        self.rf = RegularForce(device)
        self.ens = Ensemble(self.rf, None, list_cap=list_cap, capacity=capacity, max_clusters=max_clusters)
        self.eps2 = eps2
        self.eta_reg, self.eta_irr = eta_reg, eta_irr
        self.list_cap = list_cap
        self.pool = ThreadPoolExecutor(max_workers=max(1, host_threads))
        self.waiting: list[Request] = []
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.t0 = time.perf_counter()
        self.rounds = 0
        self.wave_ms = 0.0
        self.peak_active = 0

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def close(self):
        self.pool.shutdown()
        for r in self.active:
            r.ac.close()
        self.ens.close()
        self.rf.close()

    # ------------------------------------------------------------ admission
    def submit(self, req: Request):
        self.waiting.append(req)

    def _admit(self):
        still = []
        for r in self.waiting:
            if r.arrival > self.now():
                still.append(r)
                continue
            slot = self.ens.attach(r.n)
            if slot is None:
                still.append(r)  # not enough device room yet: wait for a retirement
                continue
            c = r.make_cluster()
            r.slot = slot
            r.ac = ACIntegrator(self.rf, c.x, c.v, c.m, c.r2nb, eps2=self.eps2, eta_reg=self.eta_reg,
                                eta_irr=self.eta_irr, fix_nb=r.k_nb, nb_max=self.list_cap, t_end=r.t_end,
                                threads=1)
            r.e0 = r.ac.energy()
            r.admitted = self.now()
            self.active.append(r)
        self.waiting = still

    # ------------------------------------------------------------ one round
    def round(self):
        self._admit()
        self.peak_active = max(self.peak_active, len(self.active))
        if not self.active:
            return
        # begin: irregular levels up to each integration's next regular block
        need = [r for r in self.active if r.pending is None]
        for r, res in zip(need, self.pool.map(lambda q: q.ac.begin_block(), need)):
            r.pending = res
        finished = [r for r in self.active if r.pending is None]
        live = [r for r in self.active if r.pending is not None]
        if live:
            states = list(self.pool.map(lambda q: q.ac.block_state(), live))
            for r, st in zip(live, states):
                self.ens.upload_state(r.slot, st["x"], st["v"], st["a0"], st["a1"], st["t0"], st["mass"], st["r2nb"])
            self.ens.set_wave([r.slot for r in live], [r.pending[1] for r in live], [r.pending[2] for r in live],
                              [r.pending[0] for r in live])
            self.ens.launch(self.eps2, GRAPH)
            out = self.ens.fetch()
            self.wave_ms += self.ens.last_ms()
            sp = self.ens.row_splits

            def end(i):
                r = live[i]
                a, b = sp[i], sp[i + 1]
                return r.ac.end_block(out.acc_reg[a:b], out.jerk_reg[a:b], out.acc_irr[a:b], out.jerk_irr[a:b],
                                      out.nnb[a:b], out.list[a:b])

            for i, status in enumerate(self.pool.map(end, range(len(live)))):
                r = live[i]
                if status == "redo":
                    continue  # radii shrunk; the block is recomputed next round
                r.pending = None
                r.blocks += 1
                if status == "done":
                    finished.append(r)
        for r in finished:
            self._retire(r)
        self.rounds += 1

    def _retire(self, r: Request):
        r.e1 = r.ac.energy()
        r.finished = self.now()
        r.result = dict(rid=r.rid, n=r.n, model=r.model, dE_over_E=abs((r.e1 - r.e0) / r.e0), blocks=r.blocks,
                        latency_s=r.finished - r.arrival, queue_s=r.admitted - r.arrival)
        st = r.ac.state()
        r.result["x_final"] = st["x"]
        r.ac.close()
        r.ac = None
        self.ens.detach(r.slot)
        self.active.remove(r)
        self.done.append(r)

    def run_until_idle(self, max_seconds: float = 1e9):
        while (self.waiting or self.active) and self.now() < max_seconds:
            if not self.active and self.waiting and all(r.arrival > self.now() for r in self.waiting):
                time.sleep(max(0.0, min(r.arrival for r in self.waiting) - self.now()))
            self.round()


def poisson_requests(rate: float, duration: float, nmin: int, nmax: int, seed: int = 5, t_end: float = 1.0,
                     k_nb: int = 24):
    """Seeded Poisson stream: model uniform over Plummer, King W0 in {3, 6, 9}; N log-uniform."""
    rng = np.random.default_rng(seed)
    t, rid, out = 0.0, 0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        model = ["plummer", "king3", "king6", "king9"][rng.integers(0, 4)]
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        out.append(Request(rid, t, model, n, int(rng.integers(1, 1 << 30)), t_end=t_end, k_nb=k_nb))
        rid += 1
    return out


def serve(rate: float = 200.0, duration: float = 2.0, nmin: int = 256, nmax: int = 2048, t_end: float = 0.0625,
          capacity: int = 1 << 21, seed: int = 5, host_threads: int = 16, serial: bool = False):
    """Run a Poisson stream through the server (or, with serial=True, one request at
    a time through the same code) and report latency percentiles and throughput."""
    reqs = poisson_requests(rate, duration, nmin, nmax, seed=seed, t_end=t_end)
    if serial:
        done = serve_serial(reqs, host_threads)
        rounds, wave_ms, peak = 0, 0.0, 1
        srv = None
    else:
        srv = Server(capacity=capacity, host_threads=host_threads)
        for r in reqs:
            srv.submit(r)
        srv.run_until_idle()
        done, rounds, wave_ms, peak = srv.done, srv.rounds, srv.wave_ms, srv.peak_active
        srv.close()
    wall = max(r.finished for r in done) if done else 0.0
    lat = np.array([r.result["latency_s"] for r in done])
    de = np.array([r.result["dE_over_E"] for r in done])
    res = dict(requests=len(reqs), completed=len(done), wall_s=wall,
               clusters_per_s=len(done) / wall if wall > 0 else None,
               p50_latency_s=float(np.percentile(lat, 50)) if len(lat) else None,
               p99_latency_s=float(np.percentile(lat, 99)) if len(lat) else None,
               max_dE_over_E=float(de.max()) if len(de) else None,
               median_dE_over_E=float(np.median(de)) if len(de) else None,
               rounds=rounds, gpu_wave_ms=wave_ms, peak_active=peak,
               config=dict(rate=rate, duration=duration, nmin=nmin, nmax=nmax, t_end=t_end, capacity=capacity,
                           seed=seed, serial=serial))
    return res, done


def serve_serial(reqs, host_threads: int = 16):
    """The plain baseline: the same stream, one integration at a time in arrival
    order, each through the single-cluster regular-force path (one launch per
    regular block, host threads inside the integration)."""
    rf = RegularForce(0)
    t0 = time.perf_counter()
    done = []
    for r in sorted(reqs, key=lambda q: q.arrival):
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        r.admitted = time.perf_counter() - t0
        c = r.make_cluster()
        ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=1e-8, eta_reg=0.02, eta_irr=0.01, fix_nb=r.k_nb,
                          nb_max=128, t_end=r.t_end, threads=host_threads)
        r.e0 = ac.energy()
        ac.run(1.0)
        r.e1 = ac.energy()
        r.finished = time.perf_counter() - t0
        r.result = dict(rid=r.rid, n=r.n, model=r.model, dE_over_E=abs((r.e1 - r.e0) / r.e0),
                        latency_s=r.finished - r.arrival, queue_s=r.admitted - r.arrival, x_final=ac.state()["x"])
        ac.close()
        done.append(r)
    rf.close()
    return done


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=2.0)
    ap.add_argument("--nmin", type=int, default=256)
    ap.add_argument("--nmax", type=int, default=2048)
    ap.add_argument("--t-end", type=float, default=0.0625)
    ap.add_argument("--capacity", type=int, default=1 << 21)
    ap.add_argument("--threads", type=int, default=16)
    args = ap.parse_args()
    out = {}
    for serial in (False, True):
        res, _ = serve(args.rate, args.duration, args.nmin, args.nmax, args.t_end, args.capacity,
                       host_threads=args.threads, serial=serial)
        out["serial_plain" if serial else "continuous"] = res
    out["speedup"] = out["continuous"]["clusters_per_s"] / out["serial_plain"]["clusters_per_s"]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
