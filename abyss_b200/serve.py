"""Serving loop: many cluster integrations on one GPU with continuous batching.

A request carries one cluster (Plummer, or King of a given W0; N particles;
Kroupa IMF) to be integrated with the Ahmad-Cohen scheme to code time 1.
The server keeps every admitted cluster's state resident in one ensemble arena
on the GPU and runs rounds:

  1. admit   waiting requests while the arena has a free slot and a contiguous
             particle range for them (admission by device-memory footprint;
             a request that does not fit waits, the loop never allocates);
             their initial conditions and integrator set-up run on host
             threads, each through a regular-force context of its own;
  2. run     for a slice of wall time the admitted integrations advance on
             their own: host workers run each one's irregular levels up to its
             next regular block and queue the block, the GPU runs every queued
             block -- each cluster at its own time, with its own active set --
             as back-to-back waves of ONE replayed CUDA graph (prediction, one
             persistent force launch, finalize), and a worker applies the
             corrector as soon as a block's rows are back and opens the next
             block (one native call, abyss_ac_serve_run);
  3. retire  finished integrations report energy drift (host threads) and free
             their range.

Requests arriving while others are on the GPU join the next round: their work
shares the device with the ones already running (continuous batching).  A
cluster's regular forces do not depend on what else is in a wave (its j-chunking
depends on its own size only), so its integration is the same alone and in any
mix, bit for bit.
"""
from __future__ import annotations

import argparse
import json
import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

import ctypes as C

from . import _lib, ic
from ._lib import AbyssError, _ip, ptr
from .ensemble import GRAPH, Ensemble
from .integrator import ACIntegrator
from .regforce import RegularForce


ROUND_ADVANCED, ROUND_ADVANCED_DONE, ROUND_FINISHED, ROUND_REDO = 0, 1, 2, 3  # include/abyss_ac.h


class ServeStats(C.Structure):
    _fields_ = [("wall_s", C.c_double), ("prep_s", C.c_double), ("wait_s", C.c_double), ("hand_s", C.c_double),
                ("idle_s", C.c_double), ("worker_s", C.c_double), ("rows", C.c_longlong)]


def _bind(L):
    if getattr(L, "_serve_bound", False):
        return
    L.abyss_ac_serve_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), _ip, C.c_double, C.c_int,
                                     C.c_int, C.c_double, C.c_int, _ip, _ip, C.POINTER(C.c_float),
                                     C.POINTER(C.c_int), C.POINTER(ServeStats)]
    L._serve_bound = True


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
    cluster: object = None         # the payload: initial conditions (built on admission if None)
    state: dict | None = None      # its un-predicted state, to upload
    ctx_lock: object = None        # lock of the context the integrator was set up on
    result: dict = field(default_factory=dict)

    def make_cluster(self):
        if self.cluster is not None:
            return self.cluster
        if self.model == "plummer":
            return ic.plummer(self.n, self.seed, masses="kroupa", k_nb=self.k_nb)
        return ic.king(self.n, self.seed, float(self.model[4:]), masses="kroupa", k_nb=self.k_nb)


class Server:
    def __init__(self, device: int = 0, capacity: int = 1 << 21, max_clusters: int = 512, list_cap: int = 128,
                 eps2: float = 1e-8, eta_reg: float = 0.02, eta_irr: float = 0.01, host_threads: int = 16,
                 slice_ms: float = 20.0, max_n: int = 16384, chunk_j: int = 256, device_irregular_min_n: int = 0,
                 team_min_n: int = 16384, lane_min_n: int = 0, lane_threads: int = 2, lane_team: int = 4,
                 device_blocks_min_n: int = 0, lane_wait_us: int = -1, lane_order: str = "arrival"):
        """device_irregular_min_n > 0: integrations of at least that many
        particles run their irregular levels on the GPU (include/abyss_irr.h)
        instead of on their worker thread; the results are the same.
        team_min_n: integrations of at least that many particles get a team of
        1 + n / team_min_n host threads (at most host_threads) for their host
        work; smaller ones run on their worker thread alone.
        lane_min_n > 0: requests of at least that many particles skip the waves:
        one of their regular blocks fills the GPU alone, so batching gains them
        nothing and its round trips would set their latency.  Each runs whole on
        one of lane_threads host threads, through a context of its own, with a
        team of lane_team threads and (above device_irregular_min_n) its
        irregular levels on the GPU.
        device_blocks_min_n > 0: a lane's request of at least that many
        particles runs with whole blocks on the GPU and its state kept there
        (abyss_ac_set_device_resident): the host only waits, so many lanes can
        share the GPU; the results are the same.
        lane_wait_us >= 0: a lane thread waiting for the GPU polls that long,
        then sleeps (include/abyss_reg.h abyss_set_wait), leaving its core to
        the other lanes; < 0: it spins.
        lane_order: which waiting lane request starts when a lane frees up --
        "arrival" (first come, first served) or "largest" (the most particles
        first: for a batch that arrives at once, the long integrations do not
        end up last and alone)."""
        self.rf = RegularForce(device)
        self.ens = Ensemble(self.rf, None, list_cap=list_cap, capacity=capacity, max_clusters=max_clusters)
        # short j-chunks: a serving wave is small and latency-bound, so its work
        # is spread over as many CTAs as possible
        self.ens.set_chunk(chunk_j)
        self.eps2 = eps2
        self.eta_reg, self.eta_irr = eta_reg, eta_irr
        self.device_irregular_min_n = int(device_irregular_min_n)
        self.device_blocks_min_n = int(device_blocks_min_n)
        self.team_min_n = max(1, int(team_min_n))
        self.lane_min_n = int(lane_min_n)
        self.lane_team = max(1, int(lane_team))
        self.lane_jobs: list = []  # (request, future) of large requests run whole
        self.lane_queue: list = []  # lane requests waiting for a lane
        self.lane_threads = max(1, lane_threads)
        if lane_order not in ("arrival", "largest"):
            raise ValueError("lane_order must be 'arrival' or 'largest'")
        self.lane_order = lane_order
        self.lane_pool = ThreadPoolExecutor(max_workers=max(1, lane_threads)) if self.lane_min_n > 0 else None
        self.lane_ctx: queue.Queue = queue.Queue()
        if self.lane_min_n > 0:
            for _ in range(max(1, lane_threads)):
                rf = RegularForce(device)
                if lane_wait_us >= 0:
                    rf.set_wait(int(lane_wait_us))
                self.lane_ctx.put(rf)
        self.list_cap = list_cap
        nthreads = max(1, host_threads)
        self.host_threads = nthreads
        self._L = _lib.lib()
        _bind(self._L)
        self.pool = ThreadPoolExecutor(max_workers=nthreads)
        # Integrator set-up (its initial force on the GPU) and energies run on
        # host threads, each through a context of its own: a context serves one
        # caller at a time, which its lock enforces.
        self.ctx_free: queue.Queue = queue.Queue()
        self.ctxs = [(RegularForce(device), threading.Lock()) for _ in range(nthreads)]
        # every buffer a set-up of up to max_n particles uses, allocated now: a
        # context that grew while waves run would stall the device in cudaFree
        for rf, _ in self.ctxs:
            rf.reserve(max_n, max_n, list_cap)
            # a set-up waits behind the waves on the GPU: it sleeps meanwhile,
            # leaving its core to the workers instead of spinning on it
            rf.set_wait(50)
        for c in self.ctxs:
            self.ctx_free.put(c)
        self.waiting: list[Request] = []
        self.building: list = []  # (request, future of its set-up)
        self.retiring: list = []  # (request, future of its final energy and state)
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.t0 = time.perf_counter()
        self.rounds = 0
        self.wave_ms = 0.0
        self.waves = 0
        self._st = ServeStats()
        self.run_stats = {f: 0 for f, _ in ServeStats._fields_}
        self.slice_ms = float(slice_ms)
        self.peak_active = 0
        self.phase_s = dict(admit=0.0, round=0.0, retire=0.0)
        self.build_s = dict(cluster=0.0, wait_ctx=0.0, init=0.0, energy=0.0)
        self.stat_lock = threading.Lock()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def close(self):
        self._reap(wait=True)
        self.pool.shutdown()
        if self.lane_pool is not None:
            self.lane_pool.shutdown()
            while not self.lane_ctx.empty():
                self.lane_ctx.get().close()
        for r, _ in self.building:
            if r.ac is not None:
                r.ac.close()
        for r in self.active:
            r.ac.close()
        self.ens.close()
        for rf, _ in self.ctxs:
            rf.close()
        self.rf.close()

    # ------------------------------------------------------------ admission
    def submit(self, req: Request):
        self.waiting.append(req)

    def _build(self, r: Request):
        """Initial conditions, integrator set-up and initial energy of one request."""
        t0 = time.perf_counter()
        c = r.make_cluster()
        t1 = time.perf_counter()
        ctx = self.ctx_free.get()
        try:
            rf, lock = ctx
            with lock:
                t2 = time.perf_counter()
                # one host thread per integration, except for large clusters,
                # whose per-block host work (j-set fill, corrector) would set
                # the stream's tail on one thread
                threads = 1 if r.n < self.team_min_n else min(self.host_threads, r.n // self.team_min_n + 1)
                r.ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=self.eps2, eta_reg=self.eta_reg,
                                    eta_irr=self.eta_irr, fix_nb=r.k_nb, nb_max=self.list_cap, t_end=r.t_end,
                                    threads=threads)
                if self.device_irregular_min_n > 0 and r.n >= self.device_irregular_min_n:
                    r.ac.set_device_irregular(True)
                t3 = time.perf_counter()
                r.e0 = r.ac.energy()
                t4 = time.perf_counter()
            r.ctx_lock = lock
            r.cluster = None
        finally:
            self.ctx_free.put(ctx)
        with self.stat_lock:  # thread-seconds spent per part of the set-up
            self.build_s["cluster"] += t1 - t0
            self.build_s["wait_ctx"] += t2 - t1
            self.build_s["init"] += t3 - t2
            self.build_s["energy"] += t4 - t3

    def _admit(self):
        """Requests that have arrived get an arena slot (main thread, between
        runs: the ensemble is not in use then) and their set-up is started on
        the host pool; set-ups that have finished join the active set.  Set-ups
        run while the integrations already admitted are being served."""
        still = []
        for r in self.waiting:
            if r.arrival > self.now():
                still.append(r)
                continue
            if self.lane_min_n > 0 and r.n >= self.lane_min_n:
                r.admitted = self.now()
                self.lane_queue.append(r)
                continue
            slot = self.ens.attach(r.n)
            if slot is None:
                still.append(r)  # not enough device room yet: wait for a retirement
                continue
            r.slot = slot
            self.building.append((r, self.pool.submit(self._build, r)))
        self.waiting = still
        self._pump_lanes()
        pending = []
        for r, fut in self.building:
            if fut.done():
                fut.result()  # re-raises a failed set-up
                r.admitted = self.now()
                self.active.append(r)
            else:
                pending.append((r, fut))
        self.building = pending
        if not self.active and self.building:  # nothing to serve meanwhile: wait for one set-up
            r, fut = self.building.pop(0)
            fut.result()
            r.admitted = self.now()
            self.active.append(r)

    # ------------------------------------------------------------ one round
    def round(self):
        ph = self.phase_s
        t = time.perf_counter()
        self._admit()
        ph["admit"] += time.perf_counter() - t
        self.peak_active = max(self.peak_active, len(self.active))
        if not self.active:
            return
        # the integrations advance asynchronously for a slice of wall time: host
        # workers run irregular levels and correctors, the GPU runs every queued
        # regular block in back-to-back waves (include/abyss_ac.h abyss_ac_serve_run)
        t = time.perf_counter()
        k = len(self.active)
        acs = (C.c_void_p * k)(*[r.ac._h.value for r in self.active])
        slots = np.array([r.slot for r in self.active], np.int32)
        status = np.zeros(k, np.int32)
        blocks = np.zeros(k, np.int32)
        ms = C.c_float(0.0)
        nw = C.c_int(0)
        rc = self._L.abyss_ac_serve_run(self.ens._h, k, acs, ptr(slots, _ip), self.eps2, GRAPH, self.host_threads,
                                        self.slice_ms, 0, ptr(status, _ip), ptr(blocks, _ip), C.byref(ms),
                                        C.byref(nw), C.byref(self._st))
        for f, _ in ServeStats._fields_:
            self.run_stats[f] += getattr(self._st, f)
        if rc != 0:
            raise AbyssError(rc, "serve run failed")
        self.wave_ms += float(ms.value)
        self.waves += int(nw.value)
        ph["round"] += time.perf_counter() - t
        finished = []
        for r, st, nb in zip(self.active, status, blocks):
            if st < 0:
                raise AbyssError(int(st), f"request {r.rid}: " + r.ac.last_error())
            r.blocks += int(nb)
            if st in (ROUND_ADVANCED_DONE, ROUND_FINISHED):
                finished.append(r)
        t = time.perf_counter()
        # a finished integration no longer touches the ensemble: its range is
        # freed now, its final energy and state are taken on the host pool
        for r in finished:
            self.ens.detach(r.slot)
            self.active.remove(r)
            self.retiring.append((r, self.pool.submit(self._finish, r)))
        self._reap()
        ph["retire"] += time.perf_counter() - t
        self.rounds += 1

    def _run_lane(self, r: Request):
        """A large request run whole, outside the waves (the plain single-cluster
        path on a context of this lane)."""
        c = r.make_cluster()
        rf = self.lane_ctx.get()
        try:
            ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=self.eps2, eta_reg=self.eta_reg,
                              eta_irr=self.eta_irr, fix_nb=r.k_nb, nb_max=self.list_cap, t_end=r.t_end,
                              threads=self.lane_team)
            on_device = self.device_blocks_min_n > 0 and r.n >= self.device_blocks_min_n
            if on_device:
                ac.set_device_resident(True)
            elif self.device_irregular_min_n > 0 and r.n >= self.device_irregular_min_n:
                ac.set_device_irregular(True)
            r.e0 = ac.energy()
            ac.run(1.0)
            r.e1 = ac.energy()
            r.blocks = int(ac.stats()["blocks"])
            r.finished = self.now()
            r.result = dict(rid=r.rid, n=r.n, model=r.model, dE_over_E=abs((r.e1 - r.e0) / r.e0), blocks=r.blocks,
                            latency_s=r.finished - r.arrival, queue_s=r.admitted - r.arrival,
                            device_irregular=on_device or ac.device_irregular_info()["on"], lane=True,
                            device_blocks=on_device,
                            x_final=ac.state()["x"])
            ac.close()
        finally:
            self.lane_ctx.put(rf)
        r.cluster = None

    def _pump_lanes(self):
        """Start waiting lane requests while a lane is free, in lane_order."""
        while self.lane_queue and len(self.lane_jobs) < self.lane_threads:
            if self.lane_order == "largest":
                k = max(range(len(self.lane_queue)), key=lambda q: (self.lane_queue[q].n, -q))
            else:
                k = 0
            r = self.lane_queue.pop(k)
            self.lane_jobs.append((r, self.lane_pool.submit(self._run_lane, r)))

    def _reap_lane(self, wait: bool = False):
        while True:
            still = []
            for r, fut in self.lane_jobs:
                if wait or fut.done():
                    fut.result()
                    self.done.append(r)
                else:
                    still.append((r, fut))
            self.lane_jobs = still
            self._pump_lanes()
            if not (wait and (self.lane_jobs or self.lane_queue)):
                return

    def _reap(self, wait: bool = False):
        still = []
        for r, fut in self.retiring:
            if wait or fut.done():
                fut.result()
                self.done.append(r)
            else:
                still.append((r, fut))
        self.retiring = still

    def _finish(self, r: Request):
        """Final energy and positions of a finished integration; frees it."""
        with r.ctx_lock:
            r.e1 = r.ac.energy()
        r.finished = self.now()
        r.result = dict(rid=r.rid, n=r.n, model=r.model, dE_over_E=abs((r.e1 - r.e0) / r.e0), blocks=r.blocks,
                        latency_s=r.finished - r.arrival, queue_s=r.admitted - r.arrival,
                        device_irregular=r.ac.device_irregular_info()["on"])
        r.result["x_final"] = r.ac.state()["x"]
        r.ac.close()
        r.ac = None

    def run_until_idle(self, max_seconds: float = 1e9):
        while (self.waiting or self.building or self.active or self.lane_jobs or self.lane_queue) and \
                self.now() < max_seconds:
            self._reap_lane()
            if not self.active and not self.building and self.waiting and \
                    all(r.arrival > self.now() for r in self.waiting):
                time.sleep(max(0.0, min(0.05, min(r.arrival for r in self.waiting) - self.now())))
            if not self.active and not self.building and not self.waiting and (self.lane_jobs or self.lane_queue):
                time.sleep(0.01)  # only large requests left: they run on their own threads
            self.round()
        self._reap(wait=True)
        self._reap_lane(wait=True)


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
          capacity: int = 1 << 21, seed: int = 5, host_threads: int = 16, serial: bool = False,
          chunk_j: int = 256, slice_ms: float = 20.0, device_irregular_min_n: int = 0, reqs=None,
          lane_min_n: int = 0, lane_threads: int = 2, device_blocks_min_n: int = 0, lane_wait_us: int = -1,
          lane_order: str = "arrival"):
    """Run a Poisson stream through the server (or, with serial=True, one request at
    a time through the same code) and report latency percentiles and throughput.
    `reqs` replaces the generated stream (requests with prebuilt clusters)."""
    if reqs is None:
        reqs = poisson_requests(rate, duration, nmin, nmax, seed=seed, t_end=t_end)
    # a request arrives with its particles: build the payloads before the clock starts
    for r in reqs:
        r.cluster = r.make_cluster()
    if serial:
        done, phases = serve_serial(reqs, host_threads)
        rounds, wave_ms, peak = 0, 0.0, 1
        srv = None
    else:
        srv = Server(capacity=capacity, host_threads=host_threads, max_n=max(nmax, max(r.n for r in reqs)),
                     chunk_j=chunk_j, slice_ms=slice_ms, device_irregular_min_n=device_irregular_min_n,
                     lane_min_n=lane_min_n, lane_threads=lane_threads, device_blocks_min_n=device_blocks_min_n,
                     lane_wait_us=lane_wait_us, lane_order=lane_order)
        for r in reqs:
            srv.submit(r)
        srv.run_until_idle()
        done, rounds, wave_ms, peak = srv.done, srv.rounds, srv.wave_ms, srv.peak_active
        phases = dict(srv.phase_s, build_thread_s=dict(srv.build_s), waves=srv.waves, run=dict(srv.run_stats))
        srv.close()
    wall = max(r.finished for r in done) if done else 0.0
    lat = np.array([r.result["latency_s"] for r in done])
    de = np.array([r.result["dE_over_E"] for r in done])
    blocks = int(sum(r.blocks for r in done))
    res = dict(requests=len(reqs), completed=len(done), wall_s=wall, cluster_blocks=blocks,
               cluster_blocks_per_s=blocks / wall if wall > 0 else None,
               frac_dE_below_1e6=float(np.mean(de <= 1e-6)) if len(de) else None,
               device_irregular_requests=int(sum(bool(r.result.get("device_irregular")) for r in done)),
               device_blocks_requests=int(sum(bool(r.result.get("device_blocks")) for r in done)),
               clusters_per_s=len(done) / wall if wall > 0 else None,
               p50_latency_s=float(np.percentile(lat, 50)) if len(lat) else None,
               p99_latency_s=float(np.percentile(lat, 99)) if len(lat) else None,
               max_dE_over_E=float(de.max()) if len(de) else None,
               median_dE_over_E=float(np.median(de)) if len(de) else None,
               rounds=rounds, gpu_wave_ms=wave_ms, peak_active=peak, phase_s=phases,
               config=dict(rate=rate, duration=duration, nmin=nmin, nmax=nmax, t_end=t_end, capacity=capacity,
                           seed=seed, serial=serial, device_irregular_min_n=device_irregular_min_n,
                           lane_min_n=lane_min_n, lane_threads=lane_threads,
                           device_blocks_min_n=device_blocks_min_n, lane_wait_us=lane_wait_us,
                           lane_order=lane_order))
    return res, done


def serve_serial(reqs, host_threads: int = 16):
    """The plain baseline: the same stream, one integration at a time in arrival
    order, each through the single-cluster regular-force path (one launch per
    regular block, host threads inside the integration)."""
    rf = RegularForce(0)
    t0 = time.perf_counter()
    done = []
    phases = dict(cluster=0.0, init=0.0, run=0.0)
    for r in sorted(reqs, key=lambda q: q.arrival):
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        r.admitted = time.perf_counter() - t0
        t = time.perf_counter()
        c = r.make_cluster()
        phases["cluster"] += time.perf_counter() - t
        t = time.perf_counter()
        ac = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, eps2=1e-8, eta_reg=0.02, eta_irr=0.01, fix_nb=r.k_nb,
                          nb_max=128, t_end=r.t_end, threads=host_threads)
        r.e0 = ac.energy()
        phases["init"] += time.perf_counter() - t
        t = time.perf_counter()
        ac.run(1.0)
        phases["run"] += time.perf_counter() - t
        r.blocks = int(ac.stats()["blocks"])
        r.e1 = ac.energy()
        r.finished = time.perf_counter() - t0
        r.result = dict(rid=r.rid, n=r.n, model=r.model, dE_over_E=abs((r.e1 - r.e0) / r.e0),
                        latency_s=r.finished - r.arrival, queue_s=r.admitted - r.arrival, x_final=ac.state()["x"])
        ac.close()
        done.append(r)
    rf.close()
    return done, phases


def c4_requests(k: int = 512, t_end: float = 5.0):
    """The batched-ensemble configuration as one serving job: the k equal-mass
    Plummer clusters of workloads.ensemble (N log-uniform in [256, 16384],
    seed 4, cluster i seeded 4000 + i, 24 neighbours), all arriving at once,
    each integrated to t = t_end."""
    from . import workloads

    clusters = workloads.ensemble(k=k)
    return [Request(i, 0.0, "plummer", c.n, 4000 + i, t_end=t_end, k_nb=24, cluster=c)
            for i, c in enumerate(clusters)]


# Server options of the stated configurations (run_config).  Configuration 4
# runs every integration whole on a lane with its blocks on the GPU: sixteen at
# once, sharing the GPU, in arrival order (largest first measured 4 % slower:
# sixteen large integrations at once share the GPU worse than a mix of sizes).
# Configuration 5 sends integrations of 16 384 particles and more to four such
# lanes and serves the rest in waves.
CONFIG_LANES = {"c4": dict(lane_min_n=1, lane_threads=16, device_blocks_min_n=1, lane_order="arrival"),
                "c5": dict(lane_min_n=16384, lane_threads=4, device_blocks_min_n=1, lane_order="arrival")}


def run_config(name: str, duration: float = 1.0, sample: int = 16, device_irregular_min_n: int = 4096,
               host_threads: int = 16, capacity: int = 1 << 22, lane_min_n: int | None = None,
               lane_threads: int | None = None, device_blocks_min_n: int | None = None, lane_wait_us: int = -1,
               lane_order: str | None = None, k: int = 512):
    """A stated configuration through the continuous server, and the serial
    plain form on an evenly spaced sample of the same requests (the whole
    stream one at a time would take hours): its clusters/s is the sample's
    count over the sample's back-to-back run time.
      c4: the 512 ensemble clusters to t = 5, all arriving at once;
      c5: Poisson 200 requests/s for `duration` s (seed 5), Plummer or King W0
          3/6/9, Kroupa IMF, N log-uniform in [1024, 131072], to t = 1."""
    lanes = CONFIG_LANES[name]
    lane_min_n = lanes["lane_min_n"] if lane_min_n is None else lane_min_n
    lane_threads = lanes["lane_threads"] if lane_threads is None else lane_threads
    device_blocks_min_n = lanes["device_blocks_min_n"] if device_blocks_min_n is None else device_blocks_min_n
    lane_order = lanes["lane_order"] if lane_order is None else lane_order
    if name == "c4":
        reqs = c4_requests(k)
        nmax = 16384
    else:
        reqs = poisson_requests(200.0, duration, 1024, 131072, seed=5, t_end=1.0)
        nmax = 131072
    for r in reqs:
        r.cluster = r.make_cluster()
    res, done = serve(reqs=reqs, nmax=nmax, capacity=capacity, host_threads=host_threads,
                      device_irregular_min_n=device_irregular_min_n, lane_min_n=lane_min_n,
                      lane_threads=lane_threads, device_blocks_min_n=device_blocks_min_n, lane_wait_us=lane_wait_us,
                      lane_order=lane_order)
    res.pop("phase_s", None)
    res["config"] = dict(
        name=name, requests=len(reqs), device_irregular_min_n=device_irregular_min_n, host_threads=host_threads,
        capacity=capacity, lane_min_n=lane_min_n, lane_threads=lane_threads, device_blocks_min_n=device_blocks_min_n,
        lane_wait_us=lane_wait_us, lane_order=lane_order,
        workload=(f"{k} equal-mass Plummer clusters (the first {k} of the configuration's 512), N log-uniform in "
                  "[256, 16384] (seed 4, cluster k seeded 4000 + k), eps = 1e-4, all arriving at t = 0, each to t = 5"
                  if name == "c4" else
                  f"Poisson 200 requests/s for {duration} s (seed 5), Plummer or King W0 3/6/9, Kroupa IMF, "
                  "N log-uniform in [1024, 131072], eps = 1e-4, each to t = 1"))
    de = {r.rid: r.result["dE_over_E"] for r in done}
    res["dE_over_E_by_request"] = [de[k] for k in sorted(de)]
    # serial plain on a sample (fresh requests: the served ones hold their results)
    step = max(1, len(reqs) // max(1, sample))
    pick = [r.rid for r in reqs][::step][:sample]
    if name == "c4":
        fresh = {r.rid: r for r in c4_requests(k)}
    else:
        fresh = {r.rid: r for r in poisson_requests(200.0, duration, 1024, 131072, seed=5, t_end=1.0)}
    sub = [fresh[k] for k in pick]
    for r in sub:
        r.arrival = 0.0
        r.cluster = r.make_cluster()
    sdone, phases = serve_serial(sub, host_threads)
    run_s = phases["init"] + phases["run"]
    res["serial_plain_sample"] = dict(requests=len(sub), run_s=run_s, clusters_per_s=len(sub) / run_s,
                                      dE_over_E=[r.result["dE_over_E"] for r in sdone])
    res["vs_serial_plain"] = res["clusters_per_s"] / res["serial_plain_sample"]["clusters_per_s"]
    return res


def main():
    """Serving benchmark: a seeded Poisson stream through the continuous server and
    through serial plain integrations.  The defaults (2000 requests/s for 0.5 s,
    N log-uniform in [256, 2048], t_end = 1/16) arrive faster than either can
    serve them, so clusters/s measures throughput at saturation.  With
    --config c4 or c5, the stated configuration (run_config)."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["c4", "c5"], default=None)
    ap.add_argument("--sample", type=int, default=16)
    ap.add_argument("--device-irregular-min-n", type=int, default=4096)
    ap.add_argument("--lane-min-n", type=int, default=None,
                    help="requests of at least this many particles run whole outside the waves (0: none; "
                         "default: 0, or the stated configuration's)")
    ap.add_argument("--lane-threads", type=int, default=None, help="host threads (and contexts) of the lane")
    ap.add_argument("--device-blocks-min-n", type=int, default=None,
                    help="lane requests of at least this many particles run whole blocks on the GPU (0: none)")
    ap.add_argument("--lane-wait-us", type=int, default=-1,
                    help="a lane thread polls the GPU this long, then sleeps (< 0: spins)")
    ap.add_argument("--lane-order", choices=["arrival", "largest"], default=None,
                    help="which waiting lane request starts first (default: arrival, or the configuration's)")
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--duration", type=float, default=None,
                    help="stream length in s (default 0.5; 1 for the stated configuration 5)")
    ap.add_argument("--nmin", type=int, default=256)
    ap.add_argument("--nmax", type=int, default=2048)
    ap.add_argument("--t-end", type=float, default=0.0625)
    ap.add_argument("--capacity", type=int, default=1 << 21)
    ap.add_argument("--threads", type=int, default=16)
    args = ap.parse_args()
    if args.config:
        print(json.dumps(run_config(args.config, duration=1.0 if args.duration is None else args.duration,
                                    sample=args.sample,
                                    device_irregular_min_n=args.device_irregular_min_n, host_threads=args.threads,
                                    lane_min_n=args.lane_min_n, lane_threads=args.lane_threads,
                                    device_blocks_min_n=args.device_blocks_min_n, lane_wait_us=args.lane_wait_us,
                                    lane_order=args.lane_order)))
        return
    out = {}
    duration = 0.5 if args.duration is None else args.duration
    for serial in (False, True):
        res, _ = serve(args.rate, duration, args.nmin, args.nmax, args.t_end, args.capacity,
                       host_threads=args.threads, serial=serial, lane_min_n=args.lane_min_n or 0,
                       lane_threads=args.lane_threads or 2, device_blocks_min_n=args.device_blocks_min_n or 0,
                       lane_wait_us=args.lane_wait_us, lane_order=args.lane_order or "arrival")
        res["phase_s"].pop("build_thread_s", None)
        out["serial_plain" if serial else "continuous"] = res
    out["speedup"] = out["continuous"]["clusters_per_s"] / out["serial_plain"]["clusters_per_s"]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
