"""Benchmark of the Ahmad-Cohen regular-force step on B200.

Workload (the regular-force kernel sweep configuration): a King W0 = 6 cluster of
N = 1,048,576 equal-mass particles (seed 3, FP64 positions and velocities), squared
neighbour radii set for 100 neighbours each, list capacity 256, softening
eps = 1e-4.  One step is one regular block with every particle active (m = N):
device prediction of the whole j-set, target ordering, the force kernel and the
finalize pass.  The metric is regular-force pairs per second (m * N per step).

Arms
  default            this library: `value` with inputs resident in HBM, `e2e`
                     through the public C ABI from pinned host buffers
  --impl reference   the reference's own CPU regular force
                     (Particle::computeAccelerationReg compiled from its sources,
                     oracle/_ref) on the host cores, on a bounded sample of targets

Multi-GPU (torchrun): each rank runs an independent replica of the workload;
`value` is the pairs of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_PAIR = 40          # FMA = 2, rsqrt = 1 (acc + jerk)
REF_FLOP_PER_PAIR = 60      # the reference's convention (src/cuda/cuda_my_acceleration.cu:553)
N_DEFAULT = 1 << 20
LIST_CAP = 256
EPS2 = 1e-8
K_NB = 100
def workload_name(n: int) -> str:
    return f"king_w0=6_n={n}_m=N_regular_block"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="abyss", choices=["abyss", "reference", "reference_gpu"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-ensemble, serving and energy measurements after the timed region")
    ap.add_argument("--no-stated", action="store_true",
                    help="skip the shortened configurations 4 and 5 among the extras")
    ap.add_argument("--case", type=int, nargs=2, metavar=("N", "M"),
                    help="profiling case instead of the benchmark: one regular-force call (repeated "
                         "--repeat times) of M evenly spaced targets of an N-particle cluster, 100 "
                         "neighbours each, list capacity 256, eps2 = 1e-8; prints the plan")
    ap.add_argument("--case-model", default="king", choices=["king", "plummer"],
                    help="cluster of --case: King W0 = 6 or Plummer, seed 3")
    ap.add_argument("--tuning", default="{}", help="--case launch shape as a JSON abyss_tuning object")
    ap.add_argument("--repeat", type=int, default=1, help="--case calls")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value: float, local: int) -> float:
    if pg is None:
        return value
    import torch

    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def workload(n):
    from abyss_b200 import ic

    return ic.king(n, 3, 6.0, k_nb=K_NB)


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._th = None

    def start(self):
        self._th = threading.Thread(target=self._run, daemon=True)
        self._th.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._th:
            self._th.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 4 + k and s[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# DRAM bytes of one force launch of the default workload (N = m = 2^20) with the
# default anchor plan, from one ncu capture (dram__bytes_read.sum 734.35 MB +
# dram__bytes_write.sum 997.66 MB).  The kernel is FP32-bound; these bytes are
# reported beside the FP32 roofline, not against HBM.
CAPTURED_TRAFFIC = {"n": 1 << 20, "m": 1 << 20, "kernel": 3, "mode": 1, "threads": 128, "ipt": 6,
                    "bytes": 791.76e6 + 1074.76e6}


def captured_traffic(n, m, plan):
    c = CAPTURED_TRAFFIC
    if n == c["n"] and m == c["m"] and all(plan.get(k) == c[k] for k in ("kernel", "mode", "threads", "ipt")):
        return c["bytes"]
    return None


def launches_per_step(plan) -> int:
    """Kernels one device step launches (all compiled into libabyss_reg.so):
    predict_jset; for anchor offsets the spatial ordering (target_bbox,
    target_curve_key, CUB radix sort: histogram, exclusive sum, 4 onesweep
    passes, gather_order, block_anchor); the force kernel; finalize_rows and
    relist_rows."""
    order = 10 if plan.get("mode") == 1 and plan.get("kernel") in (1, 3) else 0
    return 1 + order + 1 + 2


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


def fp32_peak_tflops(sm_count: int, mhz: float) -> float:
    return 2.0 * sm_count * 128 * mhz * 1e6 / 1e12


# ------------------------------------------------------------------ CPU baselines
def cpu_port_baseline(c, sample_targets: int, nthreads: int):
    """The FP64 oracle restatement on a bounded sample of targets (all N j)."""
    import oracle

    px, pv = c.x, c.v
    t = np.linspace(0, c.n - 1, sample_targets).astype(np.int32)
    t0 = time.perf_counter()
    oracle.reg_force_range(px, pv, c.m, c.r2nb, EPS2, t, 0, c.n, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return sample_targets * c.n / dt / 1e9, dt


def cpu_reference_baseline(c, sample_targets: int, nthreads: int):
    """Particle::computeAccelerationReg of the reference (oracle/_ref) on a sample of
    targets against the whole cluster, one target per host thread at a time."""
    import oracle

    L = oracle.ref()
    n = c.n
    L.ref_alloc(n)
    L.ref_set_globals(1.0, -30, 1 << 30)
    a_tot = np.zeros((n, 12))
    zeros = np.zeros(n)
    dt = np.full(n, 2.0 ** -10)
    L.ref_set_all(n, oracle._p(np.ascontiguousarray(c.x)), oracle._p(np.ascontiguousarray(c.v)),
                  oracle._p(c.m), oracle._p(c.r2nb), oracle._p(a_tot), oracle._p(zeros), oracle._p(zeros),
                  oracle._p(dt))
    t = np.linspace(0, n - 1, sample_targets).astype(np.int32)
    t0 = time.perf_counter()
    L.ref_compute_reg(sample_targets, oracle._p(t, oracle._ip), nthreads)
    el = time.perf_counter() - t0
    L.ref_free()
    return sample_targets * n / el / 1e9, el


def sampled_parity(st, outs, rows: int, nthreads: int) -> dict:
    """The timed workload's own outputs (the last e2e step, host copies) against
    the FP64 oracle on `rows` sampled targets: lists and counts bit-exact, and
    the force bar of the GPU tests (|da| <= 1e-6 |a| + 1e-7 A per row, jerk
    1e-5 / 1e-6, A the sum of the regular terms' magnitudes)."""
    import oracle

    c = st.cluster
    n = c.n
    acc, jerk, nnb, lst = outs
    rng = np.random.default_rng(11)
    sel = np.unique(np.concatenate([np.linspace(0, n - 1, rows // 2).astype(np.int64),
                                    rng.choice(n, rows - rows // 2, replace=False)]))
    t = sel.astype(np.int32)  # m = N with targets 0..N-1: row r is target r
    px, pv = oracle.predict(c.x, c.v, st.a0, st.a1, st.t0, st.new_time, st.time_scale)
    t_start = time.perf_counter()
    ref = oracle.reg_force(px, pv, c.m, c.r2nb, EPS2, t, LIST_CAP, nthreads=nthreads, with_irr=False)
    sa, sj = oracle.reg_scale(px, pv, c.m, c.r2nb, EPS2, t, nthreads=nthreads)
    el = time.perf_counter() - t_start
    exact = bool(np.array_equal(nnb[sel], ref["nnb"]))
    if exact:
        for k, r in enumerate(sel):
            q = min(int(ref["nnb"][k]), LIST_CAP)
            if not np.array_equal(lst[r, :q], ref["list"][k, :q]):
                exact = False
                break
    da = np.linalg.norm(acc[sel] - ref["acc_reg"], axis=1)
    dj = np.linalg.norm(jerk[sel] - ref["jerk_reg"], axis=1)
    na = np.linalg.norm(ref["acc_reg"], axis=1)
    nj = np.linalg.norm(ref["jerk_reg"], axis=1)
    use_a = float((da / (1e-6 * na + 1e-7 * sa)).max())
    use_j = float((dj / (1e-5 * nj + 1e-6 * sj)).max())
    return {"rows": int(len(sel)), "lists_and_counts_exact": exact,
            "acc_rel_max": float((da / na).max()), "acc_rel_median": float(np.median(da / na)),
            "jerk_rel_max": float((dj / nj).max()), "jerk_rel_median": float(np.median(dj / nj)),
            "bound_use_acc": use_a, "bound_use_jerk": use_j,
            "rows_needing_floor_acc": int(np.count_nonzero(da > 1e-6 * na)),
            "rows_needing_floor_jerk": int(np.count_nonzero(dj > 1e-5 * nj)),
            "pass": exact and use_a <= 1.0 and use_j <= 1.0,
            "checker": f"FP64 oracle (oracle/liboracle.so), {el:.1f} s on {nthreads} threads",
            "sample": f"{len(sel)} targets: evenly spaced and seeded random rows of the last e2e step"}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_mem_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable"):
                    return int(line.split()[1]) / 1e6
    except Exception:
        pass
    return 0.0


# ------------------------------------------------------------------ reference arm
def run_reference(args, world, rank, local, pg):
    if rank != 0:
        return
    import oracle

    n = args.n
    c = workload(n)
    threads = host_threads()
    need_gb = n * 16616 / 1e9 * 1.2
    use_ref = oracle.ref_available() and host_mem_gb() > need_gb + 8
    sample = max(threads * 2, 2048 if use_ref else 4096)
    fn = cpu_reference_baseline if use_ref else cpu_port_baseline
    # warm-up, then K timed samples
    for _ in range(max(args.warmup, 0)):
        fn(c, max(threads, 64), threads)
    vals, secs = [], []
    for _ in range(args.steps):
        v, el = fn(c, sample, threads)
        vals.append(v)
        secs.append(el)
    value = statistics.median(vals)
    kind = "reference" if use_ref else "port"
    line = {
        "impl": "reference", "metric": "regular_force_pairs_per_s", "value": value, "unit": "Gpairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(n), "n": n, "m": n, "list_cap": LIST_CAP, "eps2": EPS2,
                   "k_nb": K_NB, "sampled_targets_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "Gpairs/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} evenly spaced targets x all {n} j per step "
                                   f"({'Particle::computeAccelerationReg, oracle/_ref' if use_ref else 'FP64 restatement, oracle/liboracle.so'})"},
        "e2e": {"value": value, "unit": "Gpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ reference GPU kernel
REF_GPU_UNAVAILABLE = (
    "the reference's GPU regular force (src_mpi/cuda, float build) made an illegal memory access on "
    "B200 at N = 2^20 and is not run again: its per-chunk list buffer is sized GridDimY * NNB_per_block * "
    "target_size = 64 * 128 * 2^20 = 2^33 ints in an int argument (cuda_my_acceleration.cu:695, "
    "cuda_routines.h:124), which wraps to 0, so compute_forces writes its lists outside any allocation")


def run_reference_gpu(args, world, rank, local, pg):
    """The reference's own GPU kernel as a baseline: unavailable (see the reason)."""
    if rank != 0:
        return
    print(json.dumps({"impl": "reference_gpu", "unavailable": REF_GPU_UNAVAILABLE}), flush=True)


# ------------------------------------------------------------------ our arm
def run_ours(args, world, rank, local, pg):
    import torch

    from abyss_b200 import workloads
    from abyss_b200.regforce import RegularForce

    n = args.n
    m = n
    st = workloads.kernel_sweep_state(n)
    c = st.cluster
    a0, a1, t0 = st.a0, st.a1, st.t0
    new_time, time_scale = st.new_time, st.time_scale
    targets = np.arange(m, dtype=np.int32)
    rf = RegularForce(local)
    stream = torch.cuda.ExternalStream(rf.stream, device=torch.device("cuda", local))
    rf.upload_state(c.x, c.v, a0, a1, t0, c.m, c.r2nb)
    rf.set_targets(targets)
    rf.reserve(n, m, LIST_CAP)
    l2_flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=torch.device("cuda", local))

    def device_step():
        rf.predict(new_time, time_scale)
        rf.launch(EPS2, LIST_CAP)

    # warm-up
    rf.set_profiling(True)
    for _ in range(args.warmup):
        device_step()
    rf.synchronize()
    plan = rf.last_plan()

    # timed: device-resident inputs, L2 flushed between steps (outside the events)
    barrier(pg)
    torch.cuda.synchronize(local)
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    force_ms = []
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            l2_flush.zero_()
            ev[k][0].record(stream)
            device_step()
            ev[k][1].record(stream)
            force_ms.append(rf.last_timing()["force_ms"])
    torch.cuda.synchronize(local)
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_total = max_over_ranks(pg, sum(step_ms) / 1e3, local)
    barrier(pg)

    value = world * m * n * args.steps / t_total / 1e9
    f_ms = statistics.median(force_ms)

    # e2e through the public API: pinned host inputs in, results out, every step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hx, hv, ha0, ha1, ht0, hm, hr2 = map(pin, (c.x, c.v, a0, a1, t0, c.m, c.r2nb))
    htg = pin(targets)
    out_acc = pin(np.zeros((m, 3)))
    out_jerk = pin(np.zeros((m, 3)))
    out_airr = pin(np.zeros((m, 3)))
    out_jirr = pin(np.zeros((m, 3)))
    out_nnb = pin(np.zeros(m, np.int32))
    out_list = pin(np.zeros((m, LIST_CAP), np.int32))
    L = rf._L
    from abyss_b200._lib import ptr, _ip
    import ctypes as C

    def e2e_step():
        assert L.abyss_upload_state(rf._h, n, ptr(hx), ptr(hv), ptr(ha0), ptr(ha1), ptr(ht0), ptr(hm),
                                    ptr(hr2)) == 0
        assert L.abyss_predict(rf._h, new_time, time_scale) == 0
        ovf = C.c_int(0)
        rc = L.abyss_regular_force(rf._h, m, ptr(htg, _ip), EPS2, LIST_CAP, None, ptr(out_acc),
                                   ptr(out_jerk), ptr(out_airr), ptr(out_jirr), ptr(out_nnb, _ip),
                                   ptr(out_list, _ip), C.byref(ovf))
        assert rc >= 0, rc

    e2e_step()
    barrier(pg)
    torch.cuda.synchronize(local)
    t0w = time.perf_counter()
    e_start = torch.cuda.Event(enable_timing=True)
    e_stop = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e_stop.record(stream)
    torch.cuda.synchronize(local)
    e2e_s = max(e_start.elapsed_time(e_stop) / 1e3, time.perf_counter() - t0w)
    e2e_s = max_over_ranks(pg, e2e_s, local)
    e2e_value = world * m * n * args.steps / e2e_s / 1e9
    h2d = 8 * (3 * 4 * n + 3 * n) + 4 * m
    d2h = m * (4 * 3 * 8 + 4 + 4 * LIST_CAP) + 8

    # sweep of active-block sizes (same j-set), device-resident, kernel only
    sweep = {}
    if not args.no_sweep:
        # each call timed by two events around it (ordering, force, finalize)
        rf.set_profiling("whole")
        for mm, t in workloads.sweep_targets(n).items():
            rf.set_targets(t)
            rf.predict(new_time, time_scale)
            for _ in range(3):
                rf.launch(EPS2, LIST_CAP)
            times = []
            for _ in range(5):
                rf.launch(EPS2, LIST_CAP)
                times.append(rf.last_timing()["force_ms"])
            ms = statistics.median(times)
            sweep[str(mm)] = {"gpairs_s": mm * n / ms / 1e6, "ms": ms, "plan": rf.last_plan()}
        rf.set_targets(targets)

    peaks, peak_src = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    peak_tf = fp32_peak_tflops(sm_count, max_mhz)
    achieved_tf = FLOP_PER_PAIR * m * n / (f_ms / 1e3) / 1e12
    clk = clocks.get("sm_mhz")
    roofline = {
        "bound": "fp32", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
        "frac": achieved_tf / peak_tf, "traffic": captured_traffic(n, m, plan),
        "traffic_unit": "bytes per force launch (ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                        "launch of this workload and plan; null for any other)",
        "note": (f"FP32 CUDA-core pipe: 2 x {sm_count} SMs x 128 lanes x {max_mhz:.0f} MHz "
                 f"(sm_max_mhz of MEASURED_PEAKS.json, {peak_src}); 40 flop/pair; force kernel "
                 f"{f_ms:.1f} ms per launch by CUDA events on the launching stream"),
        "frac_at_sampled_clock": (achieved_tf / fp32_peak_tflops(sm_count, clk)) if clk else None,
    }
    line = {
        "metric": "regular_force_pairs_per_s", "value": value, "unit": "Gpairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(step_ms),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair arithmetic, f64 differencing/sums", "data": "synthetic",
        "config": {"workload": workload_name(n), "n": n, "m": m, "list_cap": LIST_CAP, "eps2": EPS2,
                   "k_nb": K_NB, "parallelism": f"replicas{world}", "plan": plan,
                   "l2": "flushed between timed steps (256 MB write)"},
        "force_kernel": {"ms": f_ms, "gpairs_s": m * n / f_ms / 1e6,
                         "pct_fp32_peak": 100 * achieved_tf / peak_tf,
                         "ref_60flop_tflops": REF_FLOP_PER_PAIR * m * n / (f_ms / 1e3) / 1e12},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "Gpairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step(plan) * args.steps,
        "clocks": clocks,
        "sweep": sweep,
    }
    rf.close()
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle

        threads = host_threads()
        sample = 2048
        if oracle.ref_available() and host_mem_gb() > n * 16616 / 1e9 * 1.2 + 8:
            v, el = cpu_reference_baseline(c, sample, threads)
            kind, what = "reference", "Particle::computeAccelerationReg of the reference, oracle/_ref"
        else:
            v, el = cpu_port_baseline(c, sample, threads)
            kind, what = "port", "FP64 restatement of ComputeAcceleration.cpp:235-299"
        line["cpu_baseline"] = {"value": v, "unit": "Gpairs/s", "cores": threads, "kind": kind,
                                "sample": f"{sample} evenly spaced targets x all {n} j ({el:.1f} s, {what})"}
        # the same CPU leg checks the timed step's outputs on sampled rows
        line["parity"] = sampled_parity(st, (out_acc, out_jerk, out_nnb, out_list), 512, threads)
    if rank == 0 and world == 1 and not args.no_extras:
        line["extras"] = extras(local, stated=not args.no_stated)
    if rank == 0:
        print(json.dumps(line), flush=True)


def extras(device: int, stated: bool = True) -> dict:
    """The rest of the headline metric, measured after the timed region on the
    same GPU: batched-ensemble throughput against one cluster per launch, the
    serving loop against serial plain integrations (throughput, p50/p99) on a
    saturated stream and, shortened to fit the benchmark's few minutes, on
    configurations 4 and 5, and the energy drift of full integrations."""
    from abyss_b200 import bench_ensemble, runs, serve, workloads
    from abyss_b200.regforce import RegularForce

    out = {}
    rf = RegularForce(device)
    clusters = workloads.ensemble(k=512)
    waves = workloads.ensemble_waves(clusters, 6)
    ens = bench_ensemble.measure(rf, clusters, waves, tune=True)
    rf.close()
    out["batched_ensemble"] = {
        "workload": "512 Plummer clusters, N log-uniform in [256, 16384], 6 waves of regular blocks",
        "cluster_blocks_per_s_graph": ens["graph"]["cluster_blocks_per_s"],
        "cluster_blocks_per_s_plain": ens["plain"]["cluster_blocks_per_s"],
        "gpairs_s_graph": ens["graph"]["gpairs_s"], "graph_vs_plain": ens["graph_vs_plain"],
        "cluster_blocks_per_s_graph_tuned": ens["graph_tuned"]["cluster_blocks_per_s"],
        "gpairs_s_graph_tuned": ens["graph_tuned"]["gpairs_s"],
        "graph_tuned_vs_plain": ens["graph_tuned_vs_plain"], "tuning": ens["tuning"]}
    kw = dict(rate=2000.0, duration=0.5, nmin=256, nmax=2048, t_end=0.0625)
    res = {}
    for serial in (False, True):
        # a short stream first, untimed, for one-time costs (host threads and
        # memory, first launches of each kernel) in either arm
        serve.serve(**dict(kw, duration=0.05, seed=6), serial=serial)
        r, _ = serve.serve(**kw, serial=serial)
        res["serial" if serial else "continuous"] = r
    c, sp = res["continuous"], res["serial"]
    out["serving"] = {
        "workload": "Poisson 2000 requests/s for 0.5 s (seed 5), Plummer or King W0 3/6/9, Kroupa IMF, "
                    "N log-uniform in [256, 2048], each integrated to t = 1/16; each arm after an untimed "
                    "0.05 s stream (seed 6)",
        "requests": c["requests"], "clusters_per_s": c["clusters_per_s"],
        "clusters_per_s_serial_plain": sp["clusters_per_s"], "vs_serial_plain": c["clusters_per_s"] / sp["clusters_per_s"],
        "p50_latency_s": c["p50_latency_s"], "p99_latency_s": c["p99_latency_s"],
        "p50_latency_s_serial_plain": sp["p50_latency_s"], "p99_latency_s_serial_plain": sp["p99_latency_s"],
        "median_dE_over_E": c["median_dE_over_E"], "max_dE_over_E": c["max_dE_over_E"]}
    c1 = runs.run("c1")
    out["energy_c1"] = {"workload": "Plummer N = 1024, eps = 1e-4, to t = 10", "dE_over_E": c1["dE_over_E"],
                        "regular_blocks": c1["stats"]["blocks"], "wall_s": c1["wall_s"]}
    if stated:
        # the stated configurations, shortened: 128 of configuration 4's 512
        # clusters, and configuration 5's stream for 0.25 s instead of 1 s; the
        # serial plain arm on 16 evenly spaced requests of each, as for the
        # whole configurations (their run times span two decades with N, so
        # the sample sets that arm's clusters/s)
        for name, kw, short in (("c4", dict(k=128), "the first 128 of the 512 clusters"),
                                ("c5", dict(duration=0.25), "the stream for 0.25 s instead of 1 s")):
            r = serve.run_config(name, sample=16, **kw)
            out[f"serving_{name}"] = {
                "workload": r["config"]["workload"] + f" (shortened to fit the benchmark: {short}; serial "
                                                      "plain arm on 16 evenly spaced requests)",
                "lanes": {k: r["config"][k] for k in ("lane_min_n", "lane_threads", "device_blocks_min_n",
                                                      "lane_order")},
                "requests": r["requests"], "clusters_per_s": r["clusters_per_s"],
                "clusters_per_s_serial_plain": r["serial_plain_sample"]["clusters_per_s"],
                "vs_serial_plain": r["vs_serial_plain"], "p50_latency_s": r["p50_latency_s"],
                "p99_latency_s": r["p99_latency_s"], "median_dE_over_E": r["median_dE_over_E"],
                "max_dE_over_E": r["max_dE_over_E"], "frac_dE_below_1e6": r["frac_dE_below_1e6"]}
    c2 = runs.run("c2", device_blocks=True)
    out["energy_c2"] = {"workload": "Plummer N = 65536, Kroupa IMF, eps = 1e-4, to t = 2, whole blocks on the GPU",
                        "dE_over_E": c2["dE_over_E"], "regular_blocks": c2["stats"]["blocks"],
                        "wall_s": c2["wall_s"], "irregular_s": c2["stats"]["sec_irr"],
                        "borderline": c2["device_blocks"]["borderline"] + c2["device_irregular"]["borderline"]}
    return out


def run_case(args):
    """One regular-force call shape for a profiler capture: the plan it ran and
    the mean neighbour count, so that a capture can be tied to its shape."""
    from abyss_b200 import ic
    from abyss_b200.regforce import RegularForce

    n, m = args.case
    c = ic.king(n, 3, 6.0, k_nb=K_NB) if args.case_model == "king" else ic.plummer(n, 3, k_nb=K_NB)
    rf = RegularForce(0)
    try:
        rf.send_to_device(c.m, c.x, c.v, c.r2nb)
        t = np.arange(0, n, max(1, n // m), dtype=np.int32)[:m]
        tu = json.loads(args.tuning)
        rf.set_profiling(True)
        ms, parts = [], []
        for _ in range(args.repeat):
            res = rf.calculate_acceleration(t, eps2=EPS2, list_cap=LIST_CAP, tuning=tu)
            tm = rf.last_timing()
            ms.append(tm["order_ms"] + tm["force_ms"] + tm["finalize_ms"])
            parts.append(tm)
        k = int(np.argmin(ms))
        # the whole call between two events (no events between its phases)
        rf.set_profiling("whole")
        whole = []
        for _ in range(args.repeat):
            rf.launch(EPS2, LIST_CAP, tu)
            whole.append(rf.last_timing()["force_ms"])
        best = min(whole)
        print(json.dumps({"case": f"{args.case_model} n={n} m={len(t)}", "plan": res.plan,
                          "mean_nnb": float(res.nnb.mean()), "best_ms": best, "best_parts_ms": parts[k],
                          "best_sum_of_parts_ms": ms[k],
                          "gpairs_s": len(t) * n / best / 1e6}), flush=True)
    finally:
        rf.close()


def main():
    args = parse()
    if args.case:
        run_case(args)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local, pg)
        elif args.impl == "reference_gpu":
            run_reference_gpu(args, world, rank, local, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
