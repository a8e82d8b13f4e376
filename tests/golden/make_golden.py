"""Generate the golden vectors in tests/golden/ from the reference itself.

The reference ships no tests, fixtures or known-answer vectors for its regular
force, so this script runs the reference's own CPU code -- compiled from its
sources into oracle/_ref/libabyss_ref.so by oracle/Makefile -- on seeded
synthetic clusters and stores inputs and outputs as compressed .npz files:

* initial FP64 forces, neighbour lists          CalculateAcceleration01 (Initialize.cpp:16-92)
* predicted positions / velocities at new_time  predictParticleSecondOrder (UpdateParticle.cpp:37-59)
* CPU regular force, new lists, a_irr, corrector computeAccelerationReg (ComputeAcceleration.cpp:197-398)
* GPU-result corrector                          updateRegularParticleCuda (ComputeAcceleration.cpp:405-661)
* timestep rules                                TimeStepRoutines.cpp:10-115
* irregular step and its new level (*_irr.npz)   computeAccelerationIrr (ComputeAcceleration.cpp:14-190),
                                                calculateTimeStepIrr (UpdateParticle.cpp:151-241)
* level rules and radius update (ref_levels)    calculateTimeStepIrr, calculateTimeStepReg
                                                (UpdateParticle.cpp:314-407), updateRadius (:108-139),
                                                initializeTimeStep (Initialize.cpp:199-230)

Run from the repository root with the reference tree present:
    make -C oracle && python tests/golden/make_golden.py
(`--irregular-only` rewrites only the last two kinds, from the committed
regular-step fixtures.)
The reference applies no softening, so every vector here has eps2 = 0.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import _p, _ip  # noqa: E402
from abyss_b200 import ic  # noqa: E402

CAP = 2000  # MaxNumberOfNeighbor, src_mpi/def.h:10


def _state_from_ref(L, n):
    x = np.zeros((n, 3)); v = np.zeros((n, 3))
    a_tot = np.zeros((n, 3, 4)); a_reg = np.zeros((n, 3, 4)); a_irr = np.zeros((n, 3, 4))
    newpos = np.zeros((n, 3)); newvel = np.zeros((n, 3)); r2 = np.zeros(n)
    nnb = np.zeros(n, np.int32); nb = np.full((n, CAP), -1, np.int32)
    new_nnb = np.zeros(n, np.int32); new_nb = np.full((n, CAP), -1, np.int32)
    for i in range(n):
        r2i = np.zeros(1); k = np.zeros(1, np.int32); k2 = np.zeros(1, np.int32)
        L.ref_get_particle(i, _p(x[i]), _p(v[i]), _p(a_tot[i]), _p(a_reg[i]), _p(a_irr[i]),
                           _p(newpos[i]), _p(newvel[i]), _p(r2i), _p(k, _ip), _p(nb[i], _ip),
                           _p(k2, _ip), _p(new_nb[i], _ip), CAP)
        r2[i] = r2i[0]; nnb[i] = k[0]; new_nnb[i] = k2[0]
    return dict(x=x, v=v, a_tot=a_tot, a_reg=a_reg, a_irr=a_irr, newpos=newpos, newvel=newvel,
                r2nb=r2, nnb=nnb, nb=nb, new_nnb=new_nnb, new_nb=new_nb)


def _load(L, st, i):
    L.ref_set_particle(i, _p(st["x"][i]), _p(st["v"][i]), float(st["m"][i]), float(st["r2nb"][i]),
                       _p(st["a_tot"][i]), _p(st["a_reg"][i]), _p(st["a_irr"][i]),
                       float(st["t_reg"][i]), float(st["t_irr"][i]), float(st["dt_reg"][i]),
                       float(st["dt_irr"][i]), int(st["nnb"][i]), _p(st["nb"][i], _ip))


def make_case(cl: ic.Cluster, time_scale: float, seed: int):
    L = oracle.ref()
    n = cl.n
    rng = np.random.default_rng(seed)
    L.ref_alloc(n)
    L.ref_set_globals(time_scale, -30, 1 << 30)
    z = np.zeros((3, 4))
    no = np.zeros(1, np.int32)
    for i in range(n):
        L.ref_set_particle(i, _p(np.ascontiguousarray(cl.x[i])), _p(np.ascontiguousarray(cl.v[i])),
                           float(cl.m[i]), float(cl.r2nb[i]), _p(z), _p(z), _p(z),
                           0.0, 0.0, 0.0, 0.0, 0, _p(no, _ip))
    for i in range(n):
        L.ref_init_acc01(i)
    init = _state_from_ref(L, n)

    # A regular-step state: targets share t_reg = 0 and dt_reg = dt; the other
    # particles sit at assorted irregular times <= new_time; a third of all
    # particles carry no neighbour list (predicted from t_reg).
    dt = 2.0 ** -7
    new_time = dt
    targets = np.sort(rng.choice(n, size=n // 2, replace=False)).astype(np.int32)
    is_t = np.zeros(n, bool); is_t[targets] = True
    st = dict(x=init["x"], v=init["v"], m=cl.m.copy(), r2nb=init["r2nb"], a_tot=init["a_tot"],
              a_reg=init["a_reg"], a_irr=init["a_irr"], nnb=init["nnb"].copy(), nb=init["nb"])
    st["nnb"][rng.uniform(size=n) < 1.0 / 3.0] = 0
    st["t_reg"] = np.zeros(n)
    st["dt_reg"] = np.where(is_t, dt, 2.0 * dt)
    lag = rng.choice([0.0, 2.0 ** -9, 2.0 ** -8, 3 * 2.0 ** -9], size=n)
    st["t_irr"] = np.where(st["nnb"] > 0, np.where(is_t, new_time, new_time - lag), 0.0)
    st["dt_irr"] = np.full(n, 2.0 ** -9)
    t0 = np.where(st["nnb"] == 0, st["t_reg"], st["t_irr"])
    for i in range(n):
        _load(L, st, i)
    # predicted state of every particle at new_time (the j-set the GPU path sees)
    px = np.zeros((n, 3)); pv = np.zeros((n, 3))
    px32 = np.zeros((n, 3), np.float32); pv32 = np.zeros((n, 3), np.float32)
    for i in range(n):
        L.ref_predict(i, new_time - t0[i], _p(px[i]), _p(pv[i]))
        L.ref_predict_f32(i, new_time - t0[i], px32[i].ctypes.data_as(oracle._fp),
                          pv32[i].ctypes.data_as(oracle._fp))
    # reference CPU regular force for the targets, every particle predicted from
    # its pre-step state (see ref_compute_reg_isolated in oracle/ref_shim)
    k = targets.shape[0]
    o_reg = np.zeros((k, 3, 4)); o_irr = np.zeros((k, 3, 4)); o_tot = np.zeros((k, 3, 4))
    o_pos = np.zeros((k, 3)); o_vel = np.zeros((k, 3)); o_nnb = np.zeros(k, np.int32)
    o_nb = np.full((k, CAP), -1, np.int32)
    L.ref_compute_reg_isolated(k, _p(targets, _ip), _p(o_reg), _p(o_irr), _p(o_tot), _p(o_pos),
                               _p(o_vel), _p(o_nnb, _ip), _p(o_nb, _ip), CAP)
    out = dict(a_reg=np.zeros((n, 3, 4)), a_irr=np.zeros((n, 3, 4)), a_tot=np.zeros((n, 3, 4)),
               newpos=np.zeros((n, 3)), newvel=np.zeros((n, 3)), new_nnb=np.zeros(n, np.int32),
               new_nb=np.full((n, CAP), -1, np.int32))
    out["a_reg"][targets] = o_reg; out["a_irr"][targets] = o_irr; out["a_tot"][targets] = o_tot
    out["newpos"][targets] = o_pos; out["newvel"][targets] = o_vel
    out["new_nnb"][targets] = o_nnb; out["new_nb"][targets] = o_nb
    # reference GPU-result corrector fed with the reference's own new list and a_new,
    # every target corrected from the pre-step state of the others
    for i in range(n):
        _load(L, st, i)
    cuda_out = dict(a_reg=np.zeros((n, 3, 4)), a_irr=np.zeros((n, 3, 4)), a_tot=np.zeros((n, 3, 4)),
                    newpos=np.zeros((n, 3)), newvel=np.zeros((n, 3)))
    for i in targets:
        k = int(out["new_nnb"][i])
        L.ref_update_reg_cuda_isolated(int(i), _p(np.ascontiguousarray(out["new_nb"][i, :k]), _ip), k,
                                       _p(np.ascontiguousarray(out["a_reg"][i, :, 0])),
                                       _p(np.ascontiguousarray(out["a_reg"][i, :, 1])),
                                       _p(cuda_out["a_reg"][i]), _p(cuda_out["a_irr"][i]),
                                       _p(cuda_out["a_tot"][i]), _p(cuda_out["newpos"][i]),
                                       _p(cuda_out["newvel"][i]))
    maxnb = int(out["new_nnb"][targets].max())
    maxold = int(st["nnb"].max())
    res = dict(
        x=st["x"], v=st["v"], m=st["m"], r2nb=st["r2nb"], a_tot=st["a_tot"], a_reg=st["a_reg"],
        a_irr=st["a_irr"], t_reg=st["t_reg"], t_irr=st["t_irr"], dt_reg=st["dt_reg"],
        dt_irr=st["dt_irr"], nnb=st["nnb"], nb=st["nb"][:, :maxold], t0=t0,
        time_scale=np.array(time_scale), new_time=np.array(new_time), targets=targets,
        px=px, pv=pv, px32=px32, pv32=pv32,
        out_a_reg=out["a_reg"][targets], out_a_irr=out["a_irr"][targets][:, :, :2],
        out_a_tot=out["a_tot"][targets], out_newpos=out["newpos"][targets],
        out_newvel=out["newvel"][targets], out_nnb=out["new_nnb"][targets],
        out_list=out["new_nb"][targets][:, :maxnb],
        cuda_a_reg=cuda_out["a_reg"][targets], cuda_a_irr=cuda_out["a_irr"][targets][:, :, :2],
        cuda_a_tot=cuda_out["a_tot"][targets], cuda_newpos=cuda_out["newpos"][targets],
        cuda_newvel=cuda_out["newvel"][targets],
        init_nnb=init["nnb"],
    )
    return res


def make_timesteps(seed: int):
    L = oracle.ref()
    rng = np.random.default_rng(seed)
    k = 64
    f = rng.normal(size=(k, 3, 4)) * 10.0 ** rng.uniform(-3, 3, size=(k, 1, 4))
    df = rng.normal(size=(k, 3, 4)) * 10.0 ** rng.uniform(-3, 3, size=(k, 1, 4))
    vv = rng.normal(size=(k, 3))
    reg = np.array([L.ref_new_time_step_reg(_p(np.ascontiguousarray(vv[i])), _p(np.ascontiguousarray(df[i])))
                    for i in range(k)])
    irr = np.array([L.ref_new_time_step_irr(_p(np.ascontiguousarray(f[i])), _p(np.ascontiguousarray(df[i])))
                    for i in range(k)])
    time_scale = 10.0
    tblock = -30
    L.ref_set_globals(time_scale, tblock, 1 << 30)
    dts = 10.0 ** rng.uniform(-9, 1, size=k)
    lv = np.zeros(k, np.int32); bl = np.zeros(k, np.uint64); stp = np.zeros(k)
    for i in range(k):
        a = np.zeros(1, np.int32); b = np.zeros(1, np.uint64); c = np.zeros(1)
        L.ref_block_time_step(float(dts[i]), _p(a, _ip), b.ctypes.data_as(oracle.C.POINTER(oracle.C.c_ulonglong)),
                              _p(c))
        lv[i] = a[0]; bl[i] = b[0]; stp[i] = c[0]
    return dict(f=f, df=df, v=vv, reg=reg, irr=irr, eta=np.array(L.ref_eta()), dts=dts,
                time_scale=np.array(time_scale), time_block=np.array(tblock), level=lv, block=bl, step=stp)


def _blocks(L, i):
    ull = np.zeros(4, np.uint64); lvl = np.zeros(2, np.int32); dts = np.zeros(2)
    L.ref_get_blocks(i, ull.ctypes.data_as(oracle.C.POINTER(oracle.C.c_ulonglong)), _p(lvl, _ip), _p(dts))
    return ull, lvl, dts


def make_irregular(base: dict, tblock: int = -30):
    """computeAccelerationIrr, then calculateTimeStepIrr (the IrrForce task of
    WorkerRoutines.cpp:46-64), for every particle of a golden regular-step state
    that has neighbours and for a few that have none, each run from the
    pre-step state of all the others."""
    L = oracle.ref()
    st = {k: np.array(base[k]) for k in ("x", "v", "m", "r2nb", "a_tot", "a_reg", "a_irr", "t_reg", "t_irr",
                                         "dt_reg", "dt_irr", "nnb", "nb")}
    st["nb"] = np.ascontiguousarray(st["nb"], np.int32)
    n = st["x"].shape[0]
    time_scale = float(base["time_scale"])
    L.ref_alloc(n)
    L.ref_set_globals(time_scale, tblock, 1 << -tblock)
    for i in range(n):
        _load(L, st, i)
    with_nb = np.flatnonzero(st["nnb"] > 0)
    without = np.flatnonzero(st["nnb"] == 0)[:8]
    idx = np.sort(np.concatenate([with_nb, without])).astype(np.int32)
    k = idx.shape[0]
    newpos = np.zeros((k, 3)); newvel = np.zeros((k, 3))
    a_irr = np.zeros((k, 3, 4)); a_tot = np.zeros((k, 3, 4))
    lv_irr = np.zeros(k, np.int32); tb_irr = np.zeros(k, np.uint64); dt_irr = np.zeros(k)
    step = 2.0 ** tblock
    lv_reg = np.round(np.log2(st["dt_reg"])).astype(np.int32)
    for r, i in enumerate(idx):
        i = int(i)
        one = np.array([i], np.int32)
        L.ref_compute_irr(1, _p(one, _ip), 1)
        cur_irr = int(round(st["t_irr"][i] / step))
        tb = int(round(st["dt_irr"][i] / step))
        L.ref_set_blocks(i, 0, cur_irr, int(round(st["dt_reg"][i] / step)), tb, int(lv_reg[i]),
                         int(round(np.log2(st["dt_irr"][i]))), cur_irr + tb)
        L.ref_time_step_irr(i)
        x = np.zeros(3); v = np.zeros(3); at = np.zeros(12); ar = np.zeros(12); ai = np.zeros(12)
        r2 = np.zeros(1); c1 = np.zeros(1, np.int32); c2 = np.zeros(1, np.int32)
        nb = np.zeros(CAP, np.int32); nb2 = np.zeros(CAP, np.int32)
        L.ref_get_particle(i, _p(x), _p(v), _p(at), _p(ar), _p(ai), _p(newpos[r]), _p(newvel[r]), _p(r2),
                           _p(c1, _ip), _p(nb, _ip), _p(c2, _ip), _p(nb2, _ip), CAP)
        a_irr[r] = ai.reshape(3, 4); a_tot[r] = at.reshape(3, 4)
        ull, lvl, dts = _blocks(L, i)
        lv_irr[r] = lvl[1]; tb_irr[r] = ull[3]; dt_irr[r] = dts[1]
        _load(L, st, i)
    # the state itself is the base fixture's
    return dict(time_block=np.array(tblock), idx=idx, out_newpos=newpos, out_newvel=newvel, out_a_irr=a_irr,
                out_a_tot=a_tot, out_lv_irr=lv_irr, out_tb_irr=tb_irr, out_dt_irr=dt_irr)


def _derivs(rng, dt, eta):
    """[3][4] derivatives whose Aarseth step is about dt: F_k ~ A w^k with
    w = sqrt(eta) / dt, randomised component by component."""
    w = np.sqrt(eta) / dt
    amp = 10.0 ** rng.uniform(-2, 2)
    return rng.normal(size=(3, 4)) * amp * w ** np.arange(4) * 10.0 ** rng.uniform(-0.5, 0.5, size=(1, 4))


def make_levels(seed: int, tblock: int = -30):
    """calculateTimeStepIrr, calculateTimeStepReg and updateRadius on seeded
    block states that reach every branch (level up, kept, one or two down, the
    clamp at the regular block's end, the end of the run), no throwing case."""
    L = oracle.ref()
    rng = np.random.default_rng(seed)
    L.ref_alloc(1)
    z = np.zeros(12)
    zx = np.zeros(3)
    nb = np.zeros(CAP, np.int32)
    eta = float(L.ref_eta())
    bmax = 1 << -tblock
    scales = np.array([0.1, 1.0, 10.0])
    res = {}
    # calculateTimeStepIrr
    k = 1000
    cols = {c: [] for c in ("scale", "has_nb", "a_tot", "a_irr", "new_cur_irr", "cur_reg", "tb_reg", "lv_reg",
                            "lv_irr", "tb_irr", "dt_irr", "out_lv_irr", "out_tb_irr", "out_dt_irr")}
    for _ in range(k):
        scale = float(rng.choice(scales))
        L.ref_set_globals(scale, tblock, bmax)
        lv_reg = int(rng.integers(-20, -2))
        tb_reg = 1 << (lv_reg - tblock)
        cur_reg = int(rng.integers(0, bmax // tb_reg)) * tb_reg
        lv_irr = lv_reg - int(rng.integers(1, 7))
        tb_irr = 1 << (lv_irr - tblock)
        cur_irr = cur_reg + int(rng.integers(0, tb_reg // tb_irr)) * tb_irr
        new_cur = cur_irr + tb_irr
        has_nb = int(rng.uniform() < 0.9)
        dt_target = 2.0 ** (lv_irr + rng.uniform(-3.5, 3.5)) * scale
        at = _derivs(rng, dt_target, eta)
        ai = _derivs(rng, dt_target, eta)
        ai[:, 0] = at[:, 0] * rng.uniform(0.2, 1.0)
        L.ref_set_particle(0, _p(zx), _p(zx), 1.0, 0.0, _p(np.ascontiguousarray(at.reshape(12))), _p(z),
                           _p(np.ascontiguousarray(ai.reshape(12))), cur_reg * 2.0 ** tblock,
                           cur_irr * 2.0 ** tblock, 2.0 ** lv_reg, 2.0 ** lv_irr, has_nb, _p(nb, _ip))
        L.ref_set_blocks(0, cur_reg, cur_irr, tb_reg, tb_irr, lv_reg, lv_irr, new_cur)
        L.ref_time_step_irr(0)
        ull, lvl, dts = _blocks(L, 0)
        for c, val in (("scale", scale), ("has_nb", has_nb), ("a_tot", at), ("a_irr", ai), ("new_cur_irr", new_cur),
                       ("cur_reg", cur_reg), ("tb_reg", tb_reg), ("lv_reg", lv_reg), ("lv_irr", lv_irr),
                       ("tb_irr", tb_irr), ("dt_irr", 2.0 ** lv_irr), ("out_lv_irr", lvl[1]),
                       ("out_tb_irr", ull[3]), ("out_dt_irr", dts[1])):
            cols[c].append(val)
    for c, val in cols.items():
        dt = np.uint64 if c in ("new_cur_irr", "cur_reg", "tb_reg", "tb_irr", "out_tb_irr") else None
        res["irr_" + c] = np.array(val, dtype=dt)
    # calculateTimeStepReg
    cols = {c: [] for c in ("scale", "has_nb", "a_reg", "t_reg", "cur_reg", "lv_reg", "tb_reg", "dt_reg",
                            "lv_irr", "out_lv_reg", "out_tb_reg", "out_dt_reg", "out_lv_irr")}
    for _ in range(k):
        scale = float(rng.choice(scales))
        L.ref_set_globals(scale, tblock, bmax)
        lv_reg = int(rng.integers(-20, -1))
        tb_reg = 1 << (lv_reg - tblock)
        u = rng.uniform()
        if u < 0.1:
            cur_reg = 0
        elif u < 0.25:  # the last steps of the run
            cur_reg = bmax - tb_reg * int(rng.integers(1, 4))
        else:
            cur_reg = int(rng.integers(0, bmax // tb_reg)) * tb_reg
        cur_reg = max(cur_reg, 0)
        t_reg = cur_reg * 2.0 ** tblock
        has_nb = int(rng.uniform() < 0.8)
        lv_irr = lv_reg - 2
        ar = _derivs(rng, 2.0 ** (lv_reg + rng.uniform(-3.5, 4.5)) * scale, eta)
        L.ref_set_particle(0, _p(zx), _p(zx), 1.0, 0.0, _p(z), _p(np.ascontiguousarray(ar.reshape(12))), _p(z),
                           t_reg, t_reg, 2.0 ** lv_reg, 2.0 ** lv_irr, has_nb, _p(nb, _ip))
        L.ref_set_blocks(0, cur_reg, cur_reg, tb_reg, 1 << (lv_irr - tblock), lv_reg, lv_irr, cur_reg)
        L.ref_time_step_reg(0)
        ull, lvl, dts = _blocks(L, 0)
        for c, val in (("scale", scale), ("has_nb", has_nb), ("a_reg", ar), ("t_reg", t_reg), ("cur_reg", cur_reg),
                       ("lv_reg", lv_reg), ("tb_reg", tb_reg), ("dt_reg", 2.0 ** lv_reg), ("lv_irr", lv_irr),
                       ("out_lv_reg", lvl[0]), ("out_tb_reg", ull[2]), ("out_dt_reg", dts[0]),
                       ("out_lv_irr", lvl[1])):
            cols[c].append(val)
    for c, val in cols.items():
        dt = np.uint64 if c in ("cur_reg", "tb_reg", "out_tb_reg") else None
        res["reg_" + c] = np.array(val, dtype=dt)
    # initializeTimeStep (Initialize.cpp:199-230) at the start of a run
    cols = {c: [] for c in ("scale", "has_nb", "a_tot", "a_reg", "a_irr", "out_lv_reg", "out_tb_reg", "out_dt_reg",
                            "out_lv_irr", "out_tb_irr", "out_dt_irr")}
    for _ in range(k):
        scale = float(rng.choice(scales))
        L.ref_set_globals(scale, tblock, bmax)
        has_nb = int(rng.uniform() < 0.85)
        lv = rng.uniform(-16, 2)  # some steps above 1, which the rule caps
        ar = _derivs(rng, 2.0 ** lv * scale, eta)
        ai = _derivs(rng, 2.0 ** (lv - rng.uniform(0, 6)) * scale, eta)
        at = ar + ai
        L.ref_set_particle(0, _p(zx), _p(zx), 1.0, 0.0, _p(np.ascontiguousarray(at.reshape(12))),
                           _p(np.ascontiguousarray(ar.reshape(12))), _p(np.ascontiguousarray(ai.reshape(12))),
                           0.0, 0.0, 0.0, 0.0, has_nb, _p(nb, _ip))
        L.ref_initialize_time_step(0)
        ull, lvl, dts = _blocks(L, 0)
        for c, val in (("scale", scale), ("has_nb", has_nb), ("a_tot", at), ("a_reg", ar), ("a_irr", ai),
                       ("out_lv_reg", lvl[0]), ("out_tb_reg", ull[2]), ("out_dt_reg", dts[0]),
                       ("out_lv_irr", lvl[1]), ("out_tb_irr", ull[3]), ("out_dt_irr", dts[1])):
            cols[c].append(val)
    for c, val in cols.items():
        dt = np.uint64 if c in ("out_tb_reg", "out_tb_irr") else None
        res["init_" + c] = np.array(val, dtype=dt)
    # updateRadius over every count from 0 to 2 NumNeighborMax
    fix, nbmax = int(L.ref_fix_num_neighbor()), int(L.ref_num_neighbor_max())
    counts = np.arange(0, min(2 * nbmax, CAP) + 1, dtype=np.int32)
    r2in = 10.0 ** rng.uniform(-6, 0, size=counts.shape[0])
    r2out = np.zeros_like(r2in)
    for q, (c, r2) in enumerate(zip(counts, r2in)):
        L.ref_set_particle(0, _p(zx), _p(zx), 1.0, float(r2), _p(z), _p(z), _p(z), 0.0, 0.0, 0.0, 0.0, int(c),
                           _p(nb, _ip))
        L.ref_update_radius(0)
        x = np.zeros(3); v = np.zeros(3); a = np.zeros(12); r2o = np.zeros(1)
        c1 = np.zeros(1, np.int32); c2 = np.zeros(1, np.int32); nb2 = np.zeros(CAP, np.int32)
        L.ref_get_particle(0, _p(x), _p(v), _p(a), _p(a), _p(a), _p(x), _p(v), _p(r2o), _p(c1, _ip),
                           _p(nb2, _ip), _p(c2, _ip), _p(nb2, _ip), CAP)
        r2out[q] = r2o[0]
    res.update(rad_counts=counts, rad_r2_in=r2in, rad_r2_out=r2out, rad_fix=np.array(fix),
               rad_nb_max=np.array(nbmax), eta=np.array(eta), time_block=np.array(tblock), block_max=np.array(bmax,
                                                                                                          np.uint64))
    return res


def main():
    oracle.build()
    here = os.path.dirname(os.path.abspath(__file__))
    if "--irregular-only" in sys.argv:
        write_irregular(here)
        return
    c1 = ic.plummer(1024, 1, k_nb=32, exact_k=True)
    np.savez_compressed(os.path.join(here, "ref_plummer1024_s1.npz"), **make_case(c1, 10.0, 11))
    c3 = ic.king(2048, 3, 6.0, k_nb=100, exact_k=True)
    np.savez_compressed(os.path.join(here, "ref_king2048_s3.npz"), **make_case(c3, 1.0, 33))
    np.savez_compressed(os.path.join(here, "ref_timesteps.npz"), **make_timesteps(7))
    write_irregular(here)
    print("golden vectors written to", here)


def write_irregular(here):
    for name in ("ref_plummer1024_s1", "ref_king2048_s3"):
        base = np.load(os.path.join(here, name + ".npz"))
        np.savez_compressed(os.path.join(here, name + "_irr.npz"), **make_irregular(base))
    np.savez_compressed(os.path.join(here, "ref_levels.npz"), **make_levels(17))


if __name__ == "__main__":
    main()
