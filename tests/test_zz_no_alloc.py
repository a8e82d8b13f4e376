"""abyss_regular_force_noalloc: the regular force for callers that cannot
allocate device memory (their GPU memory belongs to another allocator, a hard
budget, or a path where cudaMalloc may not run).  The caller owns every input
and output buffer; the library keeps its intermediates in one fixed array.

Checked through the C ABI against the ordinary context entry point on the same
inputs and against the FP64 oracle, on two calls in a row (the second with
other targets, so stale contents of the shared array would show), within the
tolerance of the other GPU tests; then on a few-row call (the launch path that
finalizes a row per block) and on calls whose lists overflow a small capacity
(exact counts, truncated ascending rows, ABYSS_WARN_OVERFLOW) through the
array's overflow list and re-list pass.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from abyss_b200 import _lib, ic
from abyss_b200.regforce import ForceResult, RegularForce
from tests.helpers import lists_equal
from tests.test_regforce_gpu import check

pytestmark = pytest.mark.gpu

EPS2 = 1e-8
CAP = 128
SAME_SHAPE = dict(kernel=3, mode=2, threads=128, ipt=2, min_blocks=4)


def _bind(L):
    vp, ip = C.c_void_p, C.c_int
    L.abyss_regular_force_noalloc.argtypes = [ip] + [vp] * 9 + [ip, vp, C.c_double, ip] + [vp] * 6 + [vp]
    L.abyss_regular_force_noalloc.restype = C.c_int


def _device_jset(torch, c):
    dev = torch.device("cuda", 0)
    f64 = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    vm = np.concatenate([c.v.astype(np.float32), c.m.astype(np.float32)[:, None]], axis=1)
    return dict(px=f64(c.x[:, 0]), py=f64(c.x[:, 1]), pz=f64(c.x[:, 2]),
                vm=torch.tensor(np.ascontiguousarray(vm), dtype=torch.float32, device=dev),
                pvx=f64(c.v[:, 0]), pvy=f64(c.v[:, 1]), pvz=f64(c.v[:, 2]), mass=f64(c.m), r2nb=f64(c.r2nb))


def _call(L, torch, js, n, targets, cap=CAP):
    dev = torch.device("cuda", 0)
    m = len(targets)
    t = torch.tensor(np.asarray(targets, np.int32), device=dev)
    out = dict(acc_reg=torch.zeros((m, 3), dtype=torch.float64, device=dev),
               jerk_reg=torch.zeros((m, 3), dtype=torch.float64, device=dev),
               acc_irr=torch.zeros((m, 3), dtype=torch.float64, device=dev),
               jerk_irr=torch.zeros((m, 3), dtype=torch.float64, device=dev),
               nnb=torch.zeros(m, dtype=torch.int32, device=dev),
               list=torch.zeros((m, cap), dtype=torch.int32, device=dev))
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.abyss_regular_force_noalloc(
        n, js["px"].data_ptr(), js["py"].data_ptr(), js["pz"].data_ptr(), js["vm"].data_ptr(),
        js["pvx"].data_ptr(), js["pvy"].data_ptr(), js["pvz"].data_ptr(), js["mass"].data_ptr(),
        js["r2nb"].data_ptr(), m, t.data_ptr(), EPS2, cap, out["acc_reg"].data_ptr(),
        out["jerk_reg"].data_ptr(), out["acc_irr"].data_ptr(), out["jerk_irr"].data_ptr(),
        out["nnb"].data_ptr(), out["list"].data_ptr(), stream)
    torch.cuda.synchronize(dev)
    host = {k: v.cpu().numpy() for k, v in out.items()}
    return rc, ForceResult(host["acc_reg"], host["jerk_reg"], host["acc_irr"], host["jerk_irr"], host["nnb"],
                           host["list"])


def test_noalloc_matches_context_entry_point_twice():
    import torch

    L = _lib.lib()
    _bind(L)
    c = ic.plummer(5000, 77, k_nb=40)
    js = _device_jset(torch, c)
    rf = RegularForce(0)
    try:
        rf.send_to_device(c.m, c.x, c.v, c.r2nb)
        rng = np.random.default_rng(13)
        for call in range(2):
            m = 3000 if call == 0 else 1777
            targets = np.sort(rng.choice(c.n, m, replace=False)).astype(np.int32)
            rc, got = _call(L, torch, js, c.n, targets)
            assert rc == 0, f"call {call}: rc {rc}"
            want = rf.calculate_acceleration(targets, eps2=EPS2, list_cap=CAP, tuning=SAME_SHAPE)
            ref = dict(acc_reg=want.acc_reg, jerk_reg=want.jerk_reg, acc_irr=want.acc_irr,
                       jerk_irr=want.jerk_irr, nnb=want.nnb, list=want.list)
            scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, EPS2, targets)
            check(got, ref, f"noalloc call {call}", scale)
            assert np.array_equal(got.nnb, want.nnb)
            # and against the FP64 oracle itself
            check(got, oracle.reg_force(c.x, c.v, c.m, c.r2nb, EPS2, targets, CAP),
                  f"noalloc call {call} vs oracle", scale)
    finally:
        rf.close()


def test_noalloc_few_rows_and_overflow():
    """m = 64 (at most two rows per SM: each row is finalized by a block of its
    own), then two overflowing calls, one few-row and one many-row, against the
    context entry point on the same shape and the oracle."""
    import torch

    L = _lib.lib()
    _bind(L)
    c = ic.plummer(3000, 79, k_nb=40)
    js = _device_jset(torch, c)
    rf = RegularForce(0)
    try:
        rf.send_to_device(c.m, c.x, c.v, c.r2nb)
        rng = np.random.default_rng(17)
        for m, cap in ((64, CAP), (50, 16), (2500, 16)):
            targets = np.sort(rng.choice(c.n, m, replace=False)).astype(np.int32)
            rc, got = _call(L, torch, js, c.n, targets, cap)
            ref = oracle.reg_force(c.x, c.v, c.m, c.r2nb, EPS2, targets, cap)
            overflowing = ref["overflow"] > 0
            assert overflowing == (cap < 40), (m, cap, ref["overflow"])
            assert rc == (_lib.ABYSS_WARN_OVERFLOW if overflowing else _lib.ABYSS_OK), (m, cap, rc)
            want = rf.calculate_acceleration(targets, eps2=EPS2, list_cap=cap, tuning=SAME_SHAPE)
            assert lists_equal(got.nnb, got.list, want.nnb, want.list), (m, cap)
            scale = oracle.reg_scale(c.x, c.v, c.m, c.r2nb, EPS2, targets)
            check(got, ref, f"noalloc m={m} cap={cap} vs oracle", scale)
    finally:
        rf.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    L = _lib.lib()
    _bind(L)
    c = ic.plummer(5000, 78, k_nb=20)
    js = _device_jset(torch, c)
    rc, _ = _call(L, torch, js, c.n, np.arange(4097, dtype=np.int32))
    assert rc == _lib.ABYSS_ERR_ARG
    # and the next call within the limit still works
    rc, got = _call(L, torch, js, c.n, np.arange(0, 4000, 2, dtype=np.int32))
    assert rc == 0 and got.nnb.shape == (2000,)
