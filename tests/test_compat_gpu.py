"""The reference's drop-in ABI on the GPU, through ctypes, with compute.

The six entry points of src_mpi/cuda/cuda_functions.h:3-10 (CUDA_REAL = float)
and the FP64 spelling of src/cuda/cuda_functions.h:3-10 are called the way the
reference's hosts call them (src_mpi/cuda/CalculateRegularAcceleration.cpp:109,151;
src/cuda/CalculateRegularAcceleration.cpp:130,149):

  * OpenDevice -> SendToDevice(float predicted j-set, the FP32 output of the
    reference's own predictParticleSecondOrder held in the golden vectors)
    -> CalculateAccelerationOnDevice into caller-owned rows of stride 1000
    (NumNeighborMax of src_mpi/def.h:20);
  * SendToDevice_f64 / CalculateAccelerationOnDevice_f64 with the row stride
    set to 200 (the serial build's NumNeighborMax), against the reference's own
    CPU outputs;
  * an overflowed call: exact NumNeighbor, truncated ascending rows, the
    status ABYSS_WARN_OVERFLOW, and the library still usable afterwards.

The float entry point widens its inputs to FP64 and computes as the context
API does; its outputs are FP32, so the force bar adds FP32 output rounding
(2^-24 relative) to the tolerance of tests/test_regforce_gpu.py.  Row entries
past a row's count are never written (checked with a sentinel).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from abyss_b200 import _lib
from tests.helpers import golden

pytestmark = pytest.mark.gpu

_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
SENTINEL = -7


def p(a, t):
    return a.ctypes.data_as(t)


@pytest.fixture(scope="module")
def L():
    lib = _lib.lib()
    r = C.c_int(0)
    lib.OpenDevice(C.byref(r))
    assert lib.abyss_compat_status() == _lib.ABYSS_OK
    yield lib
    lib.abyss_compat_set_list_stride(1000)
    lib.CloseDevice()


def send(L, dtype, m, x, v, r2):
    fn = L.SendToDevice if dtype == np.float32 else L.SendToDevice_f64
    t = _fp if dtype == np.float32 else _dp
    arrs = [np.ascontiguousarray(a, dtype) for a in (m, x, v, r2)]
    mdot = np.zeros_like(arrs[0])
    nnb = C.c_int(arrs[0].shape[0])
    fn(C.byref(nnb), *[p(a, t) for a in arrs], p(mdot, t))
    return L.abyss_compat_status()


def calc(L, dtype, targets, stride):
    fn = L.CalculateAccelerationOnDevice if dtype == np.float32 else L.CalculateAccelerationOnDevice_f64
    t = _fp if dtype == np.float32 else _dp
    m = len(targets)
    tg = np.ascontiguousarray(targets, np.int32)
    acc = np.full((m, 3), np.nan, dtype)
    adot = np.full((m, 3), np.nan, dtype)
    cnt = np.full(m, SENTINEL, np.int32)
    lst = np.full((m, stride), SENTINEL, np.int32)
    nt = C.c_int(m)
    fn(C.byref(nt), p(tg, _ip), p(acc, t), p(adot, t), p(cnt, _ip), p(lst, _ip))
    return L.abyss_compat_status(), acc, adot, cnt, lst


def check_rows(tag, cnt, lst, stride, ref_nnb, ref_list):
    assert np.array_equal(cnt, ref_nnb), f"{tag}: neighbour counts differ"
    for r in range(len(cnt)):
        k = min(int(cnt[r]), stride)
        assert np.array_equal(lst[r, :k], ref_list[r, :k]), f"{tag}: row {r} differs"
        assert np.all(lst[r, k:] == SENTINEL), f"{tag}: row {r} written past its count"


def check_force(tag, got, ref, scale, tol, out_eps):
    """Per row |d| <= tol |ref| + 0.1 tol A + out_eps |ref| (output rounding)."""
    d = np.linalg.norm(got.astype(np.float64) - ref, axis=1)
    n = np.linalg.norm(ref, axis=1)
    use = d / np.maximum((tol + out_eps) * n + 0.1 * tol * scale, 1e-300)
    rel = d / np.maximum(n, 1e-300)
    print(f"{tag}: rel max {rel.max():.2e} med {np.median(rel):.2e} bound use {use.max():.2f}")
    assert use.max() <= 1.0, f"{tag}: {use.max():.2f} x the bound"


def test_float_abi_stride_1000(L):
    g = golden("ref_plummer1024_s1.npz")
    # the reference's MPI host sends FP32: predicted x, v (predictParticleSecondOrder),
    # masses and squared neighbour radii (CalculateRegularAcceleration.cpp:360-420)
    assert send(L, np.float32, g["m"], g["px32"], g["pv32"], g["r2nb"]) == _lib.ABYSS_OK
    t = g["targets"]
    st, acc, adot, cnt, lst = calc(L, np.float32, t, 1000)
    assert st == _lib.ABYSS_OK
    # the oracle on the same float-rounded inputs, widened to FP64, no softening
    f = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    px, pv, m, r2 = f(g["px32"]), f(g["pv32"]), f(g["m"]), f(g["r2nb"])
    ref = oracle.reg_force(px, pv, m, r2, 0.0, t, 1000, with_irr=False)
    check_rows("float/1000", cnt, lst, 1000, ref["nnb"], ref["list"])
    sa, sj = oracle.reg_scale(px, pv, m, r2, 0.0, t)
    check_force("float acc", acc, ref["acc_reg"], sa, 1e-6, 2.0 ** -23)
    check_force("float adot", adot, ref["jerk_reg"], sj, 1e-5, 2.0 ** -23)


def test_f64_abi_stride_200_against_reference_outputs(L):
    """The serial build's FP64 spelling, rows of 200, against the reference's
    own CPU regular force (golden vectors, eps = 0)."""
    assert L.abyss_compat_set_list_stride(200) == _lib.ABYSS_OK
    try:
        for name in ("ref_plummer1024_s1.npz", "ref_king2048_s3.npz"):
            g = golden(name)
            assert send(L, np.float64, g["m"], g["px"], g["pv"], g["r2nb"]) == _lib.ABYSS_OK
            t = g["targets"]
            st, acc, adot, cnt, lst = calc(L, np.float64, t, 200)
            assert st == _lib.ABYSS_OK, name
            ref_list = np.full((len(t), 200), -1, np.int32)
            w = min(200, g["out_list"].shape[1])
            ref_list[:, :w] = g["out_list"][:, :w]
            check_rows(f"f64/200 {name}", cnt, lst, 200, g["out_nnb"], ref_list)
            sa, sj = oracle.reg_scale(g["px"], g["pv"], g["m"], g["r2nb"], 0.0, t)
            check_force(f"f64 acc {name}", acc, g["out_a_reg"][:, :, 0], sa, 1e-6, 0.0)
            check_force(f"f64 adot {name}", adot, g["out_a_reg"][:, :, 1], sj, 1e-5, 0.0)
    finally:
        L.abyss_compat_set_list_stride(1000)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_overflow_keeps_exact_counts_and_truncates(L, dtype):
    """Rows longer than the stride: NumNeighbor exact, the first `stride`
    neighbours in ascending order, ABYSS_WARN_OVERFLOW (the reference asserts
    in device code instead, cuda_kernels.cu:363,432); the next call is clean."""
    g = golden("ref_king2048_s3.npz")  # about 100 neighbours per target
    stride = 40
    assert L.abyss_compat_set_list_stride(stride) == _lib.ABYSS_OK
    try:
        assert send(L, dtype, g["m"], g["px"], g["pv"], g["r2nb"]) == _lib.ABYSS_OK
        t = g["targets"][:300]
        st, acc, adot, cnt, lst = calc(L, dtype, t, stride)
        assert st == _lib.ABYSS_WARN_OVERFLOW
        f = lambda a: np.asarray(a, dtype).astype(np.float64)  # noqa: E731
        px, pv, m, r2 = f(g["px"]), f(g["pv"]), f(g["m"]), f(g["r2nb"])
        ref = oracle.reg_force(px, pv, m, r2, 0.0, t, stride, with_irr=False)
        assert ref["overflow"] > 0 and np.all(cnt > stride)
        check_rows(f"overflow {dtype.__name__}", cnt, lst, stride, ref["nnb"], ref["list"])
        for r in range(len(t)):
            assert np.all(np.diff(lst[r]) > 0)
        # a regular force that excludes every listed and unlisted neighbour alike
        sa, _ = oracle.reg_scale(px, pv, m, r2, 0.0, t)
        check_force(f"overflow acc {dtype.__name__}", acc, ref["acc_reg"], sa, 1e-6,
                    2.0 ** -23 if dtype == np.float32 else 0.0)
    finally:
        L.abyss_compat_set_list_stride(1000)
    # the next call, with room, is clean
    st, *_ = calc(L, dtype, g["targets"][:10], 1000)
    assert st == _lib.ABYSS_OK


def test_bad_calls_report_status_and_keep_the_device(L):
    g = golden("ref_plummer1024_s1.npz")
    assert send(L, np.float64, g["m"], g["px"], g["pv"], g["r2nb"]) == _lib.ABYSS_OK
    # NumTarget above NNB: the reference asserts (cuda_my_acceleration.cu:104)
    st, *_ = calc(L, np.float64, np.arange(1025, dtype=np.int32) % 1024, 1000)
    assert st == _lib.ABYSS_ERR_ARG
    # a target index outside the j-set
    st, *_ = calc(L, np.float64, np.array([0, 1024], np.int32), 1000)
    assert st == _lib.ABYSS_ERR_ARG
    st, *_ = calc(L, np.float64, g["targets"][:5], 1000)
    assert st == _lib.ABYSS_OK
    # OpenDevice on an open device warns and changes nothing
    r = C.c_int(0)
    L.OpenDevice(C.byref(r))
    st, *_ = calc(L, np.float64, g["targets"][:5], 1000)
    assert st == _lib.ABYSS_OK
