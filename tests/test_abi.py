"""The C-ABI library loads and exports every function that include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re

import pytest

from abyss_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(INC)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INC, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_headers_declare_the_reference_abi():
    names = declared_functions()
    for ref in ("InitializeDevice", "OpenDevice", "CloseDevice", "ProfileDevice", "SendToDevice",
                "CalculateAccelerationOnDevice"):
        assert ref in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    L = C.CDLL(_lib.LIB_PATH)
    assert hasattr(L, name), f"{name} declared in include/ but not exported"


def test_loader_binds_everything():
    L = _lib.lib()
    for name in declared_functions():
        getattr(L, name)


def test_context_creation_without_gpu_reports_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.lib()
    h = C.c_void_p()
    rc = L.abyss_create(0, C.byref(h))
    assert rc == _lib.ABYSS_ERR_NODEVICE


def _zero_args(argtypes):
    args = []
    for t in argtypes:
        if t in (C.c_int, C.c_uint, C.c_longlong, C.c_ulonglong):
            args.append(0)
        elif t in (C.c_double, C.c_float):
            args.append(0.0)
        else:
            args.append(None)
    return args


def test_null_handles_return_errors():
    """Every call that takes a context, ensemble or integrator handle, given a
    null handle and null or zero arguments, answers with an error code (or its
    documented null result) and touches nothing: the boundary never traps."""
    from abyss_b200 import ensemble, serve

    L = _lib.lib()
    ensemble._bind(L)
    serve._bind(L)
    called = 0
    for name in declared_functions():
        if not name.startswith("abyss_") or name.startswith(("abyss_host_", "abyss_compat_")):
            continue
        f = getattr(L, name)
        if not f.argtypes:
            continue
        r = f(*_zero_args(f.argtypes))
        called += 1
        if name in ("abyss_ac_destroy", "abyss_ens_destroy"):
            assert r in (0, _lib.ABYSS_ERR_ARG), name  # deleting nothing is allowed
        elif name in ("abyss_last_error", "abyss_ac_last_error"):
            assert r and r.startswith(b"null"), name
        elif name in ("abyss_stream",):
            assert r is None
        elif name in ("abyss_ac_time", "abyss_ens_device_bytes", "abyss_ens_list_cap"):
            assert r == 0, name
        else:
            assert r == _lib.ABYSS_ERR_ARG, (name, r)
    assert called > 50


def test_reference_entry_points_with_null_arguments():
    """The reference's six entry points (void in its ABI) report bad calls
    through abyss_compat_status() instead of trapping."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.lib()
    expect = {"InitializeDevice": _lib.ABYSS_ERR_NODEVICE, "OpenDevice": _lib.ABYSS_ERR_NODEVICE,
              "SendToDevice": _lib.ABYSS_ERR_ARG, "SendToDevice_f64": _lib.ABYSS_ERR_ARG,
              "CalculateAccelerationOnDevice": _lib.ABYSS_ERR_STATE,
              "CalculateAccelerationOnDevice_f64": _lib.ABYSS_ERR_STATE}
    for name, status in expect.items():
        f = getattr(L, name)
        f(*([None] * len(f.argtypes or [])))
        assert L.abyss_compat_status() == status, name
    # with no device open these two do nothing
    for name in ("ProfileDevice", "CloseDevice"):
        f = getattr(L, name)
        f(*([None] * len(f.argtypes or [])))
