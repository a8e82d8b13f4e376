"""ctypes binding of libabyss_reg.so (include/abyss_reg.h, include/abyss_reg_compat.h).

The library is built in-tree by ``abyss_b200/csrc/Makefile``; importing this
module never builds or falls back: if the shared object is missing, ``lib()``
raises, so nothing can run the path without the CUDA code.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libabyss_reg.so")

ABYSS_OK = 0
ABYSS_WARN_OVERFLOW = 1
ABYSS_ERR_ARG = -1
ABYSS_ERR_CUDA = -2
ABYSS_ERR_OOM = -3
ABYSS_ERR_TIMEOUT = -4
ABYSS_ERR_STATE = -5
ABYSS_ERR_NODEVICE = -6

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class Tuning(C.Structure):
    """abyss_tuning: launch shape (zero = automatic)."""

    _fields_ = [("kernel", C.c_int), ("mode", C.c_int), ("threads", C.c_int), ("ipt", C.c_int),
                ("j_split", C.c_int), ("grid", C.c_int), ("unroll", C.c_int), ("min_blocks", C.c_int)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class ACParams(C.Structure):
    """abyss_ac_params (include/abyss_ac.h)."""

    _fields_ = [("eps2", C.c_double), ("eta_reg", C.c_double), ("eta_irr", C.c_double),
                ("fix_nb", C.c_int), ("nb_max", C.c_int), ("t_end", C.c_double), ("threads", C.c_int)]


class ACStats(C.Structure):
    """abyss_ac_stats (include/abyss_ac.h)."""

    _fields_ = [("blocks", C.c_longlong), ("reg_steps", C.c_longlong), ("irr_steps", C.c_longlong),
                ("irr_levels", C.c_longlong), ("radius_retries", C.c_longlong), ("pairs", C.c_double),
                ("sec_reg_gpu", C.c_double), ("sec_reg_host", C.c_double), ("sec_irr", C.c_double),
                ("sec_init", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_LIB = None


class AbyssError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"abyss error {code}: {msg}")
        self.code = code


def lib():
    """Load libabyss_reg.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                           "g.build()'` or `make -C abyss_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    L.abyss_create.argtypes = [C.c_int, C.POINTER(_vp)]
    L.abyss_destroy.argtypes = [_vp]
    L.abyss_last_error.argtypes = [_vp]
    L.abyss_last_error.restype = C.c_char_p
    L.abyss_stream.argtypes = [_vp]
    L.abyss_stream.restype = _vp
    L.abyss_synchronize.argtypes = [_vp]
    L.abyss_set_wait.argtypes = [_vp, C.c_int]
    L.abyss_reserve.argtypes = [_vp, C.c_int, C.c_int, C.c_int]
    L.abyss_upload_state.argtypes = [_vp, C.c_int] + [_dp] * 7
    L.abyss_predict.argtypes = [_vp, C.c_double, C.c_double]
    L.abyss_upload_predicted.argtypes = [_vp, C.c_int] + [_dp] * 4
    L.abyss_read_predicted.argtypes = [_vp, _dp, _dp, _fp]
    L.abyss_set_targets.argtypes = [_vp, C.c_int, _ip]
    L.abyss_launch.argtypes = [_vp, C.c_double, C.c_int, C.POINTER(Tuning)]
    L.abyss_fetch.argtypes = [_vp, _dp, _dp, _dp, _dp, _ip, _ip, _ip]
    L.abyss_regular_force.argtypes = [_vp, C.c_int, _ip, C.c_double, C.c_int, C.POINTER(Tuning),
                                      _dp, _dp, _dp, _dp, _ip, _ip, _ip]
    L.abyss_last_plan.argtypes = [_vp, C.POINTER(Tuning), _ip]
    L.abyss_last_order.argtypes = [_vp, _ip]
    L.abyss_set_profiling.argtypes = [_vp, C.c_int]
    L.abyss_last_timing.argtypes = [_vp, _fp]
    L.abyss_set_tuning_table.argtypes = [_vp, C.c_int, _ip, C.POINTER(Tuning)]
    L.abyss_energy.argtypes = [_vp, C.c_int, _dp, _dp, _dp, C.c_double, _dp]
    L.abyss_init_derivs23.argtypes = [_vp, C.c_int] + [_dp] * 6 + [C.c_double] + [_dp] * 4
    # state I/O (include/abyss_io.h)
    L.abyss_read_reference_ic.argtypes = [C.c_char_p, _ip, _dp, _dp, _dp]
    L.abyss_ac_write_snapshot.argtypes = [_vp, C.c_char_p, C.c_double, C.c_double]
    L.abyss_ac_save.argtypes = [_vp, C.c_char_p]
    L.abyss_ac_load.argtypes = [_vp, C.c_char_p, C.c_int, C.POINTER(_vp)]
    L.abyss_ac_info.argtypes = [_vp, _ip, C.POINTER(ACParams)]
    L.abyss_tile_variant.argtypes = [C.c_int, _ip]
    # reference-compatible drop-in
    L.InitializeDevice.argtypes = [_ip]
    L.OpenDevice.argtypes = [_ip]
    L.CloseDevice.argtypes = []
    L.ProfileDevice.argtypes = [_ip]
    L.SendToDevice.argtypes = [_ip, _fp, _fp, _fp, _fp, _fp]
    L.CalculateAccelerationOnDevice.argtypes = [_ip, _ip, _fp, _fp, _ip, _ip]
    L.SendToDevice_f64.argtypes = [_ip, _dp, _dp, _dp, _dp, _dp]
    L.CalculateAccelerationOnDevice_f64.argtypes = [_ip, _ip, _dp, _dp, _ip, _ip]
    L.abyss_compat_set_list_stride.argtypes = [C.c_int]
    L.abyss_compat_status.argtypes = []
    # host integrator rules (include/abyss_host.h)
    L.abyss_host_predict.argtypes = [_dp] * 4 + [C.c_double, C.c_double, _dp, _dp]
    L.abyss_host_time_step_reg.argtypes = [_dp, C.c_double]
    L.abyss_host_time_step_reg.restype = C.c_double
    L.abyss_host_time_step_irr.argtypes = [_dp, _dp, C.c_double]
    L.abyss_host_time_step_irr.restype = C.c_double
    L.abyss_host_block_time_step.argtypes = [C.c_double, C.c_double, C.c_int, _ip,
                                             C.POINTER(C.c_ulonglong), _dp]
    L.abyss_host_regular_correct.argtypes = ([C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                              C.c_double, C.c_int, C.c_double, _dp, C.c_int, _ip, C.c_int,
                                              _ip] + [_dp] * 8)
    L.abyss_host_irregular_steps.argtypes = ([C.c_int] + [_dp] * 9 + [_ip, _ip, C.c_int, C.c_double, C.c_double,
                                                                      C.c_int, _ip] + [_dp] * 4)
    L.abyss_host_time_level_irr.argtypes = [C.c_double, C.c_int, C.c_double, C.c_int, _dp, _dp, C.c_ulonglong,
                                            C.c_ulonglong, C.c_ulonglong, C.c_int, _ip, _dp,
                                            C.POINTER(C.c_ulonglong)]
    L.abyss_host_time_level_reg.argtypes = [C.c_double, C.c_int, C.c_ulonglong, C.c_double, C.c_int, _dp,
                                            C.c_double, C.c_ulonglong, _ip, _dp, C.POINTER(C.c_ulonglong), _ip]
    L.abyss_host_initial_time_steps.argtypes = [C.c_double, C.c_int, C.c_ulonglong, C.c_double, C.c_double, C.c_int,
                                                _dp, _dp, _dp, _ip, _dp, C.POINTER(C.c_ulonglong), _ip, _dp,
                                                C.POINTER(C.c_ulonglong)]
    L.abyss_host_initial_time_steps.restype = None
    L.abyss_host_update_radius.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int]
    L.abyss_host_update_radius.restype = C.c_double
    # host integrator (include/abyss_ac.h)
    L.abyss_ac_create.argtypes = [_vp, C.POINTER(ACParams), C.c_int, _dp, _dp, _dp, _dp, C.POINTER(_vp)]
    L.abyss_ac_destroy.argtypes = [_vp]
    L.abyss_ac_advance_block.argtypes = [_vp, _ip]
    L.abyss_ac_run.argtypes = [_vp, C.c_double]
    L.abyss_ac_time.argtypes = [_vp]
    L.abyss_ac_time.restype = C.c_double
    L.abyss_ac_get_state.argtypes = [_vp, _dp, _dp, _ip, _dp]
    L.abyss_ac_energy.argtypes = [_vp, _dp]
    L.abyss_ac_get_stats.argtypes = [_vp, C.POINTER(ACStats)]
    L.abyss_ac_last_regular.argtypes = [_vp, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_int]
    L.abyss_ac_begin_block.argtypes = [_vp, _ip, _dp, _dp, _ip]
    L.abyss_ac_block_targets.argtypes = [_vp, _ip]
    L.abyss_ac_block_state.argtypes = [_vp] + [_dp] * 7
    L.abyss_ac_end_block.argtypes = [_vp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_int, _ip]
    L.abyss_ac_last_error.argtypes = [_vp]
    L.abyss_ac_last_error.restype = C.c_char_p
    L.abyss_ac_host_timers.argtypes = [_vp, _dp]
    # irregular steps on the device (include/abyss_irr.h)
    _ull = C.POINTER(C.c_ulonglong)
    L.abyss_ac_set_device_irregular.argtypes = [_vp, C.c_int]
    L.abyss_ac_device_irregular_info.argtypes = [_vp, _ip, C.POINTER(C.c_longlong), _dp, C.POINTER(C.c_longlong)]
    L.abyss_ac_set_device_resident.argtypes = [_vp, C.c_int]
    L.abyss_ac_device_resident_info.argtypes = [_vp, _ip, C.POINTER(C.c_longlong), _dp]
    L.abyss_device_irregular_steps.argtypes = ([C.c_int, C.c_int] + [_dp] * 9 + [_ip, _ip, C.c_int, C.c_double,
                                               C.c_double, C.c_int, C.c_double, _ip, _ull, _ull, C.c_int, _ip] +
                                               [_dp] * 4 + [_ip, _dp, _ull])
    _LIB = L
    return L


def ptr(a, t=_dp):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)
