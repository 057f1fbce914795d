"""ctypes declarations of the C ABI in include/atvb.h (libatvb.so)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libatvb.so")

ATVB_OK = 0
ATVB_ERR_INVALID = 1
ATVB_ERR_CUDA = 2
ATVB_ERR_OVERFLOW = 3
ATVB_ERR_STATE = 4
ATVB_ERR_NOMEM = 5
ATVB_ERR_NOTFOUND = 6
ATVB_ERR_PHYSICS = 7

# atvb_scalars.status_bits (sticky until clear_status)
STATUS_ROW_OVERFLOW = 1
STATUS_BOX_RANGE = 2
STATUS_NEARQ_LOST = 4
STATUS_NONFINITE = 8
STATUS_FORCE_RANGE = 16

FP64, MIXED = 0, 1
NVE, NOSE_HOOVER, LANGEVIN = 0, 1, 2


class DeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("reserved", C.c_int * 7)]


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("box", C.c_double * 9),
        ("precision", C.c_int32),
        ("nl_cutoff", C.c_double),
        ("nl_skin", C.c_double),
        ("nl_every", C.c_int32),
        ("nl_delay", C.c_int32),
        ("nl_check", C.c_int32),
        ("lj_enabled", C.c_int32),
        ("lj_epsilon", C.c_double),
        ("lj_sigma", C.c_double),
        ("lj_cutoff", C.c_double),
        ("coul_enabled", C.c_int32),
        ("coul_alpha", C.c_double),
        ("coul_cutoff", C.c_double),
        ("pme_enabled", C.c_int32),
        ("pme_alpha", C.c_double),
        ("pme_grid_spacing", C.c_double),
        ("pme_order", C.c_int32),
        ("pme_grid", C.c_int32 * 3),
        ("dt", C.c_double),
        ("thermostat", C.c_int32),
        ("temperature", C.c_double),
        ("tau", C.c_double),
        ("damp", C.c_double),
        ("seed", C.c_uint32),
        ("stress_required", C.c_int32),
        ("history_capacity", C.c_int32),
    ]


_dp = C.POINTER(C.c_double)


class SoaView(C.Structure):
    _fields_ = [
        ("x", _dp), ("y", _dp), ("z", _dp),
        ("vx", _dp), ("vy", _dp), ("vz", _dp),
        ("fx", _dp), ("fy", _dp), ("fz", _dp),
        ("mass", _dp), ("charge", _dp),
        ("type", C.POINTER(C.c_int32)),
        ("tag", C.POINTER(C.c_int64)),
    ]


class Scalars(C.Structure):
    _fields_ = [
        ("energy", C.c_double),
        ("energy_pair", C.c_double),
        ("energy_lj", C.c_double),
        ("energy_coul", C.c_double),
        ("energy_recip", C.c_double),
        ("energy_const", C.c_double),
        ("kinetic", C.c_double),
        ("conserved", C.c_double),
        ("stress", C.c_double * 6),
        ("nh_xi", C.c_double),
        ("step", C.c_int64),
        ("rebuilds", C.c_int64),
        ("max_neighbors", C.c_int32),
        ("status", C.c_int32),
        ("list_pairs", C.c_int64),
        ("box", C.c_double * 3),
        ("pressure", C.c_double),
        ("status_bits", C.c_uint32),
        ("halted", C.c_int32),
    ]


class NptDesc(C.Structure):
    """atvb_npt_desc: md::NoseHooverNPT parameters."""
    _fields_ = [
        ("T_start", C.c_double),
        ("T_stop", C.c_double),
        ("tau_T", C.c_double),
        ("P_target", C.c_double),
        ("tau_P", C.c_double),
        ("drag", C.c_double),
        ("mtchain", C.c_int32),
        ("mpchain", C.c_int32),
        ("couple", C.c_int32 * 3),
        ("nfirst", C.c_int64),
        ("nlast", C.c_int64),
    ]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("total_ms", C.c_double), ("launches", C.c_int64)]


class RequestResult(C.Structure):
    _fields_ = [
        ("id", C.c_int64),
        ("state", C.c_int32),
        ("steps_done", C.c_int32),
        ("t_submit", C.c_double),
        ("t_start", C.c_double),
        ("t_done", C.c_double),
        ("scalars", Scalars),
    ]


# name -> (restype, argtypes); every function declared in include/atvb.h
_vp = C.c_void_p


class DeviceFrame(C.Structure):
    """atvb_device_frame: the system's device arrays as a component sees them."""
    _fields_ = [("n_atoms", C.c_int64)] + [(k, C.c_void_p) for k in (
        "x", "y", "z", "vx", "vy", "vz", "mass", "charge", "tag", "fx", "fy", "fz",
        "energy", "virial", "box")]


class LaunchCtx(C.Structure):
    """atvb_launch_ctx: stream, phase, cumulative step, device frame."""
    _fields_ = [("stream", C.c_void_p), ("phase", C.c_int32), ("reserved", C.c_int32),
                ("step", C.c_int64), ("frame", DeviceFrame)]


# atvb_component_fn: int (*)(void* user, const atvb_launch_ctx* ctx)
COMPONENT_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(LaunchCtx))
SIGNATURES = {
    "atvb_abi_version": (C.c_int, []),
    "atvb_last_error": (C.c_char_p, []),
    "atvb_ctx_create": (C.c_int, [C.POINTER(DeviceOpts), C.POINTER(_vp)]),
    "atvb_ctx_destroy": (C.c_int, [_vp]),
    "atvb_system_create": (C.c_int, [_vp, C.POINTER(SystemDesc), C.POINTER(_vp)]),
    "atvb_system_destroy": (C.c_int, [_vp]),
    "atvb_system_upload": (C.c_int, [_vp, C.POINTER(SoaView)]),
    "atvb_system_compute_forces": (C.c_int, [_vp]),
    "atvb_system_step": (C.c_int, [_vp, C.c_int32]),
    "atvb_system_step_timed": (C.c_int, [_vp, C.c_int32, _dp, _dp]),
    "atvb_system_download": (C.c_int, [_vp, C.POINTER(SoaView), C.POINTER(Scalars)]),
    "atvb_system_scalars": (C.c_int, [_vp, C.POINTER(Scalars)]),
    "atvb_system_run": (C.c_int, [_vp, C.POINTER(SoaView), C.c_int32, C.POINTER(Scalars)]),
    "atvb_system_energy_history": (C.c_int, [_vp, _dp, C.c_int32, C.POINTER(C.c_int32)]),
    "atvb_system_pairs": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.c_int64, C.POINTER(C.c_int64)]),
    "atvb_system_clear_status": (C.c_int, [_vp]),
    "atvb_system_set_stop_on_nan": (C.c_int, [_vp, C.c_int32]),
    "atvb_system_set_langevin_ramp": (C.c_int, [_vp, C.c_double, C.c_int64, C.c_int64]),
    # build / launch / destroy are COMPONENT_FN callbacks (or None)
    "atvb_system_add_component": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp]),
    "atvb_system_set_capacity": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "atvb_batch_clear_status": (C.c_int, [_vp, C.c_int32]),
    "atvb_batch_set_stop_on_nan": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "atvb_batch_set_langevin_ramp": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_int64,
                                               C.c_int64]),
    "atvb_system_profile": (C.c_int, [_vp, C.c_int32]),
    "atvb_system_profile_read": (C.c_int, [_vp, C.POINTER(KernelTime), C.c_int32,
                                           C.POINTER(C.c_int32)]),
    "atvb_system_set_pair_lanes": (C.c_int, [_vp, C.c_int32]),
    "atvb_system_launch_count": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "atvb_system_stream": (_vp, [_vp]),
    "atvb_batch_create": (C.c_int, [_vp, C.POINTER(SystemDesc), C.c_int32, C.POINTER(_vp)]),
    "atvb_batch_destroy": (C.c_int, [_vp]),
    "atvb_batch_upload": (C.c_int, [_vp, C.c_int32, C.POINTER(SoaView)]),
    "atvb_batch_compute_forces": (C.c_int, [_vp]),
    "atvb_batch_step": (C.c_int, [_vp, C.c_int32]),
    "atvb_batch_download": (C.c_int, [_vp, C.c_int32, C.POINTER(SoaView), C.POINTER(Scalars)]),
    "atvb_batch_autotune": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "atvb_batch_launch_count": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "atvb_batch_set_lj_types": (C.c_int, [_vp, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]),
    "atvb_batch_set_special_bonds": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_double),
                                               C.POINTER(C.c_double), C.c_int64,
                                               C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "atvb_system_set_npt": (C.c_int, [_vp, C.POINTER(NptDesc)]),
    "atvb_system_set_barostat": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double]),
    "atvb_system_set_nve_limit": (C.c_int, [_vp, C.c_double]),
    "atvb_system_set_deform": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "atvb_batch_set_nve_limit": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "atvb_batch_set_deform": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_double]),
    "atvb_batch_set_barostat": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "atvb_server_keep_checkpoints": (C.c_int, [_vp, C.c_int32]),
    "atvb_server_suspend": (C.c_int, [_vp, C.c_int64]),
    "atvb_server_resume": (C.c_int, [_vp, C.c_int64, C.c_int32]),
    "atvb_server_checkpoint": (C.c_int, [_vp, C.c_int64, _vp, C.c_int64,
                                         C.POINTER(C.c_int64)]),
    "atvb_server_submit_checkpoint": (C.c_int, [_vp, C.POINTER(SystemDesc), _vp, C.c_int64,
                                                C.c_int32, C.POINTER(C.c_int64)]),
    "atvb_system_set_snapshots": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "atvb_system_snapshot_poll": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int64)] +
                                  [C.POINTER(C.c_double)] * 7 +
                                  [C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "atvb_system_checkpoint_size": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "atvb_system_save": (C.c_int, [_vp, _vp, C.c_int64]),
    "atvb_system_restore": (C.c_int, [_vp, _vp, C.c_int64]),
    "atvb_batch_checkpoint_size": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int64)]),
    "atvb_batch_save": (C.c_int, [_vp, C.c_int32, _vp, C.c_int64]),
    "atvb_batch_restore": (C.c_int, [_vp, C.c_int32, _vp, C.c_int64]),
    "atvb_batch_set_npt": (C.c_int, [_vp, C.c_int32, C.POINTER(NptDesc)]),
    "atvb_system_set_lj_types": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]),
    "atvb_system_set_special_bonds": (C.c_int, [_vp, C.POINTER(C.c_double),
                                                C.POINTER(C.c_double), C.c_int64,
                                                C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "atvb_batch_profile": (C.c_int, [_vp, C.c_int32]),
    "atvb_batch_profile_read": (C.c_int, [_vp, C.POINTER(KernelTime), C.c_int32,
                                          C.POINTER(C.c_int32)]),
    "atvb_server_create": (C.c_int, [_vp, C.c_size_t, C.c_int32, C.POINTER(_vp)]),
    "atvb_server_destroy": (C.c_int, [_vp]),
    "atvb_server_submit": (C.c_int, [_vp, C.POINTER(SystemDesc), C.POINTER(SoaView),
                                     C.c_int32, C.POINTER(C.c_int64)]),
    "atvb_server_cancel": (C.c_int, [_vp, C.c_int64]),
    "atvb_server_set_limits": (C.c_int, [_vp, C.c_int64]),
    "atvb_server_tick": (C.c_int, [_vp, C.c_int32]),
    "atvb_server_poll": (C.c_int, [_vp, C.c_int64, C.POINTER(RequestResult)]),
    "atvb_server_collect": (C.c_int, [_vp, C.c_int64, C.POINTER(SoaView),
                                      C.POINTER(RequestResult)]),
    "atvb_server_stats": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_size_t)]),
    "atvb_request_bytes": (C.c_int, [C.POINTER(SystemDesc), C.POINTER(C.c_size_t)]),
    "atvb_pair_forces_static": (C.c_int, [C.POINTER(SystemDesc)] + [C.c_void_p] * 9),
}

_lib = None


class AtvbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"atvb error {code}: {msg}")
        self.code = code


class PhysicsError(AtvbError):
    """A sticky status bit is set (ATVB_ERR_PHYSICS): some step ran on wrong
    or non-finite physics.  `result` holds what the call returned anyway."""

    def __init__(self, code: int, msg: str, result=None):
        super().__init__(code, msg)
        self.result = result


def load(path: str | None = None):
    """Load libatvb.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python -m atomiverse_b200.build` "
            "(the CUDA library is the only implementation of this path)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != ATVB_OK:
        msg = load().atvb_last_error()
        text = msg.decode() if msg else ""
        if rc == ATVB_ERR_PHYSICS:
            raise PhysicsError(rc, text)
        raise AtvbError(rc, text)


def check_status(rc: int, result, strict: bool):
    """check() for calls that fill their outputs before reporting a sticky
    status bit: with strict=False that code is not an error."""
    if rc == ATVB_ERR_PHYSICS and not strict:
        return result
    try:
        check(rc)
    except PhysicsError as e:
        e.result = result
        raise
    return result
