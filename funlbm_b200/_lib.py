"""ctypes binding of ``liblbm_b200.so`` (declared in ``include/funlbm_b200.h``).

The library is the only compute path: if it is missing or cannot be loaded,
every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
# FUNLBM_B200_CHECKED=1 selects the bounds-checked build (python -m
# funlbm_b200.build --checked): same results, index checks in every kernel
LIB_PATH = os.path.join(PKG, "liblbm_b200_checked.so" if os.environ.get("FUNLBM_B200_CHECKED") == "1"
                        else "liblbm_b200.so")

LBM_OK = 0
LBM_ERR_INVALID = 1
LBM_ERR_UNSUPPORTED = 2
LBM_ERR_CUDA = 3

LBM_STATUS_RHO_BAD = 0x1
LBM_STATUS_U_BAD = 0x2
LBM_STATUS_STENCIL_EMPTY = 0x4
LBM_STATUS_WAIT_TIMEOUT = 0x8
LBM_STATUS_DRAIN_FAILED = 0x10

STORAGE = {"fp32": 0, "fp16s": 1, "bf16s": 2, "fp64": 3}
SPREAD_NOALLOC_MAX_NODES = 1 << 22
RIGID_WALL = 1
RIGID_UPDATE = 2

c_float3 = ctypes.c_float * 3


class LbmLattice(ctypes.Structure):
    _fields_ = [
        ("q", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("face", ctypes.c_int32 * 6),
        ("face_uw", (ctypes.c_float * 3) * 6),
        ("tau", ctypes.c_float),
        ("cs2", ctypes.c_float),
        ("storage", ctypes.c_int32),
        ("re_mu", ctypes.c_float),
        ("neq_profile", ctypes.c_void_p),
        ("step_nodes", ctypes.c_int32),
        ("step_threads", ctypes.c_int32),
        ("pz", ctypes.c_int32),
    ]


class LbmForce(ctypes.Structure):
    _fields_ = [
        ("old_uniform", ctypes.c_float * 3),
        ("new_uniform", ctypes.c_float * 3),
        ("old_field", ctypes.c_void_p),
        ("new_field", ctypes.c_void_p),
        ("old_chunks", ctypes.c_void_p),
        ("new_chunks", ctypes.c_void_p),
    ]


class LbmObserve(ctypes.Structure):
    _fields_ = [("f", ctypes.c_void_p), ("rho", ctypes.c_void_p), ("u", ctypes.c_void_p)]


class LbmParticles(ctypes.Structure):
    _fields_ = [
        ("n_particles", ctypes.c_int32),
        ("n_markers", ctypes.c_int32),
        ("marker_offset", ctypes.c_void_p),
        ("marker_owner", ctypes.c_void_p),
        ("lagrange", ctypes.c_void_p),
        ("lx", ctypes.c_void_p),
        ("lu", ctypes.c_void_p),
        ("lF", ctypes.c_void_p),
        ("lrou", ctypes.c_void_p),
        ("lm", ctypes.c_void_p),
        ("cx", ctypes.c_void_p),
        ("cu", ctypes.c_void_p),
        ("cw", ctypes.c_void_p),
        ("cF", ctypes.c_void_p),
        ("cT", ctypes.c_void_p),
        ("angle", ctypes.c_void_p),
        ("mass", ctypes.c_void_p),
        ("inertia", ctypes.c_void_p),
        ("rou", ctypes.c_void_p),
        ("fp64", ctypes.c_int32),
        ("extreme", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_LAT = ctypes.POINTER(LbmLattice)
_FORCE = ctypes.POINTER(LbmForce)
_OBS = ctypes.POINTER(LbmObserve)
_PART = ctypes.POINTER(LbmParticles)
I = ctypes.c_int
F = ctypes.c_float

# name -> (restype, argtypes); every name is declared in include/funlbm_b200.h
SIGNATURES = {
    "lbm_face_plane_floats": (ctypes.c_size_t, [_LAT]),
    "lbm_lattice_check": (I, [_LAT]),
    "lbm_flow_init": (I, [_LAT, _P, _P, _P, _P]),
    "lbm_flow_step": (I, [_LAT, _P, _P, _FORCE, _P, _P, _OBS, _P, _P]),
    "lbm_flow_stats": (I, [_LAT, _P, _FORCE, _P, _P, _P, _P]),
    "lbm_batch_entry_bytes": (ctypes.c_size_t, []),
    "lbm_batch_pack": (I, [_LAT, _P, _P, _FORCE, _P, _P, _P, ctypes.c_int32, _P, _P]),
    "lbm_flow_step_batch": (I, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                _P, _P, ctypes.c_int32, ctypes.c_uint32, _P]),
    "lbm_collide": (I, [_LAT, _P, _P, _P, _P, _P]),
    "lbm_stream": (I, [_LAT, _P, _P, _P, _P, _P]),
    "lbm_moments": (I, [_LAT, _P, _P, _P, _P, _P, _P, _P]),
    "lbm_add_force": (I, [_LAT, _P, _P, _P, _P]),
    "ibm_interpolate": (I, [_LAT, _P, _FORCE, _P, _P, _P, _PART, F, ctypes.c_int32, _P, _P]),
    "rigid_wall_and_update": (I, [_LAT, _PART, ctypes.c_int32, F, F, F, F, _P]),
    "ibm_spread": (I, [_LAT, _PART, ctypes.c_int32, _P, _P, _P, _P]),
    "ibm_spread_noalloc": (I, [_LAT, _PART, ctypes.c_int32, _P, _P, _P]),
    "rigid_update_markers": (I, [_PART, _P]),
    "ibm_interpolate_wall": (I, [_LAT, _P, _FORCE, _P, _PART, F, F, ctypes.c_int32, _P, _P]),
    "ibm_interpolate_wall_claim": (I, [_LAT, _P, _FORCE, _P, _PART, F, F, ctypes.c_int32, _P,
                                       _P, _P, _P, _P]),
    "ibm_spread_claimed": (I, [_LAT, _PART, _P, _P, _P, _P]),
    "rigid_step": (I, [_PART, F, F, F, _P]),
    "ibm_spread_tiled_scratch_bytes": (ctypes.c_size_t, [_LAT, ctypes.c_int32]),
    "ibm_spread_tiled": (I, [_LAT, _PART, ctypes.c_int32, _P, _P, _P, ctypes.c_size_t, _P]),
    "rigid_extremes": (I, [_PART, _P]),
    "lbm_debug_set_wait_limit": (None, [ctypes.c_int64]),
    "lbm_debug_bounds_faults": (ctypes.c_int64, [ctypes.c_int32]),
    "lbm_last_error": (ctypes.c_char_p, []),
    "lbm_version": (ctypes.c_char_p, []),
}

_lock = threading.Lock()
_lib = None


def load(path=LIB_PATH):
    """Load the library once.  Raises RuntimeError if it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                "funlbm_b200: %s is missing; build it with `python -m funlbm_b200.build` "
                "(there is no CPU fallback)" % path)
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class LbmError(RuntimeError):
    pass


def check(rc, what=""):
    """Map a library status to the reference's exception types."""
    if rc == LBM_OK:
        return
    msg = load().lbm_last_error().decode(errors="replace")
    if what:
        msg = "%s: %s" % (what, msg)
    if rc == LBM_ERR_INVALID:
        raise ValueError(msg)
    if rc == LBM_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise LbmError(msg)


def call(name, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)


def ptr(t):
    """Device address of a tensor (None for None)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(torch_mod, device=None):
    return ctypes.c_void_p(torch_mod.cuda.current_stream(device).cuda_stream)
