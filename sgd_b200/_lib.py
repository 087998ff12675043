"""ctypes binding of sgd_b200/libnetwork.so, the CUDA projector library.

The library is built in-tree (``make -C sgd_b200/csrc`` or
``__graft_entry__.build()``).  There is no CPU fallback: if it is missing or
fails to load, every projector raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnetwork.so")

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

_LIB = None


class ProjectorError(RuntimeError):
    """A failure reported by the CUDA library (sgd_last_error())."""


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ProjectorError(f"CUDA projector library not built: {LIB_PATH} (run `make -C sgd_b200/csrc`)")
    L = ctypes.CDLL(LIB_PATH)
    L.sgd_last_error.restype = ctypes.c_char_p
    L.sgd_last_error.argtypes = []
    for pre in ("b1", "SF", "b0", "h0", "hl"):
        _declare_fan2d(L, pre)
    cone = [_i] * 6 + [_d] * 7 + [_dp]
    L.b1_3d_init.restype = _vp
    L.b1_3d_init.argtypes = cone
    L.sgd_b1_3d_init.restype = _vp
    L.sgd_b1_3d_init.argtypes = [_i] + cone
    L.b1_3d_forward_projection.restype = ctypes.c_ulonglong
    L.b1_3d_forward_projection.argtypes = [_dp, _dp, _vp]
    L.sgd_b1_3d_backward_projection.restype = _i
    L.sgd_b1_3d_backward_projection.argtypes = [_dp, _dp, _vp]
    L.b1_3d_destroy.restype = None
    L.b1_3d_destroy.argtypes = [_vp]
    for n in ("sgd_b1_3d_forward_dev", "sgd_b1_3d_backward_dev"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_vp, _vp, _vp, _vp]
    L.sgd_b1_3d_count.restype = ctypes.c_ulonglong
    L.sgd_b1_3d_count.argtypes = [_vp]
    L.sgd_sf3d_init.restype = _vp
    L.sgd_sf3d_init.argtypes = [_i, _i] + cone
    for n in ("sgd_sf3d_forward_projection", "sgd_sf3d_backward_projection"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_dp, _dp, _vp]
    L.sgd_sf3d_destroy.restype = None
    L.sgd_sf3d_destroy.argtypes = [_vp]
    for n in ("sgd_sf3d_forward_dev", "sgd_sf3d_backward_dev"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_vp, _vp, _vp, _vp]
    L.sgd_b0_parallel_init.restype = _vp
    L.sgd_b0_parallel_init.argtypes = [_i, _i, _i, _i, _d, _d, _d, _dp]
    L.sgd_b1_batch_create.restype = _vp
    L.sgd_b1_batch_create.argtypes = [_i] + [_vp] * 10
    L.sgd_b1_batch_destroy.restype = None
    L.sgd_b1_batch_destroy.argtypes = [_vp]
    for n, a in (("offsets", [_vp, _vp, _vp]), ("forward", [_vp] * 4), ("backward", [_vp] * 4),
                 ("capture", [_vp] * 5), ("replay", [_vp, _vp]), ("tune", [_vp, ctypes.c_char_p, _vp, _vp]),
                 ("set_variant", [_vp, _i, _i]), ("status", [_vp])):
        f = getattr(L, f"sgd_b1_batch_{n}")
        f.restype = _i
        f.argtypes = a
    gen = [_i] * 4 + [_d] * 5 + [_dp, _i]
    for n in ("pixel_matrix_generation", "bilinear_matrix_generation"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = gen
    for pre in ("b1", "b0", "SF", "h0", "hl"):
        f = getattr(L, f"sgd_{pre}_matrix_csr")
        f.restype = ctypes.c_longlong
        f.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_longlong]
    L.sgd_hex_init.restype = _vp
    L.sgd_hex_init.argtypes = [_i] + _INIT_ARGS["h0"]
    # B1 in the reference's FP32 rounding (generic kernels)
    L.sgd_b1ref_init.restype = _vp
    L.sgd_b1ref_init.argtypes = _INIT_ARGS["b1"]
    for n in ("sgd_b1ref_forward_projection", "sgd_b1ref_backward_projection"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_dp, _dp, _vp]
    L.sgd_b1ref_destroy.restype = None
    L.sgd_b1ref_destroy.argtypes = [_vp]
    for n in ("sgd_b1ref_forward_dev", "sgd_b1ref_backward_dev"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_vp, _vp, _vp, _vp]
    L.sgd_b1ref_count.restype = ctypes.c_ulonglong
    L.sgd_b1ref_count.argtypes = [_vp]
    L.sgd_b1ref_matrix_csr.restype = ctypes.c_longlong
    L.sgd_b1ref_matrix_csr.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_longlong]
    L.sgd_proj2d_status.restype = _i
    L.sgd_proj2d_status.argtypes = [_vp]
    for n in ("sgd_b1_set_wait_limit", "sgd_proj2d_set_wait_limit", "sgd_b1_batch_set_wait_limit",
              "sgd_b1_3d_set_wait_limit", "sgd_sf3d_set_wait_limit"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_vp, ctypes.c_uint]
    L.sgd_b1_status.restype = _i
    L.sgd_b1_status.argtypes = [_vp]
    for n in ("sgd_b1_3d_status", "sgd_sf3d_status"):
        getattr(L, n).restype = _i
        getattr(L, n).argtypes = [_vp]
    L.sgd_geometry_pmi.restype = _i
    L.sgd_b1_forward_noalloc.restype = _i
    L.sgd_b1_forward_noalloc.argtypes = [_vp, _vp, _vp, _vp]
    _LIB = L
    return L


# per-prefix init argument lists (the reference's signatures)
_INIT_ARGS = {
    "b1": [_i, _i, _i, _i, _d, _d, _d, _d, _d, _dp, _dp, _dp],
    "b0": [_i, _i, _i, _i, _d, _d, _d, _d, _d, _dp, _dp, _dp],
    "SF": [_i, _i, _i, _i, _d, _d, _d, _d, _d, _dp],
    "h0": [_i, _i, _i, _i, _d, _d, _d, _d, _dp, _dp, _dp],
    "hl": [_i, _i, _i, _i, _d, _d, _d, _d, _dp, _dp, _dp],
}


def _declare_fan2d(L, pre: str) -> None:
    init = getattr(L, f"{pre}_init")
    init.restype = _vp
    init.argtypes = _INIT_ARGS[pre]
    f = getattr(L, f"{pre}_forward_projection")
    f.restype = _i
    f.argtypes = [_dp, _dp, _vp]
    b = getattr(L, f"{pre}_backward_projection")
    b.restype = None
    b.argtypes = [_dp, _dp, _vp]
    sb = getattr(L, f"sgd_{pre}_backward_projection")
    sb.restype = _i
    sb.argtypes = [_dp, _dp, _vp]
    d = getattr(L, f"{pre}_destroy")
    d.restype = None
    d.argtypes = [_vp]
    fd = getattr(L, f"sgd_{pre}_forward_dev")
    fd.restype = _i
    fd.argtypes = [_vp, _vp, _vp, _vp]
    bd = getattr(L, f"sgd_{pre}_backward_dev")
    bd.restype = _i
    bd.argtypes = [_vp, _vp, _vp, _vp]
    c = getattr(L, f"sgd_{pre}_count")
    c.restype = ctypes.c_ulonglong
    c.argtypes = [_vp]


def last_error() -> str:
    msg = lib().sgd_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str) -> None:
    if status != 0:
        raise ProjectorError(f"{what}: {last_error()}")
