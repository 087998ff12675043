"""ORACLE — test infrastructure only (tests/, smoke() and bench.py's CPU-baseline
leg).  ctypes bindings of oracle/liboracle.so, the CPU restatement of the
reference projector layer (oracle/sgd_oracle.cpp).  The product package never
imports this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        _LIB = ctypes.CDLL(path)
        L = _LIB
        L.oracle_geometry.restype = None
        L.oracle_b1_forward.restype = ctypes.c_longlong
        L.oracle_b1_backward.restype = None
        L.oracle_b1_matrix.restype = ctypes.c_longlong
        L.oracle_sf_forward.restype = None
        L.oracle_b0_forward.restype = ctypes.c_longlong
        L.oracle_b0_backward.restype = None
        L.oracle_hex_forward.restype = ctypes.c_longlong
        L.oracle_hex_backward.restype = None
        L.oracle_b1_3d_forward.restype = ctypes.c_ulonglong
        L.oracle_b1_3d_backward.restype = None
        L.oracle_sf3d_forward.restype = None
        L.oracle_exact_fan2d_matrix.restype = None
        L.oracle_exact_parallel_matrix.restype = None
        L.oracle_exact_hex_matrix.restype = None
        L.oracle_exact_hl_matrix.restype = None
        L.oracle_matrix_generation.restype = ctypes.c_longlong
        L.oracle_ref_simpson_3d.restype = None
        L.oracle_sf3d_backward.restype = None
        L.oracle_sf_backward.restype = None
        L.oracle_b1_flops.restype = None
        L.oracle_fan2d_flops.restype = None
        L.oracle_cone_flops.restype = None
    return _LIB


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _c(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def geometry(nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, dzs=None, drho=None):
    """utils/geo.cu geometry: dict of src/dtv/puv/pvv (np,3), pm (np,12), pmi (np,12) float32."""
    angles = _c(angles)
    n = len(angles)
    out = {k: np.zeros((n, 3)) for k in ("src", "dtv", "puv", "pvv")}
    out["pm"] = np.zeros((n, 12))
    out["pmi"] = np.zeros((n, 12), dtype=np.float32)
    lib().oracle_geometry(nx, ny, nz, n, nu, nv, ctypes.c_double(dx), ctypes.c_double(dy), ctypes.c_double(dz),
                          ctypes.c_double(du), ctypes.c_double(dv), ctypes.c_double(lsd), ctypes.c_double(lso),
                          _p(angles), _p(_c(dzs)), _p(_c(drho)), _p(out["src"]), _p(out["dtv"]),
                          _p(out["puv"]), _p(out["pvv"]), _p(out["pm"]), out["pmi"].ctypes.data_as(_fp))
    return out


def b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0):
    """FP64 replica (precision=0) or FP32 emulation (1) of b1_forward_projection.

    x: host layout x[ix*ny+iy]; returns (b[np*nu], footprint-evaluation count).
    """
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu)
    cnt = lib().oracle_b1_forward(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy),
                                  ctypes.c_double(du), ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles),
                                  _p(_c(dzs)), _p(_c(drho)), _p(x), _p(b), precision)
    return b, int(cnt)


def b1_backward(b, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0):
    """FP64 replica (precision=0) or FP32 emulation (1) of b1_backward_projection."""
    angles = _c(angles)
    b = _c(np.ravel(b))
    x = np.zeros(nx * ny)
    lib().oracle_b1_backward(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy), ctypes.c_double(du),
                             ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), _p(_c(dzs)), _p(_c(drho)),
                             _p(b), _p(x), precision)
    return x


def b1_flops(nx, ny, nu, dx, dy, du, lsd, lso, angles, nviews=8):
    """(range FLOPs per pixel-view, FLOPs per footprint evaluation, evaluations per pixel-view)."""
    angles = _c(angles)
    out = np.zeros(3)
    lib().oracle_b1_flops(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy), ctypes.c_double(du),
                          ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), nviews, _p(out))
    return tuple(out)


def fan2d_flops(kind, nx, ny, nu, dx, dy, du, lsd, lso, angles, nviews=8):
    """(FLOPs per cell-view, bins visited per cell-view) of the reference formula
    of kind "sf", "b0", "h0" or "hl" (lattices: nx rows x ny sites, dx = dt)."""
    k = {"sf": 1, "b0": 2, "h0": 3, "hl": 4}[kind]
    angles = _c(angles)
    out = np.zeros(2)
    lib().oracle_fan2d_flops(k, nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy),
                             ctypes.c_double(du), ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), nviews,
                             _p(out))
    return tuple(out)


def cone_flops(kind, n, nd, d, dd, lsd, lso, angles, nviews=4, stride=4):
    """(FLOPs per voxel-view, (u, v) bins per voxel-view) of the reference's
    cone-beam forward formula of kind "b1_3d" or "sf3d" on an n^3 volume of
    pitch d and an nd x nd detector of pitch dd."""
    k = {"b1_3d": 1, "sf3d": 2}[kind]
    angles = _c(angles)
    out = np.zeros(2)
    lib().oracle_cone_flops(k, n, n, n, len(angles), nd, nd, ctypes.c_double(d), ctypes.c_double(d),
                            ctypes.c_double(d), ctypes.c_double(dd), ctypes.c_double(dd), ctypes.c_double(lsd),
                            ctypes.c_double(lso), _p(angles), nviews, stride, _p(out))
    return tuple(out)


def b1_matrix(nx, ny, nu, dx, dy, du, lsd, lso, angles, views):
    """scipy CSR rows of the B1 system matrix for the listed views (FP64 replica)."""
    import scipy.sparse as sp
    angles = _c(angles)
    views = np.ascontiguousarray(views, dtype=np.int32)
    cap = int(len(views) * nx * ny * 4.5)
    while True:
        rows = np.empty(cap, dtype=np.int32)
        cols = np.empty(cap, dtype=np.int32)
        vals = np.empty(cap, dtype=np.float64)
        n = lib().oracle_b1_matrix(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy),
                                   ctypes.c_double(du), ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles),
                                   views.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(views),
                                   ctypes.c_longlong(cap), rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   cols.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(vals))
        if n <= cap:
            break
        cap = int(n)
    return sp.csr_matrix((vals[:n], (rows[:n], cols[:n])), shape=(len(views) * nu, nx * ny))


def _fan2d(name, nx, ny, nu, dx, dy, du, lsd, lso, angles, vec, out_len, precision):
    angles = _c(angles)
    vec = _c(np.ravel(vec))
    out = np.zeros(out_len)
    getattr(lib(), name)(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy), ctypes.c_double(du),
                         ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), _p(vec), _p(out), precision)
    return out


def sf_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0, chord=False):
    """FP64 replica of SF_forward_projection; returns (b, 0): the reference's SF never counts.
    chord=True (FP64) replaces the reference's amplitude dx/max(|sin|, |cos|)
    (layers/A_SF.cu:177) by the pixel's chord min(dx/|sin|, dy/|cos|)."""
    return _fan2d("oracle_sf_forward", nx, ny, nu, dx, dy, du, lsd, lso, angles, x, len(angles) * nu,
                  2 if chord else precision), 0


def sf_backward(b, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0):
    return _fan2d("oracle_sf_backward", nx, ny, nu, dx, dy, du, lsd, lso, angles, b, nx * ny, precision)


def b0_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0):
    """FP64 replica of b0_forward_projection: (b, footprint-evaluation count)."""
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu)
    cnt = lib().oracle_b0_forward(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy),
                                  ctypes.c_double(du), ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles),
                                  _p(_c(dzs)), _p(_c(drho)), _p(x), _p(b), precision)
    return b, int(cnt)


def b0_backward(b, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, precision=0):
    angles = _c(angles)
    b = _c(np.ravel(b))
    x = np.zeros(nx * ny)
    lib().oracle_b0_backward(nx, ny, len(angles), nu, ctypes.c_double(dx), ctypes.c_double(dy), ctypes.c_double(du),
                             ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), _p(_c(dzs)), _p(_c(drho)),
                             _p(b), _p(x), precision)
    return x


HEX_MODES = {"h0c": 0, "h0": 1, "hl": 2}


def hex_forward(mode, x, nl, nc, nu, dt, du, lsd, lso, angles, precision=0):
    """FP64 replica of h0_/hl_forward_projection: (b, count).  mode: 'h0' (as
    the reference), 'h0c' (true hexagon bounds), 'hl'."""
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu)
    cnt = lib().oracle_hex_forward(HEX_MODES[mode], nl, nc, len(angles), nu, ctypes.c_double(dt), ctypes.c_double(du),
                                   ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), _p(x), _p(b), precision)
    return b, int(cnt)


def hex_backward(mode, b, nl, nc, nu, dt, du, lsd, lso, angles, precision=0):
    angles = _c(angles)
    b = _c(np.ravel(b))
    x = np.zeros(nl * nc)
    lib().oracle_hex_backward(HEX_MODES[mode], nl, nc, len(angles), nu, ctypes.c_double(dt), ctypes.c_double(du),
                              ctypes.c_double(lsd), ctypes.c_double(lso), _p(angles), _p(b), _p(x), precision)
    return x


def b1_3d_forward(x, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles):
    """FP64 replica of b1_3d_forward_projection: (b[(p*nv+v)*nu+u], count)."""
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu * nv)
    d = ctypes.c_double
    cnt = lib().oracle_b1_3d_forward(nx, ny, nz, len(angles), nu, nv, d(dx), d(dy), d(dz), d(du), d(dv), d(lsd), d(lso),
                                     _p(angles), _p(x), _p(b))
    return b, int(cnt)


def b1_3d_backward(b, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, exact=False):
    """FP64 replica of b1_3d_backward_projection (exact=False) or of the exact
    transpose of the forward (exact=True)."""
    angles = _c(angles)
    b = _c(np.ravel(b))
    x = np.zeros(nx * ny * nz)
    d = ctypes.c_double
    lib().oracle_b1_3d_backward(2 if exact else 1, nx, ny, nz, len(angles), nu, nv, d(dx), d(dy), d(dz), d(du), d(dv),
                                d(lsd), d(lso), _p(angles), _p(b), _p(x))
    return x


def sf3d_forward(x, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, mode=0, trap=False):
    """FP64 replica of SF::project (mode 0) or of the corrected forward (mode 1):
    b[(p*nv+v)*nu+u] from x[(iz*ny+iy)*nx+ix]."""
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu * nv)
    d = ctypes.c_double
    lib().oracle_sf3d_forward(mode, int(trap), nx, ny, nz, len(angles), nu, nv, d(dx), d(dy), d(dz), d(du), d(dv),
                              d(lsd), d(lso), _p(angles), _p(x), _p(b))
    return b


def sf3d_backward(b, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, mode=0, trap=False):
    """FP64 replica of SF::back_project (mode 0) or the exact transpose of the
    corrected forward (mode 1)."""
    angles = _c(angles)
    b = _c(np.ravel(b))
    x = np.zeros(nx * ny * nz)
    d = ctypes.c_double
    lib().oracle_sf3d_backward(mode, int(trap), nx, ny, nz, len(angles), nu, nv, d(dx), d(dy), d(dz), d(du), d(dv),
                               d(lsd), d(lso), _p(angles), _p(b), _p(x))
    return x


def exact_fan2d_matrix(kind, nx, ny, nu, dx, dy, du, lsd, lso, angles, dzs=None, drho=None, tol=1e-10):
    """Dense exact FP64 system matrix (np*nu, nx*ny) of the pixel-indicator
    ("b0") or bilinear ("b1") basis: bin-averaged line integrals by adaptive
    Simpson (the exact projectors of python/matrix_gen/*_ref_project.py).
    Columns in the host layout ix*ny + iy."""
    angles = _c(angles)
    M = np.zeros(len(angles) * nu * nx * ny)
    d = ctypes.c_double
    lib().oracle_exact_fan2d_matrix({"b0": 0, "b1": 1}[kind], nx, ny, len(angles), nu, d(dx), d(dy), d(du), d(lsd),
                                    d(lso), _p(angles), _p(_c(dzs)), _p(_c(drho)), d(tol), _p(M))
    return M.reshape(len(angles) * nu, nx * ny)


def exact_hex_matrix(nl, nc, nu, dt, du, lsd, lso, angles, tol=1e-10):
    """Dense exact FP64 system matrix (np*nu, nc*nl) of the hexagon indicator
    (the H0 basis, layers/A_H0.cu:158-256): bin-averaged chord lengths;
    columns in the host layout ic*nl + il, absent sites zero."""
    angles = _c(angles)
    M = np.zeros(len(angles) * nu * nc * nl)
    d = ctypes.c_double
    lib().oracle_exact_hex_matrix(nl, nc, len(angles), nu, d(dt), d(du), d(lsd), d(lso), _p(angles), d(tol), _p(M))
    return M.reshape(len(angles) * nu, nc * nl)


def exact_hl_matrix(nl, nc, nu, dt, du, lsd, lso, angles, tol=1e-10):
    """Dense exact FP64 system matrix (np*nu, nc*nl) of the hexagonal linear
    element (the Hl basis, layers/A_Hl.cu:168-266: the Courant hat of the
    triangular lattice, rows 0.5 dt apart): bin-averaged line integrals;
    columns in the host layout ic*nl + il, absent sites zero."""
    angles = _c(angles)
    M = np.zeros(len(angles) * nu * nc * nl)
    d = ctypes.c_double
    lib().oracle_exact_hl_matrix(nl, nc, len(angles), nu, d(dt), d(du), d(lsd), d(lso), _p(angles), d(tol), _p(M))
    return M.reshape(len(angles) * nu, nc * nl)


def ref_simpson_3d(x, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, adaptive=False, max_depth=6,
                   eps=1e-9):
    """Ref_project_Simpson (layers/Ref_projector.cu:217-367) over a whole
    volume in FP64: voxel-indicator projections b[(p*nv+v)*nu+u], chord lengths
    averaged over each detector cell by 3x3 Simpson or adaptively."""
    angles = _c(angles)
    x = _c(np.ravel(x))
    b = np.zeros(len(angles) * nu * nv)
    d = ctypes.c_double
    lib().oracle_ref_simpson_3d(int(adaptive), max_depth, d(eps), nx, ny, nz, len(angles), nu, nv, d(dx), d(dy),
                                d(dz), d(du), d(dv), d(lsd), d(lso), _p(angles), _p(x), _p(b))
    return b


def matrix_generation(kind, np_, nu, nx, ny, dx, dy, du, lsd, lso, precision=1):
    """Replica of pixel_matrix_generation ("b0") / bilinear_matrix_generation
    ("b1"): (rows int64, cols int32, vals f64) COO in row-major order."""
    d = ctypes.c_double
    k = {"b0": 0, "b1": 1}[kind]
    L = lib()
    n = L.oracle_matrix_generation(k, np_, nu, nx, ny, d(dx), d(dy), d(du), d(lsd), d(lso), precision, 0, None,
                                   None, None)
    rows = np.zeros(n, dtype=np.int64)
    cols = np.zeros(n, dtype=np.int32)
    vals = np.zeros(n)
    L.oracle_matrix_generation(k, np_, nu, nx, ny, d(dx), d(dy), d(du), d(lsd), d(lso), precision, n,
                               rows.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                               cols.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(vals))
    return rows, cols, vals


def exact_parallel_matrix(kind, nx, ny, nu, dx, dy, du, angles, tol=1e-10):
    """Dense exact FP64 parallel-beam system matrix (np*nu, nx*ny) of the
    pixel-indicator ("b0") or bilinear ("b1") basis, columns ix*ny + iy."""
    angles = _c(angles)
    M = np.zeros(len(angles) * nu * nx * ny)
    d = ctypes.c_double
    lib().oracle_exact_parallel_matrix({"b0": 0, "b1": 1}[kind], nx, ny, len(angles), nu, d(dx), d(dy), d(du),
                                       _p(angles), d(tol), _p(M))
    return M.reshape(len(angles) * nu, nx * ny)
