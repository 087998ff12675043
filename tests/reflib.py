"""ctypes access to the reference projector library built from its own sources
(oracle/_ref/libnetwork.so, made by `make -C oracle ref`).  Test
infrastructure: it runs the reference's CUDA kernels, so only GPU tests and
the golden-vector script use it."""
import ctypes
import os

import numpy as np

from conftest import ROOT

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnetwork.so")
_dp = ctypes.POINTER(ctypes.c_double)
_L = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _L
    if _L is None:
        L = ctypes.CDLL(REF_LIB)
        for pre in ("b0", "b1", "h0", "hl"):
            init = getattr(L, f"{pre}_init")
            init.restype = ctypes.c_void_p
            f = getattr(L, f"{pre}_forward_projection")
            f.restype = ctypes.c_int
            f.argtypes = [_dp, _dp, ctypes.c_void_p]
            b = getattr(L, f"{pre}_backward_projection")
            b.restype = None
            b.argtypes = [_dp, _dp, ctypes.c_void_p]
        L.b0_init.argtypes = L.b1_init.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [_dp] * 3
        for pre in ("h0", "hl"):
            getattr(L, f"{pre}_init").argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 4 + [_dp] * 3
        L.b1_3d_init.restype = ctypes.c_void_p
        L.b1_3d_init.argtypes = [ctypes.c_int] * 6 + [ctypes.c_double] * 7 + [_dp]
        L.b1_3d_forward_projection.restype = ctypes.c_ulonglong
        L.b1_3d_forward_projection.argtypes = [_dp, _dp, ctypes.c_void_p]
        L.b1_3d_backward_projection.restype = None
        L.b1_3d_backward_projection.argtypes = [_dp, _dp, ctypes.c_void_p]
        L.SF_init.restype = ctypes.c_void_p
        L.SF_init.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [_dp]
        for n in ("SF_forward_projection",):
            getattr(L, n).restype = ctypes.c_int
            getattr(L, n).argtypes = [_dp, _dp, ctypes.c_void_p]
        L.SF_backward_projection.restype = None
        L.SF_backward_projection.argtypes = [_dp, _dp, ctypes.c_void_p]
        L.ref_b1_kernel_ms.restype = ctypes.c_float
        L.ref_b1_kernel_ms.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        _L = L
    return _L


class RefFan2D:
    """The reference's 2D fan projector `kind` (b0, b1, SF) on one geometry."""

    def __init__(self, kind, nx, ny, nu, dx, dy, du, lsd, lso, angles, dz=None, drho=None):
        L = lib()
        self.kind, self.nx, self.ny, self.nu, self.np = kind, nx, ny, nu, len(angles)
        self._ang = np.ascontiguousarray(angles, dtype=np.float64)
        self._off = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (dz, drho)]
        p = self._ang.ctypes.data_as(_dp)
        offs = [None if a is None else a.ctypes.data_as(_dp) for a in self._off]
        if kind == "SF":
            self.h = L.SF_init(nx, ny, self.np, nu, dx, dy, du, lsd, lso, p)
        else:
            self.h = getattr(L, f"{kind}_init")(nx, ny, self.np, nu, dx, dy, du, lsd, lso, p, *offs)
        assert self.h

    def forward(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        b = np.zeros(self.np * self.nu)
        cnt = getattr(lib(), f"{self.kind}_forward_projection")(b.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return b, cnt

    def backward(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        x = np.zeros(self.nx * self.ny)
        getattr(lib(), f"{self.kind}_backward_projection")(y.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return x


class RefHex:
    """The reference's hexagonal projector `kind` (h0, hl): nl rows of nc sites."""

    def __init__(self, kind, nl, nc, nu, dt, du, lsd, lso, angles):
        L = lib()
        self.kind, self.nl, self.nc, self.nu, self.np = kind, nl, nc, nu, len(angles)
        self._ang = np.ascontiguousarray(angles, dtype=np.float64)
        self.h = getattr(L, f"{kind}_init")(nl, nc, self.np, nu, dt, du, lsd, lso, self._ang.ctypes.data_as(_dp),
                                           None, None)
        assert self.h

    def forward(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        b = np.zeros(self.np * self.nu)
        cnt = getattr(lib(), f"{self.kind}_forward_projection")(b.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return b, cnt

    def backward(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        x = np.zeros(self.nl * self.nc)
        getattr(lib(), f"{self.kind}_backward_projection")(y.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return x


class RefCone:
    """The reference's A_B1_3D projector on one geometry."""

    def __init__(self, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles):
        L = lib()
        self.n = nx * ny * nz
        self.m = len(angles) * nu * nv
        self._ang = np.ascontiguousarray(angles, dtype=np.float64)
        self.h = L.b1_3d_init(nx, ny, nz, len(angles), nu, nv, dx, dy, dz, du, dv, lsd, lso,
                              self._ang.ctypes.data_as(_dp))
        assert self.h

    def forward(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        b = np.zeros(self.m)
        cnt = lib().b1_3d_forward_projection(b.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return b, cnt

    def backward(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        x = np.zeros(self.n)
        lib().b1_3d_backward_projection(y.ctypes.data_as(_dp), x.ctypes.data_as(_dp), self.h)
        return x


class RefSF3D:
    """The reference's SF_projector layer (3D separable footprint) on the
    geometry of b1_3d_init, through the test shim's ref_sf3d_* entry points."""

    def __init__(self, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles):
        L = lib()
        for n in ("ref_sf3d_init",):
            getattr(L, n).restype = ctypes.c_void_p
            getattr(L, n).argtypes = [ctypes.c_int] * 6 + [ctypes.c_double] * 7 + [_dp]
        L.ref_sf3d_forward.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        L.ref_sf3d_backward.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_sf3d_destroy.argtypes = [ctypes.c_void_p]
        self.n = nx * ny * nz
        self.nx, self.ny = nx, ny
        self.m = len(angles) * nu * nv
        self._ang = np.ascontiguousarray(angles, dtype=np.float64)
        self.h = L.ref_sf3d_init(nx, ny, nz, len(angles), nu, nv, dx, dy, dz, du, dv, lsd, lso,
                                 self._ang.ctypes.data_as(_dp))
        assert self.h

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_sf3d_destroy(self.h)
            self.h = None

    def forward(self, x, trap=False):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        b = np.zeros(self.m)
        assert lib().ref_sf3d_forward(self.h, x.ctypes.data_as(_dp), b.ctypes.data_as(_dp), int(trap)) == 0
        return b

    def backward(self, y):
        # SF_backproject has no bounds check on ix, iy (layers/SF_projector.cu:
        # 237-356): with nx or ny not a multiple of its 8 x 8 blocks, threads
        # past the edge add into other voxels and, in the last slice, past the
        # end of the volume.  Only whole blocks are run here.
        if self.nx % 8 or self.ny % 8:
            raise ValueError("the reference SF back projection writes out of bounds unless nx, ny are multiples of 8")
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        x = np.zeros(self.n)
        assert lib().ref_sf3d_backward(self.h, y.ctypes.data_as(_dp), x.ctypes.data_as(_dp)) == 0
        return x


def matrix_generation(kind, np_, nu, nx, ny, dx, dy, du, lsd, lso, buffer_size):
    """The reference's pixel_matrix_generation ("b0") or
    bilinear_matrix_generation ("b1"): (nnz, triplets (buffer_size, 3))."""
    L = lib()
    f = getattr(L, {"b0": "pixel_matrix_generation", "b1": "bilinear_matrix_generation"}[kind])
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [_dp, ctypes.c_int]
    spmat = np.zeros((buffer_size, 3))
    n = f(np_, nu, nx, ny, dx, dy, du, lsd, lso, spmat.ctypes.data_as(_dp), buffer_size)
    return n, spmat
