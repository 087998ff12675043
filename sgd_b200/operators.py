"""LinearOperator wrappers with the names, arguments and behaviour of the
reference's python/operators/operators.py.

Each ``A_*_operator`` builds its geometry once through the library's
``*_init`` entry point (the same C signature as the reference's) and applies
the CUDA forward/back projectors on FP64 numpy vectors through
``*_forward_projection`` / ``*_backward_projection``:

* ``matvec(x)``: x flat of length nx*ny in the layout x[ix*ny + iy];
  returns y of length np*nu in the layout y[p*nu + u]
  (python/operators/operators.py:201-209);
* ``rmatvec(y)``: the adjoint (operators.py:211-219).

The base class is pylops.LinearOperator when pylops is importable (as in the
reference) and scipy.sparse.linalg.LinearOperator otherwise; both take
``dtype``/``shape`` and dispatch to ``_matvec``/``_rmatvec``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import scipy.sparse

from . import _lib

try:  # the reference's base class
    from pylops import LinearOperator  # type: ignore
except ImportError:  # pragma: no cover - pylops is not installed in this image
    from scipy.sparse.linalg import LinearOperator

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


class _Fan2DOperator(LinearOperator):
    """Common body of the 2D fan-beam operators over one C entry-point prefix."""

    _prefix = ""
    _offsets = True  # the init takes per-view dz/drho

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, lsd, lso, angles, dz=None, drho=None, dtype=np.float64):
        super().__init__(dtype=dtype, shape=(nnp * nu, nx * ny))
        self.vol_shape = (nx, ny)
        self.proj_shape = (nnp, nu)
        self.lsd = lsd
        self.lso = lso
        self.dimension = (dx, dy)
        self.blur = du
        self.angles = angles
        if dz is not None and drho is None:
            # python/operators/operators.py:171-172
            raise AssertionError("Error: drho should be provided if dz is provided.")
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        if angles.shape != (nnp,):
            raise ValueError(f"angles must have shape ({nnp},), got {angles.shape}")
        self._angles = angles
        self._dz = None if dz is None else np.ascontiguousarray(dz, dtype=np.float64)
        self._drho = None if drho is None else np.ascontiguousarray(drho, dtype=np.float64)
        L = _lib.lib()
        self._L = L
        init = getattr(L, self._sym("init"))
        if self._offsets:
            self.cpointer = init(nx, ny, nnp, nu, dx, dy, du, lsd, lso, _ptr(angles), _ptr(self._dz),
                                 _ptr(self._drho))
        else:
            self.cpointer = init(nx, ny, nnp, nu, dx, dy, du, lsd, lso, _ptr(angles))
        if not self.cpointer:
            raise _lib.ProjectorError(f"{self._sym('init')}: {_lib.last_error()}")
        self._fwd = getattr(L, self._sym("forward_projection"))
        self._bwd = getattr(L, f"sgd_{self._prefix}_backward_projection")
        self._destroy = getattr(L, self._sym("destroy"))
        self.conv_count = int(getattr(L, f"sgd_{self._prefix}_count")(self.cpointer))

    def _sym(self, what):
        # the reference's names (b1_init, ...); modes without a counterpart
        # in the reference carry the library's sgd_ prefix throughout
        return f"sgd_{self._prefix}_{what}" if self._prefix == "b1ref" else f"{self._prefix}_{what}"

    def __del__(self):
        p = getattr(self, "cpointer", None)
        if p:
            self._destroy(p)
            self.cpointer = None

    def _matvec(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        if x.size != self.shape[1]:
            raise ValueError(f"expected {self.shape[1]} image values, got {x.size}")
        y = np.empty((self.shape[0],), dtype=np.float64)  # every value is written
        if self._fwd(_ptr(y), _ptr(x), self.cpointer) < 0:
            raise _lib.ProjectorError(f"{self._prefix}_forward_projection: {_lib.last_error()}")
        return y.astype(self.dtype, copy=False)

    def _rmatvec(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        if y.size != self.shape[0]:
            raise ValueError(f"expected {self.shape[0]} sinogram values, got {y.size}")
        x = np.empty((self.shape[1],), dtype=np.float64)  # every value is written
        _lib.check(self._bwd(_ptr(y), _ptr(x), self.cpointer), f"{self._prefix}_backward_projection")
        return x.astype(self.dtype, copy=False)

    def matrix(self):
        """The operator's system matrix as scipy CSR (rows p*nu + u, columns in
        the host image layout), built on the GPU from the footprints the
        projection kernels use: ``matrix() @ x`` equals ``matvec(x)``."""
        return layer_csr(self._prefix, self.cpointer, self.shape)


class A_B1_operator(_Fan2DOperator):
    """Bilinear box-spline fan-beam projector (python/operators/operators.py:156-219).

    ``reference_rounding=True`` selects the mode that repeats the reference
    layer's FP32 bin positioning and edge-ray arithmetic (layers/A_B1.cu:
    100-197), for results within a few units in the last place of the
    reference's own; the default evaluates the footprint from exact bin
    geometry."""

    _prefix = "b1"

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, lsd, lso, angles, dz=None, drho=None, dtype=np.float64,
                 reference_rounding=False):
        if reference_rounding:
            self._prefix = "b1ref"
        super().__init__(nx, ny, nnp, nu, dx, dy, du, lsd, lso, angles, dz=dz, drho=drho, dtype=dtype)


class A_SF_operator(_Fan2DOperator):
    """Separable-footprint fan-beam projector (python/operators/operators.py:351-399)."""

    _prefix = "SF"
    _offsets = False

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, lsd, lso, angles, dtype=np.float64):
        super().__init__(nx, ny, nnp, nu, dx, dy, du, lsd, lso, angles, dtype=dtype)


class A_B0_operator(_Fan2DOperator):
    """Pixel-indicator fan-beam projector (python/operators/operators.py:91-154)."""

    _prefix = "b0"


class A_B0_parallel_operator(_Fan2DOperator):
    """Pixel-indicator projector in parallel-beam geometry (no counterpart in
    the reference, whose geometry always has a point source): view angle
    beta, rays along (cos beta, sin beta), nu bins of pitch du on the axis
    (-sin beta, cos beta) through the isocentre.  Layouts as A_B0_operator."""

    _prefix = "b0"

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, angles, dtype=np.float64):
        LinearOperator.__init__(self, dtype=dtype, shape=(nnp * nu, nx * ny))
        self.vol_shape = (nx, ny)
        self.proj_shape = (nnp, nu)
        self.dimension = (dx, dy)
        self.blur = du
        self.angles = angles
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        if angles.shape != (nnp,):
            raise ValueError(f"angles must have shape ({nnp},), got {angles.shape}")
        self._angles = angles
        L = _lib.lib()
        self._L = L
        self.cpointer = L.sgd_b0_parallel_init(nx, ny, nnp, nu, dx, dy, du, _ptr(angles))
        if not self.cpointer:
            raise _lib.ProjectorError(f"sgd_b0_parallel_init: {_lib.last_error()}")
        self._fwd = L.b0_forward_projection
        self._bwd = L.sgd_b0_backward_projection
        self._destroy = L.b0_destroy
        self.conv_count = int(L.sgd_b0_count(self.cpointer))


class _HexOperator(_Fan2DOperator):
    """Common body of the hexagonal-lattice operators.  The reference names
    the lattice sizes (nx, ny) in Python and (nl, nc) in C: nx rows of ny
    sites, host layout x[ic*nl + il] (python/operators/operators.py:221-349)."""

    _mode = 1

    def __init__(self, nx, ny, nnp, nu, dt, du, lsd, lso, angles, dz=None, drho=None, dtype=np.float64):
        LinearOperator.__init__(self, dtype=dtype, shape=(nnp * nu, nx * ny))
        self.vol_shape = (nx, ny)
        self.proj_shape = (nnp, nu)
        self.lsd = lsd
        self.lso = lso
        self.dimension = dt
        self.blur = du
        self.angles = angles
        if dz is not None and drho is None:
            raise AssertionError("Error: drho should be provided if dz is provided.")
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        if angles.shape != (nnp,):
            raise ValueError(f"angles must have shape ({nnp},), got {angles.shape}")
        self._angles = angles
        self._dz = None if dz is None else np.ascontiguousarray(dz, dtype=np.float64)
        self._drho = None if drho is None else np.ascontiguousarray(drho, dtype=np.float64)
        L = _lib.lib()
        self._L = L
        self.cpointer = L.sgd_hex_init(self._mode, nx, ny, nnp, nu, dt, du, lsd, lso, _ptr(angles), _ptr(self._dz),
                                       _ptr(self._drho))
        if not self.cpointer:
            raise _lib.ProjectorError(f"{self._sym('init')}: {_lib.last_error()}")
        self._fwd = getattr(L, self._sym("forward_projection"))
        self._bwd = getattr(L, f"sgd_{self._prefix}_backward_projection")
        self._destroy = getattr(L, self._sym("destroy"))
        self.conv_count = int(getattr(L, f"sgd_{self._prefix}_count")(self.cpointer))

    def _sym(self, what):
        # the reference's names (b1_init, ...); modes without a counterpart
        # in the reference carry the library's sgd_ prefix throughout
        return f"sgd_{self._prefix}_{what}" if self._prefix == "b1ref" else f"{self._prefix}_{what}"


class A_H0_operator(_HexOperator):
    """Hexagon-indicator projector (python/operators/operators.py:221-284).

    ``exact_bounds=True`` bounds each site's true hexagon (an exact adjoint
    pair); the default reproduces the reference, whose bounds are computed at
    the 0.5 dt row pitch of its projection matrices (layers/A_H0.cu:556) and
    so drop footprint away from the centre row."""

    _prefix = "h0"

    def __init__(self, nx, ny, nnp, nu, dt, du, lsd, lso, angles, dz=None, drho=None, dtype=np.float64,
                 exact_bounds=False):
        self._mode = 0 if exact_bounds else 1
        super().__init__(nx, ny, nnp, nu, dt, du, lsd, lso, angles, dz, drho, dtype=dtype)


class A_Hl_operator(_HexOperator):
    """Hexagonal linear box-spline projector (python/operators/operators.py:286-349)."""

    _prefix = "hl"
    _mode = 2


class A_B1_3D_operator(LinearOperator):
    """Cone-beam bilinear x separable-footprint projector
    (python/operators/operators.py:401-449): x flat [z][y][x], y flat
    [p][v][u].  ``exact_adjoint=True`` makes rmatvec the exact transpose of
    matvec; the default reproduces the reference's backward."""

    def __init__(self, nx, ny, nz, nnp, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, dtype=np.float64,
                 exact_adjoint=False):
        super().__init__(dtype=dtype, shape=(nnp * nu * nv, nx * ny * nz))
        self.vol_shape = (nz, ny, nx)
        self.proj_shape = (nnp, nu, nv)
        self.lsd = lsd
        self.lso = lso
        self.dimension = (dx, dy, dz)
        self.blur = (du, dv)
        self.angles = angles
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        if angles.shape != (nnp,):
            raise ValueError(f"angles must have shape ({nnp},), got {angles.shape}")
        self._angles = angles
        L = _lib.lib()
        self._L = L
        self.cpointer = L.sgd_b1_3d_init(1 if exact_adjoint else 0, nx, ny, nz, nnp, nu, nv, dx, dy, dz, du, dv, lsd,
                                         lso, _ptr(angles))
        if not self.cpointer:
            raise _lib.ProjectorError(f"b1_3d_init: {_lib.last_error()}")
        self.conv_count = int(L.sgd_b1_3d_count(self.cpointer))

    def __del__(self):
        p = getattr(self, "cpointer", None)
        if p:
            self._L.b1_3d_destroy(p)
            self.cpointer = None

    def _matvec(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        if x.size != self.shape[1]:
            raise ValueError(f"expected {self.shape[1]} volume values, got {x.size}")
        y = np.empty((self.shape[0],), dtype=np.float64)  # every value is written
        if self._L.b1_3d_forward_projection(_ptr(y), _ptr(x), self.cpointer) == 2 ** 64 - 1:
            raise _lib.ProjectorError(f"b1_3d_forward_projection: {_lib.last_error()}")
        return y.astype(self.dtype, copy=False)

    def _rmatvec(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        if y.size != self.shape[0]:
            raise ValueError(f"expected {self.shape[0]} projection values, got {y.size}")
        x = np.empty((self.shape[1],), dtype=np.float64)  # every value is written
        _lib.check(self._L.sgd_b1_3d_backward_projection(_ptr(y), _ptr(x), self.cpointer),
                   "b1_3d_backward_projection")
        return x.astype(self.dtype, copy=False)


class SF_projector_operator(LinearOperator):
    """Cone-beam separable-footprint projector (the class SF of
    layers/SF_projector.cu, which the reference drives from C++ only): x flat
    [z][y][x], y flat [p][v][u], geometry as A_B1_3D_operator.

    ``mode=0`` reproduces the reference kernels: matvec accumulates the
    footprint of every non-zero voxel without the voxel's value or amplitude
    (layers/SF_projector.cu:190-221), bins past the u edges wrap into the
    neighbouring detector rows, and rmatvec is SF::back_project.  ``mode=1``
    is the corrected projector (value x amplitude, in-detector bins) with
    rmatvec its exact transpose.  ``trap_v`` selects SF-TT in v (the
    reference's ``tt`` flag) for the forward, and for mode 1's transpose."""

    def __init__(self, nx, ny, nz, nnp, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, dtype=np.float64, mode=0,
                 trap_v=False):
        super().__init__(dtype=dtype, shape=(nnp * nu * nv, nx * ny * nz))
        self.vol_shape = (nz, ny, nx)
        self.proj_shape = (nnp, nv, nu)
        self.lsd = lsd
        self.lso = lso
        self.dimension = (dx, dy, dz)
        self.blur = (du, dv)
        self.angles = angles
        self.mode = int(mode)
        self.trap_v = bool(trap_v)
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        if angles.shape != (nnp,):
            raise ValueError(f"angles must have shape ({nnp},), got {angles.shape}")
        self._angles = angles
        L = _lib.lib()
        self._L = L
        self.cpointer = L.sgd_sf3d_init(self.mode, int(self.trap_v), nx, ny, nz, nnp, nu, nv, dx, dy, dz, du, dv,
                                        lsd, lso, _ptr(angles))
        if not self.cpointer:
            raise _lib.ProjectorError(f"sgd_sf3d_init: {_lib.last_error()}")

    def __del__(self):
        p = getattr(self, "cpointer", None)
        if p:
            self._L.sgd_sf3d_destroy(p)
            self.cpointer = None

    def _matvec(self, x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.float64)
        if x.size != self.shape[1]:
            raise ValueError(f"expected {self.shape[1]} volume values, got {x.size}")
        y = np.empty((self.shape[0],), dtype=np.float64)  # every value is written
        _lib.check(self._L.sgd_sf3d_forward_projection(_ptr(y), _ptr(x), self.cpointer), "sgd_sf3d_forward_projection")
        return y.astype(self.dtype, copy=False)

    def _rmatvec(self, y):
        y = np.ascontiguousarray(np.ravel(y), dtype=np.float64)
        if y.size != self.shape[0]:
            raise ValueError(f"expected {self.shape[0]} projection values, got {y.size}")
        x = np.empty((self.shape[1],), dtype=np.float64)  # every value is written
        _lib.check(self._L.sgd_sf3d_backward_projection(_ptr(y), _ptr(x), self.cpointer),
                   "sgd_sf3d_backward_projection")
        return x.astype(self.dtype, copy=False)



# ---- system matrices --------------------------------------------------------

def layer_csr(prefix, handle, shape):
    """CSR system matrix of a layer handle through ``sgd_<prefix>_matrix_csr``."""
    f = getattr(_lib.lib(), f"sgd_{prefix}_matrix_csr")
    n = f(handle, None, None, None, 0)
    if n < 0:
        raise _lib.ProjectorError(f"sgd_{prefix}_matrix_csr: {_lib.last_error()}")
    rowptr = np.zeros(shape[0] + 1, dtype=np.int64)
    cols = np.zeros(max(n, 1), dtype=np.int32)
    vals = np.zeros(max(n, 1))
    m = f(handle, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, n)
    if m != n:
        raise _lib.ProjectorError(f"sgd_{prefix}_matrix_csr: {_lib.last_error()}")
    return scipy.sparse.csr_matrix((vals[:n], cols[:n], rowptr), shape=shape)


def matrix_generation(kind, nx, ny, nnp, nu, dx, dy, du, lsd, lso, buffer_size=None):
    """The reference's generators (``pixel_matrix_generation`` for "b0",
    ``bilinear_matrix_generation`` for "b1"; python/matrix_gen/A_B*_project.py)
    run on the GPU: returns (nnz, spmat) with spmat (buffer_size, 3) holding
    the (row, column, value) triplets.  Without ``buffer_size`` the buffer
    grows until the matrix fits."""
    f = getattr(_lib.lib(), {"b0": "pixel_matrix_generation", "b1": "bilinear_matrix_generation"}[kind])
    size = buffer_size or max(1024, 4 * nnp * nx * ny)
    while True:
        spmat = np.zeros((size, 3), dtype=np.float64)
        n = f(nnp, nu, nx, ny, dx, dy, du, lsd, lso, _ptr(spmat), size)
        if n >= 0:
            return n, spmat
        if buffer_size is not None or size >= 2 ** 31 - 1:
            raise _lib.ProjectorError(f"{kind} matrix generation: {_lib.last_error()}")
        size = min(2 ** 31 - 1, 2 * size)


def generate_matrix(kind, nx, ny, nnp, nu, dx, dy, du, lsd, lso):
    """scipy CSR of the reference generator's matrix, shape (nnp*nu, nx*ny)."""
    n, spmat = matrix_generation(kind, nx, ny, nnp, nu, dx, dy, du, lsd, lso)
    t = spmat[:n]
    return scipy.sparse.csr_matrix((t[:, 2], (t[:, 0].astype(np.int64), t[:, 1].astype(np.int64))),
                                   shape=(nnp * nu, nx * ny))


class _MatrixOperator(LinearOperator):
    """Operators over a stored system matrix (python/operators/operators.py:
    11-89): the reference loads ./matrixes/A_<kind>_sparse_<n1>_<n2>_<np>_<nu>.npz.
    Here ``matrix`` may be passed directly; otherwise that file is loaded when
    it exists, and else the matrix is built on the GPU (the reference's
    generator for B0/B1, the layer's matrix at uniform angles for H0/Hl)."""

    _kind = ""

    def __init__(self, n1, n2, nnp, nu, d, du, lsd, lso, dtype=np.float64, matrix=None, directory="./matrixes"):
        super().__init__(dtype=dtype, shape=(nnp * nu, n1 * n2))
        self.vol_shape = (n1, n2)
        self.proj_shape = (nnp, nu)
        self.lsd = lsd
        self.lso = lso
        self.dimension = d
        self.blur = du
        if matrix is None:
            path = os.path.join(directory, f"A_{self._kind}_sparse_{n1}_{n2}_{nnp}_{nu}.npz")
            if os.path.exists(path):
                matrix = scipy.sparse.load_npz(path)
            else:
                matrix = self._build(n1, n2, nnp, nu, d, du, lsd, lso)
        self.A = scipy.sparse.csr_matrix(matrix)

    def _matvec(self, x):
        return self.A @ np.ravel(x)

    def _rmatvec(self, y):
        return self.A.T @ np.ravel(y)


class A_B0_operator_matrix(_MatrixOperator):
    _kind = "B0"

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, lsd, lso, dtype=np.float64, **kw):
        super().__init__(nx, ny, nnp, nu, (dx, dy), du, lsd, lso, dtype=dtype, **kw)

    @staticmethod
    def _build(nx, ny, nnp, nu, d, du, lsd, lso):
        return generate_matrix("b0", nx, ny, nnp, nu, d[0], d[1], du, lsd, lso)


class A_B1_operator_matrix(_MatrixOperator):
    _kind = "B1"

    def __init__(self, nx, ny, nnp, nu, dx, dy, du, lsd, lso, dtype=np.float64, **kw):
        super().__init__(nx, ny, nnp, nu, (dx, dy), du, lsd, lso, dtype=dtype, **kw)

    @staticmethod
    def _build(nx, ny, nnp, nu, d, du, lsd, lso):
        return generate_matrix("b1", nx, ny, nnp, nu, d[0], d[1], du, lsd, lso)


class A_H0_operator_matrix(_MatrixOperator):
    _kind = "H0"
    _op = A_H0_operator

    def __init__(self, nl, nc, nnp, nu, dt, du, lsd, lso, dtype=np.float64, **kw):
        super().__init__(nl, nc, nnp, nu, dt, du, lsd, lso, dtype=dtype, **kw)

    @classmethod
    def _build(cls, nl, nc, nnp, nu, dt, du, lsd, lso):
        return cls._op(nl, nc, nnp, nu, dt, du, lsd, lso, 2 * np.pi * np.arange(nnp) / nnp).matrix()


class A_Hl_operator_matrix(A_H0_operator_matrix):
    _kind = "Hl"
    _op = A_Hl_operator
