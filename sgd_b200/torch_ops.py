"""The projectors on CUDA tensors, and their torch.autograd.Function.

PyTorch is used here for device memory and streams only: every projection runs
the hand-written kernels of ``libnetwork.so`` through the library's device
entry points, on ``torch.cuda.current_stream()``.

Layouts (FP32, contiguous):
* image    (nx, ny)  -> element (ix, iy), the reference host layout x[ix*ny+iy]
* sinogram (np, nu)  -> element (p, u), y[p*nu+u]
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


class FanProjector:
    """One fan-beam geometry bound to the current CUDA device.

    ``kind`` selects the basis ("b1" bilinear, "b1ref" bilinear in the
    reference layer's FP32 rounding, "SF" separable footprint, "b0" pixel
    indicator).  Arguments follow the reference's
    ``*_init`` entry points (layers/A_B1.cu:595-603): image nx x ny with pixel
    dx x dy, np views at ``angles`` (radians), nu bins of pitch du,
    source-detector distance lsd, source-isocentre distance lso, optional
    per-view source offsets dz/drho.
    """

    def __init__(self, kind, nx, ny, nu, dx, dy, du, lsd, lso, angles, dz=None, drho=None):
        if not torch.cuda.is_available():
            raise _lib.ProjectorError("FanProjector needs a CUDA device")
        self.kind = kind
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        self.nx, self.ny, self.np, self.nu = int(nx), int(ny), int(angles.shape[0]), int(nu)
        self.image_shape = (self.nx, self.ny)
        self.sino_shape = (self.np, self.nu)
        self.device = torch.device("cuda", torch.cuda.current_device())
        L = _lib.lib()
        self._L = L
        dz = None if dz is None else np.ascontiguousarray(dz, dtype=np.float64)
        drho = None if drho is None else np.ascontiguousarray(drho, dtype=np.float64)
        pre = "sgd_b1ref" if kind == "b1ref" else kind  # a mode without a reference counterpart
        init = getattr(L, f"{pre}_init")
        if kind == "SF":
            self.handle = init(self.nx, self.ny, self.np, self.nu, dx, dy, du, lsd, lso, _ptr(angles))
        else:
            self.handle = init(self.nx, self.ny, self.np, self.nu, dx, dy, du, lsd, lso, _ptr(angles), _ptr(dz),
                               _ptr(drho))
        if not self.handle:
            raise _lib.ProjectorError(f"{kind}_init: {_lib.last_error()}")
        # the library's kernels behind each direction, and the launches of
        # one forward + back projection (the B1 forward also transposes)
        if kind == "b1":
            self.kernels = {"forward": "b1_forward_kernel", "back": "b1_back_kernel"}
            self.launches_per_step = 3
        else:
            self.kernels = {"forward": "fan2d_forward_kernel", "back": "fan2d_back_kernel"}
            # image transpose + forward kernel + sum of its parts, back kernel
            self.launches_per_step = 4
        self._fwd = getattr(L, f"sgd_{kind}_forward_dev")
        self._bwd = getattr(L, f"sgd_{kind}_backward_dev")
        self._destroy = getattr(L, f"{pre}_destroy")
        self.conv_count = int(getattr(L, f"sgd_{kind}_count")(self.handle))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def _check(self, t, shape, name):
        if t.device != self.device or t.dtype != torch.float32 or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float32 tensor on {self.device}")
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")

    def forward(self, img: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Sinogram (np, nu) of an image (nx, ny)."""
        self._check(img, self.image_shape, "image")
        if out is None:
            out = torch.empty(self.sino_shape, dtype=torch.float32, device=self.device)
        self._check(out, self.sino_shape, "out")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._fwd(self.handle, img.data_ptr(), out.data_ptr(), s), f"sgd_{self.kind}_forward_dev")
        return out

    def backward(self, sino: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Adjoint (back projection) image (nx, ny) of a sinogram (np, nu)."""
        self._check(sino, self.sino_shape, "sinogram")
        if out is None:
            out = torch.empty(self.image_shape, dtype=torch.float32, device=self.device)
        self._check(out, self.image_shape, "out")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._bwd(self.handle, sino.data_ptr(), out.data_ptr(), s), f"sgd_{self.kind}_backward_dev")
        return out


class _HandleProjector:
    """A layer handle with FP32 device entry points ``fwd(h, in, out, stream)``
    and ``bwd(h, in, out, stream)``: the common body of the projectors below."""

    # the library's kernels behind each direction, and the launches of one
    # forward + back projection (the generic 2D kernels: the forward's image
    # transpose, kernel and sum of its parts, the back kernel)
    kernels = {"forward": "fan2d_forward_kernel", "back": "fan2d_back_kernel"}
    launches_per_step = 4

    def _setup(self, handle, fwd, bwd, destroy, image_shape, sino_shape, what):
        if not handle:
            raise _lib.ProjectorError(f"{what}: {_lib.last_error()}")
        self.handle, self._fwd, self._bwd, self._destroy = handle, fwd, bwd, destroy
        self.image_shape, self.sino_shape, self.kind = tuple(image_shape), tuple(sino_shape), what
        self.device = torch.device("cuda", torch.cuda.current_device())

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def _check(self, t, shape, name):
        if t.device != self.device or t.dtype != torch.float32 or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float32 tensor on {self.device}")
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")

    def forward(self, img, out=None):
        self._check(img, self.image_shape, "image")
        out = torch.empty(self.sino_shape, dtype=torch.float32, device=self.device) if out is None else out
        self._check(out, self.sino_shape, "out")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._fwd(self.handle, img.data_ptr(), out.data_ptr(), s), f"{self.kind} forward")
        return out

    def backward(self, sino, out=None):
        self._check(sino, self.sino_shape, "sinogram")
        out = torch.empty(self.image_shape, dtype=torch.float32, device=self.device) if out is None else out
        self._check(out, self.image_shape, "out")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._bwd(self.handle, sino.data_ptr(), out.data_ptr(), s), f"{self.kind} backward")
        return out


class HexProjector(_HandleProjector):
    """H0 / Hl on the hexagonal lattice (arguments of h0_init / hl_init).
    ``mode``: "h0c" (H0 with the true hexagon bounds: an exact adjoint pair,
    the default for autograd), "h0" (the reference's H0), "hl".  Image shape
    (nc, nl) in the host layout x[ic*nl + il]."""

    def __init__(self, nl, nc, nu, dt, du, lsd, lso, angles, mode="h0c", dz=None, drho=None):
        L = _lib.lib()
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        dz = None if dz is None else np.ascontiguousarray(dz, dtype=np.float64)
        drho = None if drho is None else np.ascontiguousarray(drho, dtype=np.float64)
        code = {"h0c": 0, "h0": 1, "hl": 2}[mode]
        pre = "hl" if mode == "hl" else "h0"
        h = L.sgd_hex_init(code, nl, nc, len(angles), nu, dt, du, lsd, lso, _ptr(angles), _ptr(dz), _ptr(drho))
        self._keep = (angles, dz, drho)
        self._setup(h, getattr(L, f"sgd_{pre}_forward_dev"), getattr(L, f"sgd_{pre}_backward_dev"),
                    getattr(L, f"{pre}_destroy"), (nc, nl), (len(angles), nu), f"hex {mode}")


class ParallelB0Projector(_HandleProjector):
    """B0 in parallel-beam geometry (sgd_b0_parallel_init); image (nx, ny)."""

    def __init__(self, nx, ny, nu, dx, dy, du, angles):
        L = _lib.lib()
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        h = L.sgd_b0_parallel_init(nx, ny, len(angles), nu, dx, dy, du, _ptr(angles))
        self._keep = angles
        self._setup(h, L.sgd_b0_forward_dev, L.sgd_b0_backward_dev, L.b0_destroy, (nx, ny), (len(angles), nu),
                    "b0 parallel")


class ConeProjector(_HandleProjector):
    """Cone-beam projectors (arguments of b1_3d_init); volume (nz, ny, nx),
    projections (np, nv, nu).  kind "b1_3d" or "sf3d"; ``exact=True`` (the
    default, needed by autograd) selects the pair whose backward is the exact
    transpose of its forward (A_B1_3D mode 1, SF_projector mode 1); False the
    reference's kernels."""

    def __init__(self, kind, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles, exact=True, trap_v=False):
        L = _lib.lib()
        angles = np.ascontiguousarray(angles, dtype=np.float64)
        m = 1 if exact else 0
        if kind == "b1_3d":
            h = L.sgd_b1_3d_init(m, nx, ny, nz, len(angles), nu, nv, dx, dy, dz, du, dv, lsd, lso, _ptr(angles))
            f, b, d = L.sgd_b1_3d_forward_dev, L.sgd_b1_3d_backward_dev, L.b1_3d_destroy
        elif kind == "sf3d":
            h = L.sgd_sf3d_init(m, int(trap_v), nx, ny, nz, len(angles), nu, nv, dx, dy, dz, du, dv, lsd, lso,
                                _ptr(angles))
            f, b, d = L.sgd_sf3d_forward_dev, L.sgd_sf3d_backward_dev, L.sgd_sf3d_destroy
        else:
            raise ValueError(f"unknown cone-beam kind {kind!r}")
        if kind == "b1_3d":
            # column transpose + forward kernel, back kernel
            self.kernels = {"forward": "b1_3d_fwd_kernel", "back": "b1_3d_back_kernel"}
        elif exact:
            # column transpose + factored forward kernel, back kernel
            self.kernels = {"forward": "sf3d_fwd_kernel", "back": "sf3d_back1_kernel"}
        else:
            # the reference's scatter + FP64-to-FP32 finish, its gather
            self.kernels = {"forward": "sf3d_forward_kernel", "back": "sf3d_back_kernel"}
        self.launches_per_step = 3
        self._keep = angles
        self._setup(h, f, b, d, (nz, ny, nx), (len(angles), nv, nu), kind)


class ProjectFunction(torch.autograd.Function):
    """y = A x with dL/dx = A^T dL/dy computed by the hand-written back projector."""

    @staticmethod
    def forward(ctx, img, projector):
        ctx.projector = projector
        return projector.forward(img.contiguous())

    @staticmethod
    def backward(ctx, grad):
        return ctx.projector.backward(grad.contiguous()), None


class BackProjectFunction(torch.autograd.Function):
    """x = A^T y with dL/dy = A dL/dx."""

    @staticmethod
    def forward(ctx, sino, projector):
        ctx.projector = projector
        return projector.backward(sino.contiguous())

    @staticmethod
    def backward(ctx, grad):
        return ctx.projector.forward(grad.contiguous()), None


def project(img: torch.Tensor, projector) -> torch.Tensor:
    """Differentiable forward projection; batched over leading dimensions."""
    if img.dim() == len(projector.image_shape):
        return ProjectFunction.apply(img, projector)
    return torch.stack([project(x, projector) for x in img])


def back_project(sino: torch.Tensor, projector) -> torch.Tensor:
    """Differentiable back projection; batched over leading dimensions."""
    if sino.dim() == len(projector.sino_shape):
        return BackProjectFunction.apply(sino, projector)
    return torch.stack([back_project(y, projector) for y in sino])
