"""Many B1 fan-beam slices of different sizes projected in one persistent
launch per direction (``sgd_b1_batch_*`` of libnetwork.so), optionally
replayed from a CUDA graph, with an autotuned launch shape.

Device arenas (FP32 CUDA tensors) hold all slices back to back: slice k's
image (nx, ny) at ``img_off[k]`` and its sinogram (np, nu) at ``sino_off[k]``;
``images()`` / ``sinograms()`` return the per-slice views.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib


class B1Batch:
    """``slices``: sequence of (nx, ny, nu, dx, dy, du, lsd, lso, angles), the
    arguments of ``b1_init`` per slice."""

    def __init__(self, slices):
        if not torch.cuda.is_available():
            raise _lib.ProjectorError("B1Batch needs a CUDA device")
        self.slices = [tuple(s) for s in slices]
        ns = len(self.slices)
        if ns == 0:
            raise ValueError("no slices")
        L = _lib.lib()
        self._L = L
        cols = list(zip(*self.slices))
        self._angles = [np.ascontiguousarray(a, dtype=np.float64) for a in cols[8]]
        ints = [np.ascontiguousarray(c, dtype=np.int32) for c in (cols[0], cols[1], [len(a) for a in self._angles],
                                                                  cols[2])]
        dbls = [np.ascontiguousarray(c, dtype=np.float64) for c in cols[3:8]]
        ptrs = (ctypes.c_void_p * ns)(*[a.ctypes.data for a in self._angles])
        self.handle = L.sgd_b1_batch_create(ns, *[a.ctypes.data for a in ints], *[a.ctypes.data for a in dbls],
                                            ctypes.cast(ptrs, ctypes.c_void_p))
        if not self.handle:
            raise _lib.ProjectorError(f"sgd_b1_batch_create: {_lib.last_error()}")
        self.img_off = np.zeros(ns + 1, dtype=np.int64)
        self.sino_off = np.zeros(ns + 1, dtype=np.int64)
        _lib.check(L.sgd_b1_batch_offsets(self.handle, self.img_off.ctypes.data, self.sino_off.ctypes.data),
                   "sgd_b1_batch_offsets")
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.shapes = [((s[0], s[1]), (len(a), s[2])) for s, a in zip(self.slices, self._angles)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._L.sgd_b1_batch_destroy(h)
            self.handle = None

    # ---- arenas -------------------------------------------------------------
    def image_arena(self):
        return torch.zeros(int(self.img_off[-1]), dtype=torch.float32, device=self.device)

    def sinogram_arena(self):
        return torch.zeros(int(self.sino_off[-1]), dtype=torch.float32, device=self.device)

    def images(self, arena):
        return [arena[self.img_off[k]:self.img_off[k + 1]].view(*self.shapes[k][0]) for k in range(len(self.slices))]

    def sinograms(self, arena):
        return [arena[self.sino_off[k]:self.sino_off[k + 1]].view(*self.shapes[k][1])
                for k in range(len(self.slices))]

    def _check(self, t, n, name):
        if t.device != self.device or t.dtype != torch.float32 or not t.is_contiguous() or t.numel() != n:
            raise ValueError(f"{name} must be a contiguous float32 arena of {n} values on {self.device}")

    # ---- projections --------------------------------------------------------
    def forward(self, img, out=None):
        self._check(img, int(self.img_off[-1]), "image arena")
        out = self.sinogram_arena() if out is None else out
        self._check(out, int(self.sino_off[-1]), "sinogram arena")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.sgd_b1_batch_forward(self.handle, img.data_ptr(), out.data_ptr(), s), "batch forward")
        return out

    def backward(self, sino, out=None):
        self._check(sino, int(self.sino_off[-1]), "sinogram arena")
        out = self.image_arena() if out is None else out
        self._check(out, int(self.img_off[-1]), "image arena")
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.sgd_b1_batch_backward(self.handle, sino.data_ptr(), out.data_ptr(), s), "batch backward")
        return out

    def capture(self, img=None, sino=None, sino_in=None, img_out=None):
        """Records forward (img -> sino) and/or backward (sino_in -> img_out)
        into a CUDA graph; the arenas must stay alive while it is replayed."""
        ptr = (lambda t: None if t is None else t.data_ptr())
        torch.cuda.synchronize(self.device)
        _lib.check(self._L.sgd_b1_batch_capture(self.handle, ptr(img), ptr(sino), ptr(sino_in), ptr(img_out)),
                   "batch capture")
        self._keep = (img, sino, sino_in, img_out)

    def replay(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.sgd_b1_batch_replay(self.handle, s), "batch replay")

    def status(self):
        _lib.check(self._L.sgd_b1_batch_status(self.handle), "batch status")

    def set_variant(self, fw, vc):
        _lib.check(self._L.sgd_b1_batch_set_variant(self.handle, int(fw), int(vc)), "batch set_variant")

    def tune(self, cache_path=None):
        """Launch shape from ``cache_path`` (default: $SGD_AUTOTUNE_CACHE or
        ~/.cache/sgd_b200/autotune.txt), measured and appended when absent.
        Returns (fw, vc, loaded)."""
        if cache_path is None:
            cache_path = os.environ.get("SGD_AUTOTUNE_CACHE",
                                        os.path.join(os.path.expanduser("~"), ".cache", "sgd_b200", "autotune.txt"))
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        fw, vc = ctypes.c_int(0), ctypes.c_int(0)
        r = self._L.sgd_b1_batch_tune(self.handle, cache_path.encode(), ctypes.addressof(fw), ctypes.addressof(vc))
        if r < 0:
            raise _lib.ProjectorError(f"batch tune: {_lib.last_error()}")
        return fw.value, vc.value, bool(r)


def uneven_slices(seed=0, n=48, lsd=1085.6, lso=595.0):
    """Uneven batch of fan-beam slices: side N ~ U{256, 384, 512} at
    0.5 * 512 / N mm (a 256 mm field), views ~ U{360, 540, 720} over 2 pi,
    ceil(1.44 N) bins at 1 mm."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.choice([256, 384, 512]))
        nv = int(rng.choice([360, 540, 720]))
        d = 0.5 * 512 / N
        out.append((N, N, math.ceil(1.44 * N), d, d, 1.0, lsd, lso, 2 * np.pi * np.arange(nv) / nv))
    return out
