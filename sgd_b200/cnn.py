"""Small residual CNN used as the ASD-POCS warm start: 5 layers of 3x3
convolutions, 32 channels, ReLU between them, output = input + last layer.
Weights are BF16 on the device (FP32 master copies for Adam), every
convolution accumulates in FP32.  Forward, backward and the optimiser step
run the library's own kernels (sgd_conv3x3_*, sgd_relu_backward,
sgd_mse_grad, sgd_adam_step); torch provides device memory only.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_vp = ctypes.c_void_p


def _declare(L):
    if getattr(L, "_cnn_declared", False):
        return
    i, ll, f = ctypes.c_int, ctypes.c_longlong, ctypes.c_float
    L.sgd_conv3x3_forward.argtypes = [_vp, _vp, _vp, _vp, i, i, i, i, i, i, _vp]
    L.sgd_conv3x3_backward_data.argtypes = [_vp, _vp, _vp, _vp, i, i, i, i, i, _vp]
    L.sgd_conv3x3_backward_weight.argtypes = [_vp, _vp, _vp, _vp, i, i, i, i, i, _vp]
    L.sgd_relu_backward.argtypes = [_vp, _vp, ll, _vp]
    L.sgd_mse_grad.argtypes = [_vp, _vp, _vp, ll, _vp, _vp]
    L.sgd_adam_step.argtypes = [_vp, _vp, _vp, _vp, _vp, ll, f, f, f, f, i, _vp]
    L.sgd_conv3x3_forward_tc.argtypes = [_vp, _vp, _vp, _vp, i, i, i, i, i, i, _vp]
    L.sgd_conv3x3_tc_status.argtypes = []
    for n in ("sgd_conv3x3_forward", "sgd_conv3x3_backward_data", "sgd_conv3x3_backward_weight",
              "sgd_relu_backward", "sgd_mse_grad", "sgd_adam_step", "sgd_conv3x3_forward_tc",
              "sgd_conv3x3_tc_status"):
        getattr(L, n).restype = i
    L._cnn_declared = True


def _stream():
    return torch.cuda.current_stream().cuda_stream


class WarmStartCNN:
    """channels: (1, 32, 32, 32, 32, 1) by default; He-initialised, seeded;
    the last layer starts at zero, so the untrained network is the identity.
    tensor_cores: the forward of 32-to-32-channel layers runs on the tensor
    cores (sgd_conv3x3_forward_tc: exact products, FP32 accumulation in
    tensor memory); the other layers and the backward pass use the FP32
    direct kernels."""

    def __init__(self, channels=(1, 32, 32, 32, 32, 1), seed=0, device=None, tensor_cores=True):
        self.tensor_cores = bool(tensor_cores)
        self.L = _lib.lib()
        _declare(self.L)
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.channels = tuple(channels)
        rng = np.random.default_rng(seed)
        self.w32, self.b = [], []
        for cin, cout in zip(self.channels[:-1], self.channels[1:]):
            std = np.sqrt(2.0 / (9 * cin))
            w = (rng.standard_normal((cout, cin, 3, 3)) * std).astype(np.float32)
            self.w32.append(torch.tensor(w, dtype=torch.float32, device=self.device))
            self.b.append(torch.zeros(cout, dtype=torch.float32, device=self.device))
        self.w32[-1].zero_()
        self.w16 = [w.to(torch.bfloat16) for w in self.w32]
        self.params = self.w32 + self.b
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0
        nmax = max(ci * co * 9 for ci, co in zip(self.channels[:-1], self.channels[1:]))
        self._flip = torch.empty(nmax, dtype=torch.bfloat16, device=self.device)

    def _conv(self, x, k, relu):
        N, C, H, W = x.shape
        cout = self.channels[k + 1]
        out = torch.empty((N, cout, H, W), dtype=torch.float32, device=self.device)
        f = self.L.sgd_conv3x3_forward
        if self.tensor_cores and C == 32 and cout == 32:
            f = self.L.sgd_conv3x3_forward_tc
        _lib.check(f(x.data_ptr(), self.w16[k].data_ptr(), self.b[k].data_ptr(), out.data_ptr(), N, C, cout, H, W,
                     int(relu), _stream()), "sgd_conv3x3_forward")
        return out

    def forward(self, x, keep=False):
        """x: (N, 1, H, W) float32 -> x + net(x).  keep=True stores the
        activations for backward()."""
        acts = [x.contiguous()]
        h = acts[0]
        nl = len(self.channels) - 1
        for k in range(nl):
            h = self._conv(h, k, relu=(k < nl - 1))
            acts.append(h)
        if keep:
            self._acts = acts
        return x + h

    def backward(self, gy):
        """Gradients of the parameters for dL/dy = gy (N, 1, H, W): weights
        (FP32), then biases."""
        acts = self._acts
        nl = len(self.channels) - 1
        gw = [torch.zeros_like(w) for w in self.w32]
        gb = [torch.zeros_like(b) for b in self.b]
        g = gy.contiguous().clone()
        for k in reversed(range(nl)):
            a_in, a_out = acts[k], acts[k + 1]
            N, C, H, W = a_in.shape
            cout = self.channels[k + 1]
            if k < nl - 1:
                _lib.check(self.L.sgd_relu_backward(g.data_ptr(), a_out.data_ptr(), g.numel(), _stream()),
                           "sgd_relu_backward")
            _lib.check(self.L.sgd_conv3x3_backward_weight(a_in.data_ptr(), g.data_ptr(), gw[k].data_ptr(),
                                                          gb[k].data_ptr(), N, C, cout, H, W, _stream()),
                       "sgd_conv3x3_backward_weight")
            if k > 0:
                gin = torch.empty_like(a_in)
                _lib.check(self.L.sgd_conv3x3_backward_data(g.data_ptr(), self.w16[k].data_ptr(),
                                                            self._flip.data_ptr(), gin.data_ptr(), N, C, cout, H, W,
                                                            _stream()),
                           "sgd_conv3x3_backward_data")
                g = gin
        return gw + gb

    def mse_grad(self, y, t):
        """(dL/dy, sum of squared errors) for L = mean((y - t)^2)."""
        g = torch.empty_like(y)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        _lib.check(self.L.sgd_mse_grad(y.data_ptr(), t.data_ptr(), g.data_ptr(), y.numel(), loss.data_ptr(),
                                       _stream()), "sgd_mse_grad")
        return g, loss

    def adam(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        nw = len(self.w32)
        for k, (p, g, m, v) in enumerate(zip(self.params, grads, self.m, self.v)):
            w16 = self.w16[k].data_ptr() if k < nw else None
            _lib.check(self.L.sgd_adam_step(p.data_ptr(), w16, g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                                            lr, b1, b2, eps, self.step_count, _stream()), "sgd_adam_step")

    def train_step(self, x, t, lr=1e-3):
        y = self.forward(x, keep=True)
        g, loss = self.mse_grad(y, t)
        self.adam(self.backward(g), lr=lr)
        return loss

    # -- checkpoints ---------------------------------------------------------

    def state_dict(self):
        """Everything training resumes from, as host tensors: the FP32
        master weights and biases, Adam's moments and its step count (the
        BF16 weights are derived from the masters)."""
        host = lambda ts: [p.detach().to("cpu", copy=True) for p in ts]  # noqa: E731
        return {"channels": list(self.channels), "w32": host(self.w32), "b": host(self.b),
                "m": host(self.m), "v": host(self.v), "step_count": int(self.step_count)}

    def load_state_dict(self, sd):
        """Inverse of state_dict(); the architecture must match."""
        if tuple(sd["channels"]) != self.channels:
            raise ValueError(f"checkpoint channels {tuple(sd['channels'])} != network channels {self.channels}")
        for key, dst in (("w32", self.w32), ("b", self.b), ("m", self.m), ("v", self.v)):
            src = sd[key]
            if len(src) != len(dst) or any(tuple(s.shape) != tuple(d.shape) for s, d in zip(src, dst)):
                raise ValueError(f"checkpoint tensor shapes of '{key}' do not match the network")
            for s, d in zip(src, dst):
                d.copy_(s)
        for w16, w32 in zip(self.w16, self.w32):
            w16.copy_(w32)
        self.step_count = int(sd["step_count"])

    def save(self, path):
        torch.save(self.state_dict(), path)

    def load(self, path):
        self.load_state_dict(torch.load(path, map_location="cpu", weights_only=True))
