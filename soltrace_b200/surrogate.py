"""Learned flux surrogate for aim-point optimisation, trained on the tracer's own output.

A small BF16 multilayer perceptron maps one heliostat's situation -- sun vector (3), field
position (2, in km), aim offset on the receiver (2, m), slope-error sigma (1, mrad) -- to the
flux image it puts on the receiver (32 x 32 bins over the cylinder: angle x height, kW per
bin at 1000 W/m2 DNI).  Summing the heliostats' images gives the field's receiver flux map,
so an aim strategy can be evaluated -- and improved by gradient steps on the aim offsets --
in one batched network pass instead of a trace.  The plain trace stays the judge: training
images come from st_sim_run with a per-source flux map (every heliostat's image in one run),
and every surrogate answer can be checked against a trace of the same configuration.

The network's forward and backward passes run on the library's own kernels
(st_b200_mlp_gemm: tcgen05 tensor-core GEMMs with fused bias/ReLU epilogues; st_b200_mlp_mse,
st_b200_mlp_colsum, st_b200_mlp_adam); PyTorch only provides the device memory and the
stream.  The reference has no counterpart (SolTrace traces every ray).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import scenes

DIMS = (8, 256, 256, 256, 256, 256, 1024)  # 6 layers, width 256, 32 x 32 output image
IMG = 32
EPI_BIAS_RELU_BF16, EPI_BIAS_F32, EPI_RELU_MASK_BF16, EPI_F32, EPI_F32_ADD = range(5)

MLP_SIGNATURES = {
    "st_b200_mlp_gemm": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p,
                                   C.c_longlong, C.c_longlong, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_void_p]),
    "st_b200_mlp_mse": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "st_b200_mlp_colsum": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "st_b200_mlp_adam": (C.c_int, [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                   C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "st_b200_mlp_to_bf16": (C.c_int, [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p]),
    "st_b200_mlp_error": (C.c_int, []),
}


def _ptr(t) -> int:
    return t.data_ptr()


class Mlp:
    """The network on the device: float master weights, their bf16 copies the GEMMs read, Adam
    moments, and the activations of the last forward pass (kept for the backward pass)."""

    def __init__(self, api, dims=DIMS, seed: int = 0, device: str = "cuda"):
        import torch
        self.torch, self.api, self.dims, self.device = torch, api, tuple(dims), device
        for name, (res, args) in MLP_SIGNATURES.items():
            fn = getattr(api.lib, name)
            fn.restype, fn.argtypes = res, args
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.w, self.b = [], []
        for din, dout in zip(dims[:-1], dims[1:]):  # He initialisation
            self.w.append((torch.randn(dout, din, generator=g) * math.sqrt(2.0 / din)).float().to(device))
            self.b.append(torch.zeros(dout, dtype=torch.float32, device=device))
        self.wb = [w.to(torch.bfloat16) for w in self.w]
        self.mw = [torch.zeros_like(w) for w in self.w]
        self.vw = [torch.zeros_like(w) for w in self.w]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step_count = 0
        self.stream = None  # the current torch stream, taken per call
        self.acts = []

    # ---- kernels ----
    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _check(self, rc, what):
        if rc != 1:
            raise RuntimeError(f"{what} failed")

    def gemm(self, m, n, k, a, lam, lak, b, lbn, lbk, c, ldc, epi, bias=None, aux=None, splits=1):
        rc = self.api.lib.st_b200_mlp_gemm(m, n, k, _ptr(a), lam, lak, _ptr(b), lbn, lbk, _ptr(c), ldc, epi,
                                           None if bias is None else _ptr(bias), None if aux is None else _ptr(aux),
                                           splits, self._s())
        self._check(rc, "st_b200_mlp_gemm")

    # ---- passes ----
    def forward(self, x):
        """x: (B, dims[0]) bf16 on the device.  Returns the output (B, dims[-1]) float; the hidden
        activations are kept for backward()."""
        torch = self.torch
        B = x.shape[0]
        acts = [x]
        n = len(self.w)
        for l in range(n):
            din, dout = self.dims[l], self.dims[l + 1]
            last = l == n - 1
            out = torch.empty(B, dout, dtype=torch.float32 if last else torch.bfloat16, device=self.device)
            self.gemm(B, dout, din, acts[-1], din, 1, self.wb[l], din, 1, out, dout,
                      EPI_BIAS_F32 if last else EPI_BIAS_RELU_BF16, bias=self.b[l])
            acts.append(out)
        self.acts = acts
        return acts[-1]

    def backward(self, dy, want_input_grad: bool = False):
        """dy: (B, dims[-1]) bf16 gradient of the loss at the output.  Returns (dW list, db list,
        dX float or None)."""
        torch = self.torch
        B = dy.shape[0]
        n = len(self.w)
        dws, dbs = [None] * n, [None] * n
        dz = dy
        dx = None
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        for l in range(n - 1, -1, -1):
            din, dout = self.dims[l], self.dims[l + 1]
            a_in = self.acts[l]
            dw = torch.zeros(dout, din, dtype=torch.float32, device=self.device)
            tiles = ((dout + 127) // 128) * ((din + 255) // 256)
            splits = max(1, min((B + 63) // 64, sms // max(tiles, 1)))
            # dW = dZ^T A: rows o of dZ^T are dZ's columns (stride dout along the batch)
            self.gemm(dout, din, B, dz, 1, dout, a_in, 1, din, dw, din, EPI_F32_ADD, splits=splits)
            db = torch.empty(dout, dtype=torch.float32, device=self.device)
            self._check(self.api.lib.st_b200_mlp_colsum(B, dout, _ptr(dz), _ptr(db), self._s()), "colsum")
            dws[l], dbs[l] = dw, db
            if l > 0:
                # dZ_prev = (dZ W) where the layer's input activation was positive; W^T read in place
                nxt = torch.empty(B, din, dtype=torch.bfloat16, device=self.device)
                self.gemm(B, din, dout, dz, dout, 1, self.wb[l], 1, din, nxt, din, EPI_RELU_MASK_BF16, aux=a_in)
                dz = nxt
            elif want_input_grad:
                dx = torch.empty(B, din, dtype=torch.float32, device=self.device)
                self.gemm(B, din, dout, dz, dout, 1, self.wb[l], 1, din, dx, din, EPI_F32)
        return dws, dbs, dx

    def loss_grad(self, y, t):
        """Mean-squared error of output y (float) against targets t (float): (loss tensor, dy bf16)."""
        torch = self.torch
        B, N = y.shape
        dy = torch.empty(B, N, dtype=torch.bfloat16, device=self.device)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._check(self.api.lib.st_b200_mlp_mse(B, N, _ptr(y), _ptr(t), t.stride(0), _ptr(dy), _ptr(loss), self._s()),
                    "mse")
        return loss / (B * N), dy

    def train_step(self, x, t, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        y = self.forward(x)
        loss, dy = self.loss_grad(y, t)
        dws, dbs, _ = self.backward(dy)
        self.step_count += 1
        for l in range(len(self.w)):
            self._check(self.api.lib.st_b200_mlp_adam(self.w[l].numel(), _ptr(self.w[l]), _ptr(dws[l]), _ptr(self.mw[l]),
                                                      _ptr(self.vw[l]), _ptr(self.wb[l]), lr, beta1, beta2, eps,
                                                      self.step_count, self._s()), "adam")
            self._check(self.api.lib.st_b200_mlp_adam(self.b[l].numel(), _ptr(self.b[l]), _ptr(dbs[l]), _ptr(self.mb[l]),
                                                      _ptr(self.vb[l]), None, lr, beta1, beta2, eps, self.step_count,
                                                      self._s()), "adam")
        return loss

    def error(self) -> int:
        return self.api.lib.st_b200_mlp_error()
