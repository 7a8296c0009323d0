"""Learned flux surrogate for aim-point optimisation, trained on the tracer's own output.

A small BF16 multilayer perceptron maps one heliostat's situation -- sun vector (3), field
position (2, in km), aim offset on the receiver (2, m), slope-error sigma (1, mrad), and eight
quantities the bisector aiming rule derives from them (see situation_features) -- to the
flux image it puts on the receiver (32 x 32 bins over the cylinder: angle x height, kW per
bin at 1000 W/m2 DNI).  Summing the heliostats' images gives the field's receiver flux map,
so an aim strategy can be evaluated -- and improved by gradient steps on the aim offsets --
in one batched network pass instead of a trace.  The plain trace stays the reference: training
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

N_FEATURES = 16
DIMS = (N_FEATURES, 256, 256, 256, 256, 256, 1024)  # 6 layers, width 256, 32 x 32 output image
HELIO_Z = 5.0  # heliostat pivot height of the field layout (m)


def situation_features(sun, x, y, ox, oy, sigma, tower_h: float, xp=np):
    """The network's 16 inputs per heliostat, as columns of an (n, 16) array of the array
    module xp (numpy, or torch for the aim optimiser, where ox and oy carry gradients): sun
    unit vector (3), position in km (2), aim offset east and up in m (2), slope sigma - 2
    mrad (1); then quantities the heliostat's geometry derives from those: distance to the
    tower base in km, the horizontal unit vector toward it (2), the mirror normal of the
    bisector aiming rule (3), the cosine of the sun on the mirror, and the vertical
    component of the unit vector toward the aim point.  The derived columns are functions of
    the first eight; they give the network the image's orientation and foreshortening
    directly (the worst held-out peak error fell from about 5 % to under 3 %)."""
    s = [float(c) for c in sun]
    sn = (s[0] ** 2 + s[1] ** 2 + s[2] ** 2) ** 0.5
    s = [c / sn for c in s]
    one = x * 0.0 + 1.0
    r = (x * x + y * y) ** 0.5
    tx, ty, tz = ox - x, -y, tower_h + oy - HELIO_Z
    tl = (tx * tx + ty * ty + tz * tz) ** 0.5
    tx, ty, tz = tx / tl, ty / tl, tz / tl
    nx, ny, nz = s[0] + tx, s[1] + ty, s[2] + tz
    nl = (nx * nx + ny * ny + nz * nz) ** 0.5
    nx, ny, nz = nx / nl, ny / nl, nz / nl
    cols = [s[0] * one, s[1] * one, s[2] * one, x / 1000.0, y / 1000.0, ox, oy, (sigma - 2.0) * one,
            r / 1000.0, -x / r, -y / r, nx, ny, nz, s[0] * nx + s[1] * ny + s[2] * nz, tz]
    return xp.stack(cols, 1)
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
    "st_b200_mlp_packed_bytes": (C.c_longlong, [C.c_int, C.c_void_p]),
    "st_b200_mlp_pack": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "st_b200_mlp_forward_fused": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                            C.c_longlong, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int,
                                            C.c_void_p]),
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
        self.acts = []
        self._packed, self._packed_step = None, -1

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

    def packed(self):
        """The bf16 weights laid out for the fused forward; rebuilt after training steps (the
        layout is a copy: edit weights through train_step, or drop _packed after editing wb)."""
        torch = self.torch
        if self._packed is None or self._packed_step != self.step_count:
            dims = (C.c_int * len(self.dims))(*self.dims)
            nbytes = self.api.lib.st_b200_mlp_packed_bytes(len(self.w), dims)
            if nbytes < 0:
                raise ValueError(f"dims {self.dims} not supported by the fused forward")
            blob = torch.empty(nbytes // 2, dtype=torch.bfloat16, device=self.device)
            ptrs = (C.c_void_p * len(self.wb))(*[w.data_ptr() for w in self.wb])
            self._check(self.api.lib.st_b200_mlp_pack(len(self.w), dims, ptrs, _ptr(blob), self._s()), "pack")
            self._packed, self._packed_step = blob, self.step_count
        return self._packed

    def forward_fused(self, x, group_rows: int = 0, scale: float = 1.0, clamp: bool = False, out=None):
        """Inference through the fused kernel (all layers in one launch).  x: (B, dims[0]) bf16.
        group_rows 0: every row's output (B, dims[-1]); otherwise the sums over consecutive
        groups of group_rows rows (ceil(B / group_rows), dims[-1]), added into `out` when given.
        Outputs are scaled by `scale` and, with clamp, clipped to >= 0 before any sum."""
        torch = self.torch
        B, n_out = x.shape[0], self.dims[-1]
        blob = self.packed()
        dims = (C.c_int * len(self.dims))(*self.dims)
        bias = (C.c_void_p * len(self.b))(*[b.data_ptr() for b in self.b])
        if out is None:
            rows = B if group_rows <= 0 else -(-B // group_rows)
            out = torch.zeros(rows, n_out, dtype=torch.float32, device=self.device)
        rc = self.api.lib.st_b200_mlp_forward_fused(len(self.w), dims, _ptr(blob), bias, B, _ptr(x), x.stride(0),
                                                     _ptr(out), 0 if group_rows <= 0 else 1, max(group_rows, 1),
                                                     float(scale), 1 if clamp else 0, self._s())
        self._check(rc, "st_b200_mlp_forward_fused")
        return out

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


# ------------------------------------------------------------------------------------
# Training data from the tracer
# ------------------------------------------------------------------------------------
RECEIVER_IMAGE = (2, 1, 1, IMG, IMG, 0.0, 4.0, -5.0, 5.0, 1)  # receiver: angle x height, absorbed rays


class FieldTracer:
    """The headline field (2,000 flat heliostats, cylindrical receiver, Buie CSR 0.1) in one
    context of the product library, re-aimed per call: every heliostat aims at the receiver
    centre plus its own offset (east, up) by the bisector rule, under a given sun and slope
    error.  trace() returns every heliostat's receiver image in kW per bin at 1000 W/m2."""

    def __init__(self, api, n_helio: int = 2000, tower_h: float = 150.0, precision: int = 1):
        self.api, self.n, self.tower_h = api, n_helio, tower_h
        self.sc = scenes.field_scene(n_helio, 1000, dynamic_group=False)
        self.xy = scenes.field_layout(n_helio)
        self.ctx = api.st_create_context()
        scenes.push(api, self.ctx, self.sc)
        api.st_b200_set_records(self.ctx, 0)
        api.st_b200_set_precision(self.ctx, precision)
        self.img = api.st_b200_add_source_flux_map(self.ctx, *RECEIVER_IMAGE)
        self.whole = api.st_b200_add_flux_map(self.ctx, *RECEIVER_IMAGE)

    def close(self):
        self.api.st_free_context(self.ctx)

    def aim(self, sun: np.ndarray, offsets: np.ndarray, sigma: float):
        api, ctx = self.api, self.ctx
        s = np.asarray(sun, dtype=np.float64) / np.linalg.norm(sun)
        api.st_sun_xyz(ctx, *(1.0e4 * s))
        for k, (x, y) in enumerate(self.xy):
            pos = np.array([x, y, 5.0])
            t = np.array([offsets[k, 0], 0.0, self.tower_h + offsets[k, 1]]) - pos
            n = s + t / np.linalg.norm(t)
            a = pos + 100.0 * n / np.linalg.norm(n)
            api.st_element_aim(ctx, 0, k, float(a[0]), float(a[1]), float(a[2]))
        from .scenes import OpticFace, OpticSet, push_optic
        push_optic(api, ctx, 0, OpticSet("helio", OpticFace("g", refl=0.9, slope=sigma), OpticFace("g", refl=0.9, slope=sigma)))

    def trace(self, sun, offsets, sigma: float, hits: int, seed: int):
        """(per-heliostat images (n, 32, 32), whole-receiver map (32, 32)), kW per bin."""
        api, ctx = self.api, self.ctx
        self.aim(sun, offsets, sigma)
        api.st_sim_params(ctx, int(hits), 2_000_000_000 - 1, 0)
        api.st_b200_set_max_sun_rays(ctx, 40 * int(hits))
        if api.run(ctx, seed) < 0:
            raise RuntimeError("; ".join(api.messages(ctx)))
        st = api.stats(ctx)
        box = api.sun_stats(ctx)
        ppr_kw = 1000.0 * (box["xmax"] - box["xmin"]) * (box["ymax"] - box["ymin"]) / st["sun_rays"] / 1000.0
        imgs = api.source_flux(ctx, self.img, self.n, IMG, IMG).astype(np.float32) * ppr_kw
        whole = api.flux(ctx, self.whole, IMG, IMG).astype(np.float64) * ppr_kw
        return imgs, whole

    def features(self, sun, offsets, sigma: float) -> np.ndarray:
        """The network's inputs per heliostat (situation_features), float32 (n, 16)."""
        off = np.asarray(offsets, dtype=np.float64)
        return situation_features(sun, self.xy[:, 0].astype(np.float64), self.xy[:, 1].astype(np.float64),
                                  off[:, 0], off[:, 1], sigma, self.tower_h).astype(np.float32)


def random_situation(rng, n: int):
    """A random sun (elevation 20-80 deg, azimuth 100-260 deg from north), aim offsets
    uniform in [-1, 1] m and slope error uniform in [1, 3] mrad."""
    sun = scenes.sun_vector(rng.uniform(20.0, 80.0), rng.uniform(100.0, 260.0))
    return sun, rng.uniform(-1.0, 1.0, size=(n, 2)), float(rng.uniform(1.0, 3.0))


def make_dataset(tracer: FieldTracer, n_traces: int, hits: int, seed: int = 0):
    """Inputs (n_traces * n, 8) float32 and target images (n_traces * n, 1024) float32 (kW per
    bin), on the device."""
    import torch
    rng = np.random.default_rng(seed)
    xs, ts = [], []
    for i in range(n_traces):
        sun, off, sig = random_situation(rng, tracer.n)
        imgs, _ = tracer.trace(sun, off, sig, hits, seed * 100_003 + i)
        xs.append(torch.from_numpy(tracer.features(sun, off, sig)).cuda())
        ts.append(torch.from_numpy(imgs.reshape(tracer.n, IMG * IMG)).cuda())
    return torch.cat(xs), torch.cat(ts)


def train(net: Mlp, x, t, steps: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0, target_scale: float = None,
          lr_final: float = 0.1):
    """Adam on random minibatches, the learning rate decayed exponentially to lr * lr_final
    over the run.  Targets are divided by target_scale (default: their 99.9th percentile) so
    the network sees O(1) values; returns (scale, loss history)."""
    import torch
    if target_scale is None:
        target_scale = float(torch.quantile(t.flatten()[:: max(1, t.numel() // 4_000_000)].float(), 0.999).item())
        target_scale = max(target_scale, 1e-6)
    g = torch.Generator(device="cuda").manual_seed(seed)
    xb = x.to(torch.bfloat16)
    hist = []
    for k in range(steps):
        idx = torch.randint(0, x.shape[0], (batch,), device="cuda", generator=g)
        step_lr = lr * (lr_final ** (k / max(steps - 1, 1)))
        loss = net.train_step(xb[idx], t[idx] / target_scale, lr=step_lr)
        if k % 50 == 0 or k == steps - 1:
            hist.append(float(loss.item()))
    return target_scale, hist


def predict_images(net: Mlp, feats, target_scale: float):
    """Per-heliostat images (n, 1024) in kW per bin (negative network outputs clipped to 0)."""
    import torch
    x = torch.as_tensor(feats).cuda().to(torch.bfloat16)
    return torch.clamp(net.forward(x), min=0.0) * target_scale


def predict_fields(net: Mlp, feats, n_helio: int, target_scale: float):
    """Field receiver maps (n_situations, 1024) in kW per bin: the per-heliostat images
    (clipped to >= 0) of every n_helio consecutive rows summed inside the fused kernel."""
    import torch
    x = torch.as_tensor(feats).cuda().to(torch.bfloat16)
    return net.forward_fused(x, group_rows=n_helio, scale=target_scale, clamp=True)


def peak_error(pred_map: np.ndarray, trace_map: np.ndarray) -> float:
    """|peak(pred) - peak(trace)| / peak(trace) of two field maps (kW per bin)."""
    return abs(float(pred_map.max()) - float(trace_map.max())) / max(float(trace_map.max()), 1e-30)


def optimise_aims(net: Mlp, tracer: "FieldTracer", sun, offsets, sigma: float, target_scale: float, iters: int = 60,
                  step: float = 0.05):
    """Aim offsets that flatten the predicted receiver map: gradient descent, through the
    network's backward kernels to its inputs and from them (torch autograd over
    situation_features) to the offsets, on sum(F^4) / sum(F)^4 of the field map F (a smooth
    stand-in for the peak over the total), offsets kept in [-1, 1] m.  Returns the offsets
    (n, 2)."""
    import torch
    x = torch.as_tensor(tracer.xy[:, 0], dtype=torch.float64, device="cuda")
    y = torch.as_tensor(tracer.xy[:, 1], dtype=torch.float64, device="cuda")
    off = torch.as_tensor(np.asarray(offsets, dtype=np.float64), device="cuda").clone()
    for _ in range(iters):
        o = off.clone().requires_grad_(True)
        feats = situation_features(sun, x, y, o[:, 0], o[:, 1], sigma, tracer.tower_h, xp=torch)
        out = net.forward(feats.detach().to(torch.bfloat16))
        yv = torch.clamp(out, min=0.0)
        f = yv.sum(0).double()
        s1, s4 = f.sum(), (f ** 4).sum()
        dldf = 4 * f ** 3 / s1 ** 4 - 4 * s4 / s1 ** 5        # d(sum F^4 / (sum F)^4) / dF
        dldf = (dldf / dldf.abs().max().clamp(min=1e-300)).float()
        # every heliostat's image adds to F: the same dL/dF for each, through the clipping
        dy = (dldf.unsqueeze(0) * (out > 0)).to(torch.bfloat16).contiguous()
        _, _, dx = net.backward(dy, want_input_grad=True)
        feats.backward(dx.double())
        g = o.grad
        g = g / g.abs().max().clamp(min=1e-30)
        off = (off - step * g).clamp(-1.0, 1.0)
    return off.cpu().numpy()


# ------------------------------------------------------------------------------------
# Fitting and judging against the trace
# ------------------------------------------------------------------------------------
def fit(tracer: FieldTracer, n_traces: int, hits: int, steps: int, seed: int = 1, dims=DIMS, batch: int = 8192,
        lr: float = 2e-3, lr_final: float = 0.1):
    """A network trained on n_traces random situations traced at `hits` first-stage hits each:
    (net, target_scale, seconds spent tracing, seconds spent training)."""
    import time

    import torch
    t0 = time.perf_counter()
    x, t = make_dataset(tracer, n_traces, hits, seed=seed)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = Mlp(tracer.api, dims=dims, seed=seed)
    scale, _ = train(net, x, t, steps=steps, batch=batch, lr=lr, lr_final=lr_final)
    torch.cuda.synchronize()
    return net, scale, t1 - t0, time.perf_counter() - t1


def evaluate(net: Mlp, tracer: FieldTracer, target_scale: float, n: int, hits: int, seed: int = 999,
          noise: list = None):
    """Field maps predicted for n held-out random situations (half of them with every aim
    offset 0) against traces of the same situations at `hits` hits: per situation the
    relative peak error |peak(pred) - peak(trace)| / peak(trace) and the relative L1 map
    error sum |pred - trace| / sum trace.  With `noise` (a list), each situation is traced a
    second time with another seed and the peak error of that repeat against the first trace
    (the judging trace's own Monte-Carlo noise in the same measure) is appended to it."""
    rng = np.random.default_rng(seed)
    peaks, l1 = [], []
    for i in range(n):
        sun, off, sig = random_situation(rng, tracer.n)
        if i % 2 == 0:
            off[:] = 0.0
        _, whole = tracer.trace(sun, off, sig, hits, 5000 + i)
        pred = predict_fields(net, tracer.features(sun, off, sig), tracer.n, target_scale)[0]
        pred = pred.reshape(IMG, IMG).double().cpu().numpy()
        peaks.append(peak_error(pred, whole))
        l1.append(float(np.abs(pred - whole).sum() / max(whole.sum(), 1e-30)))
        if noise is not None:
            _, again = tracer.trace(sun, off, sig, hits, 7000 + i)
            noise.append(peak_error(again, whole))
    return peaks, l1


def fused_flops(dims, rows: int) -> float:
    """Multiply-adds x 2 of one forward pass over `rows` inputs (the input layer at its true
    width, not the 16 the kernel pads it to)."""
    return 2.0 * rows * sum(a * b for a, b in zip(dims[:-1], dims[1:]))


def time_fields(net: Mlp, tracer: FieldTracer, target_scale: float, n_suns: int = 64, reps: int = 20, seed: int = 3):
    """Device milliseconds of one fused pass that predicts n_suns field maps of tracer.n
    heliostats each (CUDA events on the launching stream, after 3 warm-up passes)."""
    import torch
    rng = np.random.default_rng(seed)
    feats = np.concatenate([tracer.features(*random_situation(rng, tracer.n)) for _ in range(n_suns)])
    x = torch.as_tensor(feats).cuda().to(torch.bfloat16)
    out = torch.zeros(n_suns, IMG * IMG, dtype=torch.float32, device="cuda")
    for _ in range(3):
        net.forward_fused(x, group_rows=tracer.n, scale=target_scale, clamp=True, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        out.zero_()
        net.forward_fused(x, group_rows=tracer.n, scale=target_scale, clamp=True, out=out)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _time_fused_forward(rows: int = 64 * 2000, group: int = 2000, reps: int = 20) -> None:
    """Times the fused forward of a randomly initialised network on `rows` random inputs summed
    per `group` rows (the field maps of rows / group suns): device milliseconds per pass and
    TFLOP/s, with 4 warm-up passes.  `python -m soltrace_b200.surrogate`."""
    import torch

    from .lib import load
    net = Mlp(load(), seed=3)
    x = torch.randn(rows, DIMS[0], device="cuda").to(torch.bfloat16)  # random inputs: timing only
    out = torch.zeros(-(-rows // group), DIMS[-1], dtype=torch.float32, device="cuda")
    for _ in range(4):
        net.forward_fused(x, group_rows=group, scale=1.0, clamp=True, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward_fused(x, group_rows=group, scale=1.0, clamp=True, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    print(f"fused forward, {rows} rows in groups of {group}: {ms:.4f} ms per pass, "
          f"{fused_flops(DIMS, rows) / (ms / 1e3) / 1e12:.1f} TFLOP/s, error flag {net.error()}")


if __name__ == "__main__":
    _time_fused_forward()
