"""CPU oracle of the flux surrogate's network (test infrastructure only).

A plain numpy restatement of what the device's BF16 MLP kernels compute, used by the
tests to check their forward values and gradients: layers of Y = act(X W^T + b) with
X and W rounded to bfloat16 (round to nearest even, as the device converts them), the
products accumulated in float32, ReLU on the hidden layers and none on the output, and
the mean-squared-error loss against the target images.  Backward: dZ = dA * (A > 0),
dW = dZ^T X, db = sum over rows of dZ, dX = dZ W, with the activations and incoming
gradients rounded to bfloat16 where the device stores them in bfloat16.

This network has no counterpart in the reference (SolTrace traces every ray); its error is
measured against the plain trace.  Nothing in the product imports this file.
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(np.asarray(x, dtype=np.float32))
    out = r.astype(np.uint32).view(np.float32).copy()
    out[nan] = np.nan
    return out


def forward(x: np.ndarray, weights: list, biases: list):
    """Activations of every layer (bf16-rounded hidden outputs as the device stores them; the
    last layer's output in float32).  x: (B, d0); weights[l]: (d_{l+1}, d_l)."""
    acts = [bf16(x)]
    n = len(weights)
    for l, (w, b) in enumerate(zip(weights, biases)):
        z = acts[-1].astype(np.float32) @ bf16(w).T.astype(np.float32) + b.astype(np.float32)
        if l < n - 1:
            acts.append(bf16(np.maximum(z, 0.0)))
        else:
            acts.append(z.astype(np.float32))
    return acts


def loss_and_grads(x: np.ndarray, y: np.ndarray, weights: list, biases: list):
    """Mean-squared-error loss over all outputs and its gradients (dW per layer, db per layer,
    dX of the input), following the device's rounding of stored intermediates."""
    acts = forward(x, weights, biases)
    out = acts[-1]
    n_out = out.size
    diff = out - y.astype(np.float32)
    loss = float(np.sum(diff.astype(np.float64) ** 2) / n_out)
    dz = bf16(2.0 * diff / n_out)
    dws, dbs = [None] * len(weights), [None] * len(weights)
    dx = None
    for l in range(len(weights) - 1, -1, -1):
        a_in = acts[l].astype(np.float32)
        dws[l] = dz.T.astype(np.float32) @ a_in
        dbs[l] = dz.astype(np.float32).sum(axis=0)
        da = dz.astype(np.float32) @ bf16(weights[l]).astype(np.float32)
        if l > 0:
            dz = bf16(da * (acts[l] > 0))
        else:
            dx = da
    return loss, dws, dbs, dx
