"""The surrogate network's CPU oracle, pinned before it checks the device kernels (no GPU).

oracle/mlp_oracle.py restates the device's BF16 forward and backward passes; the GPU tests
compare the tcgen05 kernels with it.  Here the oracle itself is checked against independent
implementations: its bfloat16 rounding against torch's conversion (round to nearest even),
and its loss and gradients against torch autograd of the same network in float64 with the
same bfloat16 rounding points.
"""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as M  # noqa: E402


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(100_000).astype(np.float32) * 10.0 ** rng.integers(-20, 20, 100_000),
                        np.array([0.0, -0.0, np.inf, -np.inf, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8,
                                  3.0e38, -1.17549435e-38], dtype=np.float32)])
    ours = M.bf16(x)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(ours.view(np.uint32), ref.view(np.uint32))
    assert np.isnan(M.bf16(np.array([np.nan], dtype=np.float32)))[0]


def _net(rng, dims):
    ws = [M.bf16(rng.standard_normal((b, a)).astype(np.float32) / np.sqrt(a)) for a, b in zip(dims[:-1], dims[1:])]
    bs = [rng.standard_normal(b).astype(np.float32) * 0.1 for b in dims[1:]]
    return ws, bs


def _bf16_t(t):
    return t.float().to(torch.bfloat16).double()


def test_loss_and_gradients_match_autograd():
    """torch autograd in float64 with the device's rounding points made explicit: stored
    hidden activations rounded to bfloat16 in the forward pass (the rounding passed through as
    the identity in the backward pass), and the gradient reaching every layer's
    pre-activation rounded to bfloat16 (the device stores dZ in bfloat16)."""
    rng = np.random.default_rng(1)
    dims = (16, 64, 64, 32)
    ws, bs = _net(rng, dims)
    x = M.bf16(rng.standard_normal((128, dims[0])).astype(np.float32))
    y = rng.standard_normal((128, dims[-1])).astype(np.float32)
    loss, dws, dbs, dx = M.loss_and_grads(x, y, ws, bs)

    tw = [torch.tensor(w, dtype=torch.float64, requires_grad=True) for w in ws]
    tb = [torch.tensor(b, dtype=torch.float64, requires_grad=True) for b in bs]
    tx = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    a = tx
    for l, (w, b) in enumerate(zip(tw, tb)):
        z = a @ w.T + b
        z.register_hook(_bf16_t)
        if l < len(tw) - 1:
            r = torch.relu(z)
            a = r + (_bf16_t(r) - r).detach()
        else:
            a = z
    tl = ((a - torch.tensor(y, dtype=torch.float64)) ** 2).mean()
    tl.backward()

    assert abs(loss - tl.item()) <= 1e-5 * tl.item()

    def close(ours, ref, what):
        ref = ref.detach().numpy()
        err = np.linalg.norm(ours - ref) / np.linalg.norm(ref)
        assert err <= 1e-5, (what, err)

    for l in range(len(ws)):
        close(dws[l], tw[l].grad, f"dW{l}")
        close(dbs[l], tb[l].grad, f"db{l}")
    close(dx, tx.grad, "dX")
