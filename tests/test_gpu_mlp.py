"""The flux surrogate's tensor-core kernels (st_b200_mlp_*), against host references.

* GEMM (tcgen05, FP32 accumulation in tensor memory): C = epilogue(A B^T) for ragged shapes,
  operands read in place through strides (as the backward pass reads them), every epilogue
  and split-K, against float64 products of the same bf16 values (relative error 1e-5 of the
  result's scale, with bf16 rounding of the stored outputs allowed for).
* The whole network: forward output, loss and every layer's weight and bias gradients
  against the CPU oracle (oracle/mlp_oracle.py), which restates the network in float32 with
  the device's bf16 roundings; and a short training run on a fixed teacher network that must
  cut the loss tenfold.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mlp_env(product):
    import torch
    from soltrace_b200.surrogate import Mlp
    net = Mlp(product, dims=(8, 256, 256, 1024), seed=1)  # binds the kernels
    return torch, net


def _bf(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


CASES = [  # (m, n, k, transposed A, transposed B, epilogue, splits)
    (128, 256, 64, False, False, 3, 1),
    (300, 200, 100, False, False, 1, 1),
    (1000, 1024, 256, False, False, 0, 1),
    (77, 8, 256, False, True, 3, 1),       # dX of an 8-wide input layer, W read transposed
    (256, 256, 2048, True, True, 4, 8),    # dW = dZ^T X: both operands strided, split over K
    (256, 8, 1000, True, True, 4, 5),
    (513, 256, 256, False, True, 2, 1),    # dZ through the ReLU mask
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}x{c[2]}-e{c[5]}-s{c[6]}" for c in CASES])
def test_gemm_matches_host(mlp_env, case):
    torch, net = mlp_env
    m, n, k, ta, tb, epi, splits = case
    rng = np.random.default_rng(m * 7 + n + k)
    a = rng.normal(size=(m, k)).astype(np.float32)
    b = rng.normal(size=(n, k)).astype(np.float32)
    # stored the way the kernel is asked to read them: transposed operands in place
    A = _bf(torch, a.T.copy() if ta else a)
    B = _bf(torch, b.T.copy() if tb else b)
    lam, lak = (1, m) if ta else (k, 1)
    lbn, lbk = (1, n) if tb else (k, 1)
    ab = A.float().cpu().numpy()
    bb = B.float().cpu().numpy()
    ab = ab.T if ta else ab
    bb = bb.T if tb else bb
    ref = ab.astype(np.float64) @ bb.astype(np.float64).T
    bias = torch.from_numpy(rng.normal(size=n).astype(np.float32)).cuda()
    aux = _bf(torch, rng.normal(size=(m, n)))
    if epi in (0, 2):
        C = torch.zeros(m, n, dtype=torch.bfloat16, device="cuda")
    else:
        C = torch.full((m, n), 0.25 if epi == 4 else 0.0, dtype=torch.float32, device="cuda")
    net.gemm(m, n, k, A, lam, lak, B, lbn, lbk, C, n, epi, bias=bias if epi in (0, 1) else None,
             aux=aux if epi == 2 else None, splits=splits)
    torch.cuda.synchronize()
    assert net.error() == 0
    got = C.float().cpu().numpy().astype(np.float64)
    bias_h = bias.cpu().numpy().astype(np.float64)
    if epi == 0:
        want = np.maximum(ref + bias_h, 0.0)
    elif epi == 1:
        want = ref + bias_h
    elif epi == 2:
        want = np.where(aux.float().cpu().numpy() > 0, ref, 0.0)
    elif epi == 3:
        want = ref
    else:
        want = ref + 0.25
    scale = np.abs(ref).max()
    tol = (1e-5 if epi in (1, 3, 4) else 8e-3) * scale  # bf16 outputs keep 8 bits
    err = np.abs(got - want).max()
    assert err <= tol, (err, tol)


def test_network_gradients_match_oracle(product):
    import torch
    import mlp_oracle
    from soltrace_b200.surrogate import Mlp
    dims = (8, 256, 256, 256, 1024)
    net = Mlp(product, dims=dims, seed=3)
    rng = np.random.default_rng(5)
    B = 512
    x = rng.normal(size=(B, dims[0])).astype(np.float32)
    t = rng.normal(size=(B, dims[-1])).astype(np.float32)
    for b in net.b:  # non-zero biases exercise the bias path
        b.copy_(torch.from_numpy(rng.normal(scale=0.1, size=b.numel()).astype(np.float32)))
    xb = torch.from_numpy(x).to(torch.bfloat16).cuda()
    tb = torch.from_numpy(t).cuda()
    y = net.forward(xb)
    loss, dy = net.loss_grad(y, tb)
    dws, dbs, dx = net.backward(dy, want_input_grad=True)
    torch.cuda.synchronize()
    assert net.error() == 0
    ws = [w.cpu().numpy() for w in net.w]
    bs = [b.cpu().numpy() for b in net.b]
    o_loss, o_dws, o_dbs, o_dx = mlp_oracle.loss_and_grads(x, t, ws, bs)
    o_y = mlp_oracle.forward(x, ws, bs)[-1]

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))

    assert rel(y.cpu().numpy(), o_y) < 5e-3
    assert abs(loss.item() - o_loss) / o_loss < 1e-3
    for l in range(len(dims) - 1):
        assert rel(dws[l].cpu().numpy(), o_dws[l]) < 2e-2, l
        assert rel(dbs[l].cpu().numpy(), o_dbs[l]) < 2e-2, l
    assert rel(dx.cpu().numpy(), o_dx) < 2e-2


def test_network_learns_teacher(product):
    """A fixed random teacher network's outputs are learned: the loss falls tenfold in 300
    Adam steps of the device kernels."""
    import torch
    from soltrace_b200.surrogate import Mlp
    dims = (8, 256, 256, 256, 64)
    teacher = Mlp(product, dims=dims, seed=11)
    net = Mlp(product, dims=dims, seed=12)
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(8192, 8, generator=g).to(torch.bfloat16).cuda()
    t = teacher.forward(x).clone()
    first = net.train_step(x, t, lr=1e-3).item()
    for _ in range(300):
        last = net.train_step(x, t, lr=1e-3)
    torch.cuda.synchronize()
    assert net.error() == 0
    assert last.item() < first / 10, (first, last.item())


FUSED_CASES = [  # (rows, dims, group_rows)
    (77, (8, 256, 256, 1024), 0),                       # one partial tile
    (40_000, (8, 256, 256, 256, 256, 256, 1024), 0),    # more tiles than SMs: the persistent loop
    (5_000, (3, 256, 256, 256, 512), 0),
    (6_000, (8, 256, 256, 256, 256, 256, 1024), 2000),  # field sums: warps straddle group edges
    (1_000, (16, 256, 256), 7),                         # every warp straddles one
]


@pytest.mark.parametrize("case", FUSED_CASES, ids=[f"{c[0]}-{len(c[1]) - 1}L-{c[1][-1]}-g{c[2]}" for c in FUSED_CASES])
def test_fused_forward_matches_layers(product, case):
    """The fused kernel (all layers in one launch, activations kept on chip) gives the per-layer
    GEMM path's output: the same bf16 roundings between layers and the same K order in the
    accumulator, so rows agree to float rounding; group sums agree with summing those rows."""
    import torch
    from soltrace_b200.surrogate import Mlp
    rows, dims, group = case
    net = Mlp(product, dims=dims, seed=rows)
    rng = np.random.default_rng(rows)
    for b in net.b:
        b.copy_(torch.from_numpy(rng.normal(scale=0.1, size=b.numel()).astype(np.float32)))
    x = torch.from_numpy(rng.normal(size=(rows, dims[0])).astype(np.float32)).to(torch.bfloat16).cuda()
    want = net.forward(x).double()
    scale = 0.5
    got = net.forward_fused(x, group_rows=group, scale=scale, clamp=group > 0)
    torch.cuda.synchronize()
    assert net.error() == 0
    if group == 0:
        err = (got.double() - scale * want).abs().max().item()
        assert err <= 1e-5 * (scale * want).abs().max().item(), err
    else:
        per_row = (scale * want).clamp(min=0.0)
        sums = torch.stack([per_row[i:i + group].sum(0) for i in range(0, rows, group)])
        err = (got.double() - sums).abs().max().item()
        assert err <= 1e-5 * sums.abs().max().item(), err

