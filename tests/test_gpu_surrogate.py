"""The warm-start surrogate's kernels: the BF16 GEMM (every operand layout,
bias + GELU epilogue, split reduction) against float64 products of the same
BF16 values, and the network's loss and gradients against the CPU oracle
with BF16 rounding at the same points."""
import ctypes

import numpy as np
import pytest
import torch

from cudadsmc_b200 import lib
from cudadsmc_b200.surrogate import WarmStartMLP
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def dev_bf16(a, cuda):
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(cuda)
    out = torch.empty(t.shape, dtype=torch.bfloat16, device=cuda)
    assert lib().dsmc_to_bf16(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(out.data_ptr()), t.numel(),
                              None) == 0
    return out


def P(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("at,bt", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_gemm_layouts(cuda, at, bt):
    rng = np.random.default_rng(10 + 2 * at + bt)
    m, n, k = 200, 136, 72
    A = M.bf16(rng.normal(0, 1, (m, k)))
    B = M.bf16(rng.normal(0, 1, (k, n)))
    a_store = A.T if at else A
    b_store = B.T if bt else B
    a = dev_bf16(a_store, cuda)
    b = dev_bf16(b_store, cuda)
    c = torch.zeros((m, n), dtype=torch.float32, device=cuda)
    st = lib().dsmc_gemm_bf16(m, n, k, P(a), a_store.shape[1], at, P(b), b_store.shape[1], bt, P(c), n,
                              0.0, None, 0, None, 0, 1, None)
    assert st == 0
    torch.cuda.synchronize()
    ref = A @ B
    assert np.max(np.abs(c.cpu().numpy() - ref)) <= 1e-4 * np.max(np.abs(ref)) + 1e-4


def test_gemm_epilogue_and_split(cuda):
    rng = np.random.default_rng(3)
    m, n, k = 64, 256, 4096
    A = M.bf16(rng.normal(0, 1, (m, k)))
    B = M.bf16(rng.normal(0, 1, (k, n)))
    bias = rng.normal(0, 1, n).astype(np.float32)
    a, b = dev_bf16(A, cuda), dev_bf16(B, cuda)
    bias_t = torch.from_numpy(bias).to(cuda)
    z = torch.zeros((m, n), dtype=torch.float32, device=cuda)
    h = torch.empty((m, n), dtype=torch.bfloat16, device=cuda)
    assert lib().dsmc_gemm_bf16(m, n, k, P(a), k, 0, P(b), n, 0, P(z), n, 0.0, P(bias_t), 1, P(h), n, 1,
                                None) == 0
    split = torch.zeros((m, n), dtype=torch.float32, device=cuda)
    assert lib().dsmc_gemm_bf16(m, n, k, P(a), k, 0, P(b), n, 0, P(split), n, 0.0, None, 0, None, 0, 16,
                                None) == 0
    acc = torch.ones((m, n), dtype=torch.float32, device=cuda)
    assert lib().dsmc_gemm_bf16(m, n, k, P(a), k, 0, P(b), n, 0, P(acc), n, 2.0, None, 0, None, 0, 1,
                                None) == 0
    torch.cuda.synchronize()
    ref = A @ B
    tol = 1e-4 * np.max(np.abs(ref))
    assert np.max(np.abs(z.cpu().numpy() - (ref + bias))) <= tol
    assert np.max(np.abs(split.cpu().numpy() - ref)) <= tol
    assert np.max(np.abs(acc.cpu().numpy() - (ref + 2.0))) <= tol
    hg = h.float().cpu().numpy()
    assert np.max(np.abs(hg - M.bf16(M.gelu(ref + bias)))) <= 0.01 * np.max(np.abs(ref))
    # refused shapes: k not a multiple of 8
    assert lib().dsmc_gemm_bf16(m, n, 12, P(a), k, 0, P(b), n, 0, P(z), n, 0.0, None, 0, None, 0, 1,
                                None) == 1


def test_network_gradients_match_oracle(cuda):
    F, B = 640, 16
    net = WarmStartMLP(F, n_in=4, hidden=64, depth=3, modes=32, seed=5, device=cuda)
    rng = np.random.default_rng(6)
    net.set_mean(rng.normal(0, 0.3, F).astype(np.float32))
    for k in ("b0", "b1", "b2", "bout"):
        net.params[k].copy_(torch.from_numpy(rng.normal(0, 0.1, net.params[k].shape[0]).astype(np.float32)))
    x = rng.uniform(-1, 1, (B, 4)).astype(np.float32)
    t = rng.normal(0, 1, (B, F)).astype(np.float32)
    t[:, :50] = np.nan  # cells without samples
    tb = dev_bf16(t, cuda)
    acc, cnt, g, y = net.loss_and_grads(x, tb)
    torch.cuda.synchronize()
    host = {k: v.cpu().numpy().astype(np.float64) for k, v in net.params.items()}
    params = {"W": [host[f"W{l}"] for l in range(3)], "b": [host[f"b{l}"] for l in range(3)],
              "Wout": host["Wout"], "bout": host["bout"], "B": host["B"], "mean": host["mean"]}
    xpad = np.zeros((B, 16))
    xpad[:, :4] = x
    loss, go, yo = M.loss_and_grads(params, xpad, M.bf16(t), bf16_points=True)
    assert int(cnt.item()) == int(np.isfinite(t).sum())
    # FP32 against float64 accumulation; a value next to a BF16 rounding tie may
    # round the other way on one side, so the bounds allow a few such flips
    assert abs(acc.item() - loss) <= 1e-3 * loss
    assert np.max(np.abs(y.cpu().numpy() - yo)) <= 2e-3 * np.max(np.abs(yo))

    def rel(a, b):
        return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)

    for key in ("B", "mean", "Wout", "bout"):
        assert rel(g[key].cpu().numpy(), go[key]) < 5e-3, key
    for l in range(3):
        assert rel(g[f"W{l}"].cpu().numpy(), go["W"][l]) < 5e-3, l
        assert rel(g[f"b{l}"].cpu().numpy(), go["b"][l]) < 5e-3, l


def test_training_fits_a_smooth_family(cuda):
    """Fields that depend smoothly on two parameters: the trained network's
    error on held-out parameters is a small fraction of the spread."""
    F = 1024
    grid = np.linspace(0, 1, F // 2)
    rng = np.random.default_rng(7)

    def field(p):
        a, b = p
        return np.concatenate([np.tanh((grid - 0.3 - 0.4 * a) * 10), 0.5 + b * np.sin(6 * grid)])

    ptrain = rng.uniform(-1, 1, (512, 2))
    ptest = rng.uniform(-1, 1, (32, 2))
    ytrain = np.stack([field(p) for p in ptrain]).astype(np.float32)
    ytest = np.stack([field(p) for p in ptest]).astype(np.float32)
    net = WarmStartMLP(F, n_in=2, hidden=128, depth=3, modes=32, seed=1, device=cuda)
    net.set_mean(ytrain.mean(axis=0))
    tb = dev_bf16(ytrain, cuda)
    hist = net.train(ptrain.astype(np.float32), tb, epochs=150, batch=64, lr=2e-3, lr_final=1e-5)
    assert hist[-1] < 0.05 * hist[0]
    pred = net.predict(ptest.astype(np.float32)).cpu().numpy()
    err = np.linalg.norm(pred - ytest) / np.linalg.norm(ytest - ytrain.mean(axis=0))
    assert err < 0.2, err
