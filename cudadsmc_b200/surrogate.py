"""Warm-start surrogate: a small MLP that predicts the steady per-cell fields
(n, u, v, w, T) of a flow from its parameters, trained on fields that this
DSMC produces, and used to seed the particle population instead of the
free-stream fill (no counterpart in the reference).

Network: 4 inputs (zero-padded to 16) -> `depth` x `hidden` GELU layers ->
`modes` coefficients -> field = mean + coefficients x basis, the basis
(modes x cells*5) learned with the rest.  Every GEMM, activation, loss and
optimizer step runs in this library's kernels (BF16 operands, FP32
accumulation, FP32 master weights, Adam); torch only holds the device
buffers.
"""
import ctypes
import math

import numpy as np

from ._capi import check, lib

_P = ctypes.c_void_p


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class WarmStartMLP:
    IN_PAD = 16

    def __init__(self, field_size, n_in=4, hidden=512, depth=4, modes=256, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.F, self.n_in, self.hidden, self.depth, self.modes = field_size, n_in, hidden, depth, modes
        g = np.random.default_rng(seed)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.params = {}
        dims = [self.IN_PAD] + [hidden] * depth
        for l in range(depth):
            w = np.zeros((dims[l], hidden), np.float32)
            fan_in = n_in if l == 0 else dims[l]
            w[: (n_in if l == 0 else dims[l])] = g.normal(0, math.sqrt(2.0 / fan_in),
                                                           ((n_in if l == 0 else dims[l]), hidden))
            self.params[f"W{l}"] = torch.from_numpy(w).to(**f32)
            self.params[f"b{l}"] = torch.zeros(hidden, **f32)
        self.params["Wout"] = torch.from_numpy(
            g.normal(0, math.sqrt(1.0 / hidden), (hidden, modes)).astype(np.float32)).to(**f32)
        self.params["bout"] = torch.zeros(modes, **f32)
        self.params["B"] = torch.from_numpy(
            g.normal(0, 0.02, (modes, field_size)).astype(np.float32)).to(**f32)
        self.params["mean"] = torch.zeros(field_size, **f32)
        self.bf = {k: torch.empty(v.shape, dtype=torch.bfloat16, device=self.dev)
                   for k, v in self.params.items() if k.startswith("W") or k == "B"}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.t = 0
        self._refresh_bf16()

    # ------------------------------------------------------------ helpers --
    def _refresh_bf16(self):
        for k, b in self.bf.items():
            check(lib().dsmc_to_bf16(_p(self.params[k]), _p(b), b.numel(), _stream()), "to_bf16")

    def _gemm(self, m, n, k, a, lda, at, b, ldb, bt, c=None, ldc=0, beta=0.0, bias=None, act=0,
              cb=None, ldcb=0, split=1):
        check(lib().dsmc_gemm_bf16(m, n, k, _p(a), lda, at, _p(b), ldb, bt, _p(c), ldc, beta, _p(bias),
                                   act, _p(cb), ldcb, split, _stream()), "gemm_bf16")

    def set_mean(self, mean):
        """Sets the field mean (the decoder bias), e.g. the training-set mean."""
        self.params["mean"].copy_(self.torch.as_tensor(mean, dtype=self.torch.float32))

    def _inputs(self, x):
        torch = self.torch
        xb = np.zeros((len(x), self.IN_PAD), np.float32)
        xb[:, : self.n_in] = x
        xf = torch.from_numpy(xb).to(self.dev)
        out = torch.empty(xf.shape, dtype=torch.bfloat16, device=self.dev)
        check(lib().dsmc_to_bf16(_p(xf), _p(out), xf.numel(), _stream()), "to_bf16")
        return out

    # ------------------------------------------------------------ forward --
    def forward(self, x):
        """x: [batch, n_in] normalized inputs.  Returns the field [batch, F]
        (FP32, on the device) and the cache for backward."""
        torch = self.torch
        B = len(x)
        h = self._inputs(x)
        cache = {"x": [], "z": []}
        for l in range(self.depth):
            W = self.bf[f"W{l}"]
            z = torch.empty((B, self.hidden), dtype=torch.float32, device=self.dev)
            hn = torch.empty((B, self.hidden), dtype=torch.bfloat16, device=self.dev)
            self._gemm(B, self.hidden, W.shape[0], h, h.shape[1], 0, W, self.hidden, 0, z, self.hidden,
                       bias=self.params[f"b{l}"], act=1, cb=hn, ldcb=self.hidden)
            cache["x"].append(h)
            cache["z"].append(z)
            h = hn
        cache["h"] = h
        c = torch.empty((B, self.modes), dtype=torch.float32, device=self.dev)
        cb = torch.empty((B, self.modes), dtype=torch.bfloat16, device=self.dev)
        self._gemm(B, self.modes, self.hidden, h, self.hidden, 0, self.bf["Wout"], self.modes, 0, c,
                   self.modes, bias=self.params["bout"], cb=cb, ldcb=self.modes)
        cache["c"] = cb
        y = torch.empty((B, self.F), dtype=torch.float32, device=self.dev)
        self._gemm(B, self.F, self.modes, cb, self.modes, 0, self.bf["B"], self.F, 0, y, self.F,
                   bias=self.params["mean"])
        return y, cache

    # ----------------------------------------------------------- backward --
    def loss_and_grads(self, x, targets_bf16):
        """Masked MSE against BF16 targets [batch, F] (NaN = no target).
        Returns (loss, valid count, grads dict of FP32 tensors)."""
        torch = self.torch
        B = len(x)
        y, cache = self.forward(x)
        n = B * self.F
        dy = torch.empty_like(y)
        dyb = torch.empty(y.shape, dtype=torch.bfloat16, device=self.dev)
        acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=self.dev)
        check(lib().dsmc_mse_grad(_p(y), _p(targets_bf16), n, 1.0 / n, _p(dyb), _p(dy), _p(acc), _p(cnt),
                                  _stream()), "mse_grad")
        g = {}
        g["B"] = torch.empty((self.modes, self.F), dtype=torch.float32, device=self.dev)
        self._gemm(self.modes, self.F, B, cache["c"], self.modes, 1, dyb, self.F, 0, g["B"], self.F)
        g["mean"] = torch.empty(self.F, dtype=torch.float32, device=self.dev)
        check(lib().dsmc_colsum(_p(dy), B, self.F, self.F, _p(g["mean"]), _stream()), "colsum")
        dc = torch.zeros((B, self.modes), dtype=torch.float32, device=self.dev)
        split = max(1, min(64, self.F // 4096))
        self._gemm(B, self.modes, self.F, dyb, self.F, 0, self.bf["B"], self.F, 1, dc, self.modes,
                   split=split)
        dcb = torch.empty(dc.shape, dtype=torch.bfloat16, device=self.dev)
        check(lib().dsmc_to_bf16(_p(dc), _p(dcb), dc.numel(), _stream()), "to_bf16")
        g["Wout"] = torch.empty((self.hidden, self.modes), dtype=torch.float32, device=self.dev)
        self._gemm(self.hidden, self.modes, B, cache["h"], self.hidden, 1, dcb, self.modes, 0, g["Wout"],
                   self.modes)
        g["bout"] = torch.empty(self.modes, dtype=torch.float32, device=self.dev)
        check(lib().dsmc_colsum(_p(dc), B, self.modes, self.modes, _p(g["bout"]), _stream()), "colsum")
        dh = torch.empty((B, self.hidden), dtype=torch.float32, device=self.dev)
        self._gemm(B, self.hidden, self.modes, dcb, self.modes, 0, self.bf["Wout"], self.modes, 1, dh,
                   self.hidden)
        for l in range(self.depth - 1, -1, -1):
            z = cache["z"][l]
            dz = torch.empty_like(z)
            dzb = torch.empty(z.shape, dtype=torch.bfloat16, device=self.dev)
            check(lib().dsmc_gelu_backward(_p(z), _p(dh), _p(dz), _p(dzb), z.numel(), _stream()),
                  "gelu_backward")
            xin = cache["x"][l]
            din = xin.shape[1]
            g[f"W{l}"] = torch.empty((din, self.hidden), dtype=torch.float32, device=self.dev)
            self._gemm(din, self.hidden, B, xin, din, 1, dzb, self.hidden, 0, g[f"W{l}"], self.hidden)
            g[f"b{l}"] = torch.empty(self.hidden, dtype=torch.float32, device=self.dev)
            check(lib().dsmc_colsum(_p(dz), B, self.hidden, self.hidden, _p(g[f"b{l}"]), _stream()),
                  "colsum")
            if l > 0:
                dh = torch.empty((B, din), dtype=torch.float32, device=self.dev)
                self._gemm(B, din, self.hidden, dzb, self.hidden, 0, self.bf[f"W{l}"], self.hidden, 1, dh,
                           din)
        return acc, cnt, g, y

    def adam_step(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
        self.t += 1
        for k, w in self.params.items():
            check(lib().dsmc_adam_step(_p(w), _p(grads[k]), _p(self.m[k]), _p(self.v[k]),
                                       _p(self.bf.get(k)), w.numel(), lr, b1, b2, eps, self.t,
                                       weight_decay if k.startswith("W") else 0.0, _stream()),
                  "adam_step")

    def train(self, x, targets_bf16, epochs=200, batch=128, lr=1e-3, lr_final=1e-5, seed=0,
              log=None):
        """Mini-batch Adam over (x [N, n_in], targets_bf16 [N, F] on the
        device, rows in random order), cosine learning-rate decay; each epoch
        visits the contiguous batches in a new random order.  Returns the
        per-epoch mean loss."""
        N = len(x)
        nb = max(1, N // batch)
        rng = np.random.default_rng(seed)
        history = []
        steps = epochs * nb
        step = 0
        for ep in range(epochs):
            tot, cnt = 0.0, 0
            for i in rng.permutation(nb):
                lo, hi = i * batch, min(N, (i + 1) * batch)
                lr_now = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * step / steps))
                acc, c, g, _ = self.loss_and_grads(x[lo:hi], targets_bf16[lo:hi])
                self.adam_step(g, lr=lr_now)
                tot += float(acc.item())
                cnt += int(c.item())
                step += 1
            history.append(tot / max(cnt, 1))
            if log and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                log(f"epoch {ep}: mse {history[-1]:.3e}")
        return history

    def predict(self, x):
        y, _ = self.forward(np.asarray(x, np.float32))
        return y
