"""Learned queue order for the persistent sift kernel.

A small MLP (32 -> 128 -> 128 -> 2, GELU) maps 32 on-device trace features to
the predicted total sift passes and IMF count of each trace.  It is trained
on the GPU by this package's own kernels (FP32 forward / backward / Adam,
``emdb_mlp_*`` in the C ABI) on counts logged by the plain method
(``debug_n`` / ``n_imfs``), and served by a BF16-weight inference kernel.

The prediction only orders the work queue (longest predicted cost first) --
the decomposition of every trace is computed by the same kernel code on the
same data, so results are bit-identical to FIFO order, which stays the
fallback when no model is loaded.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native

N_FEAT = 32
N_OUT = 2


def _lib():
    L = _native.load()
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.emdb_features.argtypes = [P, P, I, I, P, P]
    L.emdb_mlp_num_params.argtypes = []
    L.emdb_mlp_forward.argtypes = [P, P, P, P, I, P, P, P, P, P, P]
    L.emdb_mlp_backward.argtypes = [P, P, P, P, P, P, P, P, P, P, I, P, P, P, P, P, P]
    L.emdb_mlp_adam.argtypes = [P, P, P, P, I, F, F, F, F, I, P, P]
    L.emdb_mlp_infer_bf16.argtypes = [P, P, P, P, I, P, P]
    for n in ("emdb_features", "emdb_mlp_num_params", "emdb_mlp_forward", "emdb_mlp_backward",
              "emdb_mlp_adam", "emdb_mlp_infer_bf16"):
        getattr(L, n).restype = I
    return L


def _stream(dev=None) -> int:
    import torch
    return torch.cuda.current_stream(dev).cuda_stream


def features(values, offsets=None, N: int | None = None):
    """[batch, 32] float32 features on the device.  CSR (values, offsets) or dense [batch, N]."""
    import torch
    L = _lib()
    if offsets is None:
        X = values
        B, N = X.shape
        out = torch.empty((B, N_FEAT), dtype=torch.float32, device=X.device)
        _native.check(L.emdb_features(X.data_ptr(), None, B, N, out.data_ptr(), _stream(X.device)),
                      "emdb_features")
        return out
    B = offsets.shape[0] - 1
    out = torch.empty((B, N_FEAT), dtype=torch.float32, device=values.device)
    _native.check(L.emdb_features(values.data_ptr(), offsets.data_ptr(), B, 0, out.data_ptr(),
                                  _stream(values.device)), "emdb_features")
    return out


def labels_from_debug(dbg_n, n_imfs):
    """Training targets: log2(1 + total sift passes) and IMF count."""
    import torch
    dn = dbg_n.to(torch.float32).clamp(min=0).sum(1)
    return torch.stack([torch.log2(1.0 + dn), n_imfs.to(torch.float32)], 1)


class CostModel:
    """MLP cost model with FP32 master weights on the device (+ a bf16 copy)."""

    def __init__(self, device=None, seed: int = 0):
        import torch
        self.L = _lib()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        n = self.L.emdb_mlp_num_params()
        self.n_params = n
        rng = np.random.default_rng(seed)
        parts = []
        for fi, fo in ((N_FEAT, 128), (128, 128), (128, N_OUT)):
            parts.append(rng.normal(0.0, np.sqrt(2.0 / fi), size=fi * fo))
            parts.append(np.zeros(fo))
        w = np.concatenate(parts).astype(np.float32)
        assert w.size == n
        self.params = torch.from_numpy(w).to(self.device)
        self.params_bf16 = self.params.to(torch.bfloat16)
        self.mu = torch.zeros(N_FEAT, dtype=torch.float32, device=self.device)
        self.sd = torch.ones(N_FEAT, dtype=torch.float32, device=self.device)
        self.t_mu = torch.zeros(N_OUT, dtype=torch.float32, device=self.device)
        self.t_sd = torch.ones(N_OUT, dtype=torch.float32, device=self.device)
        self.history: list[float] = []

    # -- raw kernels -----------------------------------------------------------
    def forward_train(self, X):
        import torch
        B = X.shape[0]
        f = lambda *s: torch.empty(s, dtype=torch.float32, device=self.device)
        Z1, H1, Z2, H2, Y = f(B, 128), f(B, 128), f(B, 128), f(B, 128), f(B, N_OUT)
        _native.check(self.L.emdb_mlp_forward(self.params.data_ptr(), X.data_ptr(), self.mu.data_ptr(),
                                              self.sd.data_ptr(), B, Z1.data_ptr(), H1.data_ptr(),
                                              Z2.data_ptr(), H2.data_ptr(), Y.data_ptr(),
                                              _stream(self.device)), "emdb_mlp_forward")
        return Y, (Z1, H1, Z2, H2)

    def backward(self, X, acts, Y, T):
        import torch
        B = X.shape[0]
        Z1, H1, Z2, H2 = acts
        f = lambda *s: torch.empty(s, dtype=torch.float32, device=self.device)
        dY, dZ2, dZ1 = f(B, N_OUT), f(B, 128), f(B, 128)
        grads = f(self.n_params)
        loss = f(1)
        _native.check(self.L.emdb_mlp_backward(
            self.params.data_ptr(), X.data_ptr(), self.mu.data_ptr(), self.sd.data_ptr(),
            Z1.data_ptr(), H1.data_ptr(), Z2.data_ptr(), H2.data_ptr(), Y.data_ptr(), T.data_ptr(),
            B, dY.data_ptr(), dZ2.data_ptr(), dZ1.data_ptr(), grads.data_ptr(), loss.data_ptr(),
            _stream(self.device)), "emdb_mlp_backward")
        return grads, loss

    def predict(self, X):
        """Standardised-target predictions with the bf16 inference kernel, decoded."""
        import torch
        B = X.shape[0]
        Y = torch.empty((B, N_OUT), dtype=torch.float32, device=self.device)
        _native.check(self.L.emdb_mlp_infer_bf16(self.params_bf16.data_ptr(), X.data_ptr(),
                                                 self.mu.data_ptr(), self.sd.data_ptr(), B,
                                                 Y.data_ptr(), _stream(self.device)),
                      "emdb_mlp_infer_bf16")
        return Y * self.t_sd + self.t_mu

    # -- training ----------------------------------------------------------------
    def fit(self, X, T, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
        """Adam on mean squared error of standardised targets, all on the GPU."""
        import torch
        X = X.to(self.device, torch.float32).contiguous()
        T = T.to(self.device, torch.float32)
        self.mu = X.mean(0)
        self.sd = X.std(0).clamp(min=1e-6)
        self.t_mu = T.mean(0)
        self.t_sd = T.std(0).clamp(min=1e-6)
        Ts = ((T - self.t_mu) / self.t_sd).contiguous()
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        self.params_bf16 = torch.empty(self.n_params, dtype=torch.bfloat16, device=self.device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        n = X.shape[0]
        step = 0
        self.history = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.device)
            tot = torch.zeros((), dtype=torch.float32, device=self.device)
            nb = 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb = X[idx].contiguous()
                tb = Ts[idx].contiguous()
                Y, acts = self.forward_train(xb)
                grads, loss = self.backward(xb, acts, Y, tb)
                step += 1
                _native.check(self.L.emdb_mlp_adam(
                    self.params.data_ptr(), grads.data_ptr(), m.data_ptr(), v.data_ptr(),
                    self.n_params, lr, 0.9, 0.999, 1e-8, step, self.params_bf16.data_ptr(),
                    _stream(self.device)), "emdb_mlp_adam")
                tot += loss[0]
                nb += 1
            self.history.append(float(tot.item()) / max(nb, 1))
        self.warmup()
        return self.history

    def warmup(self) -> None:
        """One cost prediction on a dummy row, so the first real one does not
        pay the one-time launch set-up of the kernels it uses (~0.4 s measured
        on B200, against ~0.3 ms for 65,536 traces once warm)."""
        import torch
        n = 4096    # large enough for the vectorised paths of every kernel used
        predicted_cost(self, torch.zeros((n, N_FEAT), dtype=torch.float32, device=self.device),
                       torch.ones(n, dtype=torch.int64, device=self.device))
        torch.cuda.synchronize(self.device)

    # -- persistence ---------------------------------------------------------------
    def state(self) -> dict:
        return {k: getattr(self, k).detach().float().cpu().numpy()
                for k in ("params", "mu", "sd", "t_mu", "t_sd")}

    def save(self, path: str) -> None:
        np.savez(path, **self.state())

    @classmethod
    def load(cls, path: str, device=None) -> "CostModel":
        import torch
        z = np.load(path)
        cm = cls(device)
        for k in ("params", "mu", "sd", "t_mu", "t_sd"):
            setattr(cm, k, torch.from_numpy(z[k]).to(cm.device))
        cm.params_bf16 = cm.params.to(torch.bfloat16)
        cm.warmup()
        return cm


def passes_from_prediction(y):
    """Predicted total sift passes per trace from the model's output."""
    import torch
    # 2^y as exp(y ln 2): torch's precompiled exp, where exp2 is compiled at run
    # time on first use of each vector width (~0.4 s inside a timed step)
    return torch.exp(y[:, 0] * 0.6931471805599453).clamp(min=1.0) - 1.0


def cost_from_prediction(y, lengths):
    """Work estimate per trace: N x predicted sift passes (only orders the
    queue and picks the tier)."""
    import torch
    return lengths.to(torch.float32) * passes_from_prediction(y).clamp(min=1.0)


def predicted_cost(model: CostModel, feats, lengths):
    """Work estimate per trace: N x predicted sift passes."""
    return cost_from_prediction(model.predict(feats), lengths)


def lpt_order(cost):
    """Longest-predicted-first permutation (int32) for the work queue."""
    import torch
    return torch.argsort(cost, descending=True, stable=True).to(torch.int32)


def learned_order(model: CostModel, signals):
    """Queue order for a dense device batch [batch, N]: features, the BF16
    cost model and longest-predicted-first, all on the device.  Pass it as
    GPUBatchEMD(...)(signals, order=...)."""
    import torch
    X = signals if signals.dtype == torch.float64 else signals.to(torch.float64)
    B, N = X.shape
    lengths = torch.full((B,), N, dtype=torch.int64, device=X.device)
    return lpt_order(predicted_cost(model, features(X), lengths))
