"""The learned slope limiter's network on the GPU (tensor-core kernels in csrc/hydro/mlp.cuh), bound through the C ABI.

A 3-layer MLP of width 64 maps 32 per-cell features to one logit per primitive variable; the slope factor is
alpha_adm * sigmoid(logit), alpha_adm the largest factor that keeps every face value of the cell inside its neighbours'
range (the plain limiter's admissible range), so monotonicity is kept by construction. Torch tensors are the device
buffers; all arithmetic is the library's kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import hydro

def lib():
    return hydro.lib()


IN, HID, OUT, USED = 32, 64, 16, 5


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class LimiterMLP:
    """FP32 master weights on the GPU, Adam state, and the kernels' forward and training step."""

    def __init__(self, params=None, seed: int = 0, device="cuda"):
        n = int(lib().luna_mlp_param_count())
        self.n_params = n
        if params is None:
            params = init_params(seed)
        self.params = torch.as_tensor(np.asarray(params, dtype=np.float32), device=device).contiguous()
        assert self.params.numel() == n
        self.grad = torch.zeros(n, dtype=torch.float32, device=device)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step_count = 0
        self._workspace = None

    def forward(self, features_bf16: torch.Tensor) -> torch.Tensor:
        n = features_bf16.shape[0]
        out = torch.empty((n, OUT), dtype=torch.float32, device=features_bf16.device)
        hydro.check(lib().luna_mlp_forward(_ptr(self.params), _ptr(features_bf16), n, _ptr(out), _stream()))
        return out

    def gradient(self, features_bf16, target, weight, scale=None) -> float:
        """The gradient of sum w (sigmoid(o) - t)^2 * scale into self.grad (scale default 1 / sum w); returns the loss."""
        n = features_bf16.shape[0]
        if scale is None:
            scale = 1.0 / max(float(weight.sum().item()), 1e-30)
        need = int(lib().luna_mlp_train_workspace_floats(n))
        if self._workspace is None or self._workspace.numel() < need:
            self._workspace = torch.empty(need, dtype=torch.float32, device=features_bf16.device)
        hydro.check(lib().luna_mlp_train_step(_ptr(self.params), _ptr(features_bf16), _ptr(target), _ptr(weight), n, scale,
                                              _ptr(self.grad), _ptr(self.loss), _ptr(self._workspace), need, _stream()))
        return self.loss

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        hydro.check(lib().luna_mlp_adam(_ptr(self.params), _ptr(self.grad), _ptr(self.m), _ptr(self.v), lr, beta1, beta2,
                                        eps, self.step_count, _stream()))

    def state(self) -> np.ndarray:
        return self.params.detach().cpu().numpy().copy()


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases (the output bias starts at logit 2: sigmoid ~ 0.88 of the admissible slope)."""
    rng = np.random.default_rng(seed)
    p = []
    p.append(rng.standard_normal((HID, IN)) * np.sqrt(2.0 / IN))
    p.append(np.zeros(HID))
    p.append(rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID))
    p.append(np.zeros(HID))
    p.append(rng.standard_normal((OUT, HID)) * np.sqrt(1.0 / HID) * 0.1)
    p.append(np.full(OUT, 2.0))
    return np.concatenate([a.ravel() for a in p]).astype(np.float32)


def trained_params() -> np.ndarray:
    """The network trained on the GPU by ``python -m luna_cpp_b200.limiter_training`` (its defaults: 48 1D Riemann strips
    and 16 2D four-quadrant problems on 256^2, each at gamma 1.4 and 5/3, labelled from the method's own 4x runs; 20
    epochs), shipped with its evaluation (data/limiter_mlp_eval.json) so the learned limiter runs without retraining."""
    import os

    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "limiter_mlp_params.npy"))
