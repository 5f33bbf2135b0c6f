"""The closure MLP on the GPU: parameters, Adam state and the training loop
around the CUDA kernels of csrc/closure.cu (through the C ABI).  Device
buffers are torch tensors (plumbing only: every operation on them here is
one of the library's kernels)."""
from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, load

KIN, HID, NOUT = 48, 64, 2


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights for the GELU layers, Glorot for the output layer,
    zero biases; the padded input rows and output columns zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(_lib.MLP_NPARAM, dtype=np.float32)
    w1 = rng.uniform(-1, 1, (KIN, HID)) * math.sqrt(6.0 / 45)
    w1[45:] = 0.0
    w2 = rng.uniform(-1, 1, (HID, HID)) * math.sqrt(6.0 / HID)
    w3 = np.zeros((HID, 8))
    w3[:, :NOUT] = rng.uniform(-1, 1, (HID, NOUT)) * math.sqrt(6.0 / (HID + NOUT))
    o_b1 = KIN * HID
    o_w2 = o_b1 + HID
    o_b2 = o_w2 + HID * HID
    o_w3 = o_b2 + HID
    p[:o_b1] = w1.ravel()
    p[o_w2:o_b2] = w2.ravel()
    p[o_w3:o_w3 + HID * 8] = w3.ravel()
    return p


class MLP:
    """Parameters (FP32 master + BF16 copy) and Adam moments on one GPU."""

    def __init__(self, params: Optional[np.ndarray] = None, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        self.params = torch.from_numpy(p.copy()).to(self.dev)
        self.wbf16 = torch.empty(_lib.MLP_NBF16, dtype=torch.bfloat16, device=self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros(_lib.MLP_NPARAM + 1, dtype=torch.float32, device=self.dev)
        self.step = 0
        self._partial = None
        self._idx = None
        check(load().inmsom_mlp_pack(_p(self.params), _p(self.wbf16), None))

    def forward(self, x):
        """x: device BF16 [n, 48] -> device FP32 [n, 2]."""
        y = self.torch.empty((x.shape[0], NOUT), dtype=self.torch.float32, device=self.dev)
        check(load().inmsom_mlp_forward(_p(x), x.shape[0], _p(self.params), _p(self.wbf16), _p(y), None))
        return y

    def loss_grad(self, x, t, idx=None, batch=None):
        """Mean squared error and gradient on the rows idx (device int32) of
        x (BF16 [n, 48]) and t (FP32 [n, 2]); returns the device gradient
        (NPARAM values, then the loss)."""
        b = int(batch if batch is not None else (idx.shape[0] if idx is not None else x.shape[0]))
        tiles = b // 128
        if self._partial is None or self._partial.numel() < tiles * _lib.MLP_PARTIAL:
            self._partial = self.torch.empty(tiles * _lib.MLP_PARTIAL, dtype=self.torch.float32, device=self.dev)
        check(load().inmsom_mlp_grad(_p(x), _p(t), None if idx is None else _p(idx), b, _p(self.params),
                                     _p(self.wbf16), _p(self._partial), _p(self.grad), None))
        return self.grad

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        check(load().inmsom_mlp_adam(_p(self.params), _p(self.wbf16), _p(self.m), _p(self.v), _p(self.grad),
                                     self.step, lr, b1, b2, eps, None))

    def train(self, x, t, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 1,
              log_every: int = 0):
        """Adam on random batches of (x, t); returns the losses logged every
        log_every steps (device reads only then)."""
        torch = self.torch
        n = x.shape[0]
        if self._idx is None or self._idx.numel() < batch:
            self._idx = torch.empty(batch, dtype=torch.int32, device=self.dev)
        lib = load()
        losses = []
        for k in range(steps):
            check(lib.inmsom_mlp_batch_indices(_p(self._idx), batch, n, seed, self.step + 1, None))
            self.loss_grad(x, t, self._idx, batch)
            self.adam(lr)
            if log_every and (k % log_every == 0 or k == steps - 1):
                losses.append((self.step, float(self.grad[-1].item())))
        return losses

    def host_params(self) -> np.ndarray:
        return self.params.cpu().numpy().copy()
