"""TEST INFRASTRUCTURE — float32 CPU oracle of the denoiser network.

A restatement of the U-Net of ``pyradmc_b200/denoiser.py`` in plain torch fp32 on
the CPU (``torch.nn.functional.conv3d`` and autograd), built from the same flat
parameter array.  The denoiser has no counterpart in pyRadMC, so this oracle is
the reference for its numerics: the CUDA kernels (bf16 operands, fp32
accumulation) are checked against it within bf16 tolerances.  Only the tests
use it.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import torch
import torch.nn.functional as F

from pyradmc_b200.denoiser import IN_CHANNELS, LEVELS, layout


def conv_weight(flat: np.ndarray, layer) -> torch.Tensor:
    """[cout][kpad] columns k = tap * cin + ci, tap = kz*9 + ky*3 + kx  ->  torch
    [cout, cin, 3, 3, 3]."""
    w = np.asarray(flat[layer.w_off:layer.w_off + layer.cout * layer.kpad], dtype=np.float32)
    w = w.reshape(layer.cout, layer.kpad)[:, :27 * layer.cin]
    w = w.reshape(layer.cout, 3, 3, 3, layer.cin).transpose(0, 4, 1, 2, 3)
    return torch.from_numpy(np.ascontiguousarray(w))


def weight_to_flat(grad_w: torch.Tensor, layer) -> np.ndarray:
    """Inverse of :func:`conv_weight` for a gradient, padded columns zero."""
    g = grad_w.detach().numpy().transpose(0, 2, 3, 4, 1).reshape(layer.cout, 27 * layer.cin)
    out = np.zeros((layer.cout, layer.kpad), dtype=np.float32)
    out[:, :27 * layer.cin] = g
    return out.ravel()


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bf16 (round to nearest even), back as float32."""
    return torch.from_numpy(np.asarray(x, dtype=np.float32)).to(torch.bfloat16).float().numpy()


class OracleUNet:
    def __init__(self, flat: np.ndarray):
        self.layers, self.head_w, self.head_b, n = layout()
        assert flat.shape == (n,)
        self.flat = np.asarray(flat, dtype=np.float32)
        self.w = {l.name: conv_weight(self.flat, l).requires_grad_(True) for l in self.layers}
        self.b = {l.name: torch.from_numpy(self.flat[l.b_off:l.b_off + l.cout].copy()).requires_grad_(True)
                  for l in self.layers}
        c0 = LEVELS[0]
        self.hw = torch.from_numpy(self.flat[self.head_w:self.head_w + c0].copy()).requires_grad_(True)
        self.hb = torch.from_numpy(self.flat[self.head_b:self.head_b + 1].copy()).requires_grad_(True)

    def _conv(self, x, name):
        return F.relu(F.conv3d(x, self.w[name], self.b[name], padding=1))

    def forward(self, dose: torch.Tensor, density: torch.Tensor, sigma=None) -> torch.Tensor:
        """dose, density, sigma (optional) [B, D, H, W] -> prediction [B, D, H, W]."""
        b = dose.shape[0]
        x = torch.zeros((b, IN_CHANNELS) + tuple(dose.shape[1:]), dtype=torch.float32)
        x[:, 0] = dose
        x[:, 1] = density
        if sigma is not None:
            x[:, 2] = sigma
        e0 = self._conv(self._conv(x, "enc0a"), "enc0b")
        e1 = self._conv(self._conv(F.avg_pool3d(e0, 2), "enc1a"), "enc1b")
        e2 = self._conv(self._conv(F.avg_pool3d(e1, 2), "enc2a"), "enc2b")
        m = self._conv(self._conv(F.avg_pool3d(e2, 2), "mid_a"), "mid_b")
        up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")  # noqa: E731
        d2 = self._conv(self._conv(torch.cat([up(m), e2], 1), "dec2a"), "dec2b")
        d1 = self._conv(self._conv(torch.cat([up(d2), e1], 1), "dec1a"), "dec1b")
        d0 = self._conv(self._conv(torch.cat([up(d1), e0], 1), "dec0a"), "dec0b")
        head = torch.einsum("bcdhw,c->bdhw", d0, self.hw) + self.hb[0]
        return dose + head

    @staticmethod
    def loss(pred, target, weight, lam: float) -> torch.Tensor:
        w = 1.0 + lam * (weight if weight is not None else torch.zeros_like(target))
        return (torch.abs(pred - target) * w).mean()

    def gradients(self, dose, density, target, weight, lam: float, sigma=None):
        """(loss, flat fp32 gradient in the kernels' parameter layout)."""
        pred = self.forward(dose, density, sigma)
        loss = self.loss(pred, target, weight, lam)
        loss.backward()
        g = np.zeros_like(self.flat)
        for l in self.layers:
            g[l.w_off:l.w_off + l.cout * l.kpad] = weight_to_flat(self.w[l.name].grad, l)
            g[l.b_off:l.b_off + l.cout] = self.b[l.name].grad.numpy()
        c0 = LEVELS[0]
        g[self.head_w:self.head_w + c0] = self.hw.grad.numpy()
        g[self.head_b] = self.hb.grad.numpy()[0]
        return float(loss.detach()), g


def conv3d_reference(x_ndhwc: np.ndarray, w_flat: np.ndarray, bias, cin: int, cout: int,
                     kpad: int, relu: bool) -> np.ndarray:
    """One convolution in the kernels' layouts: x [N, D, H, W, cin] float32,
    weights [cout][kpad] -> y [N, D, H, W, cout] float32."""
    layer = SimpleNamespace(cin=cin, cout=cout, kpad=kpad, w_off=0)
    w = conv_weight(np.asarray(w_flat, dtype=np.float32).ravel(), layer)
    x = torch.from_numpy(np.ascontiguousarray(np.asarray(x_ndhwc, dtype=np.float32).transpose(0, 4, 1, 2, 3)))
    b = None if bias is None else torch.from_numpy(np.asarray(bias, dtype=np.float32))
    y = F.conv3d(x, w, b, padding=1)
    if relu:
        y = F.relu(y)
    return y.numpy().transpose(0, 2, 3, 4, 1).copy()
