"""3D U-Net denoiser of Dij columns, trained and run on the project's own kernels.

No counterpart in pyRadMC (the reference has no learned component).  The network
maps a low-history dose column and its Monte Carlo sigma, both normalized by
the column's maximum, plus the density to an estimate of the high-history
column; plain Monte Carlo stays its fallback and
the judge of its error.

Architecture: four levels of 16-32-64-128 channels.  Each level is two 3x3x3
convolutions with ReLU; the encoder halves the grid with 2x2x2 average pooling,
the decoder doubles it by nearest upsampling and joins the encoder's output of
the same level by channel concatenation.  A 1x1x1 head maps the last 16 channels
to one, added to the (normalized) input dose, so the network learns a
correction and starts (zero head) as the identity.  Activations and weights are
bf16 with fp32 accumulation; the master weights, their gradients and Adam's
moments are fp32.

Every convolution, its data and weight gradient, pooling, joining, the head, the
loss and Adam run as the sm_100a kernels of ``csrc/denoise.cu`` behind
``include/pyradmc_b200_denoise.h``; torch only allocates the device buffers and
supplies the stream.  Spatial sizes must be multiples of 8 (three poolings).
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib

IN_CHANNELS = 8          # dose, density, MC sigma, five zero channels (16-byte voxel rows)
LEVELS = (16, 32, 64, 128)
ALIGN = 64               # parameter blocks start on 64-element boundaries


def kpad_for(cin: int) -> int:
    """Padded K of a 3x3x3 convolution over `cin` channels (27 * cin -> multiple of 64)."""
    return -(-27 * cin // 64) * 64


@dataclass(frozen=True)
class ConvLayer:
    name: str
    cin: int
    cout: int
    w_off: int           # offset of the [cout][kpad] weights in the flat parameters
    b_off: int           # offset of the [cout] bias

    @property
    def kpad(self) -> int:
        return kpad_for(self.cin)

    @property
    def kpad_d(self) -> int:
        """K of the data-gradient convolution (over cout channels)."""
        return kpad_for(self.cout)


def _round_up(x: int, a: int = ALIGN) -> int:
    return -(-x // a) * a


def layout() -> tuple[list[ConvLayer], int, int, int]:
    """The convolution layers with their parameter offsets, the head's weight
    and bias offsets, and the total parameter count."""
    c0, c1, c2, c3 = LEVELS
    specs = [
        ("enc0a", IN_CHANNELS, c0), ("enc0b", c0, c0),
        ("enc1a", c0, c1), ("enc1b", c1, c1),
        ("enc2a", c1, c2), ("enc2b", c2, c2),
        ("mid_a", c2, c3), ("mid_b", c3, c3),
        ("dec2a", c3 + c2, c2), ("dec2b", c2, c2),
        ("dec1a", c2 + c1, c1), ("dec1b", c1, c1),
        ("dec0a", c1 + c0, c0), ("dec0b", c0, c0),
    ]
    layers, off = [], 0
    for name, cin, cout in specs:
        w_off = off
        off = _round_up(off + cout * kpad_for(cin))
        b_off = off
        off = _round_up(off + cout)
        layers.append(ConvLayer(name, cin, cout, w_off, b_off))
    head_w = off
    off = _round_up(off + c0)
    head_b = off
    off = _round_up(off + 1)
    return layers, head_w, head_b, off


def forward_flops_per_voxel() -> float:
    """Useful multiply-add FLOPs of one forward pass per full-resolution voxel
    (the convolutions' 2 * 27 * cin * cout at their level's voxel fraction),
    the input layer counted on its 3 real channels (dose, sigma, density), not
    the 5 zero channels that pad its voxel rows to 16 bytes."""
    layers, *_ = layout()
    level = {"enc0": 0, "enc1": 1, "enc2": 2, "mid_": 3, "dec2": 2, "dec1": 1, "dec0": 0}
    return float(sum(2 * 27 * (3 if l.name == "enc0a" else l.cin) * l.cout / 8 ** level[l.name[:4]]
                     for l in layers))


def init_parameters(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights (zero in the K padding), zero biases and a
    zero head, as one flat float32 array."""
    layers, head_w, head_b, n = layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    for layer in layers:
        k = 27 * layer.cin
        w = np.zeros((layer.cout, layer.kpad), dtype=np.float32)
        w[:, :k] = rng.normal(0.0, np.sqrt(2.0 / k), size=(layer.cout, k))
        p[layer.w_off:layer.w_off + w.size] = w.ravel()
    return p


def _check(code: int, what: str) -> None:
    if code == -1:
        raise ValueError(f"{what}: shape not supported by the denoiser kernels")
    if code != 0:
        raise RuntimeError(f"{what}: kernel launch failed ({code})")


class _Workspace:
    """Device buffers of one input shape: activations kept for the backward pass
    and their gradients."""

    def __init__(self, torch, device, shape: tuple[int, int, int, int]):
        b, d, h, w = shape
        if d % 8 or h % 8 or w % 8:
            raise ValueError(f"spatial size {shape[1:]} must be a multiple of 8")
        self.shape = shape
        c0, c1, c2, c3 = LEVELS
        bf = torch.bfloat16
        self.dims = [(b, d >> i, h >> i, w >> i) for i in range(4)]
        vox = [b * (d >> i) * (h >> i) * (w >> i) for i in range(4)]
        self.m = vox[0]

        def act(level: int, c: int):
            return torch.empty((vox[level], c), dtype=bf, device=device)

        self.x0 = act(0, IN_CHANNELS)
        self.base = torch.empty(vox[0], dtype=torch.float32, device=device)
        self.out = torch.empty(vox[0], dtype=torch.float32, device=device)
        self.gout = torch.empty(vox[0], dtype=torch.float32, device=device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.a = {
            "e0a": act(0, c0), "e0": act(0, c0), "p0": act(1, c0),
            "e1a": act(1, c1), "e1": act(1, c1), "p1": act(2, c1),
            "e2a": act(2, c2), "e2": act(2, c2), "p2": act(3, c2),
            "ma": act(3, c3), "mb": act(3, c3),
            "u2": act(2, c3 + c2), "d2a": act(2, c2), "d2": act(2, c2),
            "u1": act(1, c2 + c1), "d1a": act(1, c1), "d1": act(1, c1),
            "u0": act(0, c1 + c0), "d0a": act(0, c0), "d0": act(0, c0),
        }
        self._torch = torch
        self.g: dict | None = None

    def grads(self):
        if self.g is None:
            self.g = {k: self._torch.empty_like(v) for k, v in self.a.items()}
        return self.g


class UNet3D:
    """The denoiser network on one CUDA device.

    ``train_step`` runs forward, loss, backward and an Adam step entirely on the
    device and returns the loss as a device scalar; ``predict`` runs the
    forward pass.  Inputs are float32 device tensors of shape [B, D, H, W].
    """

    def __init__(self, device: str = "cuda:0", seed: int = 0, lr: float = 1.0e-3,
                 loss_lambda: float = 1.0, params: np.ndarray | None = None):
        import torch

        self.torch = torch
        self.device = torch.device(device)
        if self.device.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("the denoiser runs on a CUDA device only (there is no CPU fallback)")
        self.lib = _lib.load()
        self.layers, self.head_w, self.head_b, self.n_params = layout()
        self._by_name = {layer.name: layer for layer in self.layers}
        self.lr = float(lr)
        self.loss_lambda = float(loss_lambda)
        self.beta1, self.beta2, self.eps = 0.9, 0.999, 1.0e-8
        host = init_parameters(seed) if params is None else np.asarray(params, dtype=np.float32)
        if host.shape != (self.n_params,):
            raise ValueError(f"expected {self.n_params} parameters, got {host.shape}")
        with torch.cuda.device(self.device):
            self.p32 = torch.from_numpy(host.copy()).to(self.device)
            self.p16 = self.p32.to(torch.bfloat16)
            self.grad = torch.zeros_like(self.p32)
            self.m1 = torch.zeros_like(self.p32)
            self.m2 = torch.zeros_like(self.p32)
            self.flipped = {
                layer.name: torch.zeros((layer.cin, layer.kpad_d), dtype=torch.bfloat16,
                                        device=self.device)
                for layer in self.layers[1:]
            }
        self.steps = 0
        self._ws: dict[tuple, _Workspace] = {}
        self.launches = 0
        self.fuse_head = True  # predict: the head in the last convolution's epilogue

    # ---- parameters -------------------------------------------------------------------
    def parameters(self) -> np.ndarray:
        return self.p32.cpu().numpy()

    def save(self, path: str | Path) -> None:
        np.savez_compressed(path, params=self.parameters(), levels=np.array(LEVELS),
                            steps=np.int64(self.steps))

    @classmethod
    def load(cls, path: str | Path, device: str = "cuda:0", **kw) -> "UNet3D":
        with np.load(path) as z:
            if tuple(int(c) for c in z["levels"]) != LEVELS:
                raise ValueError(f"{path}: network levels {tuple(z['levels'])} != {LEVELS}")
            net = cls(device=device, params=z["params"], **kw)
            net.steps = int(z["steps"])
        return net

    # ---- helpers --------------------------------------------------------------------
    def _stream(self) -> int:
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _ptr16(self, off: int) -> int:
        return self.p16.data_ptr() + 2 * off

    @staticmethod
    def _ptr32(t, off: int = 0) -> int:
        return t.data_ptr() + 4 * off

    def workspace(self, shape: tuple[int, int, int, int]) -> _Workspace:
        ws = self._ws.get(shape)
        if ws is None:
            ws = self._ws[shape] = _Workspace(self.torch, self.device, shape)
        return ws

    def release_workspaces(self) -> None:
        self._ws.clear()

    def _conv(self, x, layer: ConvLayer, y, dims, relu: int = 1) -> None:
        n, d, h, w = dims
        _check(self.lib.pmd_conv3d(x.data_ptr(), self._ptr16(layer.w_off),
                                   self._ptr32(self.p32, layer.b_off), y.data_ptr(), n, d, h, w,
                                   layer.cin, layer.cout, layer.kpad, relu, self._stream()),
               f"conv {layer.name}")
        self.launches += 1

    def _dgrad(self, g, layer: ConvLayer, gx, dims) -> None:
        n, d, h, w = dims
        _check(self.lib.pmd_conv3d(g.data_ptr(), self.flipped[layer.name].data_ptr(), None,
                                   gx.data_ptr(), n, d, h, w, layer.cout, layer.cin,
                                   layer.kpad_d, 0, self._stream()),
               f"dgrad {layer.name}")
        self.launches += 1

    def _wgrad(self, x, g, layer: ConvLayer, dims) -> None:
        n, d, h, w = dims
        _check(self.lib.pmd_conv3d_wgrad(x.data_ptr(), g.data_ptr(),
                                         self._ptr32(self.grad, layer.w_off),
                                         self._ptr32(self.grad, layer.b_off), n, d, h, w,
                                         layer.cin, layer.cout, layer.kpad, self._stream()),
               f"wgrad {layer.name}")
        self.launches += 1

    def _relu_mask(self, g, y) -> None:
        _check(self.lib.pmd_relu_mask(g.data_ptr(), y.data_ptr(), y.numel(), self._stream()),
               "relu mask")
        self.launches += 1

    def _pool(self, x, y, dims, c) -> None:
        _check(self.lib.pmd_avgpool(x.data_ptr(), y.data_ptr(), *dims, c, self._stream()), "pool")
        self.launches += 1

    def _pool_grad(self, gy, gx, dims, c) -> None:
        _check(self.lib.pmd_avgpool_grad(gy.data_ptr(), gx.data_ptr(), *dims, c, 1, self._stream()),
               "pool grad")
        self.launches += 1

    def _upcat(self, up, skip, out, dims, c_up, c_skip) -> None:
        _check(self.lib.pmd_upcat(up.data_ptr(), skip.data_ptr(), out.data_ptr(), *dims, c_up,
                                  c_skip, self._stream()), "upcat")
        self.launches += 1

    def _upcat_grad(self, gout, gup, gskip, dims, c_up, c_skip) -> None:
        _check(self.lib.pmd_upcat_grad(gout.data_ptr(), gup.data_ptr(), gskip.data_ptr(), *dims,
                                       c_up, c_skip, 0, self._stream()), "upcat grad")
        self.launches += 1

    # ---- passes ---------------------------------------------------------------------
    def pack(self, ws: _Workspace, dose, density, colmax=None, density_shared: bool = False,
             sigma=None) -> None:
        """Network input from float32 device tensors: dose [B, D, H, W] and its
        Monte Carlo sigma (optional; both scaled by 1 / colmax[b] when colmax is
        given) and density ([D, H, W] shared by the batch when density_shared,
        else [B, D, H, W])."""
        vox = ws.m // ws.shape[0]
        _check(self.lib.pmd_pack_input(dose.data_ptr(), density.data_ptr(),
                                       None if sigma is None else sigma.data_ptr(),
                                       None if colmax is None else colmax.data_ptr(), vox,
                                       int(density_shared), ws.x0.data_ptr(), ws.base.data_ptr(),
                                       ws.m, self._stream()), "pack input")
        self.launches += 1

    def _conv_head(self, x, layer: ConvLayer, ws: _Workspace, dims) -> bool:
        """The last convolution with the 1x1x1 head in its epilogue (ws.out
        directly, its features not stored); False where the kernel does not
        cover the shape and nothing ran."""
        n, d, h, w = dims
        code = self.lib.pmd_conv3d_head(x.data_ptr(), self._ptr16(layer.w_off),
                                        self._ptr32(self.p32, layer.b_off),
                                        self._ptr32(self.p32, self.head_w),
                                        self._ptr32(self.p32, self.head_b), ws.base.data_ptr(),
                                        ws.out.data_ptr(), n, d, h, w, layer.cin, layer.cout,
                                        layer.kpad, 1, self._stream())
        if code == -1:
            return False
        _check(code, f"conv {layer.name} + head")
        self.launches += 1
        return True

    def forward(self, ws: _Workspace, keep_features: bool = True) -> None:
        """keep_features False (inference): the last convolution's output is not
        needed by a backward pass, so the head is fused into it where the
        kernel allows; the prediction is the same either way."""
        a, L = ws.a, self._by_name
        c0, c1, c2, c3 = LEVELS
        d0, d1, d2, d3 = ws.dims
        self._conv(ws.x0, L["enc0a"], a["e0a"], d0)
        self._conv(a["e0a"], L["enc0b"], a["e0"], d0)
        self._pool(a["e0"], a["p0"], d0, c0)
        self._conv(a["p0"], L["enc1a"], a["e1a"], d1)
        self._conv(a["e1a"], L["enc1b"], a["e1"], d1)
        self._pool(a["e1"], a["p1"], d1, c1)
        self._conv(a["p1"], L["enc2a"], a["e2a"], d2)
        self._conv(a["e2a"], L["enc2b"], a["e2"], d2)
        self._pool(a["e2"], a["p2"], d2, c2)
        self._conv(a["p2"], L["mid_a"], a["ma"], d3)
        self._conv(a["ma"], L["mid_b"], a["mb"], d3)
        self._upcat(a["mb"], a["e2"], a["u2"], d2, c3, c2)
        self._conv(a["u2"], L["dec2a"], a["d2a"], d2)
        self._conv(a["d2a"], L["dec2b"], a["d2"], d2)
        self._upcat(a["d2"], a["e1"], a["u1"], d1, c2, c1)
        self._conv(a["u1"], L["dec1a"], a["d1a"], d1)
        self._conv(a["d1a"], L["dec1b"], a["d1"], d1)
        self._upcat(a["d1"], a["e0"], a["u0"], d0, c1, c0)
        self._conv(a["u0"], L["dec0a"], a["d0a"], d0)
        if not keep_features and self.fuse_head and self._conv_head(a["d0a"], L["dec0b"], ws, d0):
            return
        self._conv(a["d0a"], L["dec0b"], a["d0"], d0)
        _check(self.lib.pmd_head(a["d0"].data_ptr(), self._ptr32(self.p32, self.head_w),
                                 self._ptr32(self.p32, self.head_b), ws.base.data_ptr(),
                                 ws.out.data_ptr(), ws.m, c0, self._stream()), "head")
        self.launches += 1

    def backward(self, ws: _Workspace) -> None:
        """Parameter gradients (added into self.grad) from ws.gout = dloss/dout."""
        a, g, L = ws.a, ws.grads(), self._by_name
        c0, c1, c2, c3 = LEVELS
        d0, d1, d2, d3 = ws.dims
        st = self._stream()
        for layer in self.layers[1:]:
            _check(self.lib.pmd_flip_weights(self._ptr16(layer.w_off),
                                             self.flipped[layer.name].data_ptr(), layer.cin,
                                             layer.cout, layer.kpad, layer.kpad_d, st), "flip")
            self.launches += 1
        _check(self.lib.pmd_head_grad(a["d0"].data_ptr(), self._ptr32(self.p32, self.head_w),
                                      ws.gout.data_ptr(), g["d0"].data_ptr(),
                                      self._ptr32(self.grad, self.head_w),
                                      self._ptr32(self.grad, self.head_b), ws.m, c0, st),
               "head grad")
        self.launches += 1

        def pair(x_in, name_a, name_b, act_a, act_b, dims, g_in):
            # act_b = relu(conv_b(act_a)), act_a = relu(conv_a(x_in)): both
            # convolutions' gradients from g[act_b]; g[g_in] (unless None)
            # receives the gradient with respect to x_in.
            self._relu_mask(g[act_b], a[act_b])
            self._wgrad(a[act_a], g[act_b], L[name_b], dims)
            self._dgrad(g[act_b], L[name_b], g[act_a], dims)
            self._relu_mask(g[act_a], a[act_a])
            self._wgrad(x_in, g[act_a], L[name_a], dims)
            if g_in is not None:
                self._dgrad(g[act_a], L[name_a], g[g_in], dims)

        pair(a["u0"], "dec0a", "dec0b", "d0a", "d0", d0, "u0")
        self._upcat_grad(g["u0"], g["d1"], g["e0"], d0, c1, c0)
        pair(a["u1"], "dec1a", "dec1b", "d1a", "d1", d1, "u1")
        self._upcat_grad(g["u1"], g["d2"], g["e1"], d1, c2, c1)
        pair(a["u2"], "dec2a", "dec2b", "d2a", "d2", d2, "u2")
        self._upcat_grad(g["u2"], g["mb"], g["e2"], d2, c3, c2)
        pair(a["p2"], "mid_a", "mid_b", "ma", "mb", d3, "p2")
        self._pool_grad(g["p2"], g["e2"], d2, c2)
        pair(a["p1"], "enc2a", "enc2b", "e2a", "e2", d2, "p1")
        self._pool_grad(g["p1"], g["e1"], d1, c1)
        pair(a["p0"], "enc1a", "enc1b", "e1a", "e1", d1, "p0")
        self._pool_grad(g["p0"], g["e0"], d0, c0)
        pair(ws.x0, "enc0a", "enc0b", "e0a", "e0", d0, None)

    def loss(self, ws: _Workspace, target, weight=None) -> None:
        _check(self.lib.pmd_loss(ws.out.data_ptr(), target.data_ptr(),
                                 None if weight is None else weight.data_ptr(), self.loss_lambda,
                                 ws.gout.data_ptr(), ws.loss.data_ptr(), ws.m, self._stream()),
               "loss")
        self.launches += 1

    def adam(self) -> None:
        self.steps += 1
        _check(self.lib.pmd_adam(self.p32.data_ptr(), self.grad.data_ptr(), self.m1.data_ptr(),
                                 self.m2.data_ptr(), self.p16.data_ptr(), self.n_params, self.lr,
                                 self.beta1, self.beta2, self.eps, self.steps, self._stream()),
               "adam")
        self.launches += 1

    # ---- public ---------------------------------------------------------------------
    def gradients(self, dose, density, target, weight=None, sigma=None):
        """Loss and flat parameter gradient (device tensors) for one batch,
        without updating the parameters."""
        ws = self.workspace(tuple(dose.shape))
        self.grad.zero_()
        ws.loss.zero_()
        self.pack(ws, dose, density, sigma=sigma)
        self.forward(ws)
        self.loss(ws, target, weight)
        self.backward(ws)
        return ws.loss, self.grad

    def train_step(self, dose, density, target, weight=None, sigma=None):
        """One Adam step on a batch; returns the batch loss (device scalar,
        before the step)."""
        loss, _ = self.gradients(dose, density, target, weight, sigma)
        self.adam()
        return loss

    def predict(self, dose, density, colmax=None, density_shared: bool = False, sigma=None):
        """Denoised, normalized dose [B, D, H, W] (a view of the workspace,
        overwritten by the next call of the same shape)."""
        ws = self.workspace(tuple(dose.shape))
        self.pack(ws, dose, density, colmax, density_shared, sigma)
        self.forward(ws, keep_features=False)
        return ws.out.view(dose.shape)


def loss_weight(target, sigma, precision: float = 0.02):
    """Per-voxel weight of the sigma-weighted loss term: min(1, precision *
    target / sigma), i.e. 1 where the high-history target is known to better
    than `precision` and proportionally less where it is noisier."""
    import torch

    w = precision * target / sigma.clamp_min(1.0e-30)
    return torch.where(sigma > 0, w.clamp(max=1.0), (target > 0).to(target.dtype))
