"""Float64 CPU reference of the surrogate network (plain torch autograd), the
checker of the hand-written kernels in dosecuda_b200/csrc/dc_net.cu.

Weight layouts follow the C ABI: conv weights [taps][cin][cout] with tap =
(dz*k + dy)*k + dx, transposed-conv weights [8][cout][cin]."""
from __future__ import annotations

import torch
import torch.nn.functional as F

from dosecuda_b200.surrogate import ARCH


def bf16(t: torch.Tensor) -> torch.Tensor:
    """Round to bf16 and return as float64."""
    return t.to(torch.bfloat16).to(torch.float64)


def conv3_weight(w: torch.Tensor) -> torch.Tensor:
    """[27][cin][cout] -> torch conv3d weight (cout, cin, 3, 3, 3)."""
    _, cin, cout = w.shape
    return w.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2).contiguous()


def down_weight(w: torch.Tensor) -> torch.Tensor:
    """[8][cin][cout] -> torch conv3d weight (cout, cin, 2, 2, 2)."""
    _, cin, cout = w.shape
    return w.reshape(2, 2, 2, cin, cout).permute(4, 3, 0, 1, 2).contiguous()


def up_weight(w: torch.Tensor) -> torch.Tensor:
    """[8][cout][cin] -> torch conv_transpose3d weight (cin, cout, 2, 2, 2)."""
    _, cout, cin = w.shape
    return w.reshape(2, 2, 2, cout, cin).permute(4, 3, 0, 1, 2).contiguous()


class _RoundValue(torch.autograd.Function):
    """Forward: round to bf16 (an activation the kernels store in bf16);
    backward: pass the gradient through."""

    @staticmethod
    def forward(ctx, x):
        return bf16(x)

    @staticmethod
    def backward(ctx, g):
        return g


class _RoundGrad(torch.autograd.Function):
    """Forward: identity; backward: round the gradient to bf16 (a gradient
    the kernels store in bf16)."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        return bf16(g)


def stored(x, on: bool):
    """A tensor the kernels keep in bf16, with its gradient also in bf16."""
    return _RoundGrad.apply(_RoundValue.apply(x)) if on else x


def ncdhw(x):
    return x.permute(0, 4, 1, 2, 3)


def ndhwc(x):
    return x.permute(0, 2, 3, 4, 1)


def norm_act(y, gamma, beta, eps, slope):
    """Instance norm (biased variance) + affine + LeakyReLU, NCDHW."""
    mean = y.mean(dim=(2, 3, 4), keepdim=True)
    var = ((y - mean) ** 2).mean(dim=(2, 3, 4), keepdim=True)
    z = (y - mean) / torch.sqrt(var + eps) * gamma.view(1, -1, 1, 1, 1) + beta.view(1, -1, 1, 1, 1)
    return F.leaky_relu(z, slope)


def forward(params: dict, x8: torch.Tensor, slope: float, eps: float, inter: dict | None = None,
            bf16_points: bool = False) -> torch.Tensor:
    """g0 features (NCDHW, float64) of the encoder-decoder; params are float64
    tensors (weights already rounded to bf16 by the caller).  ``inter``
    (optional) receives the intermediate activations, with retain_grad.
    With ``bf16_points`` every tensor the kernels store in bf16 (convolution
    outputs, norm outputs, skip sums, and the gradients of each) is rounded
    the same way, so the result follows the kernels' arithmetic up to fp32
    versus fp64 accumulation."""
    def block(name, kind, x):
        w = params[name + ".w"]
        y = F.conv3d(x, conv3_weight(w), padding=1) if kind == "conv3" else F.conv3d(x, down_weight(w), stride=2)
        y = stored(y, bf16_points)
        return stored(norm_act(y, params[name + ".gamma"], params[name + ".beta"], eps, slope), bf16_points)

    def up(name, x, skip):
        return stored(F.conv_transpose3d(x, up_weight(params[name + ".w"]), stride=2) + skip, bf16_points)

    x = ncdhw(x8)
    e0 = block("enc0", "conv3", x)
    d0 = block("down0", "down", e0)
    e1 = block("enc1", "conv3", d0)
    d1 = block("down1", "down", e1)
    e2 = block("enc2", "conv3", d1)
    d2 = block("down2", "down", e2)
    b = block("bott", "conv3", d2)
    g2 = block("dec2", "conv3", up("up2", b, e2))
    g1 = block("dec1", "conv3", up("up1", g2, e1))
    u0 = up("up0", g1, e0)
    g0 = block("dec0", "conv3", u0)
    if inter is not None:
        for k, v in dict(e0=e0, d0=d0, e1=e1, d1=d1, e2=e2, d2=d2, b=b, g2=g2, g1=g1, u0=u0, g0=g0).items():
            if v.requires_grad:
                v.retain_grad()
            inter[k] = v
    return g0


def loss(params, x8, target, inv_count, slope, eps, inter=None, bf16_points=False):
    """The network's squared-error loss (target < 0: masked voxel)."""
    g0 = ndhwc(forward(params, x8, slope, eps, inter, bf16_points)).reshape(-1, 16)
    pred = g0 @ params["head.w"] + params["head.b"]
    active = target >= 0
    diff = torch.where(active, pred - target, torch.zeros_like(pred))
    return (diff * diff).sum() * inv_count


__all__ = ["ARCH", "bf16", "stored", "conv3_weight", "down_weight", "up_weight", "ncdhw", "ndhwc", "norm_act", "forward",
           "loss"]
