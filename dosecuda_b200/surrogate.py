"""Learned photon-dose surrogate with collapsed-cone fallback.

A 4-level 3D convolutional encoder-decoder (16, 32, 64, 128 channels) maps
(TERMA, relative density) of one photon control point to its CCCS dose.
Every layer runs on hand-written sm_100a kernels of libdosecuda.so (C ABI
``dc_net_*``): bf16 implicit-GEMM convolutions on the tensor cores with fp32
accumulation (forward, backward-data, backward-weight), instance norm +
LeakyReLU forward/backward, the output head and the squared-error loss.
torch holds the tensors and runs Adam on the fp32 master weights.

Architecture (channels-last bf16 activations; ``u_k`` adds the encoder skip):

    x  = (TERMA*terma_scale, density, 0 x 6)                  8 @ D
    e0 = NA(conv3 8->16)      d0 = NA(down 16->32)            16 @ D, 32 @ D/2
    e1 = NA(conv3 32->32)     d1 = NA(down 32->64)            32 @ D/2, 64 @ D/4
    e2 = NA(conv3 64->64)     d2 = NA(down 64->128)           64 @ D/4, 128 @ D/8
    b  = NA(conv3 128->128)                                   128 @ D/8
    u2 = up(b) + e2,  g2 = NA(conv3 64->64)                   64 @ D/4
    u1 = up(g2) + e1, g1 = NA(conv3 32->32)                   32 @ D/2
    u0 = up(g1) + e0, g0 = NA(conv3 16->16)                   16 @ D
    dose = dose_unit * (w . g0 + b) where TERMA > 0.01, else 0

NA = instance norm (per sample and channel, affine) + LeakyReLU; conv3 =
3x3x3 stride 1 pad 1; down = 2x2x2 stride 2; up = transposed 2x2x2 stride 2.
The zero outside TERMA > 0.01 is the CCCS mask of the reference engine
(IMRTClasses.cu:270-273), so masked voxels are exact.

``PhotonSurrogate`` runs the accept/fallback path for one control point:
TERMA -> network -> CCCS on a sparse probe (rays from the source through the
field and lateral profiles) -> gamma(2 %/2 mm) of the network dose at the
probe points -> accept when the pass rate reaches the threshold, otherwise run
the full CCCS from the same TERMA.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from collections import OrderedDict

import numpy as np
import torch

from . import _lib

CONV3 = 0
DOWN2 = 1
IN_CHANNELS = 8
LEVELS = (16, 32, 64, 128)

# (name, kind, cin, cout); kinds: conv3, down, up
ARCH = (
    ("enc0", "conv3", 8, 16),
    ("down0", "down", 16, 32),
    ("enc1", "conv3", 32, 32),
    ("down1", "down", 32, 64),
    ("enc2", "conv3", 64, 64),
    ("down2", "down", 64, 128),
    ("bott", "conv3", 128, 128),
    ("up2", "up", 128, 64),
    ("dec2", "conv3", 64, 64),
    ("up1", "up", 64, 32),
    ("dec1", "conv3", 32, 32),
    ("up0", "up", 32, 16),
    ("dec0", "conv3", 16, 16),
)
_KIND = {name: (kind, cin, cout) for name, kind, cin, cout in ARCH}
_TAPS = {"conv3": 27, "down": 8, "up": 8}


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class NetOps:
    """Thin torch-tensor wrappers of the ``dc_net_*`` entry points (enqueued
    on the current torch stream of ``device``)."""

    def __init__(self, device="cuda"):
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.gpu = dev.index
        self.lib = _lib.load()

    def _s(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _act(self, shape):
        return torch.empty(shape, dtype=torch.bfloat16, device=self.device)

    def pack(self, master, flip=0, trans=0, out=None):
        T, A, B = master.shape
        k, n = (B, A) if trans else (A, B)
        frags = self.lib.dc_net_packed_fragments(T, k, n)
        if frags < 0:
            raise ValueError("invalid weight shape for packing")
        if out is None:
            out = torch.empty(frags, dtype=torch.int64, device=self.device)
        elif out.numel() != frags:
            raise ValueError("packed weight buffer has the wrong size")
        _lib.raise_for(self.lib.dc_net_pack_weights(self.gpu, _ptr(master), T, A, B, flip, trans, _ptr(out),
                                                    self._s()))
        return out

    def conv(self, mode, x, wpk, cout, stats=None, out=None):
        n, d, h, w, cin = x.shape
        od, oh, ow = (d, h, w) if mode == CONV3 else (d // 2, h // 2, w // 2)
        y = out if out is not None else self._act((n, od, oh, ow, cout))
        _lib.raise_for(self.lib.dc_net_conv(self.gpu, mode, _ptr(x), n, d, h, w, cin, _ptr(wpk), wpk.numel(), cout,
                                            _ptr(y), _ptr(stats), self._s()))
        return y

    def pack_tc(self, master, flip=0, trans=0, out=None):
        """Weights packed for the tensor-core (tcgen05) 3x3x3 convolution."""
        T, A, B = master.shape
        cin, cout = (B, A) if trans else (A, B)
        nbytes = self.lib.dc_net_packed_tc_bytes(cin, cout)
        if nbytes < 0:
            raise ValueError("no tensor-core convolution for %d -> %d channels" % (cin, cout))
        if out is None:
            out = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        _lib.raise_for(self.lib.dc_net_pack_weights_tc(self.gpu, _ptr(master), T, A, B, flip, trans, _ptr(out),
                                                       self._s()))
        return out

    @staticmethod
    def tc_supported(shape, cin, cout):
        d, h, w = shape
        return w == 128 and d % 2 == 0 and h % 2 == 0 and cout == 16 and cin in (8, 16)

    def conv_tc(self, x, wtc, cout, stats=None, out=None):
        n, d, h, w, cin = x.shape
        y = out if out is not None else self._act((n, d, h, w, cout))
        _lib.raise_for(self.lib.dc_net_conv_tc(self.gpu, _ptr(x), n, d, h, w, cin, _ptr(wtc), wtc.numel(), cout,
                                               _ptr(y), _ptr(stats), self._s()))
        return y

    def tc_error(self):
        flag = C.c_int()
        _lib.raise_for(self.lib.dc_net_tc_error(self.gpu, C.byref(flag)))
        return flag.value

    def tc_selftest(self):
        """Runs the tensor-core wait self-test (MMAs withheld); 1 when the
        bounded wait expired and was reported."""
        flag = C.c_int()
        _lib.raise_for(self.lib.dc_net_tc_selftest(self.gpu, C.byref(flag)))
        return flag.value

    def conv_up(self, x, wpk, cout, addend=None, out=None):
        n, d, h, w, cin = x.shape
        y = out if out is not None else self._act((n, 2 * d, 2 * h, 2 * w, cout))
        _lib.raise_for(self.lib.dc_net_conv_up(self.gpu, _ptr(x), n, d, h, w, cin, _ptr(wpk), wpk.numel(), cout,
                                               _ptr(addend), _ptr(y), self._s()))
        return y

    def wgrad(self, mode, p, q, ca, out=None):
        n, d, h, w, cb = q.shape
        taps = 27 if mode == CONV3 else 8
        g = out if out is not None else torch.empty((taps, ca, cb), dtype=torch.float32, device=self.device)
        _lib.raise_for(self.lib.dc_net_wgrad(self.gpu, mode, _ptr(p), _ptr(q), n, d, h, w, ca, cb, _ptr(g),
                                             self._s()))
        return g

    def norm_finalize(self, stats, count, gamma, beta, eps):
        n, c = stats.shape[:2]
        coef = torch.empty((n, c, 4), dtype=torch.float32, device=self.device)
        _lib.raise_for(self.lib.dc_net_norm_finalize(self.gpu, _ptr(stats), n, c, int(count), _ptr(gamma),
                                                     _ptr(beta), float(eps), _ptr(coef), self._s()))
        return coef

    def norm_act(self, y, coef, slope, out=None):
        n, c = y.shape[0], y.shape[-1]
        vox = y.numel() // (n * c)
        a = out if out is not None else torch.empty_like(y)
        _lib.raise_for(self.lib.dc_net_norm_act(self.gpu, _ptr(y), n, vox, c, _ptr(coef), float(slope), _ptr(a),
                                                self._s()))
        return a

    def norm_stats_act(self, y, stats, count, gamma, beta, eps, slope, out=None):
        """Instance norm from the convolution's statistics + LeakyReLU in one
        pass; returns (activation, coef)."""
        n, c = y.shape[0], y.shape[-1]
        vox = y.numel() // (n * c)
        a = out if out is not None else torch.empty_like(y)
        coef = torch.empty((n, c, 4), dtype=torch.float32, device=self.device)
        _lib.raise_for(self.lib.dc_net_norm_stats_act(self.gpu, _ptr(y), n, vox, c, _ptr(stats), int(count),
                                                      _ptr(gamma), _ptr(beta), float(eps), float(slope), _ptr(coef),
                                                      _ptr(a), self._s()))
        return a, coef

    def norm_act_bwd(self, y, da, coef, gamma, slope):
        n, c = y.shape[0], y.shape[-1]
        vox = y.numel() // (n * c)
        red = torch.empty((n, c, 2), dtype=torch.float64, device=self.device)
        dy = torch.empty_like(y)
        dg = torch.empty(c, dtype=torch.float32, device=self.device)
        db = torch.empty(c, dtype=torch.float32, device=self.device)
        _lib.raise_for(self.lib.dc_net_norm_act_bwd(self.gpu, _ptr(y), _ptr(da), n, vox, c, _ptr(coef), _ptr(gamma),
                                                    float(slope), _ptr(red), _ptr(dy), _ptr(dg), _ptr(db),
                                                    self._s()))
        return dy, dg, db

    def pack_input(self, terma, density, terma_scale, out=None):
        vox = terma.numel()
        x8 = out if out is not None else self._act((1,) + tuple(terma.shape[-3:]) + (IN_CHANNELS,))
        _lib.raise_for(self.lib.dc_net_pack_input(self.gpu, _ptr(terma), _ptr(density), vox, float(terma_scale),
                                                  _ptr(x8), self._s()))
        return x8

    def head(self, g, w, b, mask, mask_thr, scale, out=None):
        c = g.shape[-1]
        vox = g.numel() // c
        out = out if out is not None else torch.empty(vox, dtype=torch.float32, device=self.device)
        _lib.raise_for(self.lib.dc_net_head(self.gpu, _ptr(g), vox, c, _ptr(w), _ptr(b), _ptr(mask),
                                            float(mask_thr), float(scale), _ptr(out), self._s()))
        return out

    def head_loss_bwd(self, g, w, pred, target, inv_count):
        """inv_count: a float, or a one-element float32 device tensor (read at
        run time, so a captured graph can be replayed with new values)."""
        c = g.shape[-1]
        vox = g.numel() // c
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        dg = torch.empty_like(g)
        dw = torch.empty(c, dtype=torch.float32, device=self.device)
        db = torch.empty(1, dtype=torch.float32, device=self.device)
        inv_dev = inv_count if isinstance(inv_count, torch.Tensor) else None
        inv_val = 0.0 if inv_dev is not None else float(inv_count)
        _lib.raise_for(self.lib.dc_net_head_loss_bwd(self.gpu, _ptr(g), vox, c, _ptr(w), _ptr(pred), _ptr(target),
                                                     inv_val, _ptr(inv_dev), _ptr(loss), _ptr(dg), _ptr(dw),
                                                     _ptr(db), self._s()))
        return loss, dg, dw, db


def weight_shape(kind, cin, cout):
    """Master weight layout of a layer (see the C ABI): [taps][cin][cout], or
    [8][cout][cin] for the transposed convolution."""
    return (8, cout, cin) if kind == "up" else (_TAPS[kind], cin, cout)


class SurrogateNet:
    """Parameters and forward/backward passes of the encoder-decoder."""

    def __init__(self, device="cuda", seed=0, slope=0.01, eps=1e-5, terma_scale=1.0, dose_unit=1.0):
        self.ops = NetOps(device)
        self.device = self.ops.device
        self.slope, self.eps = float(slope), float(eps)
        self.terma_scale, self.dose_unit = float(terma_scale), float(dose_unit)
        gen = torch.Generator().manual_seed(int(seed))
        p = OrderedDict()
        for name, kind, cin, cout in ARCH:
            shape = weight_shape(kind, cin, cout)
            fan_in = cin * (1 if kind == "up" else _TAPS[kind])
            p[name + ".w"] = torch.randn(shape, generator=gen) * math.sqrt(2.0 / fan_in)
            if kind != "up":
                p[name + ".gamma"] = torch.ones(cout)
                p[name + ".beta"] = torch.zeros(cout)
        p["head.w"] = torch.randn(16, generator=gen) * 0.1
        p["head.b"] = torch.zeros(1)
        self.params = OrderedDict((k, v.to(self.device, torch.float32).contiguous()) for k, v in p.items())
        self._fw, self._bw, self._tc = {}, {}, {}
        self.use_tc = True  # tcgen05 convolutions where the grid allows them
        self.repack()

    # -- parameters ----------------------------------------------------------
    def repack(self):
        """bf16 fragment-order copies of the master weights: forward, and the
        backward-data form (flipped/transposed) of each layer.  The packed
        buffers are allocated once and rewritten in place, so CUDA graphs
        captured over the forward/backward see every update."""
        ops = self.ops
        forms = {"conv3": ((0, 0), (1, 1)), "down": ((0, 0), (0, 1)), "up": ((0, 1), (0, 0))}
        for name, kind, _, _ in ARCH:
            w = self.params[name + ".w"]
            (ff, ft), (bf, bt) = forms[kind]
            self._fw[name] = ops.pack(w, ff, ft, out=self._fw.get(name))
            if name != "enc0":
                self._bw[name] = ops.pack(w, bf, bt, out=self._bw.get(name))
            if name == "enc0":  # the 8 -> 16 input layer also runs on tcgen05 (x extent 128)
                self._tc[name] = ops.pack_tc(w, 0, 0, out=self._tc.get(name))

    def parameters(self):
        return list(self.params.values())

    def state_dict(self):
        sd = {k: v.detach().cpu().numpy() for k, v in self.params.items()}
        sd["meta"] = np.array([self.slope, self.eps, self.terma_scale, self.dose_unit], np.float64)
        return sd

    def load_state_dict(self, sd):
        meta = np.asarray(sd["meta"], np.float64)
        self.slope, self.eps, self.terma_scale, self.dose_unit = (float(v) for v in meta[:4])
        for k in self.params:
            if k not in sd:
                raise ValueError("missing parameter %r" % k)
            v = torch.as_tensor(np.asarray(sd[k], np.float32))
            if tuple(v.shape) != tuple(self.params[k].shape):
                raise ValueError("parameter %r has shape %s, expected %s" % (k, tuple(v.shape),
                                                                            tuple(self.params[k].shape)))
            self.params[k].copy_(v.to(self.device))
        self.repack()

    def save(self, path):
        np.savez_compressed(path, **self.state_dict())

    @classmethod
    def load(cls, path, device="cuda"):
        sd = dict(np.load(path))
        net = cls(device=device)
        net.load_state_dict(sd)
        return net

    @staticmethod
    def flops(shape):
        """Forward FLOPs (2 per multiply-add) of the convolution stack and head
        for a (d, h, w) input, counted from the layer shapes (the 8 padded input
        channels of the first layer included)."""
        d, h, w = shape
        vox = {0: d * h * w, 1: d * h * w // 8, 2: d * h * w // 64, 3: d * h * w // 512}
        lvl = {"enc0": 0, "down0": 1, "enc1": 1, "down1": 2, "enc2": 2, "down2": 3, "bott": 3, "up2": 2, "dec2": 2,
               "up1": 1, "dec1": 1, "up0": 0, "dec0": 0}
        total = 0
        for name, kind, cin, cout in ARCH:
            v = vox[lvl[name]]  # output voxels
            total += 2 * v * cout * cin * (1 if kind == "up" else _TAPS[kind])
        return total + 2 * 16 * d * h * w

    # -- passes ---------------------------------------------------------------
    def _block(self, name, x, cache):
        kind, cin, cout = _KIND[name]
        ops = self.ops
        n = x.shape[0]
        stats = torch.empty((n, cout, 2), dtype=torch.float64, device=self.device)
        if self.use_tc and name in self._tc and ops.tc_supported(tuple(x.shape[1:4]), cin, cout):
            y = ops.conv_tc(x, self._tc[name], cout, stats=stats)
        else:
            y = ops.conv(CONV3 if kind == "conv3" else DOWN2, x, self._fw[name], cout, stats=stats)
        count = y.shape[1] * y.shape[2] * y.shape[3]
        a, coef = ops.norm_stats_act(y, stats, count, self.params[name + ".gamma"], self.params[name + ".beta"],
                                     self.eps, self.slope)
        if cache is not None:
            cache[name] = (x, y, coef)
        return a

    def features(self, x8, cache=None):
        """Forward pass to the 16-channel output features g0."""
        ops = self.ops
        e0 = self._block("enc0", x8, cache)
        d0 = self._block("down0", e0, cache)
        e1 = self._block("enc1", d0, cache)
        d1 = self._block("down1", e1, cache)
        e2 = self._block("enc2", d1, cache)
        d2 = self._block("down2", e2, cache)
        b = self._block("bott", d2, cache)
        u2 = ops.conv_up(b, self._fw["up2"], 64, addend=e2)
        g2 = self._block("dec2", u2, cache)
        u1 = ops.conv_up(g2, self._fw["up1"], 32, addend=e1)
        g1 = self._block("dec1", u1, cache)
        u0 = ops.conv_up(g1, self._fw["up0"], 16, addend=e0)
        g0 = self._block("dec0", u0, cache)
        if cache is not None:
            cache.update(b=b, g2=g2, g1=g1, g0=g0)
        return g0

    def predict(self, terma, density, out=None, x8=None):
        """Dose (same units as the training target times dose_unit) of one
        control point from its TERMA and density volumes (float32 (d,h,w))."""
        x8 = self.ops.pack_input(terma, density, self.terma_scale, out=x8)
        g0 = self.features(x8)
        out = self.ops.head(g0, self.params["head.w"], self.params["head.b"], terma, 0.01, self.dose_unit,
                            out=None if out is None else out.view(-1))
        return out.view(terma.shape)

    def _block_bwd(self, name, da, cache, grads, keep=None):
        kind, cin, cout = _KIND[name]
        x, y, coef = cache[name]
        dy, dg, db = self.ops.norm_act_bwd(y, da, coef, self.params[name + ".gamma"], self.slope)
        if keep is not None:
            keep("dy." + name, dy)
        grads[name + ".gamma"], grads[name + ".beta"] = dg, db
        grads[name + ".w"] = self.ops.wgrad(CONV3 if kind == "conv3" else DOWN2, x, dy, cin)
        return dy

    def backward(self, cache, dg0, trace=None):
        """Gradients of every parameter given d(loss)/d(g0).  ``trace`` (a
        dict, optional) receives the gradients of the intermediate
        activations (keys as the forward's names: u0, g1, ..., e0)."""
        ops, fw, bw = self.ops, self._fw, self._bw
        grads = {}
        keep = (lambda k, v: trace.__setitem__(k, v)) if trace is not None else (lambda k, v: None)
        dy = self._block_bwd("dec0", dg0, cache, grads, keep)
        du0 = ops.conv(CONV3, dy, bw["dec0"], 16)
        grads["up0.w"] = ops.wgrad(DOWN2, du0, cache["g1"], 16)
        dg1 = ops.conv(DOWN2, du0, bw["up0"], 32)
        dy = self._block_bwd("dec1", dg1, cache, grads, keep)
        du1 = ops.conv(CONV3, dy, bw["dec1"], 32)
        grads["up1.w"] = ops.wgrad(DOWN2, du1, cache["g2"], 32)
        dg2 = ops.conv(DOWN2, du1, bw["up1"], 64)
        dy = self._block_bwd("dec2", dg2, cache, grads, keep)
        du2 = ops.conv(CONV3, dy, bw["dec2"], 64)
        grads["up2.w"] = ops.wgrad(DOWN2, du2, cache["b"], 64)
        dbt = ops.conv(DOWN2, du2, bw["up2"], 128)
        # encoder; d(e_k) starts as d(u_k) (the skip) and gains the down path
        if trace is not None:  # d(u_k) before the in-place accumulation
            trace.update(u0=du0.clone(), u1=du1.clone(), u2=du2.clone(), g1=dg1, g2=dg2, b=dbt)
        de2, de1, de0 = du2, du1, du0
        dy = self._block_bwd("bott", dbt, cache, grads, keep)
        dd2 = ops.conv(CONV3, dy, bw["bott"], 128)
        dy = self._block_bwd("down2", dd2, cache, grads, keep)
        ops.conv_up(dy, bw["down2"], 64, addend=de2, out=de2)
        dy = self._block_bwd("enc2", de2, cache, grads, keep)
        dd1 = ops.conv(CONV3, dy, bw["enc2"], 64)
        dy = self._block_bwd("down1", dd1, cache, grads, keep)
        ops.conv_up(dy, bw["down1"], 32, addend=de1, out=de1)
        dy = self._block_bwd("enc1", de1, cache, grads, keep)
        dd0 = ops.conv(CONV3, dy, bw["enc1"], 32)
        dy = self._block_bwd("down0", dd0, cache, grads, keep)
        ops.conv_up(dy, bw["down0"], 16, addend=de0, out=de0)
        self._block_bwd("enc0", de0, cache, grads, keep)
        if trace is not None:
            trace.update(d2=dd2, e2=de2, d1=dd1, e1=de1, d0=dd0, e0=de0)
        return grads

    def loss_and_grads(self, x8, target, inv_count, trace=None):
        """Squared-error loss (times inv_count) over voxels with target >= 0 and
        the gradient of every parameter.  target: float32 (d*h*w), dose /
        dose_unit, negative where the voxel is masked."""
        cache = {}
        g0 = self.features(x8, cache)
        w, b = self.params["head.w"], self.params["head.b"]
        pred = self.ops.head(g0, w, b, target, -0.5, 1.0)
        loss, dg0, dw, db = self.ops.head_loss_bwd(g0, w, pred, target, inv_count)
        grads = self.backward(cache, dg0, trace)
        if trace is not None:
            trace["g0"] = dg0
        grads["head.w"], grads["head.b"] = dw, db
        return loss, grads


# ---------------------------------------------------------------------------
# Training data: phantoms and fields of the surrogate workload
# ---------------------------------------------------------------------------
def random_phantom_hu(rng: np.random.Generator, shape=(128, 128, 128), spacing=2.5, device="cuda") -> torch.Tensor:
    """HU volume: air, a water body ellipsoid, 1-5 random rotated ellipsoids
    with HU uniform in [-900, 1500] inside it."""
    nz, ny, nx = shape
    dev = torch.device(device)
    z = (torch.arange(nz, device=dev, dtype=torch.float32) - (nz - 1) / 2) * spacing
    y = (torch.arange(ny, device=dev, dtype=torch.float32) - (ny - 1) / 2) * spacing
    x = (torch.arange(nx, device=dev, dtype=torch.float32) - (nx - 1) / 2) * spacing
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    ext = np.array([nx, ny, nz], np.float64) * spacing
    hu = torch.full(shape, -1000.0, device=dev)
    body_ax = ext * rng.uniform(0.32, 0.46, size=3)
    body_c = rng.uniform(-0.04, 0.04, size=3) * ext
    body = ((X - body_c[0]) / body_ax[0]) ** 2 + ((Y - body_c[1]) / body_ax[1]) ** 2 + \
           ((Z - body_c[2]) / body_ax[2]) ** 2 <= 1.0
    hu[body] = 0.0
    for _ in range(int(rng.integers(1, 6))):
        ax = rng.uniform(8.0, 60.0, size=3)
        c = body_c + rng.uniform(-0.6, 0.6, size=3) * body_ax
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        R = torch.as_tensor(q, dtype=torch.float32, device=dev)
        dx, dy, dz = X - float(c[0]), Y - float(c[1]), Z - float(c[2])
        u = (R[0, 0] * dx + R[0, 1] * dy + R[0, 2] * dz) / float(ax[0])
        v = (R[1, 0] * dx + R[1, 1] * dy + R[1, 2] * dz) / float(ax[1])
        w = (R[2, 0] * dx + R[2, 1] * dy + R[2, 2] * dz) / float(ax[2])
        hu[(u * u + v * v + w * w <= 1.0) & body] = float(rng.uniform(-900.0, 1500.0))
    return hu


def hu_to_density(hu: torch.Tensor, table_hu, table_density) -> torch.Tensor:
    """Piecewise-linear HU -> relative density with end clamping (the
    np.interp of IMRTDoseGrid.DensityFromHU, plan_imrt.py:114-124)."""
    xp = torch.as_tensor(np.array(table_hu, np.float64), dtype=torch.float64, device=hu.device)
    fp = torch.as_tensor(np.array(table_density, np.float64), dtype=torch.float64, device=hu.device)
    h = hu.to(torch.float64).clamp(float(xp[0]), float(xp[-1]))
    i = torch.searchsorted(xp, h, right=True).clamp(1, len(xp) - 1)
    x0, x1, f0, f1 = xp[i - 1], xp[i], fp[i - 1], fp[i]
    t = (h - x0) / (x1 - x0)
    return (f0 + t * (f1 - f0)).to(torch.float32)


def random_field(rng: np.random.Generator):
    """(gantry deg, field x cm, field y cm): gantry uniform over 0-355 in 5
    degree steps; square or rectangular fields of 2-20 cm per side."""
    gantry = 5.0 * float(rng.integers(0, 72))
    fx = float(rng.uniform(2.0, 20.0))
    fy = fx if rng.random() < 0.5 else float(rng.uniform(2.0, 20.0))
    return gantry, fx, fy


class SampleMaker:
    """Generates (density, TERMA, CCCS dose) samples of the surrogate workload
    with this engine: seeded phantom -> density -> PhotonBeam TERMA + CCCS."""

    def __init__(self, shape=(128, 128, 128), spacing=2.5, machine="VarianTrueBeamHF", device="cuda", mu=100.0):
        import pandas as pd

        from . import engine
        from .lookup import table_path
        from .plan_imrt import IMRTPlan

        self.shape, self.spacing, self.mu = tuple(shape), float(spacing), float(mu)
        self.device = torch.device(device)
        df = pd.read_csv(table_path("photons", machine, "HU_Density.csv"))
        self.table = (df["HU"].to_numpy(), df["Density"].to_numpy())
        self.plan = IMRTPlan(machine)
        self.model = self.plan.beam_models[0]
        nz, ny, nx = self.shape

        class _G:
            pass

        g = _G()
        g.spacing = np.array([spacing] * 3, np.float64)
        g.origin = np.array([-nx * spacing / 2.0, -ny * spacing / 2.0, -nz * spacing / 2.0])
        self.grid = g
        self.beam = engine.PhotonBeam(g, self.shape, device=self.device)
        self._mv = None

    def control_point(self, gantry, fx, fy):
        self.plan.addSquareField("6", fx, fy, mu=self.mu, gantry_angle=gantry)
        return self.plan.beam_list[-1].cp_list[0]

    def views(self, cp):
        from .dose_kernels import ControlPointView, PhotonModelView
        if self._mv is None:
            self._mv = PhotonModelView(self.model)
        return self._mv, ControlPointView(cp)

    def dose_scale(self, cp):
        return float(self.model.mu_calibration) * float(cp.mu)

    def make(self, seed):
        rng = np.random.default_rng(seed)
        hu = random_phantom_hu(rng, self.shape, self.spacing, self.device)
        density = hu_to_density(hu, *self.table).contiguous()
        cp = self.control_point(*random_field(rng))
        self.beam.set_density(density)
        terma = self.beam.terma(self.model, cp, out=True, views=self.views(cp))
        dose = self.beam.dose()
        return density, terma, dose, cp


# ---------------------------------------------------------------------------
# Training
# ---------------------------------------------------------------------------
class Dataset:
    """Samples resident on the device: TERMA (f32), density (bf16) and the
    normalised target (dose/(dose_scale*dose_unit), -1 where masked)."""

    def __init__(self, maker: SampleMaker, seeds, dose_unit=1.0, log=None):
        self.maker = maker
        self.seeds = list(seeds)
        n = len(self.seeds)
        shape = maker.shape
        dev = maker.device
        self.terma = torch.empty((n,) + shape, dtype=torch.float32, device=dev)
        self.density = torch.empty((n,) + shape, dtype=torch.bfloat16, device=dev)
        self.target = torch.empty((n,) + shape, dtype=torch.float32, device=dev)
        self.inv_count = np.zeros(n)
        self.scale = np.zeros(n)
        t0 = time.time()
        for i, s in enumerate(self.seeds):
            density, terma, dose, cp = maker.make(s)
            ds = maker.dose_scale(cp) * dose_unit
            self.terma[i] = terma
            self.density[i] = density.to(torch.bfloat16)
            active = terma > 0.01
            self.target[i] = torch.where(active, dose / ds, torch.full_like(dose, -1.0))
            self.inv_count[i] = 1.0 / max(int(active.sum()), 1)
            self.scale[i] = ds
            if log and (i + 1) % 100 == 0:
                log("generated %d/%d samples (%.1f s)" % (i + 1, n, time.time() - t0))

    def __len__(self):
        return len(self.seeds)


class Trainer:
    """One training step (input packing, forward, loss, backward, Adam,
    weight repacking) on static device buffers, captured once in a CUDA graph
    and replayed per sample; eager when capture is disabled."""

    def __init__(self, net: SurrogateNet, shape, lr=1e-3, use_graph=True):
        self.net = net
        dev = net.device
        self.shape = tuple(shape)
        self.terma = torch.zeros(self.shape, dtype=torch.float32, device=dev)
        self.density = torch.zeros(self.shape, dtype=torch.float32, device=dev)
        self.target = torch.full((int(np.prod(self.shape)),), -1.0, dtype=torch.float32, device=dev)
        self.inv = torch.ones(1, dtype=torch.float32, device=dev)
        self.x8 = None
        self.lr = torch.tensor(float(lr), dtype=torch.float32, device=dev)
        for p in net.parameters():
            p.grad = torch.zeros_like(p)
        self.opt = torch.optim.Adam(net.parameters(), lr=self.lr, capturable=True)
        self.loss_sum = torch.zeros((), dtype=torch.float64, device=dev)
        self.use_graph = use_graph
        self.graph = None
        self.steps = 0  # steps taken by this training run (restored on resume)
        self._calls = 0  # steps taken by this instance

    def _step(self):
        net = self.net
        self.x8 = net.ops.pack_input(self.terma, self.density, net.terma_scale, out=self.x8)
        loss, grads = net.loss_and_grads(self.x8, self.target, self.inv)
        for k, p in net.params.items():
            p.grad.copy_(grads[k])
        self.opt.step()
        net.repack()
        self.loss_sum += loss[0]

    def _adam_state(self, p):
        """Adam's per-parameter state, created here (as the capturable
        optimiser would on its first step) so that it can be restored in
        place before any step."""
        st = self.opt.state[p]
        if not st:
            st["step"] = torch.zeros((), dtype=torch.float32, device=p.device)
            st["exp_avg"] = torch.zeros_like(p, memory_format=torch.preserve_format)
            st["exp_avg_sq"] = torch.zeros_like(p, memory_format=torch.preserve_format)
        return st

    def state(self):
        """Host copy of everything the next step depends on: master weights,
        Adam's moments and step counts, the learning rate and the running
        loss sum."""
        net = self.net
        adam = {}
        for k, p in net.params.items():
            st = self._adam_state(p)
            adam[k] = {n: st[n].detach().cpu().clone() for n in ("step", "exp_avg", "exp_avg_sq")}
        return {"params": {k: v.detach().cpu().clone() for k, v in net.params.items()},
                "meta": [net.slope, net.eps, net.terma_scale, net.dose_unit], "adam": adam,
                "lr": float(self.lr), "loss_sum": float(self.loss_sum), "steps": self.steps}

    def restore(self, state):
        """Copies a ``state()`` back into the live tensors (in place, so a
        captured step graph stays valid) and repacks the weights."""
        net = self.net
        if set(state["params"]) != set(net.params):
            raise ValueError("checkpoint parameters do not match the network")
        slope, eps, ts, du = (float(v) for v in state["meta"])
        net.slope, net.eps, net.terma_scale, net.dose_unit = slope, eps, ts, du
        for k, p in net.params.items():
            src = state["params"][k]
            if tuple(src.shape) != tuple(p.shape):
                raise ValueError("parameter %r has shape %s, expected %s" % (k, tuple(src.shape), tuple(p.shape)))
            p.data.copy_(src.to(p.device))
            st = self._adam_state(p)
            for n in ("step", "exp_avg", "exp_avg_sq"):
                st[n].copy_(state["adam"][k][n].to(p.device))
        net.repack()
        self.lr.fill_(float(state["lr"]))
        self.loss_sum.fill_(float(state["loss_sum"]))
        self.steps = int(state["steps"])

    def load(self, terma, density, target, inv_count):
        self.terma.copy_(terma)
        self.density.copy_(density)
        self.target.copy_(target.reshape(-1))
        self.inv.fill_(float(inv_count))

    def step(self):
        """One step on the loaded sample."""
        if self.use_graph and self.graph is None and self._calls >= 3:
            # capture after three eager steps of this instance (Adam's state
            # and every lazily allocated buffer exist by then)
            side = torch.cuda.Stream(self.net.device)
            side.wait_stream(torch.cuda.current_stream(self.net.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(side):
                with torch.cuda.graph(g, stream=side):
                    self._step()
            torch.cuda.current_stream(self.net.device).wait_stream(side)
            self.graph = g
        if self.graph is not None:
            self.graph.replay()
        else:
            self._step()
        self.steps += 1
        self._calls += 1


def save_training_state(path, trainer: "Trainer", progress: dict):
    """Writes a resumable training checkpoint: the trainer's ``state()`` plus
    the loop's progress (step, epoch, position in the epoch's sample order,
    the generator state the order was drawn from, the schedule, the log
    history).  Written to a temporary file and renamed, so an interrupted
    write leaves the previous checkpoint intact."""
    blob = {"version": 1, "trainer": trainer.state(), "progress": progress}
    tmp = str(path) + ".tmp"
    torch.save(blob, tmp)
    os.replace(tmp, str(path))


def load_training_state(path):
    blob = torch.load(str(path), map_location="cpu", weights_only=True)
    if blob.get("version") != 1:
        raise ValueError("unsupported training checkpoint %r" % str(path))
    return blob


def train(net: SurrogateNet, data: Dataset, epochs=1, lr=1e-3, seed=0, log=None, max_steps=None,
          time_budget_s=None, checkpoint=None, cosine=True, lr_min=1e-5, use_graph=True, state_path=None,
          state_every=None, resume=None, session_steps=None, on_step=None):
    """Adam (lr, cosine-decayed to lr_min over the planned steps when
    ``cosine``) on the squared error of the normalised dose, one sample per
    step, samples shuffled each epoch.  Returns a list of (step, epoch, mean
    loss of the last log interval, seconds).

    ``checkpoint``: weights (.npz) written at each epoch end.
    ``state_path``: a resumable training checkpoint written every
    ``state_every`` steps (default: at each epoch end) and when the loop
    stops.  ``resume``: such a checkpoint to continue from; the schedule
    (epochs, lr, lr_min, planned steps, seed) is taken from it, and the loop
    continues at the same sample of the same epoch order.
    ``session_steps``: stop after this many steps of this call (a time slice
    of a longer run; the schedule still spans the planned steps).
    ``on_step(step, epoch, sample_index, lr)`` is called before each step."""
    tr = Trainer(net, data.maker.shape, lr=lr, use_graph=use_graph)
    step, last, ep0, pos0 = 0, 0, 0, 0
    hist = []
    rng = np.random.default_rng(seed)
    if resume is not None:
        blob = load_training_state(resume)
        pr = blob["progress"]
        if int(pr["n_samples"]) != len(data):
            raise ValueError("checkpoint was written for %d samples, the dataset has %d" % (pr["n_samples"],
                                                                                          len(data)))
        tr.restore(blob["trainer"])
        epochs, lr, lr_min, cosine = int(pr["epochs"]), float(pr["lr"]), float(pr["lr_min"]), bool(pr["cosine"])
        max_steps = pr["max_steps"]
        step, last, ep0, pos0 = int(pr["step"]), int(pr["last"]), int(pr["epoch"]), int(pr["pos"])
        hist = [tuple(h) for h in pr["hist"]]
        rng.bit_generator.state = pr["rng_state"]
    total = epochs * len(data)
    if max_steps:
        total = min(total, max_steps)
    t0 = time.time()
    stop = False
    step0 = step

    def progress(ep, pos, rng_state):
        return {"step": step, "last": last, "epoch": ep, "pos": pos, "rng_state": rng_state, "epochs": epochs,
                "lr": lr, "lr_min": lr_min, "cosine": cosine, "max_steps": max_steps, "n_samples": len(data),
                "hist": [list(h) for h in hist]}

    for ep in range(ep0, epochs):
        rng_state = rng.bit_generator.state  # the order of this epoch is drawn from here
        order = rng.permutation(len(data))
        pos = pos0 if ep == ep0 else 0
        while pos < len(order):
            if step >= total:  # a resumed run that had already finished
                stop = True
                break
            i = order[pos]
            pos += 1
            lr_now = lr
            if cosine:
                frac = min(step / max(total, 1), 1.0)
                lr_now = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * frac))
                tr.lr.fill_(lr_now)
            if on_step:
                on_step(step, ep, int(i), lr_now)
            tr.load(data.terma[i], data.density[i], data.target[i], data.inv_count[i])
            tr.step()
            step += 1
            if log and step % 500 == 0:
                m = float(tr.loss_sum) / (step - last)
                tr.loss_sum.zero_()
                last = step
                hist.append((step, ep, m, time.time() - t0))
                log("step %d epoch %d loss %.4e (%.1f s)" % (step, ep, m, time.time() - t0))
            if step >= total or (time_budget_s and time.time() - t0 > time_budget_s):
                stop = True
            if session_steps and step - step0 >= session_steps:
                stop = True
            if state_path and (stop or (state_every and step % state_every == 0)):
                save_training_state(state_path, tr, progress(ep, pos, rng_state))
            if stop:
                break
        if checkpoint:
            net.save(checkpoint)
        if state_path and not state_every and not stop:
            save_training_state(state_path, tr, progress(ep + 1, 0, rng.bit_generator.state))
        if stop:
            break
    torch.cuda.synchronize(net.device)
    return hist


# ---------------------------------------------------------------------------
# Accept / fall back
# ---------------------------------------------------------------------------
class PhotonSurrogate:
    """Surrogate dose of one photon control point with CCCS fallback.

    ``dose(density, cp)`` runs TERMA, the network (one CUDA-graph replay),
    the CCCS probe and the probe gamma; it returns (dose, accepted,
    pass_rate, n_probe_points).  A rejected control point gets the full CCCS
    dose from the same TERMA."""

    def __init__(self, net: SurrogateNet, grid, shape, model, accept_rate=0.99, dta_mm=2.0, dd_frac=0.02,
                 cutoff_frac=0.1, use_graph=True):
        from . import engine
        self.net, self.model = net, model
        self.grid, self.shape = grid, tuple(shape)
        self.accept_rate, self.dta, self.dd, self.cutoff = accept_rate, dta_mm, dd_frac, cutoff_frac
        dev = net.device
        self.beam = engine.PhotonBeam(grid, shape, device=dev)
        self.terma = torch.zeros(self.shape, dtype=torch.float32, device=dev)
        self.density = torch.zeros(self.shape, dtype=torch.float32, device=dev)
        self.pred = torch.zeros(self.shape, dtype=torch.float32, device=dev)
        self.counts = torch.zeros(4, dtype=torch.int32, device=dev)
        self._x8 = None
        self._mv = None
        self.use_graph = use_graph
        self.graph = None
        self._runs = 0

    def _network(self):
        """pred = network dose / dose_scale (masked where TERMA <= 0.01)."""
        net = self.net
        self._x8 = net.ops.pack_input(self.terma, self.density, net.terma_scale, out=self._x8)
        g0 = net.features(self._x8)
        net.ops.head(g0, net.params["head.w"], net.params["head.b"], self.terma, 0.01, net.dose_unit,
                     out=self.pred.view(-1))

    def run_network(self):
        if self.use_graph and self.graph is None and self._runs >= 1:
            dev = self.net.device
            side = torch.cuda.Stream(dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(side):
                with torch.cuda.graph(g, stream=side):
                    self._network()
            torch.cuda.current_stream(dev).wait_stream(side)
            self.graph = g
        if self.graph is not None:
            self.graph.replay()
        else:
            self._network()
        self._runs += 1

    def dose(self, density: torch.Tensor, cp, force_fallback=False):
        from . import engine
        from .dose_kernels import ControlPointView, PhotonModelView
        if self._mv is None:
            self._mv = PhotonModelView(self.model)
        views = (self._mv, ControlPointView(cp))
        scale = float(self.model.mu_calibration) * float(cp.mu)
        self.beam.set_density(density)
        self.density.copy_(density)
        self.beam.terma(self.model, cp, out=self.terma, views=views)
        self.run_network()
        vp, n, _ = self.beam.probe_voxels(host=False)  # selected and uploaded by terma
        probe = self.beam.probe()
        probe.mul_(1.0 / scale)  # to the network's units (gamma is scale-free)
        engine.gamma_counts(self.pred, self.grid.spacing, probe, vp, n, 0.0, self.dta, self.dd, self.cutoff,
                            counts=self.counts)
        ev, ps = (int(v) for v in self.counts[:2].cpu())
        rate = ps / ev if ev else 0.0
        accepted = (ev > 0 and rate >= self.accept_rate) and not force_fallback
        if accepted:
            return self.pred.mul_(scale), True, rate, n
        return self.beam.dose(), False, rate, n
