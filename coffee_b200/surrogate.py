"""Learned warm start for the rotating-star problem: a small 3D convolutional
network (a two-level U-Net) that maps a star's vacuum dipole to the
magnetosphere it settles into, so that a run can start near its steady
state instead of from the dipole.  No counterpart in the reference (its
drivers always start from the vacuum dipole, ``src/user_pulsar3d_EZ.hpp``).

Every arithmetic step of training and inference runs on the library's
kernels (include/coffee_surrogate.h): BF16 tensor-core convolutions with
FP32 accumulation for the forward pass and both gradients, and the
pooling, activation, loss and Adam kernels.  torch provides the device
memory only.  The training set is made by the flat solver itself: oblique
rotators run from their vacuum dipoles at full resolution and averaged onto
the network's coarser grid (rotator_training_set); rotator_study measures
the wall time to a settled spindown luminosity from the cold and the warm
start.

Network (channels-last, 3x3x3 convolutions, leaky ReLU with slope 0.1):

    x (16) -> c1 (16) -> c2 (16) = s  -> pool -> c3 (32) -> c4 (32) -> up
    [up (32), s (16)] -> c5 (16) -> c6 (16, linear) = output

Inputs: the dipole B scaled by (r / R)^3, the coordinates over the box
size, the star mask, sin and cos of the inclination.  Output: the change of
E, B, P from the dipole state, scaled the same way, outside 1.5 star radii.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib, problems
from ._lib import CoffeeError, check

SLOPE = 0.1
CIN, C1, C2, COUT = 16, 16, 32, 16
# the prediction is trained and applied outside STAR_EDGE star radii; inside,
# the star's own boundary condition sets the fields
STAR_EDGE = 1.5


def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ---------------------------------------------------------------- kernels

def conv_forward(x, w_bf16, bias, k, act, z=None, a=None):
    """x: (N, D, H, W, C) BF16; returns (z FP32 or None, a BF16 or None)."""
    n, d, h, ww, c = x.shape
    check(_lib.load().coffee_conv3d_forward(_ptr(x), n, d, h, ww, c, _ptr(w_bf16), k, _ptr(bias),
                                            _ptr(z), _ptr(a), int(act), SLOPE, _stream()))
    return z, a


def conv_forward_tc(x, w_bf16, bias, k, act, z=None, a=None):
    """conv_forward on the tcgen05 tensor cores (K = 16, 32, 48 or 64)."""
    n, d, h, ww, c = x.shape
    check(_lib.load().coffee_conv3d_forward_tc(_ptr(x), n, d, h, ww, c, _ptr(w_bf16), k,
                                               _ptr(bias), _ptr(z), _ptr(a), int(act), SLOPE,
                                               _stream()))
    return z, a


def use_tc(c, k):
    """True where the tcgen05 convolution runs (it is the faster one for every
    layer of the network, the 48-channel input included since two CTAs share
    an SM); its results are those of the mma.sync kernel."""
    return c in (16, 32, 48, 64) and k in (16, 32, 48, 64)


def use_tc_wgrad(c, k):
    """True where the weight gradient runs on the tcgen05 kernel: inputs of
    16, 32, 48 or 64 channels and 16, 32 or 64 outputs (the results agree
    with the mma.sync kernel's to FP32 rounding)."""
    return c in (16, 32, 48, 64) and k in (16, 32, 64)


def tc_fault(clear=True):
    """True if a wait of the tcgen05 convolution ran out of time (results invalid)."""
    flag = ctypes.c_int(0)
    check(_lib.load().coffee_conv3d_tc_fault(ctypes.byref(flag), int(clear)))
    return bool(flag.value)


def check_tc():
    """Raise if a tcgen05 convolution ran out of time since the last check
    (synchronises).  A timeout also makes every later tcgen05 launch fail
    with COFFEE_E_TIMEOUT, so a training loop stops at its next launch; this
    covers the last launches of a run."""
    if tc_fault(clear=False):
        raise CoffeeError(_lib.COFFEE_E_TIMEOUT,
                          "a tcgen05 convolution ran out of time: its results are invalid")


def conv_backward_data(dy, wt_bf16, c, dx):
    n, d, h, w, k = dy.shape
    check(_lib.load().coffee_conv3d_backward_data(_ptr(dy), n, d, h, w, k, _ptr(wt_bf16), c,
                                                  _ptr(dx), _stream()))
    return dx


def conv_backward_weight(dy, x, dw, workspace):
    n, d, h, w, k = dy.shape
    c = x.shape[-1]
    check(_lib.load().coffee_conv3d_backward_weight(_ptr(dy), _ptr(x), n, d, h, w, k, c,
                                                    _ptr(dw), _ptr(workspace), _stream()))
    return dw


def conv_backward_weight_tc(dy, x, dw, workspace):
    """The weight gradient on the tcgen05 kernel (C in 16, 32, 48, 64)."""
    n, d, h, w, k = dy.shape
    c = x.shape[-1]
    check(_lib.load().coffee_conv3d_backward_weight_tc(_ptr(dy), _ptr(x), n, d, h, w, k, c,
                                                       _ptr(dw), _ptr(workspace), _stream()))
    return dw


def flip_weights(w_bf16, wt):
    k, _, c = w_bf16.shape
    check(_lib.load().coffee_conv3d_flip_weights(_ptr(w_bf16), k, c, _ptr(wt), _stream()))


def to_bf16(src, dst):
    check(_lib.load().coffee_to_bf16(_ptr(src), src.numel(), _ptr(dst), _stream()))
    return dst


def workspace_bytes(k, c):
    return int(_lib.load().coffee_conv3d_backward_weight_workspace(k, c))


# ------------------------------------------------------------------ model

class Conv:
    """One 3x3x3 layer: FP32 master weights (K, 27, C) and bias, their Adam
    moments and gradients, the BF16 copy and its tap-reversed transpose."""

    def __init__(self, cin, cout, gen, dev):
        torch = _torch()
        std = math.sqrt(2.0 / (27 * cin))
        self.cin, self.cout = cin, cout
        self.w = (torch.randn(cout, 27, cin, generator=gen) * std).to(dev)
        self.b = torch.zeros(cout, device=dev)
        self.gw, self.gb = torch.zeros_like(self.w), torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.wb = torch.empty(cout, 27, cin, dtype=torch.bfloat16, device=dev)
        self.wt = torch.empty(cin, 27, cout, dtype=torch.bfloat16, device=dev)
        self.refresh()

    def refresh(self):
        to_bf16(self.w, self.wb)
        flip_weights(self.wb, self.wt)

    def adam(self, lr, t, b1=0.9, b2=0.999, eps=1e-8):
        lib = _lib.load()
        check(lib.coffee_adam(_ptr(self.w), _ptr(self.gw), _ptr(self.mw), _ptr(self.vw),
                              self.w.numel(), lr, b1, b2, eps, t, _ptr(self.wb), _stream()))
        check(lib.coffee_adam(_ptr(self.b), _ptr(self.gb), _ptr(self.mb), _ptr(self.vb),
                              self.b.numel(), lr, b1, b2, eps, t, None, _stream()))
        flip_weights(self.wb, self.wt)


class UNet:
    """The two-level U-Net of the module docstring on the library's kernels."""

    def __init__(self, seed=0, device="cuda"):
        torch = _torch()
        gen = torch.Generator().manual_seed(seed)
        self.dev = torch.device(device)
        self.layers = [Conv(CIN, C1, gen, self.dev), Conv(C1, C1, gen, self.dev),
                       Conv(C1, C2, gen, self.dev), Conv(C2, C2, gen, self.dev),
                       Conv(C2 + C1, C1, gen, self.dev), Conv(C1, COUT, gen, self.dev)]
        self.t = 0
        self._ws = None

    def _conv(self, i, x, act):
        torch = _torch()
        L = self.layers[i]
        shape = x.shape[:4] + (L.cout,)
        z = torch.empty(shape, dtype=torch.float32, device=self.dev)
        a = torch.empty(shape, dtype=torch.bfloat16, device=self.dev) if act else None
        fwd = conv_forward_tc if use_tc(L.cin, L.cout) else conv_forward
        fwd(x, L.wb, L.b, L.cout, act, z, a)
        return z, a

    def forward(self, x):
        """x: (N, D, H, W, 16) BF16, D, H, W even.  Returns the FP32 output
        (N, D, H, W, 16) and keeps what the backward pass needs."""
        torch = _torch()
        lib = _lib.load()
        n, d, h, w, _ = x.shape
        s = {"x": x}
        s["z1"], s["a1"] = self._conv(0, x, True)
        s["z2"], s["a2"] = self._conv(1, s["a1"], True)
        p2 = torch.empty((n, d // 2, h // 2, w // 2, C1), dtype=torch.bfloat16, device=self.dev)
        check(lib.coffee_pool2_forward(_ptr(s["a2"]), n, d, h, w, C1, _ptr(p2), _stream()))
        s["p2"] = p2
        s["z3"], s["a3"] = self._conv(2, p2, True)
        s["z4"], s["a4"] = self._conv(3, s["a3"], True)
        cat = torch.empty((n, d, h, w, C2 + C1), dtype=torch.bfloat16, device=self.dev)
        check(lib.coffee_up2_forward(_ptr(s["a4"]), n, d // 2, h // 2, w // 2, C2, _ptr(cat),
                                     C2 + C1, 0, _stream()))
        check(lib.coffee_channels_copy(_ptr(s["a2"]), n * d * h * w, C1, _ptr(cat), C2 + C1, C2,
                                       _stream()))
        s["cat"] = cat
        s["z5"], s["a5"] = self._conv(4, cat, True)
        out, _ = self._conv(5, s["a5"], False)
        self._saved = s
        return out

    def _layer_grads(self, i, dz, dzb, x_in):
        """Bias and weight gradients of layer i from dz (FP32 and BF16) and its input."""
        lib = _lib.load()
        torch = _torch()
        L = self.layers[i]
        npts = dz.numel() // L.cout
        check(lib.coffee_bias_grad(_ptr(dz), npts, L.cout, _ptr(L.gb), _stream()))
        need = workspace_bytes(L.cout, L.cin)
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.dev)
        wgrad = conv_backward_weight_tc if use_tc_wgrad(L.cin, L.cout) else conv_backward_weight
        wgrad(dzb, x_in, L.gw, self._ws)

    def backward(self, dout):
        """Gradients of every layer for dL/dout (FP32, the output's shape)."""
        torch = _torch()
        lib = _lib.load()
        s = self._saved
        n, d, h, w, _ = dout.shape
        full = n * d * h * w

        def bf(t):
            return to_bf16(t, torch.empty(t.shape, dtype=torch.bfloat16, device=self.dev))

        def leaky_bwd(da, z):
            dz = torch.empty_like(da)
            dzb = torch.empty(da.shape, dtype=torch.bfloat16, device=self.dev)
            check(lib.coffee_leaky_backward(_ptr(da), _ptr(z), da.numel(), SLOPE, _ptr(dz),
                                            _ptr(dzb), _stream()))
            return dz, dzb

        def dgrad(i, dzb, like):
            L = self.layers[i]
            dx = torch.empty(like.shape[:4] + (L.cin,), dtype=torch.float32, device=self.dev)
            if use_tc(L.cout, L.cin):
                return conv_forward_tc(dzb, L.wt, None, L.cin, False, dx, None)[0]
            return conv_backward_data(dzb, L.wt, L.cin, dx)

        dzb6 = bf(dout)
        self._layer_grads(5, dout, dzb6, s["a5"])
        da5 = dgrad(5, dzb6, dout)
        dz5, dzb5 = leaky_bwd(da5, s["z5"])
        self._layer_grads(4, dz5, dzb5, s["cat"])
        dcat = dgrad(4, dzb5, dout)
        da4 = torch.empty((n, d // 2, h // 2, w // 2, C2), dtype=torch.float32, device=self.dev)
        check(lib.coffee_up2_backward(_ptr(dcat), n, d // 2, h // 2, w // 2, C2, C2 + C1, 0,
                                      _ptr(da4), _stream()))
        da2 = torch.zeros((n, d, h, w, C1), dtype=torch.float32, device=self.dev)
        check(lib.coffee_channels_add(_ptr(dcat), full, C2 + C1, C2, C1, _ptr(da2), _stream()))
        dz4, dzb4 = leaky_bwd(da4, s["z4"])
        self._layer_grads(3, dz4, dzb4, s["a3"])
        da3 = dgrad(3, dzb4, da4)
        dz3, dzb3 = leaky_bwd(da3, s["z3"])
        self._layer_grads(2, dz3, dzb3, s["p2"])
        dp2 = dgrad(2, dzb3, da4)
        check(lib.coffee_pool2_backward_add(_ptr(dp2), n, d, h, w, C1, _ptr(da2), _stream()))
        dz2, dzb2 = leaky_bwd(da2, s["z2"])
        self._layer_grads(1, dz2, dzb2, s["a1"])
        da1 = dgrad(1, dzb2, da2)
        dz1, dzb1 = leaky_bwd(da1, s["z1"])
        self._layer_grads(0, dz1, dzb1, s["x"])

    def step(self, lr):
        self.t += 1
        for L in self.layers:
            L.adam(lr, self.t)

    def loss(self, out, target, mask):
        """Masked mean-square error over the output channels: (loss, dL/dout)."""
        torch = _torch()
        npts = out.numel() // COUT
        count = float(mask.sum().item()) * COUT
        dout = torch.empty_like(out)
        buf = torch.empty(257, dtype=torch.float64, device=self.dev)
        check(_lib.load().coffee_mse(_ptr(out), _ptr(target), _ptr(mask), npts, COUT, count,
                                     _ptr(dout), _ptr(buf), _stream()))
        return buf[0], dout


# ------------------------------------------------------ the star problem

def _coords(p):
    Z, Y, X = problems._xyz(p, np.float32)
    return X, Y, Z


def features(p, fields, inclination_deg, omega_ref=0.15):
    """Input channels (D, H, W, 16) of the interior: B r^3 / R^3 of the
    dipole state, x, y, z / half size, the star mask, sin and cos of the
    inclination, the spin omega / omega_ref, zeros."""
    g = p.guard[0]
    X, Y, Z = (c[g:-g, g:-g, g:-g] for c in _coords(p))
    R = np.sqrt(X * X + Y * Y + Z * Z)
    scale = np.minimum((np.maximum(R, p.radius) / p.radius) ** 3, 1e4).astype(np.float32)
    out = np.zeros(X.shape + (CIN,), np.float32)
    for c in range(3):
        out[..., c] = fields[3 + c][g:-g, g:-g, g:-g] * scale
    L = p.size[0] / 2
    out[..., 3], out[..., 4], out[..., 5] = X / L, Y / L, Z / L
    out[..., 6] = (R < p.radius).astype(np.float32)
    a = math.radians(inclination_deg)
    out[..., 7], out[..., 8] = math.sin(a), math.cos(a)
    out[..., 9] = p.omega / omega_ref
    return out


def target_and_mask(p, start, steady):
    """Output channels (D, H, W, 16): (steady - start) for E, B, P scaled
    by r^3 / R^3, and the loss mask (outside 1.5 radii, inside the
    absorbing layer's inner edge)."""
    g = p.guard[0]
    X, Y, Z = (c[g:-g, g:-g, g:-g] for c in _coords(p))
    R = np.sqrt(X * X + Y * Y + Z * Z)
    scale = np.minimum((np.maximum(R, p.radius) / p.radius) ** 3, 1e4).astype(np.float32)
    out = np.zeros(X.shape + (COUT,), np.float32)
    for c in range(7):
        out[..., c] = (steady[c] - start[c])[g:-g, g:-g, g:-g] * scale
    edge = p.size[0] / 2 - p.pml[0] * p.size[0] / p.N[0]
    mask = ((R > STAR_EDGE * p.radius) & (np.abs(X) < edge) & (np.abs(Y) < edge) &
            (np.abs(Z) < edge)).astype(np.float32)
    return out, mask


# --------------------------------------------------------- warm-start study

def star_run(p, fields, steps, lum_radius, every=10, prepare=None, timing=None):
    """Run the flat solver (GPU build's arithmetic) from `fields` for
    `steps` steps; returns the final fields and the luminosity through the
    sphere r = lum_radius every `every` steps: [(step, L), ...].
    prepare(data), if given, changes the uploaded fields on the device before
    the run; its wall time (synchronised) goes to timing["prepare_s"]."""
    import time
    from .solver import FieldSolverEZ, SimData, SimEnvironment
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(fields)
    if prepare is not None:
        torch = _torch()
        torch.cuda.synchronize()
        t0 = time.time()
        prepare(data)
        torch.cuda.synchronize()
        if timing is not None:
            timing["prepare_s"] = time.time() - t0
    s = FieldSolverEZ(data, env, "gpu")
    dt = np.float32(p.dt)
    t = np.float32(0.0)
    hist = [(0, s.luminosity(lum_radius))]
    done = 0
    while done < steps:
        n = min(every, steps - done)
        s.step(float(t), n)
        for _ in range(n):
            t = np.float32(t + dt)
        done += n
        hist.append((done, s.luminosity(lum_radius)))
    out = data.download()
    s.close()
    data.close()
    env.close()
    return out, hist


def settle_step(series, l_ref, tol=0.02):
    """The first step of `series` [(step, value)] from which the value stays
    within tol of l_ref to the end."""
    settled = series[-1][0]
    for step, lum in reversed(series):
        if abs(lum - l_ref) > tol * abs(l_ref):
            break
        settled = step
    return settled


# ------------------------------------------ the configured oblique rotator
# The warm-start configuration: a star of radius 12 cells with light
# cylinder R_LC = 60 cells in a 384^3 box with an absorbing outer layer,
# inclination in [0, 90] degrees, and a network on a 128^3 grid whose
# prediction is trilinearly upsampled to 384^3.  The reference's star
# boundary blends the star over 4 cells (d1 = 4 delta,
# field_solver_EZ.cu:394-528), so the solver needs the star resolved by
# about 12 cells: the same box run at 128^3 (a 4-cell star) gives a spindown
# luminosity 12 times too large, at 192^3 4 times (measured).  The training
# steady states are therefore full-resolution 384^3 runs, averaged over 3^3
# cells onto the network's 128^3 grid of the same box; the network sees the
# vacuum dipole there and predicts the change to the steady state.

ROT_N = 384
ROT_COARSE = 3
ROT_RADIUS = 12.0
ROT_RLC_TRAIN = (40.0, 80.0)
ROT_RLC_TEST = 60.0
ROT_OMEGA_REF = 1.0 / 60.0


def rotator_params(N, inclination_deg, r_lc, pml=None):
    """The oblique rotator on an N^3 box of unit cells centred on the star:
    radius 12 cells, surface field of order 1 (b0 = R^3), light cylinder r_lc
    cells, dipole inclined by inclination_deg to the spin axis, absorbing
    layer pml cells (N/16 by default), dt = 0.4 cells."""
    p = problems.pulsar_params(N=N, guard=3, half_size=N / 2.0, radius=ROT_RADIUS,
                               omega=1.0 / r_lc, b0=ROT_RADIUS ** 3,
                               pml=pml if pml is not None else max(8, N // 16))
    a = math.radians(inclination_deg)
    p.p1, p.p2, p.p3 = math.sin(a), 0.0, math.cos(a)
    return p


def coarse_params(p, coarse=ROT_COARSE):
    """The network's grid of the box of p: N / coarse points whose point m is
    the centre of the fine cells coarse m .. coarse m + coarse - 1."""
    import copy
    pc = copy.deepcopy(p)
    pc.N = [n // coarse for n in p.N]
    pc.lower = [l + 0.5 * (coarse - 1) for l in p.lower]
    pc.pml = [max(1, m // coarse) for m in p.pml]
    return pc


def period_steps(p):
    """Steps per rotation period."""
    return 2 * math.pi / (p.omega * float(np.float32(p.dt)))


def _pool(fine, p, coarse=ROT_COARSE):
    """Mean over coarse^3 cells of the interior of a fine array (with guards),
    returned with the coarse grid's guard cells (zeros)."""
    g = p.guard[0]
    a = fine[g:-g, g:-g, g:-g]
    n = a.shape[0] // coarse
    m = a.reshape(n, coarse, n, coarse, n, coarse).mean(axis=(1, 3, 5))
    out = np.zeros((n + 2 * g,) * 3, dtype=fine.dtype)
    out[g:-g, g:-g, g:-g] = m
    return out


_DIPOLE_BASIS = {}


def dipole_start(p):
    """The vacuum-dipole start of a rotator (pulsar_fields), from a cached
    pair of basis fields: the dipole is linear in its moment (sin a, 0, cos a),
    so each inclination costs one combination instead of a new evaluation
    (which takes seconds at 384^3).  Agrees with pulsar_fields to FP32
    rounding."""
    key = (tuple(p.N), tuple(p.lower), p.b0, p.radius)
    if key not in _DIPOLE_BASIS:
        import copy
        q = copy.deepcopy(p)
        q.p1, q.p2, q.p3 = 1.0, 0.0, 0.0
        bx = problems.pulsar_fields(q, np.float32)[3:6]
        q.p1, q.p3 = 0.0, 1.0
        bz = problems.pulsar_fields(q, np.float32)[3:6]
        _DIPOLE_BASIS.clear()
        _DIPOLE_BASIS[key] = (bx, bz)
    bx, bz = _DIPOLE_BASIS[key]
    zero = np.zeros_like(bx[0])
    b = [(np.float32(p.p1) * bx[c] + np.float32(p.p3) * bz[c]).astype(np.float32)
         for c in range(3)]
    return [zero, zero.copy(), zero.copy()] + b + [zero.copy()]


def rotator_sample(incl, r_lc, periods=2.0, N=ROT_N):
    """One training sample: the N^3 rotator run `periods` of its rotation
    periods from the vacuum dipole; returns the network's input, target and
    mask on its coarse grid (host arrays)."""
    p = rotator_params(N, incl, r_lc)
    pc = coarse_params(p)
    start = dipole_start(p)
    steps = int(round(periods * period_steps(p)))
    steady, _ = star_run(p, start, steps, 0.75 * r_lc, steps)
    start_c = problems.pulsar_fields(pc, np.float32)
    steady_c = [start_c[c] + _pool(steady[c] - start[c], p) for c in range(7)]
    x = features(pc, start_c, incl, ROT_OMEGA_REF)
    t, m = target_and_mask(pc, start_c, steady_c)
    return x, t, m


def rotator_training_set(n, periods=2.0, seed=20261203, N=ROT_N, r_lc_range=ROT_RLC_TRAIN):
    """n samples with seeded inclinations in [0, 90] degrees and R_LC drawn
    from r_lc_range (cells), on the GPU."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    xs, ts, ms, pairs = [], [], [], []
    for _ in range(n):
        incl = float(rng.uniform(0.0, 90.0))
        r_lc = float(rng.uniform(*r_lc_range))
        x, t, m = rotator_sample(incl, r_lc, periods, N)
        xs.append(torch.from_numpy(x[None]).cuda().to(torch.bfloat16))
        ts.append(torch.from_numpy(t[None]).cuda())
        ms.append(torch.from_numpy(m[None]).cuda())
        pairs.append((incl, r_lc))
    return xs, ts, ms, pairs


def train_stream(net, xs, ts, ms, iters, lr=2e-3, batch=2, seed=0, log_every=100):
    """Adam over random mini-batches of the samples (xs, ts, ms on the GPU)."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    losses = []
    for it in range(iters):
        idx = rng.choice(len(xs), size=min(batch, len(xs)), replace=False)
        x = torch.cat([xs[i] for i in idx])
        t = torch.cat([ts[i] for i in idx])
        m = torch.cat([ms[i] for i in idx])
        out = net.forward(x)
        loss, dout = net.loss(out, t, m)
        net.backward(dout)
        net.step(lr * (0.1 ** (it / max(1, iters))))
        if it % log_every == 0 or it == iters - 1:
            losses.append((it, float(loss)))
    check_tc()
    return losses


def upsampled_warm_start(net, p, start, incl):
    """The warm start of the rotator p: the network's prediction on the
    coarse grid, trilinearly upsampled to p's grid on the GPU and added to
    the vacuum dipole outside 1.5 star radii and inside the absorbing layer.
    Returns host arrays."""
    torch = _torch()
    pc = coarse_params(p)
    start_c = problems.pulsar_fields(pc, np.float32)
    x = torch.from_numpy(features(pc, start_c, incl, ROT_OMEGA_REF)[None]).cuda()
    out = net.forward(x.to(torch.bfloat16))  # (1, n, n, n, 16): scaled corrections
    check_tc()
    g = p.guard[0]
    Z, Y, X = (c[g:-g, g:-g, g:-g] for c in problems._xyz(p, np.float32))
    R = np.sqrt(X * X + Y * Y + Z * Z)
    edge = p.size[0] / 2 - p.pml[0] * p.size[0] / p.N[0]
    keep = ((R > STAR_EDGE * p.radius) & (np.abs(X) < edge) & (np.abs(Y) < edge) &
            (np.abs(Z) < edge))
    gc = pc.guard[0]
    Zc, Yc, Xc = (c[gc:-gc, gc:-gc, gc:-gc] for c in problems._xyz(pc, np.float32))
    Rc = np.sqrt(Xc * Xc + Yc * Yc + Zc * Zc)
    scale_c = np.minimum((np.maximum(Rc, p.radius) / p.radius) ** 3, 1e4).astype(np.float32)
    corr = out[0, ..., :7].permute(3, 0, 1, 2) / torch.from_numpy(scale_c).cuda()
    up = torch.nn.functional.interpolate(corr[None], scale_factor=ROT_COARSE, mode="trilinear",
                                         align_corners=False)[0].cpu().numpy()
    warm = [a.copy() for a in start]
    for c in range(7):
        inner = warm[c][g:-g, g:-g, g:-g]
        warm[c][g:-g, g:-g, g:-g] = np.where(keep, inner + up[c], inner)
    return warm


class _DeviceArray:
    """A device buffer of the library seen by torch (zero-copy)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def warm_start_on_device(net, p, data, incl, alpha=1.0, comps=range(7)):
    """Add the network's correction to the fields in `data` (the rotator's
    vacuum dipole, already on the device), in place and on the GPU: the
    prediction on the coarse grid, trilinearly upsampled, scaled back by
    (R / R*)^-3 and added outside STAR_EDGE star radii and inside the
    absorbing layer's inner edge.  The same fields as upsampled_warm_start
    without the host round trip of the full-resolution grid.  alpha scales
    the correction and comps selects the fields it is added to (0-2 E,
    3-5 B, 6 P)."""
    from .config import Grid
    torch = _torch()
    pc = coarse_params(p)
    start_c = problems.pulsar_fields(pc, np.float32)
    x = torch.from_numpy(features(pc, start_c, incl, ROT_OMEGA_REF)[None]).cuda()
    out = net.forward(x.to(torch.bfloat16))  # (1, n, n, n, 16): scaled corrections
    check_tc()

    def coords(q):  # interior coordinates per axis (x, y, z), as problems._xyz has them
        gq = Grid.from_params(q, np.float32)
        g = q.guard[0]
        return [torch.from_numpy(gq.coords(a, np.float64)[g:-g]).cuda() for a in range(3)]

    xc, yc, zc = coords(pc)
    Rc = torch.sqrt(zc[:, None, None] ** 2 + yc[None, :, None] ** 2 + xc[None, None, :] ** 2)
    scale_c = torch.clamp((torch.clamp(Rc, min=p.radius) / p.radius) ** 3, max=1e4).float()
    corr = out[0, ..., :7].permute(3, 0, 1, 2) / scale_c
    up = torch.nn.functional.interpolate(corr[None], scale_factor=ROT_COARSE, mode="trilinear",
                                         align_corners=False)[0]
    xf, yf, zf = coords(p)
    R = torch.sqrt(zf[:, None, None] ** 2 + yf[None, :, None] ** 2 + xf[None, None, :] ** 2)
    edge = p.size[0] / 2 - p.pml[0] * p.size[0] / p.N[0]
    keep = ((R > STAR_EDGE * p.radius) & (zf.abs()[:, None, None] < edge) &
            (yf.abs()[None, :, None] < edge) & (xf.abs()[None, None, :] < edge))
    g = p.guard[0]
    for c in comps:
        f = torch.as_tensor(_DeviceArray(data.dev_ptr(c), data.shape), device="cuda")
        inner = f[g:-g, g:-g, g:-g]
        add = up[c] if alpha == 1.0 else up[c] * alpha
        inner += torch.where(keep, add, torch.zeros_like(add))


def rotator_study(n_train=40, iters=2000, batch=2, train_periods=2.0, N=ROT_N,
                  test_incl=(38.0, 68.0), r_lc=ROT_RLC_TEST, periods=3.0, seed=0,
                  r_lc_train=ROT_RLC_TRAIN):
    """The configured warm-start study.  Train on n_train N^3 runs pooled to
    the network's grid, then for each test inclination run the N^3 rotator
    (R_LC = r_lc) from its vacuum dipole (cold) and from the network's warm
    start for `periods` rotation periods, record the FP64 Poynting
    luminosity through the sphere r = 0.75 R_LC every 1/40 period, and
    compare the wall time until it stays within 2% of the cold run's steady
    value (the mean over its last period): inference (input features, the
    network, the upsampling and the upload) included for the warm start,
    step time measured with CUDA events without the diagnostics."""
    import time
    torch = _torch()
    t0 = time.time()
    xs, ts, ms, pairs = rotator_training_set(n_train, train_periods, N=N, r_lc_range=r_lc_train)
    torch.cuda.synchronize()
    t_gen = time.time() - t0
    net = UNet(seed=seed)
    t1 = time.time()
    losses = train_stream(net, xs, ts, ms, iters, batch=batch)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    del xs, ts, ms
    results = []
    for incl in test_incl:
        p = rotator_params(N, incl, r_lc)
        per = period_steps(p)
        steps = int(round(periods * per))
        every = max(1, int(per // 40))
        lum_r = 0.75 * r_lc
        start = problems.pulsar_fields(p, np.float32)
        step_ms = _step_ms(p, start)
        cold, hist_c = star_run(p, start, steps, lum_r, every)
        tw = {}
        warm_final, hist_w = star_run(
            p, start, steps, lum_r, every, timing=tw,
            prepare=lambda data: warm_start_on_device(net, p, data, incl))
        t_infer = tw["prepare_s"]
        warm0 = upsampled_warm_start(net, p, start, incl)  # the same fields, on the host
        nper = int(round(per / every))
        l_ref = float(np.mean([l for _, l in hist_c[-nper:]]))
        sc, sw = settle_step(hist_c, l_ref), settle_step(hist_w, l_ref)
        wall_c = sc * step_ms / 1e3
        wall_w = t_infer + sw * step_ms / 1e3
        g = p.guard[0]
        sl = (slice(g, -g),) * 3

        def err(f):
            num = sum(float(((f[c] - cold[c])[sl].astype(np.float64) ** 2).sum()) for c in range(6))
            den = sum(float((cold[c][sl].astype(np.float64) ** 2).sum()) for c in range(6))
            return math.sqrt(num / den)
        results.append({
            "inclination": incl, "R_LC": r_lc, "N": N, "L_steady": l_ref,
            "period_steps": per, "steps": steps,
            "settle_step_cold": sc, "settle_step_warm": sw,
            "settle_periods_cold": sc / per, "settle_periods_warm": sw / per,
            "step_ms": step_ms, "seconds_inference": t_infer,
            "wall_to_settle_cold_s": wall_c, "wall_to_settle_warm_s": wall_w,
            "gain": wall_c / max(wall_w, 1e-9),
            "field_error_dipole": err(start), "field_error_warm": err(warm0),
            "L_cold": [round(l, 5) for _, l in hist_c[::4]],
            "L_warm": [round(l, 5) for _, l in hist_w[::4]]})
    return {"train": {"n": n_train, "periods": train_periods, "grid": N,
                      "network_grid": N // ROT_COARSE, "R_LC": list(r_lc_train),
                      "iters": iters, "batch": batch, "loss": losses,
                      "seconds_generate": t_gen, "seconds_train": t_train},
            "test": results}


def _step_ms(p, fields, steps=100):
    """Device milliseconds per step of the flat solver on p (CUDA events)."""
    from .solver import FieldSolverEZ, SimData, SimEnvironment
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(fields)
    s = FieldSolverEZ(data, env, "gpu")
    s.step(0.0, 5)
    s.set_timing(True)
    s.step(0.0, steps)
    ms = s.last_timing()["total_ms"] / steps
    s.close()
    data.close()
    env.close()
    return ms
