"""Learned warm start for the rotating-star problem: a small 3D convolutional
network (a two-level U-Net) that maps a star's vacuum dipole to the
magnetosphere it settles into, so that a run can start near its steady
state instead of from the dipole.  No counterpart in the reference (its
drivers always start from the vacuum dipole, ``src/user_pulsar3d_EZ.hpp``).

Every arithmetic step of training and inference runs on the library's
kernels (include/coffee_surrogate.h): BF16 tensor-core convolutions with
FP32 accumulation for the forward pass and both gradients, and the
pooling, activation, loss and Adam kernels.  torch provides the device
memory only.  The training set is made by the flat solver itself: one
rotating-star run per inclination.

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
    """True where the tcgen05 convolution is the faster one: inputs of 16, 32
    or 64 channels (one TMA box of 16, 32 or 64 channels per tap); the results
    are those of the mma.sync kernel."""
    return c in (16, 32, 64) and k in (16, 32, 48, 64)


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
        conv_backward_weight(dzb, x_in, L.gw, self._ws)

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

def star_params(N=64, inclination_deg=30.0, omega=0.15):
    """The rotating-star configuration of the warm-start study: an inclined
    dipole star of radius 1.5 turning at omega (0.15: light cylinder 6.7) in a
    box of half size 12 with an absorbing layer."""
    p = problems.pulsar_params(N=N, guard=3, half_size=12.0, radius=1.5, omega=omega, pml=8)
    a = math.radians(inclination_deg)
    p.p1, p.p2, p.p3 = math.sin(a), 0.0, math.cos(a)
    return p


def _coords(p):
    Z, Y, X = problems._xyz(p, np.float32)
    return X, Y, Z


def features(p, fields, inclination_deg):
    """Input channels (D, H, W, 16) of the interior: B r^3 / R^3 of the
    dipole state, x, y, z / half size, the star mask, sin and cos of the
    inclination, the spin omega / 0.15, zeros."""
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
    out[..., 9] = p.omega / 0.15
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


def apply_prediction(p, start, pred):
    """The warm-start fields: start + pred / scale outside 1.5 radii (the
    star's own boundary condition sets the fields inside)."""
    g = p.guard[0]
    X, Y, Z = _coords(p)
    R = np.sqrt(X * X + Y * Y + Z * Z)
    scale = np.minimum((np.maximum(R, p.radius) / p.radius) ** 3, 1e4).astype(np.float32)
    keep = R > STAR_EDGE * p.radius
    out = [a.copy() for a in start]
    for c in range(7):
        full = np.zeros_like(start[c])
        full[g:-g, g:-g, g:-g] = pred[..., c]
        out[c] = np.where(keep, start[c] + full / scale, start[c]).astype(start[c].dtype)
    return out


# --------------------------------------------------------- warm-start study

def star_run(p, fields, steps, lum_radius, every=10):
    """Run the flat solver (GPU build's arithmetic) from `fields` for
    `steps` steps; returns the final fields and the luminosity through the
    sphere r = lum_radius every `every` steps: [(step, L), ...]."""
    from .solver import FieldSolverEZ, SimData, SimEnvironment
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(fields)
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


def rotation_mean(hist, period):
    """The luminosity averaged over the last rotation period at every
    recorded step that has a full period behind it.  The flux of an oblique
    rotator through a sphere is steady only on average: on a Cartesian grid
    it is modulated at the rotation period."""
    steps = np.array([s for s, _ in hist], float)
    lums = np.array([l for _, l in hist], float)
    out = []
    for s in steps:
        if s < period:
            continue
        sel = (steps > s - period) & (steps <= s)
        out.append((int(s), float(lums[sel].mean())))
    return out


def settle_step(series, l_ref, tol=0.02):
    """The first step of `series` [(step, value)] from which the value stays
    within tol of l_ref to the end."""
    settled = series[-1][0]
    for step, lum in reversed(series):
        if abs(lum - l_ref) > tol * abs(l_ref):
            break
        settled = step
    return settled


def _batch(samples):
    torch = _torch()
    xs, ts, ms = [], [], []
    for p, incl, start, steady in samples:
        xs.append(features(p, start, incl))
        t, m = target_and_mask(p, start, steady)
        ts.append(t)
        ms.append(m)
    x = torch.from_numpy(np.stack(xs)).cuda().to(torch.bfloat16)
    return x, torch.from_numpy(np.stack(ts)).cuda(), torch.from_numpy(np.stack(ms)).cuda()


def train(net, samples, iters, lr=2e-3, log_every=50):
    """Full-batch Adam on the library's kernels over samples
    [(params, inclination, start fields, target fields)]; returns the loss
    history."""
    x, tgt, mask = _batch(samples)
    losses = []
    for it in range(iters):
        out = net.forward(x)
        loss, dout = net.loss(out, tgt, mask)
        net.backward(dout)
        rate = lr * (0.1 ** (it / max(1, iters)))
        net.step(rate)
        if it % log_every == 0 or it == iters - 1:
            losses.append((it, float(loss)))
    check_tc()
    return losses


def predict(net, p, start, incl):
    torch = _torch()
    x = torch.from_numpy(features(p, start, incl)[None]).cuda().to(torch.bfloat16)
    out = net.forward(x)
    check_tc()
    return apply_prediction(p, start, out[0].cpu().numpy())


def warm_start_study(N=64, train_set=((0, 0.15), (15, 0.15), (30, 0.15), (45, 0.15), (60, 0.15),
                                   (75, 0.15), (90, 0.15)),
                     test_set=((38, 0.15), (68, 0.15)), periods=4.0, iters=2000, lum_radius=4.5,
                     seed=0):
    """Train the network on rotating-star runs at the (inclination in
    degrees, spin) pairs of `train_set`, each run `periods` rotation periods from
    its dipole; then for every held-out pair of `test_set` run the plain cold
    start and the warm start for as long and compare when their spindown
    luminosity (the mean over the last rotation period) settles within 2% of
    the cold run's final value, and how far each start is from the cold
    run's final fields."""
    import time

    def period_steps(p):
        return int(round(2 * math.pi / (p.omega * float(np.float32(p.dt)))))
    t0 = time.time()
    samples = []
    for incl, om in train_set:
        p = star_params(N, incl, om)
        period = period_steps(p)
        start = problems.pulsar_fields(p, np.float32)
        steady, _ = star_run(p, start, int(round(periods * period)), lum_radius,
                             max(1, period // 20))
        samples.append((p, float(incl), start, steady))
    t_gen = time.time() - t0
    net = UNet(seed=seed)
    t1 = time.time()
    losses = train(net, samples, iters)
    _torch().cuda.synchronize()
    t_train = time.time() - t1
    results = []
    for incl, om in test_set:
        p = star_params(N, incl, om)
        period = period_steps(p)
        steps = int(round(periods * period))
        every = max(1, period // 20)
        start = problems.pulsar_fields(p, np.float32)
        cold, hist_c = star_run(p, start, steps, lum_radius, every)
        t2 = time.time()
        warm0 = predict(net, p, start, incl)
        t_infer = time.time() - t2
        _, hist_w = star_run(p, warm0, steps, lum_radius, every)
        mean_c, mean_w = rotation_mean(hist_c, period), rotation_mean(hist_w, period)
        l_ref = mean_c[-1][1]
        g = p.guard[0]
        sl = (slice(g, -g),) * 3
        _, mask = target_and_mask(p, start, cold)

        def err(f):
            num = sum(float(((f[c] - cold[c])[sl] ** 2 * mask).sum()) for c in range(6))
            den = sum(float((cold[c][sl] ** 2 * mask).sum()) for c in range(6))
            return math.sqrt(num / den)
        sc, sw = settle_step(mean_c, l_ref), settle_step(mean_w, l_ref)
        # the instantaneous luminosity (steady for an aligned rotator; an
        # oblique one's is modulated at the rotation period)
        ic, iw = settle_step(hist_c, l_ref), settle_step(hist_w, l_ref)
        results.append({"inclination": incl, "omega": om, "L_steady": l_ref,
                        "period_steps": period, "steps": steps,
                        "settle_step_cold": sc, "settle_step_warm": sw, "gain": sc / max(sw, 1),
                        "settle_step_cold_instantaneous": ic,
                        "settle_step_warm_instantaneous": iw,
                        "gain_instantaneous": ic / max(iw, 1),
                        "L_cold_history": [round(l, 6) for _, l in hist_c[:40]],
                        "L_warm_history": [round(l, 6) for _, l in hist_w[:40]],
                        "L_first_period_cold": mean_c[0][1], "L_first_period_warm": mean_w[0][1],
                        "field_error_dipole": err(start), "field_error_warm": err(warm0),
                        "seconds_inference": t_infer})
    return {"N": N, "periods": periods, "train": [list(x) for x in train_set], "test": results,
            "loss": losses, "seconds_generate": t_gen, "seconds_train": t_train}
