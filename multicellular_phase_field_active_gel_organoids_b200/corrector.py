"""Learned coarse-grid corrector: the organoid at half resolution with a small
convolutional network restoring the fine grid's interface dynamics.

The coarse method is the same step (fused path, FP32) on a grid of half the
sites per side (dx = 2, dt 4x the fine one, zone_size (z+1)/2, the same
physical constants).  Every `interval` (10) coarse steps the network takes
each cell's FFT box of the coarse state -- phi, rho and the step's velocity
(vx, vy) -- and returns a correction to phi and rho on that box
(pfag_corrector_gather / pfag_conv3x3 x 5 / pfag_corrector_apply).

Network: five 3x3 convolutions, 4 (padded to 16) -> 32 -> 32 -> 32 -> 32 -> 2
(padded to 16) channels, GELU after the first four, BF16 weights and
activations with FP32 accumulation on the tensor cores (csrc/
pfag_corrector.cu); trained on the GPU by the same kernels (input and weight
gradients, Adam on FP32 master weights).

Training pairs (`make_pairs`): a fine trajectory of a seeded organoid (16-96
cells) from the plain method's step; at each checkpoint t the fine state F_t
is restricted (2 x 2 block mean) to the coarse grid, the coarse method
advances it one interval, and the target is R(F_{t + 4 interval}) minus that
coarse state on each cell's box (the fine method covers the same physical
time in four times as many steps).  Scales: features and targets are
normalised by their standard deviations over the training set.

Fallback (`CorrectedRun`): every `check_every` corrected intervals, a fine-grid
check prolongs the corrected coarse state to the fine grid, advances the
fine method one interval, restricts it and compares per-cell areas with the
corrected coarse interval from the same state; above the error budget the run
continues on the fine grid (the plain fine method is also the judge of the
corrector's error in the tests).

torch provides device memory and data plumbing only; every numerical kernel
of the network and of the step is this library's.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import capi
from .params import OrganoidConfig, jittered_hex_organoid

try:
    import torch
except ImportError:  # pragma: no cover - the corrector needs torch for device buffers
    torch = None

LAYERS = [(16, 32, True), (32, 32, True), (32, 32, True), (32, 32, True), (32, 16, False)]
REAL_IN, REAL_OUT = 4, 2


def _p(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ---------------------------------------------------------------------------
class ConvNet:
    """The corrector network: FP32 master weights, BF16 copies, Adam moments."""

    def __init__(self, seed: int = 0, device: str = "cuda"):
        g = torch.Generator().manual_seed(seed)
        self.W, self.b, self.Wb = [], [], []
        for k, (cin, cout, _) in enumerate(LAYERS):
            fan_in = 9 * (REAL_IN if k == 0 else cin)
            w = torch.randn((cout, 9, cin), generator=g) * math.sqrt(2.0 / fan_in)
            if k == 0:
                w[:, :, REAL_IN:] = 0.0
            if k == len(LAYERS) - 1:
                w *= 0.1
                w[REAL_OUT:] = 0.0
            self.W.append(w.to(device))
            self.b.append(torch.zeros(cout, device=device))
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.t = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self._bufs = {}

    def _buf(self, key, shape, dtype=torch.bfloat16):
        t = self._bufs.get(key)
        if t is None or tuple(t.shape) != tuple(shape):
            t = torch.zeros(shape, dtype=dtype, device="cuda")   # halos stay zero: the kernels never write them
            self._bufs[key] = t
        return t

    def forward(self, x, B, H, W, train=False):
        """x: BF16 [B][H+2][W+2][16] -> output BF16 [B][H+2][W+2][16]
        (channels 0, 1: the scaled corrections).  With train, keeps the
        activations and pre-activations for backward."""
        L = capi.lib()
        a = x
        self.acts, self.pres = [x], []
        for k, (cin, cout, act) in enumerate(LAYERS):
            y = self._buf(("a", k, train), (B, H + 2, W + 2, cout))
            pre = self._buf(("p", k), (B, H + 2, W + 2, cout)) if (train and act) else None
            capi.check(L.pfag_conv3x3(_p(a), _p(self.Wb[k]), _p(self.b[k]), _p(y), _p(pre) if pre is not None else None,
                                      B, H, W, cin, cout, 1 if act else 0, _p(self.err), _stream()))
            a = y
            if train:
                self.acts.append(y)
                self.pres.append(pre)
        return a

    def train_step(self, x, target, B, H, W, lr=1e-3):
        """One Adam step on a batch; returns the mean squared error (a device scalar)."""
        L = capi.lib()
        out = self.forward(x, B, H, W, train=True)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        dout = self._buf("dout", out.shape)
        capi.check(L.pfag_conv_mse(_p(out), _p(target), _p(dout), _p(loss), B, H, W, 16, REAL_OUT,
                                   1.0 / (B * H * W * REAL_OUT), _stream()))
        dz = dout
        grads = []
        for k in range(len(LAYERS) - 1, -1, -1):
            cin, cout, act = LAYERS[k]
            dw = torch.zeros_like(self.W[k])
            db = torch.zeros_like(self.b[k])
            capi.check(L.pfag_conv3x3_wgrad(_p(self.acts[k]), _p(dz), _p(dw), _p(db), B, H, W, cin, cout,
                                            _p(self.err), _stream()))
            grads.append((k, dw, db))
            if k == 0:
                break
            wt = self._buf(("wt", k), (cin, 9, cout))
            capi.check(L.pfag_conv_flip(_p(self.Wb[k]), _p(wt), cin, cout, _stream()))
            da = self._buf(("da", k), (B, H + 2, W + 2, cin))
            zero_b = self._buf(("zb", cin), (cin,), torch.float32)
            capi.check(L.pfag_conv3x3(_p(dz), _p(wt), _p(zero_b), _p(da), None, B, H, W, cout, cin, 0, _p(self.err),
                                      _stream()))
            pcin, pcout, pact = LAYERS[k - 1]
            dz = self._buf(("dz", k - 1), (B, H + 2, W + 2, pcout))
            capi.check(L.pfag_conv_act_bwd(_p(da), _p(self.pres[k - 1]), _p(dz), B, H, W, pcout, 1 if pact else 0,
                                           _stream()))
        self.t += 1
        for k, dw, db in grads:
            capi.check(L.pfag_adam(_p(self.W[k]), _p(dw), _p(self.mW[k]), _p(self.vW[k]), _p(self.Wb[k]), None,
                                   self.W[k].numel(), lr, 0.9, 0.999, 1e-8, self.t, _stream()))
            capi.check(L.pfag_adam(_p(self.b[k]), _p(db), _p(self.mb[k]), _p(self.vb[k]), None, None,
                                   self.b[k].numel(), lr, 0.9, 0.999, 1e-8, self.t, _stream()))
        return loss / (B * H * W * REAL_OUT)

    def check_err(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a convolution kernel's bounded wait for its tensor-core work ran out")

    def state_dict(self):
        return {"W": [w.cpu() for w in self.W], "b": [b.cpu() for b in self.b]}


# ---------------------------------------------------------------------------
def coarse_config(fine: OrganoidConfig) -> OrganoidConfig:
    """The same organoid on the coarse grid: half the sites per side, dx = 2,
    dt 4x, zone (z+1)/2, physical constants unchanged."""
    over = dict(fine.overrides)
    over.update({"dx": 2.0, "dt": 4e-3})
    return OrganoidConfig(fine.name + "_coarse", fine.N // 2, fine.centres / 2.0, fine.radius,
                          (fine.zone_size + 1) // 2, fine.seed, fine.steps, overrides=over)


def fine_config(ncells: int, seed: int, N: int = 1024, zone_size: int = 129) -> OrganoidConfig:
    """A seeded fine organoid of the cfg1 family (R = 24, jittered hexagonal
    lattice), its lattice clipped so that every zone stays on the grid; the
    cell count is capped at what that circle holds."""
    clip = min(220.0, N / 2.0 - zone_size - 4.0)
    for n in range(ncells, 0, -1):
        try:
            return jittered_hex_organoid(name=f"fine{seed}", N=N, ncells=n, zone_size=zone_size, seed=seed,
                                         clip=clip)
        except ValueError:
            continue
    raise ValueError(f"no lattice point within {clip} of the centre")


def _field(sim, name):
    ptr, n = sim.device_field(name)
    return ptr, n


def _to_torch(sim, name, shape):
    """Copy a context's device array into a new torch tensor (device to device)."""
    ptr, n = _field(sim, name)
    dt = torch.float32 if sim.precision == 32 else torch.float64
    out = torch.empty(shape, dtype=dt, device="cuda")
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    sim.sync()
    assert rt.cudaMemcpy(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ptr), out.numel() * out.element_size(), 3) == 0
    return out


def state_tensors(sim):
    n, N = sim.ncells, sim.N
    return (_to_torch(sim, "phi", (n, N, N)), _to_torch(sim, "rho", (n, N, N)), _to_torch(sim, "lum", (N, N)),
            _to_torch(sim, "ECM", (N, N)))


def restrict(t):
    """2 x 2 block mean of the last two axes."""
    s = t.shape
    return t.reshape(*s[:-2], s[-2] // 2, 2, s[-1] // 2, 2).mean(dim=(-3, -1))


def prolong(t):
    """Each coarse value onto its 2 x 2 fine block."""
    return t.repeat_interleave(2, dim=-2).repeat_interleave(2, dim=-1)


def upload_tensors(sim, fields):
    fields = [f.contiguous() for f in fields]
    torch.cuda.synchronize()
    sim.upload_device(*[f.data_ptr() for f in fields])


def boxes_of(t, xc, yc, z, M):
    """[Ntot][N][N] -> each cell's FFT box [Ntot][M][M] ([xc-z+1, xc+z-2])."""
    out = torch.empty((t.shape[0], M, M), dtype=t.dtype, device=t.device)
    for n in range(t.shape[0]):
        bi, bj = int(xc[n]) - z + 1, int(yc[n]) - z + 1
        out[n] = t[n, bi:bi + M, bj:bj + M]
    return out


class Scales:
    def __init__(self, s_v=1.0, t_phi=1.0, t_rho=1.0):
        self.s_v, self.t_phi, self.t_rho = float(s_v), float(t_phi), float(t_rho)

    def as_dict(self):
        return {"s_v": self.s_v, "t_phi": self.t_phi, "t_rho": self.t_rho}


def coarse_interval(sim, it0: int, interval: int):
    """`interval` coarse steps, the last with the velocity captured."""
    if interval > 1:
        sim.step(it0, interval - 1)
    sim.set_debug(1)
    sim.step(it0 + interval - 1, 1)
    sim.set_debug(0)


def make_pairs(seeds, ncells_range=(16, 96), checkpoints=4, interval=10, N=1024, zone_size=129,
               warm=40, relax_cap=100000, log=None):
    """Training pairs from fine trajectories: per seed, `checkpoints` fine
    checkpoints `4 interval` fine steps apart (after `warm` steps); returns
    per-pair lists of (features [Ntot][M+2][M+2][16] BF16 with unit scales,
    target [Ntot][M][M][2] FP32 unscaled)."""
    feats, targs = [], []
    for seed in seeds:
        rng = np.random.default_rng(10_000 + seed)
        ncells = int(rng.integers(ncells_range[0], ncells_range[1] + 1))
        fcfg = fine_config(ncells, seed, N, zone_size)
        ccfg = coarse_config(fcfg)
        with capi.Simulation(fcfg.params(), 32, capi.PATH_FUSED) as fs, \
                capi.Simulation(ccfg.params(), 32, capi.PATH_FUSED) as cs:
            fs.set_relax_cap(relax_cap)
            cs.set_relax_cap(relax_cap)
            fs.upload(*fcfg.initial_state(np.float32))
            fs.step(0, warm)
            it = warm
            for _ in range(checkpoints):
                F = state_tensors(fs)
                upload_tensors(cs, [restrict(f) for f in F])
                coarse_interval(cs, 0, interval)
                fs.step(it, 4 * interval)
                it += 4 * interval
                x0 = torch.zeros((cs.ncells, cs.M + 2, cs.M + 2, 16), dtype=torch.bfloat16, device="cuda")
                capi.check(capi.lib().pfag_corrector_gather(cs.h, ctypes.c_void_p(x0.data_ptr()), 1.0, 1.0, 1.0))
                C = state_tensors(cs)
                F2 = state_tensors(fs)
                xc, yc = cs.centres()
                z, M = int(ccfg.zone_size), cs.M
                dphi = boxes_of(restrict(F2[0]) - C[0], xc, yc, z, M)
                drho = boxes_of(restrict(F2[1]) - C[1], xc, yc, z, M)
                feats.append(x0)
                targs.append(torch.stack([dphi, drho], dim=-1).float().contiguous())
            if log:
                log(f"seed {seed}: {ncells} cells, {checkpoints} pairs")
    return feats, targs


def fit_scales(feats, targs) -> Scales:
    v = torch.cat([f[..., 2:4].float().reshape(-1) for f in feats])
    tp = torch.cat([t[..., 0].reshape(-1) for t in targs])
    tr = torch.cat([t[..., 1].reshape(-1) for t in targs])
    sd = lambda a: float(a.std().item()) or 1.0
    return Scales(1.0 / max(sd(v), 1e-12), 1.0 / max(sd(tp), 1e-12), 1.0 / max(sd(tr), 1e-12))


def scaled(feats, targs, sc: Scales):
    X = torch.cat(feats)
    X = X.float()
    X[..., 2:4] *= sc.s_v
    X = X.to(torch.bfloat16)
    T = torch.cat(targs).clone()
    T[..., 0] *= sc.t_phi
    T[..., 1] *= sc.t_rho
    return X, T.contiguous()


def train(net: ConvNet, X, T, iters=400, batch=16, lr=1e-3, seed=0, log=None):
    """Adam on random minibatches of boxes; returns the loss history (host floats)."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    n, Hp, Wp, _ = X.shape
    H, W = Hp - 2, Wp - 2
    hist = []
    for k in range(iters):
        idx = torch.randint(0, n, (batch,), generator=g, device="cuda")
        xb = X[idx].contiguous()
        tb = T[idx].contiguous()
        loss = net.train_step(xb, tb, batch, H, W, lr=lr)
        if k % 20 == 0 or k == iters - 1:
            hist.append(float(loss.item()))
            if log:
                log(f"iter {k}: mse {hist[-1]:.4g}")
    net.check_err()
    return hist


def predict(net: ConvNet, X, batch=32):
    """Network output (scaled corrections, channels 0 and 1) for every box."""
    n, Hp, Wp, _ = X.shape
    outs = []
    for s in range(0, n, batch):
        xb = X[s:s + batch].contiguous()
        o = net.forward(xb, xb.shape[0], Hp - 2, Wp - 2)
        outs.append(o[:, 1:-1, 1:-1, :2].float().clone())
    net.check_err()
    return torch.cat(outs)


class CorrectedRun:
    """A coarse run with the corrector every `interval` steps and the fine
    fallback (module docstring)."""

    def __init__(self, net: ConvNet, sc: Scales, fine: OrganoidConfig, interval=10, check_every=0, budget=0.01,
                 relax_cap=100000):
        self.net, self.sc, self.interval = net, sc, interval
        self.check_every, self.budget = check_every, budget
        self.fcfg, self.ccfg = fine, coarse_config(fine)
        self.cs = capi.Simulation(self.ccfg.params(), 32, capi.PATH_FUSED)
        self.cs.set_relax_cap(relax_cap)
        self.fs = None
        self.relax_cap = relax_cap
        self.on_fine = False
        self.corrections = 0
        self.fallbacks = 0
        self.x0 = torch.zeros((self.cs.ncells, self.cs.M + 2, self.cs.M + 2, 16), dtype=torch.bfloat16, device="cuda")

    def start_from_fine(self, fine_state):
        upload_tensors(self.cs, [restrict(f) for f in fine_state])

    def correct(self):
        L = capi.lib()
        capi.check(L.pfag_corrector_gather(self.cs.h, ctypes.c_void_p(self.x0.data_ptr()), 1.0, 1.0, self.sc.s_v))
        torch.cuda.synchronize()
        out = self.net.forward(self.x0, self.cs.ncells, self.cs.M, self.cs.M)
        torch.cuda.synchronize()
        capi.check(L.pfag_corrector_apply(self.cs.h, ctypes.c_void_p(out.data_ptr()), 1.0 / self.sc.t_phi,
                                          1.0 / self.sc.t_rho))
        self.cs.sync()
        self.corrections += 1

    def _fine_sim(self):
        if self.fs is None:
            self.fs = capi.Simulation(self.fcfg.params(), 32, capi.PATH_FUSED)
            self.fs.set_relax_cap(self.relax_cap)
        return self.fs

    def fine_check(self, it: int) -> bool:
        """True when the corrected coarse interval stays within the budget of
        the fine method over the same interval from the same state."""
        start = state_tensors(self.cs)
        fs = self._fine_sim()
        upload_tensors(fs, [prolong(f) for f in start])
        fs.step(it * 4, 4 * self.interval)
        ref_s = restrict(state_tensors(fs)[0]).sum(dim=(1, 2)) * (2.0 * 2.0)
        coarse_interval(self.cs, it, self.interval)
        self.correct()
        got_s = state_tensors(self.cs)[0].sum(dim=(1, 2)) * (2.0 * 2.0)
        rel = float(((got_s - ref_s).abs() / ref_s.abs()).max().item())
        self.last_check = rel
        if rel > self.budget:
            self.on_fine = True
            self.fallbacks += 1
        return rel <= self.budget

    def run(self, nintervals: int, it0: int = 0, corrected: bool = True):
        it = it0
        for k in range(nintervals):
            if self.on_fine:
                self.fs.step(4 * it, 4 * self.interval)
            elif corrected and self.check_every and (k + 1) % self.check_every == 0:
                self.fine_check(it)
            else:
                coarse_interval(self.cs, it, self.interval)
                if corrected:
                    self.correct()
            it += self.interval
        return it

    def state_on_coarse(self):
        if self.on_fine:
            return [restrict(f) for f in state_tensors(self.fs)]
        return list(state_tensors(self.cs))

    def close(self):
        self.cs.close()
        if self.fs is not None:
            self.fs.close()


def shape_errors(coarse_phi, fine_phi_restricted, dx=2.0):
    """Per-cell relative errors of area and perimeter of a coarse state against
    the restricted fine state (both [Ntot][n][n] on the coarse grid)."""
    def perim(p):
        gi = 0.5 * (torch.roll(p, -1, 1) - torch.roll(p, 1, 1))
        gj = 0.5 * (torch.roll(p, -1, 2) - torch.roll(p, 1, 2))
        return torch.sqrt(gi * gi + gj * gj).sum(dim=(1, 2)) * dx
    a, b = coarse_phi.double(), fine_phi_restricted.double()
    area = ((a.sum(dim=(1, 2)) - b.sum(dim=(1, 2))).abs() / b.sum(dim=(1, 2)).abs()).max().item()
    pa, pb = perim(a), perim(b)
    per = ((pa - pb).abs() / pb.abs()).max().item()
    return float(area), float(per)
