"""Seeded synthetic PIV frame pairs with analytic ground-truth displacement.

The reference ships one 512x512 pair without ground truth and names no public dataset,
so these stand in for its workloads: Gaussian particle images (peak A*exp(-8 r^2/d^2),
d the e^-2 diameter, A ~ U(128, 255)) rendered at pixel centres, frame 2 holding the same
particles moved by an analytic field evaluated at each particle (x' = x + u(x)), additive
Gaussian noise, rounded and clipped to uint8.  Pixel (i, j) has its centre at (x=j, y=i);
U is the +x (column) displacement and V the +y (row) displacement, the reference's
convention.
"""
from __future__ import annotations

import numpy as np

LAMB_OSEEN_PEAK = None


def _lamb_oseen_peak():
    global LAMB_OSEEN_PEAK
    if LAMB_OSEEN_PEAK is None:
        s = np.linspace(0.5, 3.0, 200001)
        LAMB_OSEEN_PEAK = float(np.max((1.0 / s) * (1.0 - np.exp(-s * s))))
    return LAMB_OSEEN_PEAK


class Flow:
    """An analytic displacement field u(x, y), v(x, y) in pixels."""

    def __init__(self, kind, H, W, max_disp=4.0, rng=None, core_radius=60.0, modes=32, kmin=1, kmax=8):
        self.kind, self.H, self.W, self.max_disp = kind, H, W, float(max_disp)
        self.rc = float(core_radius)
        if kind == "fourier":
            rng = rng or np.random.default_rng(0)
            L = float(max(H, W))
            kk = []
            while len(kk) < modes:
                k = rng.integers(-kmax, kmax + 1, size=2)
                n = np.hypot(*k)
                if kmin <= n <= kmax:
                    kk.append(k)
            self.k = np.array(kk, dtype=np.float64) * (2 * np.pi / L)
            self.phi = rng.uniform(0, 2 * np.pi, modes)
            self.amp = rng.normal(0, 1, modes) / np.maximum(np.hypot(self.k[:, 0], self.k[:, 1]), 1e-9)
            u, v = self._fourier_grid()
            self.scale = self.max_disp / max(np.max(np.hypot(u, v)), 1e-12)
        elif kind not in ("poiseuille", "lamb_oseen", "uniform"):
            raise ValueError(kind)

    def _fourier_raw(self, x, y):
        u = np.zeros_like(x)
        v = np.zeros_like(x)
        for (kx, ky), a, p in zip(self.k, self.amp, self.phi):
            c = a * np.cos(kx * x + ky * y + p)
            u += c * ky      # d psi / d y
            v -= c * kx      # -d psi / d x
        return u, v

    def _fourier_grid(self):
        """The unscaled field on the pixel grid, separably: cos(kx x + ky y + p) =
        cos(kx x) cos(ky y + p) - sin(kx x) sin(ky y + p), one matrix product per component."""
        x = np.arange(self.W, dtype=np.float64)
        y = np.arange(self.H, dtype=np.float64)
        ax = np.outer(self.k[:, 0], x)                      # modes x W
        by = np.outer(self.k[:, 1], y) + self.phi[:, None]  # modes x H
        L = np.concatenate([np.cos(by), np.sin(by)]).T      # H x 2M
        R = np.concatenate([np.cos(ax), -np.sin(ax)])       # 2M x W
        wu = np.concatenate([self.amp * self.k[:, 1]] * 2)
        wv = np.concatenate([-self.amp * self.k[:, 0]] * 2)
        return (L * wu) @ R, (L * wv) @ R

    def __call__(self, x, y):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        if self.kind == "uniform":
            return np.full_like(x, self.max_disp), np.zeros_like(x)
        if self.kind == "poiseuille":
            eta = 2.0 * y / self.H - 1.0
            return self.max_disp * (1.0 - eta * eta), np.zeros_like(x)
        if self.kind == "lamb_oseen":
            dx, dy = x - self.W / 2.0, y - self.H / 2.0
            r = np.maximum(np.hypot(dx, dy), 1e-9)
            ut = self.max_disp * (self.rc / r) * (1.0 - np.exp(-(r / self.rc) ** 2)) / _lamb_oseen_peak()
            return -ut * dy / r, ut * dx / r
        u, v = self._fourier_raw(x, y)
        return u * self.scale, v * self.scale

    def ground_truth(self):
        if self.kind == "fourier":
            u, v = self._fourier_grid()
            return (u * self.scale).astype(np.float32), (v * self.scale).astype(np.float32)
        yy, xx = np.mgrid[0:self.H, 0:self.W].astype(np.float64)
        u, v = self(xx, yy)
        return u.astype(np.float32), v.astype(np.float32)


def _render(H, W, px, py, amp, diam, radius):
    off = 2 * radius + 2
    img = np.zeros((H + 2 * off, W + 2 * off), np.float64)
    ix = np.floor(px).astype(np.int64)
    iy = np.floor(py).astype(np.int64)
    keep = (ix >= -radius - 1) & (ix <= W + radius) & (iy >= -radius - 1) & (iy <= H + radius)
    px, py, amp, diam, ix, iy = px[keep], py[keep], amp[keep], diam[keep], ix[keep], iy[keep]
    inv = -8.0 / (diam * diam)
    Wp = W + 2 * off
    o = np.arange(-radius, radius + 2)
    jx = ix[:, None, None] + o[None, None, :]
    jy = iy[:, None, None] + o[None, :, None]
    val = amp[:, None, None] * np.exp(inv[:, None, None] * ((jx - px[:, None, None]) ** 2 +
                                                            (jy - py[:, None, None]) ** 2))
    img += np.bincount(((jy + off) * Wp + jx + off).ravel(), weights=val.ravel(), minlength=img.size).reshape(img.shape)
    return img[off:off + H, off:off + W]


def piv_pair(H, W, flow="poiseuille", seed=0, density=0.05, diameter=2.5, noise=2.0, max_disp=4.0, **flow_kw):
    """Returns (frame1 u8, frame2 u8, U_gt f32, V_gt f32).

    diameter: a number or a (lo, hi) range drawn uniformly per particle."""
    rng = np.random.default_rng(seed)
    fl = flow if isinstance(flow, Flow) else Flow(flow, H, W, max_disp, rng=rng, **flow_kw)
    dmax = float(np.max(diameter))
    pad = int(np.ceil(fl.max_disp + 3 * dmax)) + 2
    n = int(round(density * (H + 2 * pad) * (W + 2 * pad)))
    px = rng.uniform(-pad, W + pad, n)
    py = rng.uniform(-pad, H + pad, n)
    amp = rng.uniform(128, 255, n)
    if np.ndim(diameter):
        diam = rng.uniform(diameter[0], diameter[1], n)
    else:
        diam = np.full(n, float(diameter))
    u, v = fl(px, py)
    radius = int(np.ceil(dmax)) + 1
    f1 = _render(H, W, px, py, amp, diam, radius)
    f2 = _render(H, W, px + u, py + v, amp, diam, radius)
    f1 = f1 + rng.normal(0, noise, f1.shape) if noise > 0 else f1
    f2 = f2 + rng.normal(0, noise, f2.shape) if noise > 0 else f2
    f1 = np.clip(np.round(f1), 0, 255).astype(np.uint8)
    f2 = np.clip(np.round(f2), 0, 255).astype(np.uint8)
    U, V = fl.ground_truth()
    return f1, f2, U, V


def epe(U, V, Ug, Vg, crop=0):
    """Mean endpoint error; `crop` pixels are dropped on every side."""
    if crop:
        sl = (slice(crop, -crop), slice(crop, -crop))
        U, V, Ug, Vg = U[sl], V[sl], Ug[sl], Vg[sl]
    return float(np.mean(np.hypot(np.asarray(U, np.float64) - Ug, np.asarray(V, np.float64) - Vg)))


# Workloads: the five reference calibrations with their synthetic inputs.
def config_pair(cfg, seed=0, size=None):
    """Frame pair of one named workload: 'hs256', 'lk512', 'fbls1024' (sizes overridable)."""
    if cfg == "hs256":
        n = size or 256
        return piv_pair(n, n, "poiseuille", seed, density=0.05, diameter=2.5, noise=2.0)
    if cfg == "lk512":
        n = size or 512
        return piv_pair(n, n, "lamb_oseen", seed, density=0.08, diameter=2.5, noise=2.0)
    if cfg == "fbls1024":
        n = size or 1024
        return piv_pair(n, n, "fourier", seed, density=0.05, diameter=(2.0, 3.0), noise=2.0)
    raise ValueError(cfg)
