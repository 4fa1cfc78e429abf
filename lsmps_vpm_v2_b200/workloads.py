"""Seeded synthetic vorticity fields with the shapes the velocity step is
benchmarked on. No dataset is involved: every field is generated here.

Each generator returns a dict with positions, particle size ``s``, vorticity,
the active mark and the FMM source strength computed the way the reference's
velocity manager packs it:

* 2D: ``q = -omega * s**2 / (2 pi)``
  (src/velocity_calculation/velocity_calc.cpp:477)
* 3D: ``alpha = omega * s**3 / (4 pi)`` per component
  (src/velocity_calculation/velocity_calc.cpp:2434-2436)
"""
from __future__ import annotations

import math

import numpy as np


def _q2d(omega, s):
    return -omega * np.power(s, 2.0) / (2 * math.pi)


def _lattice(x0, x1, y0, y1, h):
    """Cell-centred lattice covering [x0,x1) x [y0,y1) with spacing h."""
    nx = int(math.floor((x1 - x0) / h + 1e-9))
    ny = int(math.floor((y1 - y0) / h + 1e-9))
    xs = x0 + (np.arange(nx) + 0.5) * h
    ys = y0 + (np.arange(ny) + 0.5) * h
    gx, gy = np.meshgrid(xs, ys, indexing="xy")
    return gx.ravel(), gy.ravel()


def lamb_oseen_2d(n_side: int = 256, extent: float = 10.0, gamma: float = 1.0, sigma: float = 1.0,
                  jitter: float = 0.1, noise: float = 1e-3, seed: int = 0):
    """Lamb-Oseen vortex on a jittered n_side x n_side lattice over
    [-extent, extent]^2: omega = Gamma/(pi sigma^2) exp(-r^2/sigma^2) plus
    Gaussian noise. n_side=256 is the 65,536-particle case (h = 0.078125)."""
    rng = np.random.default_rng(seed)
    h = 2 * extent / n_side
    x, y = _lattice(-extent, extent, -extent, extent, h)
    x = x + rng.uniform(-jitter * h, jitter * h, x.size)
    y = y + rng.uniform(-jitter * h, jitter * h, y.size)
    r2 = x * x + y * y
    omega = gamma / (math.pi * sigma ** 2) * np.exp(-r2 / sigma ** 2) + rng.normal(0.0, noise, x.size)
    s = np.full(x.size, h)
    return dict(x=x, y=y, s=s, omega=omega, active=np.ones(x.size, np.uint8), q=_q2d(omega, s),
                name=f"lamb_oseen_{x.size}")


def boundary_layer_2d(scale: float = 0.66, extent: float = 10.0, u_inf: float = 1.0, delta: float = 0.02,
                      perturb: float = 0.2, seed: int = 1):
    """Multi-resolution boundary-layer field over a flat plate x in [-1,1], y=0.

    Spacings (0.005, 0.02, 0.04) * scale: fine inside |y|<0.1 over the plate,
    mid inside |y|<1, coarse elsewhere; cell-centred lattices, each zone
    excluding the finer zone it surrounds. scale=0.66 gives ~780k particles
    (the literal spacings give ~340k). omega = -(U/delta) exp(-|y|/delta)
    times a lognormal(0, perturb) factor."""
    rng = np.random.default_rng(seed)
    hf, hm, hc = 0.005 * scale, 0.02 * scale, 0.04 * scale
    fx, fy = _lattice(-1.0, 1.0, -0.1, 0.1, hf)
    mx, my = _lattice(-extent, extent, -1.0, 1.0, hm)
    keep = ~((np.abs(mx) < 1.0) & (np.abs(my) < 0.1))
    mx, my = mx[keep], my[keep]
    cx, cy = _lattice(-extent, extent, -extent, extent, hc)
    keep = np.abs(cy) >= 1.0
    cx, cy = cx[keep], cy[keep]
    x = np.concatenate([fx, mx, cx])
    y = np.concatenate([fy, my, cy])
    s = np.concatenate([np.full(fx.size, hf), np.full(mx.size, hm), np.full(cx.size, hc)])
    omega = -(u_inf / delta) * np.exp(-np.abs(y) / delta) * rng.lognormal(0.0, perturb, x.size)
    return dict(x=x, y=y, s=s, omega=omega, active=np.ones(x.size, np.uint8), q=_q2d(omega, s),
                name=f"boundary_layer_{x.size}")


def multi_vortex_2d(n: int, seed: int, extent: float = 10.0, jitter: float = 0.1):
    """Sum of 1-8 Lamb-Oseen vortices (centres U[-8,8]^2, Gamma U[-2,2],
    sigma U[0.2,1.5]) on a jittered lattice of about n particles."""
    rng = np.random.default_rng(seed)
    n_side = max(2, int(round(math.sqrt(n))))
    h = 2 * extent / n_side
    x, y = _lattice(-extent, extent, -extent, extent, h)
    x = x + rng.uniform(-jitter * h, jitter * h, x.size)
    y = y + rng.uniform(-jitter * h, jitter * h, y.size)
    k = int(rng.integers(1, 9))
    omega = np.zeros(x.size)
    for _ in range(k):
        cx, cy = rng.uniform(-8, 8, 2)
        g = rng.uniform(-2, 2)
        sg = rng.uniform(0.2, 1.5)
        omega += g / (math.pi * sg * sg) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (sg * sg))
    s = np.full(x.size, h)
    return dict(x=x, y=y, s=s, omega=omega, active=np.ones(x.size, np.uint8), q=_q2d(omega, s),
                name=f"multi_vortex_{x.size}_{seed}")


def batched_2d(n_solves: int = 64, lo: int = 4096, hi: int = 400_000, seed: int = 3):
    """Uneven batch: n_solves multi-vortex fields, N log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), n_solves)).astype(int)
    return [multi_vortex_2d(int(m), seed=seed * 1000 + i) for i, m in enumerate(sizes)]


def vortex_ring_3d(h: float = 0.02, ring_r: float = 1.0, sigma: float = 0.1, gamma: float = 1.0,
                   extent: float = 2.0, jitter: float = 0.1, noise: float = 1e-3, seed: int = 5):
    """Thin vortex ring: jittered cubic lattice on [-extent, extent]^3 keeping
    points within 3 sigma of the circle of radius ring_r in the z=0 plane.
    Vorticity is tangential, magnitude Gamma/(pi sigma^2) exp(-d^2/sigma^2)
    plus noise. h=0.02 gives ~222k particles, h=0.0096 about 2M."""
    rng = np.random.default_rng(seed)
    n = int(math.floor(2 * extent / h + 1e-9))
    axis = -extent + (np.arange(n) + 0.5) * h
    # Only lattice planes that can hold ring points are generated.
    zs = axis[np.abs(axis) <= 3 * sigma + h]
    xs = axis[np.abs(axis) <= ring_r + 3 * sigma + h]
    gx, gy, gz = np.meshgrid(xs, xs, zs, indexing="ij")
    x, y, z = gx.ravel(), gy.ravel(), gz.ravel()
    rho = np.sqrt(x * x + y * y)
    d2 = (rho - ring_r) ** 2 + z * z
    keep = d2 < (3 * sigma) ** 2
    x, y, z, rho, d2 = x[keep], y[keep], z[keep], rho[keep], d2[keep]
    x = x + rng.uniform(-jitter * h, jitter * h, x.size)
    y = y + rng.uniform(-jitter * h, jitter * h, x.size)
    z = z + rng.uniform(-jitter * h, jitter * h, x.size)
    mag = gamma / (math.pi * sigma ** 2) * np.exp(-d2 / sigma ** 2) + rng.normal(0.0, noise, x.size)
    rs = np.maximum(rho, 1e-12)
    wx, wy, wz = -y / rs * mag, x / rs * mag, np.zeros_like(mag)
    s = np.full(x.size, h)
    c = np.power(s, 3.0) / (4 * math.pi)
    return dict(x=x, y=y, z=z, s=s, wx=wx, wy=wy, wz=wz, active=np.ones(x.size, np.uint8),
                ax=wx * c, ay=wy * c, az=wz * c, name=f"vortex_ring_{x.size}")


def sample_targets(n: int, m: int = 4096, seed: int = 7) -> np.ndarray:
    """m distinct seeded target indices (all of them when n <= m)."""
    if n <= m:
        return np.arange(n, dtype=np.int64)
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=m, replace=False)).astype(np.int64)


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2 over stacked components."""
    a = np.concatenate([np.ravel(v) for v in a]) if isinstance(a, (tuple, list)) else np.ravel(a)
    b = np.concatenate([np.ravel(v) for v in b]) if isinstance(b, (tuple, list)) else np.ravel(b)
    den = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (den if den > 0 else 1.0)
