"""Seeded 2D particle sets shared by the parity tests (small enough for the
oracle to finish in seconds), including the edge cases the reference's list
logic is sensitive to."""
import os

import numpy as np

from lsmps_vpm_v2_b200 import workloads as w
from lsmps_vpm_v2_b200.state import read_particle_state

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _field(x, y, active=None, seed=0):
    rng = np.random.default_rng(seed)
    n = x.size
    omega = rng.normal(0.0, 1.0, n)
    s = np.full(n, 0.05)
    a = np.ones(n, np.uint8) if active is None else active.astype(np.uint8)
    return dict(x=x, y=y, s=s, omega=omega, active=a, q=-omega * s * s / (2 * np.pi))


def lamb_small():
    return w.lamb_oseen_2d(n_side=64)


def lamb_mid():
    return w.lamb_oseen_2d(n_side=128, seed=3)


def plate_small():
    return w.boundary_layer_2d(scale=3.0)


def clustered():
    """Two dense Gaussian blobs in a sparse background: leaves on many levels
    (lists 3 and 4 non-empty)."""
    rng = np.random.default_rng(11)
    a = rng.normal([-2, 1], 0.05, (3000, 2))
    b = rng.normal([3, -2], 0.3, (3000, 2))
    c = rng.uniform(-10, 10, (2000, 2))
    p = np.concatenate([a, b, c])
    return _field(p[:, 0], p[:, 1], seed=11)


def deep():
    """A tight blob in a wide background: leaves down to level 15, below
    the level-12 digits the cooperative sort tries first (it must detect that
    and sort the full keys)."""
    rng = np.random.default_rng(12)
    a = rng.normal([0.3, -0.2], 1.5e-3, (1500, 2))
    c = rng.uniform(-10, 10, (1500, 2))
    p = np.concatenate([a, c])
    return _field(p[:, 0], p[:, 1], seed=12)


def partly_inactive():
    """A third of the particles inactive, including whole inactive regions."""
    d = w.lamb_oseen_2d(n_side=80, seed=4)
    act = d["active"].copy()
    act[d["x"] > 3.0] = 0
    rng = np.random.default_rng(4)
    act[rng.random(act.size) < 0.15] = 0
    d = dict(d)
    d["active"] = act
    return d


def boundary_aligned():
    """Exact lattice on cell boundaries of the tree (no jitter): coordinates
    that land on the reference's index boundaries."""
    h = 20.0 / 96
    xs = -10 + np.arange(96) * h
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    return _field(gx.ravel().copy(), gy.ravel().copy(), seed=5)


def aspect():
    """Extreme aspect ratio: a 100 x 0.5 strip."""
    rng = np.random.default_rng(6)
    x = rng.uniform(-50, 50, 6000)
    y = rng.uniform(-0.25, 0.25, 6000)
    return _field(x, y, seed=6)


def duplicates():
    """A few coincident particle pairs (the reference's P2P gives NaN there)."""
    d = w.lamb_oseen_2d(n_side=40, seed=7)
    x, y = d["x"].copy(), d["y"].copy()
    x[100:105] = x[200:205]
    y[100:105] = y[200:205]
    d = dict(d)
    d["x"], d["y"] = x, y
    return d


def state500():
    """Every 8th particle of the reference solver's own flow state at step 500
    (tests/golden/particle_state_00500_sub8.csv; 2,716 particles of several
    sizes, some inactive), with the reference's source strength -omega s^2/(2 pi)
    (velocity_calc.cpp:477)."""
    p = read_particle_state(os.path.join(GOLDEN, "particle_state_00500_sub8.csv"))
    return dict(x=p["x"], y=p["y"], s=p["s"], omega=p["vorticity"], active=p["active"],
                q=-p["vorticity"] * p["s"] * p["s"] / (2 * np.pi))


def tiny(n, seed=8):
    rng = np.random.default_rng(seed)
    return _field(rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), seed=seed)


CASES = {
    "lamb_small": lamb_small,
    "lamb_mid": lamb_mid,
    "plate_small": plate_small,
    "clustered": clustered,
    "deep": deep,
    "partly_inactive": partly_inactive,
    "boundary_aligned": boundary_aligned,
    "aspect": aspect,
    "duplicates": duplicates,
    "state500": state500,
    "tiny2": lambda: tiny(2),
    "tiny17": lambda: tiny(17),
    "tiny76": lambda: tiny(76),
    "tiny300": lambda: tiny(300),
}
