"""Synthetic workload generators: sizes and determinism."""
import numpy as np

from lsmps_vpm_v2_b200 import workloads as w


def test_lamb_oseen_size_and_seed():
    a, b = w.lamb_oseen_2d(), w.lamb_oseen_2d()
    assert a["x"].size == 65536 and np.array_equal(a["x"], b["x"]) and np.array_equal(a["omega"], b["omega"])
    # q = -omega s^2 / (2 pi), velocity_calc.cpp:477
    assert np.allclose(a["q"], -a["omega"] * a["s"] ** 2 / (2 * np.pi))


def test_boundary_layer_sizes():
    assert w.boundary_layer_2d(scale=1.0)["x"].size == 340_000
    n = w.boundary_layer_2d(scale=0.66)["x"].size
    assert 770_000 < n < 790_000


def test_ring_3d():
    r = w.vortex_ring_3d(h=0.05)
    d = np.sqrt((np.hypot(r["x"], r["y"]) - 1.0) ** 2 + r["z"] ** 2)
    assert r["x"].size > 1000 and d.max() < 0.3 + 0.05


def test_batched_sizes():
    b = w.batched_2d(n_solves=8, lo=4096, hi=40000)
    assert len(b) == 8 and all(3000 <= s["x"].size <= 45000 for s in b)
