"""The oracle restatement against the live reference (oracle/_ref, compiled
from the reference sources) on seeded cases; skipped where the reference
build is absent (e.g. on the GPU box when it was not shipped)."""
import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import workloads
from lsmps_vpm_v2_b200.workloads import rel_l2

oracle = pytest.importorskip("oracle")
pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def ref():
    return oracle.Reference()


@pytest.mark.parametrize("name", ["lamb_mid", "plate_small", "duplicates", "tiny17", "tiny76"])
def test_port_matches_reference(port, ref, name):
    d = cases2d.CASES[name]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    tp, tr = port.tree2d(x, y, a), ref.tree2d(x, y, a)
    for k in ("ids", "level", "par", "src", "leaf", "active", "centers", "leaf_ids", "leaf_offs", "leaf_pids", "geom"):
        assert np.array_equal(getattr(tp, k), getattr(tr, k)), k
    ex, ey = port.fmm2d_field(x, y, q, a)
    rx, ry = ref.fmm2d_field(x, y, q, a)
    fin = np.isfinite(rx) & np.isfinite(ry)
    assert np.array_equal(fin, np.isfinite(ex) & np.isfinite(ey))   # NaN where two particles coincide
    assert rel_l2((ex[fin], ey[fin]), (rx[fin], ry[fin])) <= 1e-12


def test_reference_binomials_overflow(port, ref):
    """The reference's 32-bit binComb wraps for the top M2L orders; the port
    reproduces it (exact binomials differ at the 1e-7 level)."""
    d = cases2d.lamb_small()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    rx, ry = ref.fmm2d_field(x, y, q, a, p=12)
    ex, ey = port.fmm2d_field(x, y, q, a, p=12)
    gx, gy = port.fmm2d_field(x, y, q, a, p=12, exact_binom=True)
    assert rel_l2((ex, ey), (rx, ry)) <= 1e-12
    assert rel_l2((gx, gy), (rx, ry)) > 1e-9


def test_reference_3d(port, ref):
    r = workloads.vortex_ring_3d(h=0.06)
    args = [r[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u, v, w = port.fmm3d_velocity(*args, r["active"])
    ru, rv, rw = ref.fmm3d_velocity(*args, r["active"])
    assert rel_l2((u, v, w), (ru, rv, rw)) <= 1e-12


@pytest.mark.parametrize("caps", [(30, 50), (8, 12)])
def test_reference_treecell3d(port, ref, caps):
    """3D TreeCell path, cells and velocities, with inactive particles and a
    target subset."""
    r = workloads.vortex_ring_3d(h=0.07, seed=3)
    n = r["x"].size
    act = r["active"].copy()
    act[::6] = 0
    tgt = (np.arange(n) % 5 == 0).astype(np.uint8)
    ms, mp = caps
    tp = port.treecell3d(r["x"], r["y"], r["z"], act, max_src=ms, max_par=mp)
    tr = ref.treecell3d(r["x"], r["y"], r["z"], act, max_src=ms, max_par=mp)
    for a, b in zip(tp[:3], tr[:3]):
        assert np.array_equal(a, b)
    assert all(np.array_equal(a, b) for a, b in zip(tp[3], tr[3]))
    args = [r[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    for t in (None, tgt):
        u = port.treecell3d_velocity(*args, act, t, max_src=ms, max_par=mp)
        ru = ref.treecell3d_velocity(*args, act, t, max_src=ms, max_par=mp)
        assert rel_l2(u, ru) <= 1e-12


def test_treecell3d_port_refuses_level1_leaf(port):
    """A level-1 leaf in a deeper TreeCell: the reference's traversal throws
    (inside its OpenMP loop, which ends the process, so it is not run here);
    the port reports an error."""
    rng = np.random.default_rng(2)
    x, y, z = rng.uniform(-1, 1, (3, 400))
    x[:3] += 10.0          # three particles alone in a level-1 cell
    a = rng.normal(size=(3, 400))
    with pytest.raises(RuntimeError, match="level-1"):
        port.treecell3d_velocity(x, y, z, *a, np.ones(400, np.uint8))


@pytest.mark.parametrize("which", ["all_inactive", "max_level_1"])
def test_reference_treecell3d_edges(port, ref, which):
    """All particles inactive (every cell inactive, zero velocity), and a tree
    whose level-1 cells are all leaves (the traversal loop does not run)."""
    rng = np.random.default_rng(4)
    n = 1000 if which == "all_inactive" else 40
    x, y, z = rng.uniform(-1, 1, (3, n))
    a = rng.normal(size=(3, n))
    act = np.zeros(n, np.uint8) if which == "all_inactive" else np.ones(n, np.uint8)
    tp = port.treecell3d(x, y, z, act)
    tr = ref.treecell3d(x, y, z, act)
    for p_, r_ in zip(tp[:3], tr[:3]):
        assert np.array_equal(p_, r_)
    u = port.treecell3d_velocity(x, y, z, *a, act)
    ru = ref.treecell3d_velocity(x, y, z, *a, act)
    for p_, r_ in zip(u, ru):
        assert np.array_equal(p_, r_) and not np.any(r_)
