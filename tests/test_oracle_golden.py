"""The oracle restatement against the golden fixtures generated from the
reference's own FMM (tests/golden/make_golden.py): tree, leafList, parIDList
and lists 1-4 bit-exact; field and potential within 1e-12 relative L2."""
import glob
import os

import numpy as np
import pytest

from lsmps_vpm_v2_b200.workloads import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX2 = sorted(glob.glob(os.path.join(GOLD, "fmm2d_*.npz")))


@pytest.fixture(params=FIX2, ids=[os.path.basename(f)[6:-4] for f in FIX2], scope="module")
def fx(request):
    return dict(np.load(request.param))


def test_tree_bit_exact(port, fx):
    t = port.tree2d(fx["x"], fx["y"], fx["active"], max_src=int(fx["max_src"]), max_par=int(fx["max_par"]))
    assert np.array_equal(t.ids, fx["ids"])
    ints = np.stack([t.level, t.ix, t.iy, t.par, t.src, t.leaf.astype(np.int32) | (t.active.astype(np.int32) << 1)], 1)
    assert np.array_equal(ints, fx["ints"])
    assert np.array_equal(t.centers, fx["centers"])          # cell centres bit for bit
    assert np.array_equal(t.geom, fx["geom"])                # box, rootLength, pivot, min/max level
    assert np.array_equal(t.leaf_ids, fx["leaf_ids"])        # leafList order
    assert np.array_equal(t.leaf_offs, fx["leaf_offs"])
    assert np.array_equal(t.leaf_pids, fx["leaf_pids"])      # parIDList


@pytest.mark.parametrize("which", [1, 2, 3, 4])
def test_lists_bit_exact(port, fx, which):
    cells = fx[f"l{which}_cells"]
    offs, ids = port.lists2d(fx["x"], fx["y"], fx["active"], which, cells, max_src=int(fx["max_src"]),
                             max_par=int(fx["max_par"]))
    ro, ri = fx[f"l{which}_offs"], fx[f"l{which}_ids"]
    assert np.array_equal(offs, ro)
    for k in range(cells.size):
        assert sorted(ids[offs[k]:offs[k + 1]]) == sorted(ri[ro[k]:ro[k + 1]])


def test_field(port, fx):
    ex, ey = port.fmm2d_field(fx["x"], fx["y"], fx["q"], fx["active"], p=int(fx["p"]), max_src=int(fx["max_src"]),
                              max_par=int(fx["max_par"]))
    assert rel_l2((ex, ey), (fx["ex"], fx["ey"])) <= 1e-12


def test_potential(port, fx):
    pot = port.fmm2d_potential(fx["x"], fx["y"], fx["q"], fx["active"], p=int(fx["p"]), max_src=int(fx["max_src"]),
                               max_par=int(fx["max_par"]))
    assert rel_l2(pot, fx["pot"]) <= 1e-12


def test_3d_treecode():
    f = dict(np.load(os.path.join(GOLD, "fmm3d_ring_h005.npz")))
    from oracle import Port
    P = Port()
    ints, geom = P.tree3d(f["x"], f["y"], f["z"], f["active"])
    # Cell order differs only if creation order differs; both are creation order.
    assert np.array_equal(ints, f["ints"]) and np.array_equal(geom, f["geom"])
    u, v, w = P.fmm3d_velocity(f["x"], f["y"], f["z"], f["ax"], f["ay"], f["az"], f["active"])
    assert rel_l2((u, v, w), (f["u"], f["v"], f["w"])) <= 1e-12


def test_treecell3d_port_matches_golden():
    """3D TreeCell path: cells by ID (counts, flags, levels, centres, lengths),
    leaf particle lists, calcVelocity and calcVelocityNearBody."""
    f = dict(np.load(os.path.join(GOLD, "treecell3d_ring_h005_30_50.npz")))
    from oracle import Port
    P = Port()
    ids, ints, geom, leaves = P.treecell3d(f["x"], f["y"], f["z"], f["active"], max_src=30, max_par=50)
    assert np.array_equal(ids, f["ids"]) and np.array_equal(ints, f["ints"]) and np.array_equal(geom, f["geom"])
    offs = f["leaf_offs"]
    for k, lst in enumerate(leaves):
        assert np.array_equal(lst, f["leaf_pids"][offs[k]:offs[k + 1]])
    args = [f[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u, v, w = P.treecell3d_velocity(*args, f["active"], None, max_src=30, max_par=50)
    assert rel_l2((u, v, w), (f["u"], f["v"], f["w"])) <= 1e-12
    u, v, w = P.treecell3d_velocity(*args, f["active"], f["target"], max_src=30, max_par=50)
    assert rel_l2((u, v, w), (f["u_nb"], f["v_nb"], f["w_nb"])) <= 1e-12
    off = f["target"] == 0
    assert not np.any(u[off]) and not np.any(v[off]) and not np.any(w[off])
