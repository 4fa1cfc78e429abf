"""3D TreeCell path on the GPU (vpm_fmm3d_velocity_treecell, the reference's
VELOCITY_3D_TYPE 2) against the oracle and the reference's golden vectors:
every cell by reference ID (counts, leaf and active flags, level, parent,
bit-exact centres and lengths) and every leaf's particle list, velocities
within 1e-10 of the oracle for every particle (calcVelocity) and for a target
subset with exact zeros elsewhere (calcVelocityNearBody), the mixed form
within 1e-5 of the plain one, and the two inputs the reference cannot run
(a level-1 leaf of a deeper tree, a tree deeper than level 10) reported as
errors."""
import os

import numpy as np
import pytest

from lsmps_vpm_v2_b200 import workloads
from lsmps_vpm_v2_b200._lib import PREC_MIXED, default_params

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10          # plain form vs the oracle / the reference
TOL_MIXED = 1e-5     # mixed form vs the plain form

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.concatenate([np.ravel(v) for v in a])
    b = np.concatenate([np.ravel(v) for v in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def params(ms=30, mp=50, mixed=False):
    p = default_params(max_src=ms, max_par=mp)
    if mixed:
        p.precision = PREC_MIXED
    return p


def parent_id(cid, level):
    """Reference parent ID of cell `cid` on `level` (treeCell.cpp:336-370)."""
    start = (8 ** level - 1) // 7
    loc = cid - start
    m = 1 << level
    ix, iy, iz = loc % m, (loc // m) % m, loc // (m * m)
    L = level - 1
    return (8 ** L - 1) // 7 + (ix >> 1) + ((iy >> 1) << L) + ((iz >> 1) << (2 * L))


def gpu_treecell(ctx, d, ms, mp):
    ctx.build_treecell3d(d["x"], d["y"], d["z"], d["active"], params(ms, mp))
    t = ctx.dump_tree3d()
    ids = ctx.tree3d_cell_ids()
    return ids, t


def assert_same_treecell(ids, t, ref):
    rids, rints, rgeom, rleaves = ref
    order = np.argsort(ids, kind="stable")
    assert np.array_equal(ids[order], rids)
    nc = ids.size
    leaf = (t["chd"] == 0) & (np.arange(nc) > 0)
    assert np.array_equal(t["npar"][order], rints[:, 0])
    assert np.array_equal(leaf[order].astype(np.int32), rints[:, 2])
    assert np.array_equal(t["active"][order].astype(np.int32), rints[:, 3])
    assert np.array_equal(t["level"][order], rints[:, 4])
    assert t["depth"] == rints[0, 5]
    assert np.array_equal(t["geom"][order], rgeom)                 # bit-exact centres and lengths
    assert t["n_leaves"] == int(rints[:, 2].sum())
    par = t["parent"]
    for k in range(1, nc):
        assert ids[par[k]] == parent_id(int(ids[k]), int(t["level"][k]))
    offs, pids = t["leaf_offs"], t["leaf_pids"]
    for r, k in enumerate(order):
        assert np.array_equal(pids[offs[k]:offs[k + 1]], rleaves[r]), int(ids[k])


def cube(n, seed, inactive=0.0):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(-1.0, 1.5, n) for _ in range(3))
    ax, ay, az = (rng.normal(0, 1e-3, n) for _ in range(3))
    act = (rng.uniform(size=n) >= inactive).astype(np.uint8)
    return dict(x=x, y=y, z=z, ax=ax, ay=ay, az=az, active=act)


def clustered(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, 3)) * np.array([1.0, 0.3, 0.1])
    c[: n // 3] *= 0.3
    ax, ay, az = (rng.normal(0, 1e-3, n) for _ in range(3))
    act = (rng.uniform(size=n) >= 0.2).astype(np.uint8)
    return dict(x=c[:, 0], y=c[:, 1], z=c[:, 2], ax=ax, ay=ay, az=az, active=act)


def ring(seed, inactive_every=0):
    r = workloads.vortex_ring_3d(h=0.06, seed=seed)
    if inactive_every:
        r["active"] = r["active"].copy()
        r["active"][::inactive_every] = 0
    return r


CASES = {
    "cube3k": lambda: cube(3000, 1),
    "cube_inactive": lambda: cube(6000, 2, inactive=0.5),
    "clustered": lambda: clustered(20000, 3),
    "ring_inactive": lambda: ring(4, inactive_every=4),
}


def test_golden_treecell(ctx):
    f = dict(np.load(os.path.join(GOLD, "treecell3d_ring_h005_30_50.npz")))
    ids, t = gpu_treecell(ctx, f, 30, 50)
    offs = f["leaf_offs"]
    leaves = [f["leaf_pids"][offs[k]:offs[k + 1]] for k in range(f["ids"].size)]
    assert_same_treecell(ids, t, (f["ids"], f["ints"], f["geom"], leaves))
    args = [f[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u = ctx.velocity3d_treecell(*args, f["active"], None, params())
    assert rel_l2(u, (f["u"], f["v"], f["w"])) <= TOL
    ub = ctx.velocity3d_treecell(*args, f["active"], f["target"], params())
    assert rel_l2(ub, (f["u_nb"], f["v_nb"], f["w_nb"])) <= TOL
    off = f["target"] == 0
    assert all(not np.any(c[off]) for c in ub)


@pytest.mark.parametrize("caps", [(30, 50), (8, 12), (200, 300)])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tree_and_velocity_vs_oracle(ctx, port, name, caps):
    d = CASES[name]()
    ms, mp = caps
    ids, t = gpu_treecell(ctx, d, ms, mp)
    assert_same_treecell(ids, t, port.treecell3d(d["x"], d["y"], d["z"], d["active"], max_src=ms, max_par=mp))
    args = [d[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u = ctx.velocity3d_treecell(*args, d["active"], None, params(ms, mp))
    assert rel_l2(u, port.treecell3d_velocity(*args, d["active"], None, max_src=ms, max_par=mp)) <= TOL
    tgt = (np.arange(d["x"].size) % 3 == 1).astype(np.uint8)
    ub = ctx.velocity3d_treecell(*args, d["active"], tgt, params(ms, mp))
    assert rel_l2(ub, port.treecell3d_velocity(*args, d["active"], tgt, max_src=ms, max_par=mp)) <= TOL
    assert all(not np.any(c[tgt == 0]) for c in ub)


def test_mixed_vs_plain(ctx):
    d = CASES["clustered"]()
    args = [d[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u = ctx.velocity3d_treecell(*args, d["active"], None, params())
    um = ctx.velocity3d_treecell(*args, d["active"], None, params(mixed=True))
    assert rel_l2(um, u) <= TOL_MIXED


def test_shallow_tree_gives_zero(ctx, port):
    """Every level-1 cell a leaf (max_level 1): the reference's traversal loop
    does not run and every velocity is zero."""
    d = cube(40, 9)
    args = [d[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u = ctx.velocity3d_treecell(*args, d["active"], None, params())
    ref = port.treecell3d_velocity(*args, d["active"], None)
    for a, b in zip(u, ref):
        assert np.array_equal(a, b) and not np.any(a)


def test_device_entry_point(ctx):
    import torch
    d = CASES["cube_inactive"]()
    n = d["x"].size
    tgt = (np.arange(n) % 2).astype(np.uint8)
    dev = [torch.tensor(d[k], device="cuda") for k in ("x", "y", "z", "ax", "ay", "az")]
    act = torch.tensor(d["active"], device="cuda")
    tg = torch.tensor(tgt, device="cuda")
    out = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx.velocity3d_treecell_device(n, *[t.data_ptr() for t in dev], act.data_ptr(), tg.data_ptr(),
                                       *[t.data_ptr() for t in out], params())
        ctx.sync()
    finally:
        ctx.set_stream(None)
    u = ctx.velocity3d_treecell(*[d[k] for k in ("x", "y", "z", "ax", "ay", "az")], d["active"], tgt, params())
    for a, b in zip(out, u):
        assert np.array_equal(a.cpu().numpy(), b)


def test_inputs_the_reference_cannot_run_report_errors(ctx, port):
    from lsmps_vpm_v2_b200 import VpmError
    rng = np.random.default_rng(2)
    # a level-1 leaf (three particles alone in an octant) in a deeper tree
    x, y, z = rng.uniform(-1, 1, (3, 400))
    x[:3] += 10.0
    a = rng.normal(size=(3, 400))
    act = np.ones(400, np.uint8)
    with pytest.raises(VpmError, match="level-1"):
        ctx.velocity3d_treecell(x, y, z, *a, act, None, params())
    with pytest.raises(RuntimeError):
        port.treecell3d_velocity(x, y, z, *a, act)
    # more than max_par coincident particles: deeper than level 10
    x, y, z = rng.uniform(-1, 1, (3, 200))
    for c in (x, y, z):
        c[:60] = 0.123
    a = rng.normal(size=(3, 200))
    act = np.ones(200, np.uint8)
    with pytest.raises(VpmError, match="level 10"):
        ctx.velocity3d_treecell(x, y, z, *a, act, None, params())
    with pytest.raises(RuntimeError):
        port.treecell3d_velocity(x, y, z, *a, act)
    # the context stays usable
    d = cube(3000, 1)
    args = [d[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u = ctx.velocity3d_treecell(*args, d["active"], None, params())
    assert rel_l2(u, port.treecell3d_velocity(*args, d["active"], None)) <= TOL


@pytest.mark.parametrize("name", ["ring_inactive", "clustered"])
def test_stricter_far_test_vs_oracle(ctx, port, name):
    """support_3d = 3.5 on the TreeCell path: the oracle's walk with the same
    factor, within 1e-10, for all particles and for a target subset."""
    d = CASES[name]()
    args = [d[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    p = params()
    p.support_3d = 3.5
    u = ctx.velocity3d_treecell(*args, d["active"], None, p)
    assert rel_l2(u, port.treecell3d_velocity(*args, d["active"], None, support=3.5)) <= TOL
    tgt = (np.arange(d["x"].size) % 5 == 2).astype(np.uint8)
    ub = ctx.velocity3d_treecell(*args, d["active"], tgt, p)
    assert rel_l2(ub, port.treecell3d_velocity(*args, d["active"], tgt, support=3.5)) <= TOL
