"""3D treecode on the GPU against the oracle and the reference's golden
vectors: the octree cell for cell (bit-exact centres, sizes, counts, child
flags, active flags), velocities within 1e-10 (plain form), and the mixed
form against the plain form and the FP64 direct sum."""
import os

import numpy as np
import pytest

from lsmps_vpm_v2_b200 import workloads
from lsmps_vpm_v2_b200._lib import PREC_MIXED, default_params

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10          # plain form vs the reference's treecode
TOL_MIXED = 1e-5     # mixed form vs the plain form

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.concatenate([np.ravel(v) for v in a])
    b = np.concatenate([np.ravel(v) for v in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def canon(npar, chd, parent, active, level, geom):
    """Cells sorted by (level, z, y, x) with each cell's parent centre, so
    trees numbered in different orders compare row by row."""
    order = np.lexsort((geom[:, 0], geom[:, 1], geom[:, 2], level))
    pc = np.full((len(npar), 3), np.nan)
    has = parent >= 0
    pc[has] = geom[parent[has], :3]
    return dict(npar=npar[order], chd=chd[order], active=active[order].astype(bool), level=level[order],
                geom=geom[order], pgeom=pc[order])


def assert_same_tree(dump, ints, geom):
    g = canon(dump["npar"], dump["chd"], dump["parent"], dump["active"], dump["level"], dump["geom"])
    r = canon(ints[:, 0], ints[:, 1], ints[:, 2], ints[:, 3], ints[:, 4], geom)
    assert len(dump["npar"]) == len(ints)
    assert dump["depth"] == ints[0, 5]
    for k in ("npar", "chd", "active", "level"):
        assert np.array_equal(g[k], r[k]), k
    assert np.array_equal(g["geom"], r["geom"])          # bit-exact centres and sizes
    assert np.array_equal(g["pgeom"], r["pgeom"], equal_nan=True)


def params(leaf_cap=30, mixed=False):
    p = default_params(leaf_cap_3d=leaf_cap)
    if mixed:
        p.precision = PREC_MIXED
    return p


def uniform_cube(n, seed, inactive=0.0):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(-1.0, 1.5, n) for _ in range(3))
    ax, ay, az = (rng.normal(0, 1e-3, n) for _ in range(3))
    act = (rng.uniform(size=n) >= inactive).astype(np.uint8)
    return dict(x=x, y=y, z=z, ax=ax, ay=ay, az=az, active=act)


def clustered(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-3, 3, (6, 3))
    k = rng.integers(0, 6, n)
    p = c[k] + rng.normal(0, 0.05, (n, 3)) * rng.uniform(0.1, 2.0, (n, 1))
    ax, ay, az = (rng.normal(0, 1e-3, n) for _ in range(3))
    return dict(x=p[:, 0].copy(), y=p[:, 1].copy(), z=p[:, 2].copy(), ax=ax, ay=ay, az=az,
                active=np.ones(n, np.uint8))


def ring(h):
    r = workloads.vortex_ring_3d(h=h)
    return dict(x=r["x"], y=r["y"], z=r["z"], ax=r["ax"], ay=r["ay"], az=r["az"], active=r["active"])


def test_golden_ring_tree_and_velocity(ctx):
    f = dict(np.load(os.path.join(GOLD, "fmm3d_ring_h005.npz")))
    u, v, w = ctx.velocity3d_alpha(f["x"], f["y"], f["z"], f["ax"], f["ay"], f["az"], f["active"], params())
    assert rel_l2((u, v, w), (f["u"], f["v"], f["w"])) <= TOL
    ctx.build_tree3d(f["x"], f["y"], f["z"], f["active"], params())
    assert_same_tree(ctx.dump_tree3d(), f["ints"], f["geom"])


CASES = {
    "ring_h006": lambda: ring(0.06),
    "cube_20k_inactive": lambda: uniform_cube(20000, 1, inactive=0.2),
    "clustered_30k": lambda: clustered(30000, 2),
    "tiny_100": lambda: uniform_cube(100, 3),
    "pair": lambda: uniform_cube(2, 4),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("leaf_cap", [30, 8, 50])
def test_tree_and_velocity_vs_oracle(ctx, port, name, leaf_cap):
    d = CASES[name]()
    args = (d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"])
    ru, rv, rw = port.fmm3d_velocity(*args, d["active"], leaf_cap=leaf_cap)
    u, v, w, st = ctx.velocity3d_alpha(*args, d["active"], params(leaf_cap), stats=True)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(v)) and np.all(np.isfinite(w))
    if np.linalg.norm(np.concatenate([ru, rv, rw])) == 0:
        assert max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max()) == 0
    else:
        assert rel_l2((u, v, w), (ru, rv, rw)) <= TOL
    ints, geom = port.tree3d(d["x"], d["y"], d["z"], d["active"], leaf_cap=leaf_cap)
    ctx.build_tree3d(d["x"], d["y"], d["z"], d["active"], params(leaf_cap))
    dump = ctx.dump_tree3d()
    assert_same_tree(dump, ints, geom)
    assert st.n_cells == len(ints)
    # every particle sits in exactly one leaf, ascending within the leaf
    pids = dump["leaf_pids"]
    assert np.array_equal(np.sort(pids), np.arange(d["x"].size))
    offs = dump["leaf_offs"]
    for k in np.flatnonzero(np.diff(offs) > 1)[:200]:
        seg = pids[offs[k]:offs[k + 1]]
        assert np.all(np.diff(seg) > 0)


def test_reference_velocity_3d(ctx):
    """Against the reference's own treecode where it was built here."""
    from oracle import Reference, ref_available
    if not ref_available():
        pytest.skip("reference library not built")
    d = ring(0.06)
    args = (d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"])
    ru, rv, rw = Reference().fmm3d_velocity(*args, d["active"])
    u, v, w = ctx.velocity3d_alpha(*args, d["active"], params())
    assert rel_l2((u, v, w), (ru, rv, rw)) <= TOL


def test_mixed_vs_plain_and_direct(ctx, port):
    d = ring(0.04)
    args = (d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"])
    u, v, w = ctx.velocity3d_alpha(*args, d["active"], params())
    um, vm, wm = ctx.velocity3d_alpha(*args, d["active"], params(mixed=True))
    assert rel_l2((um, vm, wm), (u, v, w)) <= TOL_MIXED
    tg = np.random.default_rng(0).choice(d["x"].size, 512, replace=False)
    du, dv, dw = port.direct3d_velocity(*args, d["active"], tg)
    e64 = rel_l2((u[tg], v[tg], w[tg]), (du, dv, dw))
    e32 = rel_l2((um[tg], vm[tg], wm[tg]), (du, dv, dw))
    # the treecode's own truncation error dominates both forms
    assert e64 < 5e-2 and abs(e32 - e64) <= 1e-4 + 0.01 * e64


def test_velocity3d_from_vorticity(ctx, port):
    """alpha = omega s^3 / (4 pi) plus the free stream (velocity_calc.cpp:2432-2434, 226-236)."""
    r = workloads.vortex_ring_3d(h=0.06)
    s = r["s"]
    four_pi = 4 * np.pi
    a = [r[k] * s ** 3 / four_pi for k in ("wx", "wy", "wz")]
    ru, rv, rw = port.fmm3d_velocity(r["x"], r["y"], r["z"], *a, r["active"])
    u, v, w = ctx.velocity3d(r["x"], r["y"], r["z"], r["wx"], r["wy"], r["wz"], s, r["active"], 1.0, -0.5, 0.25,
                             params())
    assert rel_l2((u - 1.0, v + 0.5, w - 0.25), (ru, rv, rw)) <= TOL


def test_device_entry_point(ctx):
    import torch
    d = uniform_cube(5000, 7)
    dev = [torch.tensor(d[k], device="cuda") for k in ("x", "y", "z", "ax", "ay", "az")]
    act = torch.tensor(d["active"], device="cuda")
    out = [torch.empty(5000, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx.velocity3d_device(5000, *[t.data_ptr() for t in dev], act.data_ptr(), *[t.data_ptr() for t in out],
                              params())
        ctx.sync()
    finally:
        ctx.set_stream(None)
    u, v, w = ctx.velocity3d_alpha(d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"], d["active"], params())
    assert np.array_equal(out[0].cpu().numpy(), u)
    assert np.array_equal(out[1].cpu().numpy(), v)
    assert np.array_equal(out[2].cpu().numpy(), w)


def test_coincident_particles_report_error(ctx):
    from lsmps_vpm_v2_b200 import VpmError
    d = uniform_cube(64, 8)
    for k in ("x", "y", "z"):
        d[k][:40] = 0.25
    with pytest.raises(VpmError):
        ctx.velocity3d_alpha(d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"], d["active"], params())


def test_direct3d_device_matches_oracle(ctx, port):
    """The library's FP64 3D direct sum (the yardstick of the 3D error in the
    bench) against the oracle's on sampled targets of a partly inactive ring."""
    import ctypes as C
    import torch
    from lsmps_vpm_v2_b200._lib import lib
    r = workloads.vortex_ring_3d(h=0.05)
    act = r["active"].copy()
    act[::7] = 0
    args = (r["x"], r["y"], r["z"], r["ax"], r["ay"], r["az"], act)
    tg = workloads.sample_targets(r["x"].size, 777, seed=2)
    dev = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in args]
    t = torch.from_numpy(tg).cuda()
    out = [torch.empty(tg.size, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx._check(lib().vpm_direct3d_velocity_device(ctx._h, *[C.c_void_p(v.data_ptr()) for v in dev], r["x"].size,
                                                       C.c_void_p(t.data_ptr()), tg.size,
                                                       *[C.c_void_p(o.data_ptr()) for o in out]))
        torch.cuda.synchronize()
    finally:
        ctx.set_stream(None)
    ref = port.direct3d_velocity(*args, tg)
    got = [o.cpu().numpy() for o in out]
    assert workloads.rel_l2(got, ref) <= 1e-13


@pytest.mark.parametrize("support", [3.0, 3.5, 4.0])
@pytest.mark.parametrize("name", ["ring_h006", "clustered_30k", "cube_20k_inactive"])
def test_stricter_far_test_vs_oracle(ctx, port, name, support):
    """The far test R > support x size with a factor above the reference's 2
    (support_3d): the same per-target walk as the oracle's with that factor,
    within 1e-10, and closer to the FP64 direct sum than the factor-2 walk."""
    d = CASES[name]()
    args = (d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"])
    p = params()
    p.support_3d = support
    u, v, w = ctx.velocity3d_alpha(*args, d["active"], p)
    ru, rv, rw = port.fmm3d_velocity(*args, d["active"], support=support)
    assert rel_l2((u, v, w), (ru, rv, rw)) <= TOL
    tg = np.random.default_rng(1).choice(d["x"].size, 512, replace=False)
    du, dv, dw = port.direct3d_velocity(*args, d["active"], tg)
    u2, v2, w2 = ctx.velocity3d_alpha(*args, d["active"], params())
    assert rel_l2((u[tg], v[tg], w[tg]), (du, dv, dw)) < rel_l2((u2[tg], v2[tg], w2[tg]), (du, dv, dw))


def test_support_factor_validation(ctx):
    from lsmps_vpm_v2_b200 import VpmError
    d = ring(0.06)
    args = (d["x"], d["y"], d["z"], d["ax"], d["ay"], d["az"])
    p = params()
    p.support_3d = 0.0                    # taken as the reference's 2.0
    assert rel_l2(ctx.velocity3d_alpha(*args, d["active"], p), ctx.velocity3d_alpha(*args, d["active"], params())) == 0
    for bad in (0.5, float("nan"), float("inf")):
        p.support_3d = bad
        with pytest.raises(VpmError) as e:
            ctx.velocity3d_alpha(*args, d["active"], p)
        assert e.value.status == 22
