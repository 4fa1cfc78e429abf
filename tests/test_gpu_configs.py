"""The named workloads at their own sizes, through the C ABI.

* Lamb-Oseen, 256 x 256 jittered lattice (N = 65,536), p = 10, caps 50/75:
  tree, leafList, parIDList and lists 1-4 bit-exact against the oracle, field
  within 1e-10 of the oracle.
* Boundary layer (N = 778,377) at p = 16, mixed form (per-parent M2L on the
  FP32 pipes, and on the tensor cores): within 1e-4 of the FP64 direct sum on
  4,096 sampled targets and within 1e-5 of the same form with the FP64 M2L;
  plain FP64 at p = 16 within 1e-10 of the oracle.
* 64 uneven solves (N log-uniform in 4,096..400,000, multi-vortex fields),
  p = 12, mixed: every solve of the batch equal to the same solve run alone,
  bit for bit, and sampled solves within 1e-4 of the direct sum.
* Vortex ring at h = 0.0096 (N = 2,009,183): the octree treecode within 1e-10
  of the oracle's per-target traversal on 4,096 sampled targets; the mixed
  form within 1e-5 of the plain one; with the far test R > 3.5 size
  (support_3d) both forms within 1e-4 of the FP64 direct sum.
"""
import numpy as np
import pytest

from lsmps_vpm_v2_b200 import PREC_MIXED, default_params, workloads
from lsmps_vpm_v2_b200._lib import PREC_MIXED_FP64_M2L, PREC_MIXED_TC
from lsmps_vpm_v2_b200.workloads import rel_l2, sample_targets

pytestmark = pytest.mark.gpu
TOL = 1e-10        # plain form against the oracle
TOL_MIXED = 1e-5   # mixed form against the same form with FP64 M2L / the plain form
TOL_DIRECT = 1e-4  # chosen forms against the FP64 direct sum


def test_lamb_oseen_65536_tree_lists_field(ctx, port):
    d = workloads.lamb_oseen_2d(n_side=256)
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    assert x.size == 65536
    ex, ey = ctx.field2d(x, y, q, a)
    g = ctx.dump_tree2d()
    t = port.tree2d(x, y, a)
    for k, v in (("ids", t.ids), ("par", t.par), ("src", t.src), ("leaf", t.leaf), ("active", t.active),
                 ("centers", t.centers), ("leaf_ids", t.leaf_ids), ("leaf_offs", t.leaf_offs),
                 ("leaf_pids", t.leaf_pids), ("level", t.level), ("ix", t.ix), ("iy", t.iy)):
        assert np.array_equal(g[k], v), k
    for which in (1, 2, 3, 4):
        cid, offs, out = g["lists"][which]
        po, pv = port.lists2d(x, y, a, which, cid)
        assert np.array_equal(offs, po), which
        for k in range(cid.size):
            assert np.array_equal(np.sort(out[offs[k]:offs[k + 1]]), np.sort(pv[po[k]:po[k + 1]])), (which, cid[k])
    rx, ry = port.fmm2d_field(x, y, q, a)
    assert rel_l2((ex, ey), (rx, ry)) <= TOL


@pytest.fixture(scope="module")
def plate():
    return workloads.boundary_layer_2d(scale=0.66)


def test_boundary_layer_p16_mixed(ctx, port, plate):
    d = plate
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ref = ctx.field2d(x, y, q, a, default_params(p=16, precision=PREC_MIXED_FP64_M2L, binom=1))
    tg = sample_targets(x.size, 4096)
    dx, dy = port.direct2d_field(x, y, q, a, tg)
    for prec in (PREC_MIXED, PREC_MIXED_TC):
        f = ctx.field2d(x, y, q, a, default_params(p=16, precision=prec, binom=1))
        assert rel_l2(f, ref) <= TOL_MIXED, prec
        assert rel_l2((f[0][tg], f[1][tg]), (dx, dy)) <= TOL_DIRECT, prec


def test_boundary_layer_p16_fp64(ctx, port, plate):
    d = plate
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a, default_params(p=16))
    rx, ry = port.fmm2d_field(x, y, q, a, p=16)
    assert rel_l2((ex, ey), (rx, ry)) <= TOL


def test_batch_64_uneven_solves(ctx, port):
    fields = workloads.batched_2d(n_solves=64, lo=4096, hi=400_000, seed=3)
    solves = [(f["x"], f["y"], f["q"], f["active"]) for f in fields]
    sizes = [s[0].size for s in solves]
    assert len(solves) == 64 and min(sizes) >= 3500 and max(sizes) <= 410_000
    prm = default_params(p=12, precision=PREC_MIXED, binom=1)
    out = ctx.field2d_batched(solves, prm)
    for s, (ex, ey) in zip(solves, out):
        rx, ry = ctx.field2d(*s, prm)
        assert np.array_equal(ex, rx) and np.array_equal(ey, ry)
    for i in (int(np.argmin(sizes)), int(np.argmax(sizes)), 17):
        x, y, q, a = solves[i]
        tg = sample_targets(x.size, 1024, seed=i)
        dx, dy = port.direct2d_field(x, y, q, a, tg)
        assert rel_l2((out[i][0][tg], out[i][1][tg]), (dx, dy)) <= TOL_DIRECT, i


def test_vortex_ring_2m(ctx, port):
    r = workloads.vortex_ring_3d(h=0.0096)
    args = (r["x"], r["y"], r["z"], r["ax"], r["ay"], r["az"], r["active"])
    assert r["x"].size > 2_000_000
    u, v, w = ctx.velocity3d_alpha(*args)
    tg = sample_targets(r["x"].size, 4096)
    ou, ov, ow = port.fmm3d_velocity_at(*args, tg)
    assert rel_l2((u[tg], v[tg], w[tg]), (ou, ov, ow)) <= TOL
    um, vm, wm = ctx.velocity3d_alpha(*args, params=default_params(precision=PREC_MIXED))
    assert rel_l2((um, vm, wm), (u, v, w)) <= TOL_MIXED


def test_vortex_ring_2m_within_1e4_of_direct(ctx, port):
    r = workloads.vortex_ring_3d(h=0.0096)
    args = (r["x"], r["y"], r["z"], r["ax"], r["ay"], r["az"], r["active"])
    tg = sample_targets(r["x"].size, 1024, seed=3)
    du, dv, dw = port.direct3d_velocity(*args, tg)
    for prec in (0, PREC_MIXED):
        u, v, w = ctx.velocity3d_alpha(*args, params=default_params(precision=prec, support_3d=3.5))
        assert rel_l2((u[tg], v[tg], w[tg]), (du, dv, dw)) <= TOL_DIRECT, prec
