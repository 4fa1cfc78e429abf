"""CUDA FP64 2D path against the oracle, through the C ABI: tree, leafList,
parIDList and lists 1-4 bit-exact; field within 1e-10 relative L2 with the
reference's binomials (and with exact ones), NaN exactly where the reference
gives NaN; full-size workload and linearity."""
import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import BINOM_EXACT, VpmError, default_params, workloads
from lsmps_vpm_v2_b200.workloads import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _tree_equal(g, t):
    for k, v in (("ids", t.ids), ("par", t.par), ("src", t.src), ("leaf", t.leaf), ("active", t.active),
                 ("centers", t.centers), ("leaf_ids", t.leaf_ids), ("leaf_offs", t.leaf_offs),
                 ("leaf_pids", t.leaf_pids)):
        assert np.array_equal(g[k], v), k
    assert np.array_equal(g["level"], t.level) and np.array_equal(g["ix"], t.ix) and np.array_equal(g["iy"], t.iy)


@pytest.mark.parametrize("name", list(cases2d.CASES))
def test_tree_and_lists_bit_exact(ctx, port, name):
    d = cases2d.CASES[name]()
    x, y, a = d["x"], d["y"], d["active"]
    ctx.build_tree2d(x, y, a)
    g = ctx.dump_tree2d()
    _tree_equal(g, port.tree2d(x, y, a))
    for which in (1, 2, 3, 4):
        cid, offs, out = g["lists"][which]
        po, pv = port.lists2d(x, y, a, which, cid)
        assert np.array_equal(offs, po), which
        for k in range(cid.size):
            assert sorted(out[offs[k]:offs[k + 1]]) == sorted(pv[po[k]:po[k + 1]]), (which, cid[k])


@pytest.mark.parametrize("name", list(cases2d.CASES))
def test_field_fp64(ctx, port, name):
    d = cases2d.CASES[name]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a)
    rx, ry = port.fmm2d_field(x, y, q, a)
    fin = np.isfinite(rx) & np.isfinite(ry)
    assert np.array_equal(fin, np.isfinite(ex) & np.isfinite(ey))
    assert rel_l2((ex[fin], ey[fin]), (rx[fin], ry[fin])) <= TOL


@pytest.mark.parametrize("p,caps", [(4, (50, 75)), (12, (50, 75)), (16, (20, 30)), (20, (100, 150)), (30, (50, 75))])
def test_field_orders_and_caps(ctx, port, p, caps):
    d = cases2d.clustered()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    prm = default_params(p=p, max_src=caps[0], max_par=caps[1])
    ex, ey = ctx.field2d(x, y, q, a, prm)
    rx, ry = port.fmm2d_field(x, y, q, a, p=p, max_src=caps[0], max_par=caps[1])
    assert rel_l2((ex, ey), (rx, ry)) <= TOL


def test_exact_binomials(ctx, port):
    d = cases2d.plate_small()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a, default_params(p=16, binom=BINOM_EXACT))
    rx, ry = port.fmm2d_field(x, y, q, a, p=16, exact_binom=True)
    assert rel_l2((ex, ey), (rx, ry)) <= TOL


def test_golden_fixtures(ctx):
    import glob
    import os
    for f in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "fmm2d_*.npz"))):
        g = dict(np.load(f))
        prm = default_params(p=int(g["p"]), max_src=int(g["max_src"]), max_par=int(g["max_par"]))
        ex, ey = ctx.field2d(g["x"], g["y"], g["q"], g["active"], prm)
        assert rel_l2((ex, ey), (g["ex"], g["ey"])) <= TOL, f
        d = ctx.dump_tree2d()
        assert np.array_equal(d["ids"], g["ids"]) and np.array_equal(d["leaf_ids"], g["leaf_ids"]), f


def test_velocity_entry(ctx):
    d = workloads.lamb_oseen_2d(n_side=96, seed=2)
    ex, ey = ctx.field2d(d["x"], d["y"], d["q"], d["active"])
    u, v = ctx.velocity2d(d["x"], d["y"], d["omega"], d["s"], d["active"], 0.5, -0.25)
    # u = Ey + u_inf, v = -Ex + v_inf (velocity_calc.cpp:572-575, 226-230)
    assert np.max(np.abs(u - (ey + 0.5))) <= 1e-12 * np.max(np.abs(ey)) + 1e-15
    assert np.max(np.abs(v - (-ex - 0.25))) <= 1e-12 * np.max(np.abs(ex)) + 1e-15


def test_full_size_workload(ctx, port):
    d = workloads.boundary_layer_2d(scale=0.66)
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey, st = ctx.field2d(x, y, q, a, stats=True)
    assert st.depth_retry == 0 and st.n_cells > 20000
    rx, ry = port.fmm2d_field(x, y, q, a)
    assert rel_l2((ex, ey), (rx, ry)) <= TOL
    # linearity in the sources (size-independent property)
    ex2, ey2 = ctx.field2d(x, y, 2.5 * q, a)
    assert rel_l2((ex2, ey2), (2.5 * ex, 2.5 * ey)) <= 1e-13


def test_errors(ctx):
    with pytest.raises(VpmError) as e:
        ctx.field2d(np.zeros(1), np.zeros(1), np.ones(1), np.ones(1, np.uint8))
    assert e.value.status == 22
    x = np.linspace(0, 1, 100)
    y = x.copy()
    y[5] = np.nan
    with pytest.raises(VpmError) as e:
        ctx.field2d(x, y, np.ones(100), np.ones(100, np.uint8))
    assert e.value.status == 22
    with pytest.raises(VpmError):
        ctx.field2d(x, x, np.ones(100), np.ones(100, np.uint8), default_params(p=31))
    # still usable after errors
    d = cases2d.CASES["tiny300"]()
    ctx.field2d(d["x"], d["y"], d["q"], d["active"])


def test_coincident_cluster_retries_deeper_keys(ctx, port):
    """More than max_par particles in a cell of size 2^-16 root: the 16-level
    keys cannot separate them, the host entry point rebuilds with 31 levels."""
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-1, 1, 500), 0.3 + rng.uniform(0, 1e-7, 200)])
    y = np.concatenate([rng.uniform(-1, 1, 500), 0.2 + rng.uniform(0, 1e-7, 200)])
    q = rng.normal(0, 1, x.size)
    a = np.ones(x.size, np.uint8)
    ex, ey, st = ctx.field2d(x, y, q, a, stats=True)
    assert st.depth_retry == 1
    rx, ry = port.fmm2d_field(x, y, q, a)
    assert rel_l2((ex, ey), (rx, ry)) <= TOL


def test_inactive_large_cell_after_active_evaluation(ctx, port):
    """A cell of more than 1024 particles, all of them inactive, under an active
    parent: its moments must be zero, also when the same context evaluated the
    particles active just before (the arena then holds that cell's old moments),
    in both precision settings' upward passes."""
    rng = np.random.default_rng(77)
    xb, yb = rng.uniform(0.0, 1.0, 40_000), rng.uniform(0.0, 1.0, 40_000)
    keep = ~((xb > 0.08) & (xb < 0.18) & (yb > 0.08) & (yb < 0.18))   # no active particle near the cluster
    xb, yb = xb[keep], yb[keep]
    xc, yc = rng.uniform(0.10, 0.16, 12_000), rng.uniform(0.10, 0.16, 12_000)
    x, y = np.concatenate([xb, xc]), np.concatenate([yb, yc])
    q = rng.normal(0.0, 1.0, x.size) * 1e-3
    on = np.ones(x.size, np.uint8)
    off = on.copy()
    off[xb.size:] = 0
    for prm in (default_params(), default_params(precision=1, binom=BINOM_EXACT, p=8, max_src=100, max_par=150)):
        ctx.field2d(x, y, q, on, prm)
        ex, ey = ctx.field2d(x, y, q, off, prm)
        rx, ry = port.fmm2d_field(x, y, q, off, p=prm.p, max_src=prm.max_src, max_par=prm.max_par,
                                  exact_binom=prm.binom == BINOM_EXACT)
        tol = TOL if prm.precision == 0 else 1e-5
        assert rel_l2((ex, ey), (rx, ry)) <= tol, prm.precision


@pytest.mark.parametrize("prec", [0, 1])
def test_reused_context_matches_fresh(ctx, prec):
    """One context evaluating a sequence of different particle sets (sizes,
    clustering, inactive regions) gives, for each, the bits a fresh context
    gives: nothing read from the arena outlives the evaluation that wrote it.
    Eager launches and graph replay both."""
    from lsmps_vpm_v2_b200 import Context
    seq = [cases2d.clustered(), cases2d.partly_inactive(), cases2d.plate_small(), cases2d.deep()]
    d = dict(cases2d.clustered())
    a = d["active"].copy()
    a[(d["x"] > np.median(d["x"])) & (d["y"] > np.median(d["y"]))] = 0   # one inactive quadrant
    d["active"] = a
    seq.append(d)
    seq.append(cases2d.clustered())
    for use_graph in (0, 1):
        prm = default_params(use_graph=use_graph) if prec == 0 else \
            default_params(precision=1, binom=BINOM_EXACT, p=8, max_src=100, max_par=150, use_graph=use_graph)
        for k, d in enumerate(seq):
            x, y, q, act = d["x"], d["y"], d["q"], d["active"]
            ex, ey = ctx.field2d(x, y, q, act, prm)
            fresh = Context(0)
            fx, fy = fresh.field2d(x, y, q, act, prm)
            del fresh
            assert np.array_equal(ex, fx, equal_nan=True) and np.array_equal(ey, fy, equal_nan=True), (use_graph, k)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("use_graph", [0, 1])
def test_host_entry_matches_device_entry(ctx, prec, use_graph):
    """The host entry points upload positions first and gather the strengths
    into tree order after the sort; the device entry point sorts with them.
    Both give the same bits, for the field and (through vpm_velocity2d) the
    velocity, from page-locked and from ordinary host memory."""
    import torch
    d = cases2d.clustered()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    prm = default_params(use_graph=use_graph) if prec == 0 else \
        default_params(precision=1, binom=BINOM_EXACT, p=8, max_src=100, max_par=150, use_graph=use_graph)
    dev = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (x, y, q, a)]
    ex_d, ey_d = torch.empty_like(dev[0]), torch.empty_like(dev[0])
    ctx.field2d_device(*dev, ex_d, ey_d, prm)
    ctx.sync()
    ex_d, ey_d = ex_d.cpu().numpy(), ey_d.cpu().numpy()
    ex, ey = ctx.field2d(x, y, q, a, prm)
    assert np.array_equal(ex, ex_d) and np.array_equal(ey, ey_d)
    pinned = [torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy() for v in (x, y, q, a)]
    ex2, ey2 = ctx.field2d(*pinned, prm)
    assert np.array_equal(ex2, ex_d) and np.array_equal(ey2, ey_d)
    # velocity: q = -omega s^2 / (2 pi) formed on the upload stream; u = Ey, v = -Ex
    s = np.full(x.size, 0.02)
    omega = -q * 2.0 * np.pi / (s * s)
    u, v = ctx.velocity2d(x, y, omega, s, a, 0.0, 0.0, prm)
    assert rel_l2((u, v), (ey_d, -ex_d)) <= 1e-14
