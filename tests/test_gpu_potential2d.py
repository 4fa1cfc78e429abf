"""2D FMM potential (fmm2D::calcPotential) on the GPU against the oracle and
the reference's golden potentials: within 1e-10 relative L2 (the golden
fixtures come from the reference's own FMM)."""
import glob
import os

import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import default_params, fmm2D
from lsmps_vpm_v2_b200.workloads import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-10
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX2 = sorted(glob.glob(os.path.join(GOLD, "fmm2d_*.npz")))


@pytest.mark.parametrize("path", FIX2, ids=[os.path.basename(f)[6:-4] for f in FIX2])
def test_potential_golden(ctx, path):
    f = dict(np.load(path))
    prm = default_params(p=int(f["p"]), max_src=int(f["max_src"]), max_par=int(f["max_par"]))
    phi = ctx.potential2d(f["x"], f["y"], f["q"], f["active"], prm)
    fin = np.isfinite(f["pot"])
    assert np.array_equal(fin, np.isfinite(phi))
    assert rel_l2(phi[fin], f["pot"][fin]) <= TOL


@pytest.mark.parametrize("name", list(cases2d.CASES))
def test_potential_vs_oracle(ctx, port, name):
    d = cases2d.CASES[name]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    phi = ctx.potential2d(x, y, q, a)
    ref = port.fmm2d_potential(x, y, q, a)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(phi))
    assert rel_l2(phi[fin], ref[fin]) <= TOL


def test_potential_operator_mirror(ctx, port):
    """fmm2D.calcPotential / get_Potential, as the pressure Poisson caller uses them."""
    d = cases2d.CASES["lamb_small"]()
    pos = np.stack([d["x"], d["y"]], 1)
    f = fmm2D(ctx, default_params(p=12))
    f.calcPotential(None, pos, d["active"], d["q"])
    ref = port.fmm2d_potential(d["x"], d["y"], d["q"], d["active"], p=12)
    assert rel_l2(f.get_Potential(), ref) <= TOL


def test_potential_and_field_share_a_context(ctx, port):
    """Alternating field and potential calls (different graphs and b_0 handling)."""
    d = cases2d.CASES["clustered"]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    rx, ry = port.fmm2d_field(x, y, q, a)
    rp = port.fmm2d_potential(x, y, q, a)
    for _ in range(2):
        ex, ey = ctx.field2d(x, y, q, a)
        phi = ctx.potential2d(x, y, q, a)
        assert rel_l2((ex, ey), (rx, ry)) <= TOL
        assert rel_l2(phi, rp) <= TOL
