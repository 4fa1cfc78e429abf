"""Host logic of the fmm3D mirror (lsmps_vpm_v2_b200.fmm.fmm3D) on CPU: the
reference's calcVelocity / calcVelocityNearBody signatures reach the TreeCell
entry point with the positions split into coordinates, no target flags for
calcVelocity, the caller's flags for calcVelocityNearBody, and the
reference's 3D leaf caps (30 active, 50 particles; global.cpp:778-779) unless
the caller gives its own parameters. The context is a recording fake; the
device path itself is covered by test_gpu_treecell3d.py."""
import numpy as np
import pytest

from lsmps_vpm_v2_b200 import fmm


class FakeCtx:
    def __init__(self):
        self.calls = []

    def velocity3d_treecell(self, x, y, z, ax, ay, az, active, target, params, stats=False):
        self.calls.append(dict(x=x, y=y, z=z, ax=ax, active=active, target=target, params=params))
        n = len(x)
        return np.full(n, 1.0), np.full(n, 2.0), np.full(n, 3.0), "stats"


@pytest.fixture
def lib_params(monkeypatch):
    """Parameter defaults without loading the CUDA library."""
    def fake_default(**over):
        p = fmm.Params()
        p.p, p.max_src, p.max_par, p.exp_tree_pct = 10, 50, 75, 1.0
        for k, v in over.items():
            setattr(p, k, v)
        return p
    monkeypatch.setattr(fmm, "default_params", fake_default)
    monkeypatch.setattr(fmm, "treecell3d_params", lambda **o: fake_default(max_src=30, max_par=50, **o))


def test_calc_velocity_all_targets(lib_params):
    ctx = FakeCtx()
    f = fmm.fmm3D(ctx)
    pos = np.arange(12, dtype=float).reshape(4, 3)
    f.calcVelocity(None, pos, [True, False, True, True], [1.0] * 4, [2.0] * 4, [3.0] * 4)
    c = ctx.calls[0]
    assert np.array_equal(c["x"], pos[:, 0]) and np.array_equal(c["z"], pos[:, 2])
    assert c["target"] is None
    assert (c["params"].max_src, c["params"].max_par) == (30, 50)
    assert np.array_equal(f.get_Field_x(), np.ones(4)) and np.array_equal(f.get_Field_z(), np.full(4, 3.0))


def test_calc_velocity_near_body_passes_flags(lib_params):
    ctx = FakeCtx()
    f = fmm.fmm3D(ctx)
    pos = np.zeros((3, 3))
    flags = [False, True, False]
    f.calcVelocityNearBody(None, pos, [True] * 3, flags, [0.0] * 3, [0.0] * 3, [0.0] * 3)
    assert ctx.calls[0]["target"] == flags


def test_caller_params_are_kept(lib_params):
    ctx = FakeCtx()
    p = fmm.default_params(max_src=7, max_par=9)
    f = fmm.fmm3D(ctx, p)
    f.calcVelocity(None, np.zeros((2, 3)), [True] * 2, [0.0] * 2, [0.0] * 2, [0.0] * 2)
    assert ctx.calls[0]["params"] is p
