"""List-2 M2L of the mixed form against the FP64 M2L of the same mixed form
and against the plain form, over the supported orders, in both variants: per
parent on the FP32 pipes (VPM_PREC_MIXED, orders up to 16; per offset on the
tensor cores above) and on the tensor cores (VPM_PREC_MIXED_TC: tcgen05
kind::tf32, 3xTF32 split, TMEM accumulation); graph replay is bit-identical
to eager launches."""
import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import PREC_MIXED, default_params, workloads
from lsmps_vpm_v2_b200._lib import PREC_MIXED_FP64_M2L, PREC_MIXED_TC
from lsmps_vpm_v2_b200.workloads import rel_l2, sample_targets

pytestmark = pytest.mark.gpu
TOL_TC = 1e-5   # tensor-core M2L vs FP64 M2L, same near field


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_MIXED_TC])
def test_tc_small_case_first(ctx, prec):
    d = cases2d.CASES["lamb_small"]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    tc = ctx.field2d(x, y, q, a, default_params(precision=prec))
    ref = ctx.field2d(x, y, q, a, default_params(precision=PREC_MIXED_FP64_M2L))
    assert np.all(np.isfinite(tc[0])) and np.all(np.isfinite(tc[1]))
    assert rel_l2(tc, ref) <= TOL_TC


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_MIXED_TC])
@pytest.mark.parametrize("p", [1, 4, 8, 10, 12, 16, 20])
@pytest.mark.parametrize("name", ["clustered", "plate_small"])
def test_tc_orders(ctx, name, p, prec):
    d = cases2d.CASES[name]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    tc = ctx.field2d(x, y, q, a, default_params(p=p, precision=prec))
    ref = ctx.field2d(x, y, q, a, default_params(p=p, precision=PREC_MIXED_FP64_M2L))
    fp64 = ctx.field2d(x, y, q, a, default_params(p=p))
    assert rel_l2(tc, ref) <= TOL_TC
    assert rel_l2(tc, fp64) <= TOL_TC


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_MIXED_TC])
def test_tc_full_size_vs_direct(ctx, port, prec):
    d = workloads.boundary_layer_2d(scale=0.66)
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a, default_params(precision=prec))
    rx, ry = ctx.field2d(x, y, q, a, default_params(precision=PREC_MIXED_FP64_M2L))
    assert rel_l2((ex, ey), (rx, ry)) <= TOL_TC
    tg = sample_targets(x.size, 4096)
    dx, dy = port.direct2d_field(x, y, q, a, tg)
    assert rel_l2((ex[tg], ey[tg]), (dx, dy)) <= 1e-4


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_MIXED_TC])
def test_tc_graph_replay_bit_identical(ctx, prec):
    import torch
    d = cases2d.CASES["plate_small"]()
    dev = [torch.from_numpy(np.ascontiguousarray(d[k])).cuda() for k in ("x", "y", "q", "active")]
    n = dev[0].numel()
    e1, f1 = torch.empty(n, dtype=torch.float64, device="cuda"), torch.empty(n, dtype=torch.float64, device="cuda")
    e2, f2 = torch.empty_like(e1), torch.empty_like(f1)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx.field2d_device(*dev, e1, f1, default_params(precision=prec))
        ctx.sync()
        for _ in range(3):
            ctx.field2d_device(*dev, e2, f2, default_params(precision=prec, use_graph=1))
            ctx.sync()
            assert torch.equal(e1, e2) and torch.equal(f1, f2)
    finally:
        ctx.set_stream(None)
