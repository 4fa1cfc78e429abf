"""Batched independent 2D solves: every solve of the batch equals the same
solve run alone (bit for bit in FP64), the graph replay of the whole batch
equals the eager batch, and empty solves and errors behave."""
import numpy as np
import pytest

from lsmps_vpm_v2_b200 import PREC_MIXED, VpmError, default_params, workloads

pytestmark = pytest.mark.gpu


def _solves(n_solves, lo, hi, seed):
    return [(d["x"], d["y"], d["q"], d["active"])
            for d in workloads.batched_2d(n_solves=n_solves, lo=lo, hi=hi, seed=seed)]


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_batch_matches_single_solves(ctx, precision):
    solves = _solves(12, 2000, 60000, 4)
    prm = default_params(p=12, precision=precision)
    out = ctx.field2d_batched(solves, prm)
    for s, (ex, ey) in zip(solves, out):
        rx, ry = ctx.field2d(*s, prm)
        assert np.array_equal(ex, rx) and np.array_equal(ey, ry)


def test_batch_graph_replay(ctx):
    import torch
    solves = _solves(10, 3000, 40000, 6)
    offs = np.zeros(len(solves) + 1, np.int64)
    offs[1:] = np.cumsum([s[0].size for s in solves])
    dev = [torch.from_numpy(np.concatenate([s[k] for s in solves]).astype(np.float64)).cuda() for k in range(3)]
    act = torch.from_numpy(np.concatenate([s[3] for s in solves]).astype(np.uint8)).cuda()
    N = int(offs[-1])
    e1, f1 = torch.zeros(N, dtype=torch.float64, device="cuda"), torch.zeros(N, dtype=torch.float64, device="cuda")
    e2, f2 = torch.zeros_like(e1), torch.zeros_like(f1)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        prm = default_params(p=12, precision=PREC_MIXED)
        ctx.field2d_batched_device(offs, *[t.data_ptr() for t in dev], act.data_ptr(), e1.data_ptr(),
                                   f1.data_ptr(), prm)
        ctx.sync()
        pg = default_params(p=12, precision=PREC_MIXED, use_graph=1)
        for _ in range(3):
            e2.zero_(); f2.zero_()
            ctx.field2d_batched_device(offs, *[t.data_ptr() for t in dev], act.data_ptr(), e2.data_ptr(),
                                       f2.data_ptr(), pg)
            ctx.sync()
            assert torch.equal(e1, e2) and torch.equal(f1, f2)
    finally:
        ctx.set_stream(None)
    single = ctx.field2d(*solves[3], prm)
    o = offs[3]
    assert np.array_equal(e1[o:offs[4]].cpu().numpy(), single[0])


def test_batch_empty_and_invalid(ctx):
    solves = _solves(3, 2000, 5000, 8)
    empty = (np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0, np.uint8))
    out = ctx.field2d_batched([solves[0], empty, solves[1]])
    assert out[1][0].size == 0
    rx, _ = ctx.field2d(*solves[1])
    assert np.array_equal(out[2][0], rx)
    one = (np.ones(1), np.ones(1), np.ones(1), np.ones(1, np.uint8))
    with pytest.raises(VpmError):
        ctx.field2d_batched([solves[0], one])
