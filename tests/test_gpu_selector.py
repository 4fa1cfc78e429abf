"""Learned (caps, p) selector: the GPU forward and backward kernels against
the NumPy oracle, BF16 inference, training on the GPU, the features against
a NumPy recomputation, the GPU direct sum against the oracle's, and - with
the committed weights - what the trained network gains over the reference's
fixed caps and order on fields it was not trained on."""
import math
import os

import numpy as np
import pytest

import cases2d
from lsmps_vpm_v2_b200 import default_params, workloads
from lsmps_vpm_v2_b200.selector import N_CAND, N_FEAT, N_OUT, REFERENCE_PAIR, WEIGHTS, Selector, candidates
from lsmps_vpm_v2_b200.workloads import rel_l2, sample_targets

pytestmark = pytest.mark.gpu


def test_grads_match_oracle(ctx):
    from mlp import forward, loss_and_grads
    sel = Selector(ctx)
    sel.init(3)
    w = sel.get_params().astype(np.float64)
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (48, N_FEAT)).astype(np.float32)
    Y = rng.normal(0, 1, (48, N_OUT)).astype(np.float32)
    M = (rng.uniform(size=Y.shape) > 0.1).astype(np.float32)
    loss, g = sel.grads(X, Y, M)
    rl, rg = loss_and_grads(w, X.astype(np.float64), Y.astype(np.float64), M.astype(np.float64))
    assert abs(loss - rl) <= 1e-5 * abs(rl)
    assert np.linalg.norm(g - rg) <= 1e-4 * np.linalg.norm(rg)
    out = sel.forward(X)
    ref, _ = forward(w, X.astype(np.float64))
    assert np.max(np.abs(out - ref)) <= 1e-4 * max(1.0, np.max(np.abs(ref)))
    ob = sel.forward(X, bf16=True)
    assert np.linalg.norm(ob - ref) <= 3e-2 * np.linalg.norm(ref)   # BF16 weights, FP32 accumulation


def test_training_fits_a_smooth_map(ctx):
    sel = Selector(ctx)
    sel.init(5)
    rng = np.random.default_rng(4)
    X = rng.normal(0, 1, (2048, N_FEAT)).astype(np.float32)
    A = rng.normal(0, 1.0 / math.sqrt(N_FEAT), (N_FEAT, N_OUT))
    Y = np.tanh(X @ A).astype(np.float32)
    hist = sel.train(X, Y, None, batch=128, steps=1500, lr=2e-3, seed=1)
    assert hist[-50:].mean() < 0.25 * hist[:10].mean()


def _features_numpy(x, y, q, target):
    mnx, mxx, mny, mxy = x.min(), x.max(), y.min(), y.max()
    ln = max(mxx - mnx, mxy - mny) * 1.01
    x0, y0 = 0.5 * (mnx + mxx) - 0.5 * ln, 0.5 * (mny + mxy) - 0.5 * ln
    f = [math.log10(x.size), math.log10(ln), math.log10(np.abs(q).max()), math.log10(target)]
    G = 512
    ix = np.clip(((x - x0) / ln * G).astype(np.int64), 0, G - 1)
    iy = np.clip(((y - y0) / ln * G).astype(np.int64), 0, G - 1)
    cnt = np.zeros((G, G), np.int64)
    np.add.at(cnt, (iy, ix), 1)
    for L in range(9, 2, -1):
        c = cnt[cnt > 0]
        b = np.minimum(31, np.floor(np.log2(c)).astype(int))
        h = np.bincount(b, minlength=32)[:32] / c.size
        f.extend(h.tolist())
        cnt = cnt.reshape(cnt.shape[0] // 2, 2, cnt.shape[1] // 2, 2).sum(axis=(1, 3))
    out = np.zeros(N_FEAT, np.float32)
    out[:4] = f[:4]
    hist = np.array(f[4:]).reshape(7, 32)      # levels 9 .. 3
    for k, L in enumerate(range(9, 2, -1)):
        out[4 + (L - 3) * 32: 4 + (L - 2) * 32] = hist[k]
    return out


def test_features_match_numpy(ctx):
    d = cases2d.CASES["clustered"]()
    sel = Selector(ctx)
    f = sel.features(d["x"], d["y"], d["q"], d["active"], 1e-4)
    r = _features_numpy(d["x"], d["y"], d["q"], 1e-4)
    assert np.allclose(f[:4], r[:4], rtol=1e-6)
    assert np.allclose(f[4:], r[4:], atol=1e-6)


def test_direct_sum_matches_oracle(ctx, port):
    import torch
    from lsmps_vpm_v2_b200._lib import lib
    d = cases2d.CASES["partly_inactive"]()
    tg = sample_targets(d["x"].size, 512)
    dev = [torch.from_numpy(np.ascontiguousarray(d[k], dtype=np.float64)).cuda() for k in ("x", "y", "q")]
    a = torch.from_numpy(d["active"].astype(np.uint8)).cuda()
    t = torch.from_numpy(tg).cuda()
    ex = torch.empty(tg.size, dtype=torch.float64, device="cuda")
    ey = torch.empty_like(ex)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx._check(lib().vpm_direct2d_field_device(ctx._h, *[v.data_ptr() for v in dev], a.data_ptr(),
                                                   d["x"].size, t.data_ptr(), tg.size, ex.data_ptr(),
                                                   ey.data_ptr()))
        ctx.sync()
    finally:
        ctx.set_stream(None)
    rx, ry = port.direct2d_field(d["x"], d["y"], d["q"], d["active"], tg)
    assert rel_l2((ex.cpu().numpy(), ey.cpu().numpy()), (rx, ry)) <= 1e-13


def test_untrained_selection_falls_back(ctx):
    from lsmps_vpm_v2_b200 import Context
    c = Context(0)
    try:
        sel = Selector(c)
        (ms, mp, p), _ = sel.choose(np.zeros(N_FEAT, np.float32), 1e-4)
        assert (ms, mp, p) == REFERENCE_PAIR
    finally:
        c.close()


def _graph_ms(ctx, dev_bufs, prm, reps=5):
    """Median CUDA-event time of replays of one evaluation's CUDA graph (the
    way a time-stepping caller runs it), device buffers in and out."""
    import torch
    x, y, q, a = dev_bufs
    ex = torch.empty_like(x)
    ey = torch.empty_like(x)
    st = torch.cuda.current_stream()
    ctx.set_stream(st.cuda_stream)
    try:
        g = default_params(**{f: getattr(prm, f) for f, _ in prm._fields_})
        g.use_graph = 1
        for _ in range(2):
            ctx.field2d_device(x, y, q, a, ex, ey, g)
        ctx.sync()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            ctx.field2d_device(x, y, q, a, ex, ey, g)
            e1.record(st)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ctx.sync()
        return float(np.median(ts)), (ex.cpu().numpy(), ey.cpu().numpy())
    finally:
        ctx.set_stream(None)


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained weights committed")
def test_trained_selector_gain(ctx, port):
    """Held-out fields (seeds outside the training range) at two error
    targets: the chosen caps and order meet the target against the FP64 direct
    sum, and their evaluations together take less device time than the
    reference's fixed pair (caps 50/75, p = 10) in the same mixed form; the
    selection itself (device features and BF16 inference) costs less than one
    evaluation."""
    import time
    import torch
    sel = Selector(ctx)
    assert sel.load()
    fields = [workloads.boundary_layer_2d(scale=0.66, seed=9001), workloads.multi_vortex_2d(300_000, seed=9002),
              workloads.boundary_layer_2d(scale=1.2, seed=9003), workloads.multi_vortex_2d(1_200_000, seed=9004)]
    ref = default_params(precision=1, binom=1)
    t_sel = t_ref = 0.0
    rows = []
    for d in fields:
        x, y, q, a = d["x"], d["y"], d["q"], d["active"]
        dev = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (x, y, q, a)]
        tg = sample_targets(x.size, 4096)
        dx, dy = port.direct2d_field(x, y, q, a, tg)
        t_r, _ = _graph_ms(ctx, dev, ref)
        for target in (1e-4, 1e-3):
            sel.params_for(*dev, target)                      # warm (first call allocates)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            prm = sel.params_for(*dev, target)
            t_choice = (time.perf_counter() - t0) * 1e3
            t_s, (ex, ey) = _graph_ms(ctx, dev, prm)
            assert rel_l2((ex[tg], ey[tg]), (dx, dy)) <= target, (d["name"], target, prm.max_src, prm.p)
            assert t_choice < t_r, (t_choice, t_r)           # selection cheaper than one evaluation
            t_sel += t_s
            t_ref += t_r
            rows.append((d["name"], target, prm.max_src, prm.max_par, prm.p, t_s, t_r, t_choice))
    for r in rows:
        print("%-26s target %.0e: caps %d/%d p %d  %.3f ms vs reference pair %.3f ms (selection %.3f ms)" % r)
    print(f"gain over the reference pair: {t_ref / t_sel:.3f}x")
    assert t_sel < t_ref
