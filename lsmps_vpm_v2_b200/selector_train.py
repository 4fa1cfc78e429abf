"""Generate the selector's training data with the FMM itself and train it on
the GPU (python -m lsmps_vpm_v2_b200.selector_train).

Each random 2D field (multi-vortex lattices, boundary-layer plates at random
resolution, Gaussian clusters; N log-uniform in [10k, 2M]) is evaluated by
the mixed form at all 35 (caps, p) candidates: the label of a candidate is
its measured device time (CUDA events around a replay of the evaluation's
CUDA graph, the way a time-stepping caller runs it; median of three after
the capture) and
its relative L2 error against the FP64 direct sum on 4,096 sampled targets
(the library's direct-sum kernel). One field gives one row of 228 features
and 70 labels; the target-error feature is drawn at random per row (the
labels do not depend on it). Training is minibatch Adam in the library's
kernels; the weights and normalisation go to selector_weights.npz.
"""
from __future__ import annotations

import argparse
import math
import os
import time

import numpy as np

from . import workloads
from ._lib import default_params, lib
from .fmm import Context
from .selector import N_CAND, N_FEAT, N_OUT, REFERENCE_PAIR, WEIGHTS, Selector, candidates


def clustered_field(n: int, seed: int):
    """Gaussian clusters of mixed widths in a sparse background (multi-resolution)."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(2, 10))
    centres = rng.uniform(-8, 8, (k, 2))
    widths = np.exp(rng.uniform(math.log(0.05), math.log(2.0), k))
    share = rng.dirichlet(np.ones(k + 1))
    counts = np.maximum(1, (share * n).astype(int))
    pts = [rng.uniform(-10, 10, (counts[0], 2))]
    for i in range(k):
        pts.append(centres[i] + rng.normal(0, widths[i], (counts[i + 1], 2)))
    p = np.concatenate(pts)
    x, y = p[:, 0].copy(), p[:, 1].copy()
    omega = np.zeros(x.size)
    for i in range(k):
        g = rng.uniform(-2, 2)
        s2 = widths[i] ** 2
        omega += g / (math.pi * s2) * np.exp(-((x - centres[i][0]) ** 2 + (y - centres[i][1]) ** 2) / s2)
    h = np.full(x.size, 20.0 / math.sqrt(n))
    q = -omega * h * h / (2 * math.pi)
    return dict(x=x, y=y, q=q, active=np.ones(x.size, np.uint8))


def random_field(rng, i: int):
    n = int(math.exp(rng.uniform(math.log(10_000), math.log(2_000_000))))
    kind = rng.uniform()
    if kind < 0.45:
        d = workloads.multi_vortex_2d(n, seed=100_000 + i)
    elif kind < 0.7:
        scale = 0.66 * math.sqrt(781_937 / n)
        d = workloads.boundary_layer_2d(scale=scale, seed=200_000 + i)
    else:
        d = clustered_field(n, 300_000 + i)
    return d


def label_field(ctx, sel, d, cands, rng, torch):
    """Features and the 35 (log10 error, log10 ms) labels of one field."""
    dev = torch.device("cuda", 0)
    x, y, q = (torch.from_numpy(np.ascontiguousarray(d[k], dtype=np.float64)).to(dev) for k in ("x", "y", "q"))
    a = torch.from_numpy(np.ascontiguousarray(d["active"], dtype=np.uint8)).to(dev)
    n = x.numel()
    tg = np.sort(rng.choice(n, size=min(4096, n), replace=False)).astype(np.int64)
    tgt = torch.from_numpy(tg).to(dev)
    dx = torch.empty(tg.size, dtype=torch.float64, device=dev)
    dy = torch.empty_like(dx)
    ctx._check(lib().vpm_direct2d_field_device(ctx._h, x.data_ptr(), y.data_ptr(), q.data_ptr(), a.data_ptr(), n,
                                               tgt.data_ptr(), tg.size, dx.data_ptr(), dy.data_ptr()))
    ex = torch.empty(n, dtype=torch.float64, device=dev)
    ey = torch.empty_like(ex)
    den = torch.sqrt((dx * dx).sum() + (dy * dy).sum()).item()
    labels = np.zeros(N_OUT, np.float32)
    mask = np.ones(N_OUT, np.float32)
    st = torch.cuda.current_stream()
    for k, (ms, mp, p) in enumerate(cands):
        prm = default_params(max_src=ms, max_par=mp, p=p, precision=1, binom=1, use_graph=1)
        times = []
        ok = True
        for rep in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            r = lib().vpm_fmm2d_field_device(ctx._h, x.data_ptr(), y.data_ptr(), q.data_ptr(), a.data_ptr(), n,
                                              prm, ex.data_ptr(), ey.data_ptr())
            e1.record(st)
            if r != 0 or lib().vpm_ctx_sync(ctx._h) != 0:
                ok = False
                break
            if rep:
                times.append(e0.elapsed_time(e1))
        if not ok:
            mask[k] = mask[N_CAND + k] = 0.0
            continue
        num = torch.sqrt(((ex[tgt] - dx) ** 2).sum() + ((ey[tgt] - dy) ** 2).sum()).item()
        err = num / den if den > 0 else 0.0
        labels[k] = math.log10(max(err, 1e-12))
        labels[N_CAND + k] = math.log10(max(float(np.median(times)), 1e-3))
    feat = sel.features_device(x, y, q, a, 1e-4)
    return feat, labels, mask


def build_dataset(ctx, sel, n_fields: int, seed: int, log=print):
    import torch
    torch.cuda.set_stream(torch.cuda.Stream())
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(seed)
    cands = candidates()
    F = np.zeros((n_fields, N_FEAT), np.float32)
    L = np.zeros((n_fields, N_OUT), np.float32)
    M = np.zeros((n_fields, N_OUT), np.float32)
    t0 = time.time()
    for i in range(n_fields):
        d = random_field(rng, i)
        F[i], L[i], M[i] = label_field(ctx, sel, d, cands, rng, torch)
        if (i + 1) % 25 == 0:
            log(f"[data] {i + 1}/{n_fields} fields, {time.time() - t0:.0f} s")
    ctx.set_stream(None)
    return F, L, M


def normalise(F, L, M):
    in_mean = F.mean(0)
    in_std = np.maximum(F.std(0), 1e-3)
    out_mean = np.array([L[M[:, k] > 0, k].mean() if (M[:, k] > 0).any() else 0.0 for k in range(N_OUT)], np.float32)
    out_std = np.array([max(L[M[:, k] > 0, k].std(), 1e-2) if (M[:, k] > 0).any() else 1.0 for k in range(N_OUT)],
                       np.float32)
    return in_mean.astype(np.float32), in_std.astype(np.float32), out_mean, out_std


def augment(F, L, M, copies: int, rng):
    """Rows with the target-error feature drawn log-uniform in [1e-7, 1e-2]."""
    Fs, Ls, Ms = [], [], []
    for _ in range(copies):
        f = F.copy()
        f[:, 3] = rng.uniform(-7, -2, F.shape[0])
        Fs.append(f)
        Ls.append(L)
        Ms.append(M)
    return np.concatenate(Fs), np.concatenate(Ls), np.concatenate(Ms)


def evaluate_choice(sel, F, L, M, target: float, margin: float):
    """Held-out fields: rate of meeting the target and time against the reference pair."""
    cands = candidates()
    ref = cands.index(REFERENCE_PAIR)
    met = 0
    t_sel = t_ref = 0.0
    for i in range(F.shape[0]):
        f = F[i].copy()
        f[3] = math.log10(target)
        (ms, mp, p), _ = sel.choose(f, target, margin)
        k = cands.index((ms, mp, p))
        met += int(L[i, k] <= math.log10(target))
        t_sel += 10 ** L[i, N_CAND + k]
        t_ref += 10 ** L[i, N_CAND + ref]
    return met / max(1, F.shape[0]), t_ref / max(t_sel, 1e-12)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--fields", type=int, default=600)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--data", default=None, help="npz to write (or read with --reuse) the labelled fields")
    ap.add_argument("--reuse", action="store_true")
    ap.add_argument("--out", default=WEIGHTS)
    args = ap.parse_args(argv)
    ctx = Context(0)
    sel = Selector(ctx)
    if args.reuse and args.data and os.path.exists(args.data):
        z = np.load(args.data)
        F, L, M = z["F"], z["L"], z["M"]
    else:
        F, L, M = build_dataset(ctx, sel, args.fields, args.seed)
        if args.data:
            np.savez(args.data, F=F, L=L, M=M)
    rng = np.random.default_rng(args.seed)
    order = rng.permutation(F.shape[0])
    n_val = max(1, F.shape[0] // 10)
    val, tr = order[:n_val], order[n_val:]
    Ftr, Ltr, Mtr = augment(F[tr], L[tr], M[tr], 8, rng)
    in_mean, in_std, out_mean, out_std = normalise(Ftr, Ltr, Mtr)
    sel.init(args.seed)
    sel.set_norm(in_mean, in_std, out_mean, out_std)
    Xn = (Ftr - in_mean) / in_std
    Yn = np.where(Mtr > 0, (Ltr - out_mean) / out_std, 0.0).astype(np.float32)
    hist = sel.train(Xn, Yn, Mtr, batch=256, steps=args.steps, lr=1e-3, seed=args.seed)
    # validation loss in label units
    Fv = F[val].copy()
    Fv[:, 3] = -4.0
    Yv = sel.forward((Fv - in_mean) / in_std) * out_std + out_mean
    mv = M[val] > 0
    rmse_err = float(np.sqrt(np.mean((Yv[:, :N_CAND] - L[val, :N_CAND])[mv[:, :N_CAND]] ** 2)))
    rmse_time = float(np.sqrt(np.mean((Yv[:, N_CAND:] - L[val, N_CAND:])[mv[:, N_CAND:]] ** 2)))
    report = {}
    for target in (1e-3, 1e-4, 1e-5):
        rate, speed = evaluate_choice(sel, F[val], L[val], M[val], target, 0.3)
        report[f"{target:g}"] = (rate, speed)
    print(f"[train] loss {hist[0]:.4f} -> {hist[-1]:.4f}; validation RMSE log10 error {rmse_err:.3f}, "
          f"log10 time {rmse_time:.3f}")
    for k, (rate, speed) in report.items():
        print(f"[select] target {k}: meets target on {rate * 100:.0f}% of held-out fields, "
              f"{speed:.2f}x faster than the reference pair in total")
    sel.save(args.out, loss=hist, val_rmse=np.array([rmse_err, rmse_time]), fields=np.array(F.shape[0]))


if __name__ == "__main__":
    main()
