"""The NumPy restatement of the selector network (oracle/mlp.py) checks
itself by central finite differences, so it can check the GPU kernels."""
import numpy as np

from mlp import DIMS, forward, loss_and_grads, param_count


def test_param_count_matches_layout():
    assert param_count() == sum(DIMS[l + 1] * (DIMS[l] + 1) for l in range(len(DIMS) - 1))


def test_gradient_by_finite_differences():
    rng = np.random.default_rng(0)
    P = param_count()
    w = rng.normal(0, 0.1, P)
    X = rng.normal(0, 1, (5, DIMS[0]))
    Y = rng.normal(0, 1, (5, DIMS[-1]))
    M = (rng.uniform(size=Y.shape) > 0.2).astype(float)
    _, g = loss_and_grads(w, X, Y, M)
    idx = rng.choice(P, 40, replace=False)
    h = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        num = (loss_and_grads(wp, X, Y, M)[0] - loss_and_grads(wm, X, Y, M)[0]) / (2 * h)
        assert abs(num - g[k]) <= 1e-6 + 1e-5 * abs(num)


def test_forward_shapes():
    rng = np.random.default_rng(1)
    out, cache = forward(rng.normal(0, 0.1, param_count()), rng.normal(0, 1, (3, DIMS[0])))
    assert out.shape == (3, DIMS[-1]) and len(cache) == len(DIMS) - 1
