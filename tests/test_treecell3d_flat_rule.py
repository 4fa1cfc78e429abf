"""The construction rule of the GPU's 3D TreeCell build, restated in NumPy and
checked against the oracle's level-by-level TreeCell (treeCell.cpp:1043-1243
with DIM 3) on random inputs, including duplicate lattices, coincident blocks
and extreme leaf caps.

The rule (build_treecell3d in csrc/tree3d.cu): sort particles by their
level-10 Morton key; for particle j, lvl = the first level at which it starts
a run of equal prefixes, big = the deepest level at which that run is split
(particle j + max_par, or the (max_src + 1)-th active particle from j, shares
the prefix); j starts the cells of levels lvl .. min(10, max(lvl, big + 1))
when the parent run of its level-lvl run is split, the last one a leaf when
big < last; a split run at level 10 is an error (the reference's cell IDs
overflow past level 10). The test compares every cell (ID, particle count,
active count, leaf flag, level) with the oracle, and errors with errors."""
import numpy as np
import pytest

K = 10


def spread(v):
    k = np.zeros_like(v, dtype=np.int64)
    for b in range(K):
        k |= ((v >> b) & 1) << (3 * b)
    return k


def lcp(a, b):
    """Equal leading 3-bit digits of two 30-bit keys."""
    d = a ^ b
    out = np.full(d.shape, K)
    nz = d != 0
    hb = np.floor(np.log2(d[nz].astype(np.float64))).astype(np.int64)
    out[nz] = (29 - hb) // 3
    return out


def flat_cells(x, y, z, act, max_src, max_par, exp_pct=1.0):
    p = (x, y, z)
    mn = [c.min() for c in p]
    mx = [c.max() for c in p]
    root = max(abs(b - a) for a, b in zip(mn, mx)) * (1.0 + exp_pct / 100.0)
    piv = [(b + a - root) / 2.0 for a, b in zip(mn, mx)]
    size = root / 1024.0
    ix = [((c - pv) / size).astype(np.int64) for c, pv in zip(p, piv)]
    key = spread(ix[0]) | (spread(ix[1]) << 1) | (spread(ix[2]) << 2)
    order = np.argsort(key, kind="stable")
    key = key[order]
    n = key.size
    asc = np.concatenate([[0], np.cumsum(act[order].astype(np.int64))])
    lvl = np.empty(n, np.int64)
    lvl[0] = 1
    lvl[1:] = lcp(key[:-1], key[1:]) + 1
    big = np.full(n, -1)
    j = np.arange(n)
    m1 = j + max_par < n
    big[m1] = lcp(key[m1], key[j[m1] + max_par])
    target = asc[:-1] + max_src + 1
    has = asc[n] >= target
    m = np.searchsorted(asc, target[has], side="left")
    big[has] = np.maximum(big[has], lcp(key[has], key[m - 1]))
    cells = {}
    for i in range(n):
        L = int(lvl[i])
        if L > K:
            continue
        if L > 1:
            sh = 3 * (K - (L - 1))
            sp = np.searchsorted(key >> sh, key[i] >> sh, side="left")
            if big[sp] < L - 1:
                continue
        if big[i] >= K:
            return None
        last = min(K, max(L, int(big[i]) + 1))
        for LL in range(L, last + 1):
            sh = 3 * (K - LL)
            pre = int(key[i] >> sh)
            hi = int(np.searchsorted(key >> sh, pre, side="right"))
            c = [0, 0, 0]
            for b in range(LL):
                for d in range(3):
                    c[d] |= ((pre >> (3 * b + d)) & 1) << b
            cid = (8 ** LL - 1) // 7 + c[0] + (c[1] << LL) + (c[2] << (2 * LL))
            cells[cid] = (hi - i, int(asc[hi] - asc[i]), int(LL == last and big[i] < last), LL)
    return cells


def case(rng, trial):
    n = int(rng.integers(2, 3000))
    kind = trial % 4
    if kind == 0:
        x, y, z = rng.uniform(-1, 1, (3, n))
    elif kind == 1:
        x, y, z = np.round(rng.uniform(-1, 1, (3, n)) * 8) / 8
    elif kind == 2:
        x, y, z = rng.normal(size=(3, n)) * np.array([[1.0], [0.1], [0.01]])
    else:
        x, y, z = rng.uniform(-1, 1, (3, n))
        x[: n // 4], y[: n // 4], z[: n // 4] = 0.3, -0.2, 0.1
    act = (rng.uniform(size=n) < rng.uniform(0, 1)).astype(np.uint8)
    ms = int(rng.choice([0, 1, 3, 30, 100, 5000]))
    mp = int(rng.choice([1, 2, 8, 50, 300, 10 ** 9]))
    if kind in (1, 3) and trial % 8 < 4:
        ms, mp = max(ms, n // 3), max(mp, n // 3)
    return x, y, z, act, ms, mp


@pytest.mark.parametrize("seed", [1, 7])
def test_flat_rule_gives_the_reference_cells(port, seed):
    rng = np.random.default_rng(seed)
    built = 0
    for trial in range(100):
        x, y, z, act, ms, mp = case(rng, trial)
        try:
            ids, ints, _, _ = port.treecell3d(x, y, z, act, ms, mp)
            ref = {int(c): (int(r[0]), int(r[1]), int(r[2]), int(r[4])) for c, r in zip(ids[1:], ints[1:])}
        except RuntimeError:
            ref = None
        got = flat_cells(x, y, z, act, ms, mp)
        assert (got is None) == (ref is None), (trial, ms, mp)
        assert got == ref, (trial, ms, mp)
        built += ref is not None
    assert built >= 50
