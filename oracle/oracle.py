"""ORACLE — test infrastructure only.

ctypes front end for the CPU checkers, importable only by tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline / reference legs:

* ``Port``      — oracle/liboracle.so, the restatement in oracle2d.cpp and
                  oracle3d.cpp (always built by ``make -C oracle port``);
* ``Reference`` — oracle/_ref/libref2d.so and libref3d.so, the reference's own
                  FMM compiled from its sources by ``make -C oracle ref`` (present
                  only where the reference tree was available at build time).

Both expose the same methods so a test can run against either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_PORT = os.path.join(HERE, "liboracle.so")
_REF2 = os.path.join(HERE, "_ref", "libref2d.so")
_REF3 = os.path.join(HERE, "_ref", "libref3d.so")

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Build the checker libraries (port always; reference when present)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all" if ref else "port"])


def ref_available() -> bool:
    return os.path.exists(_REF2) and os.path.exists(_REF3)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8a(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


def _treecell_dump(call):
    """Run a TreeCell dump entry twice (size, then fill); cells sorted by ID."""
    nc = call(None, None, None, None, None)
    if nc < 0:
        return None
    ids = np.zeros(nc, np.int64)
    ints = np.zeros((nc, 6), np.int32)
    geom = np.zeros((nc, 4))
    offs = np.zeros(nc + 1, np.int64)
    call(None, None, None, _vp(offs), None)
    pids = np.zeros(max(int(offs[-1]), 1), np.int32)
    call(_vp(ids), _vp(ints), _vp(geom), _vp(offs), _vp(pids))
    order = np.argsort(ids, kind="stable")
    leaves = [pids[offs[k]:offs[k + 1]] for k in order]
    ints_s = ints[order].copy()
    ints_s[:, 5] = 0
    ints_s[0, 5] = ints[:, 5].max()
    return ids[order], ints_s, geom[order], leaves


class Tree2D:
    """A 2D tree dump in the reference's vocabulary (cell IDs, leafList)."""

    def __init__(self, ids, ints, centers, leaf_ids, leaf_offs, leaf_pids, geom):
        self.ids = ids                      # int64, ascending cell IDs
        self.level = ints[:, 0].copy()
        self.ix = ints[:, 1].copy()
        self.iy = ints[:, 2].copy()
        self.par = ints[:, 3].copy()
        self.src = ints[:, 4].copy()
        self.leaf = (ints[:, 5] & 1).astype(bool)
        self.active = (ints[:, 5] & 2).astype(bool)
        self.centers = centers
        self.leaf_ids = leaf_ids            # reference leafList order
        self.leaf_offs = leaf_offs
        self.leaf_pids = leaf_pids
        self.geom = geom                    # minx maxx miny maxy root pivx pivy
        lv = int(geom[7])
        self.min_level, self.max_level = lv & 0xFFFF, lv >> 16


class Port:
    """The oracle restatement (liboracle.so)."""

    kind = "port"

    def __init__(self, path: str = _PORT):
        if not os.path.exists(path):
            build(ref=False)
        L = self.lib = C.CDLL(path)
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_tree2d_build.restype = C.c_void_p
        L.orc_tree2d_build.argtypes = [_d, _d, _u8, C.c_int64, C.c_int, C.c_int, C.c_double]
        L.orc_tree2d_free.argtypes = [C.c_void_p]
        L.orc_tree2d_ncells.restype = C.c_int64
        L.orc_tree2d_ncells.argtypes = [C.c_void_p]
        L.orc_tree2d_nleaves.restype = C.c_int64
        L.orc_tree2d_nleaves.argtypes = [C.c_void_p]
        L.orc_tree2d_geom.argtypes = [C.c_void_p, _d]
        L.orc_tree2d_cells.argtypes = [C.c_void_p, _i64, _i32, _d]
        L.orc_tree2d_leaves.argtypes = [C.c_void_p, _i64, _i64, _i32]
        L.orc_tree2d_list.argtypes = [C.c_void_p, C.c_int, _i64, C.c_int64, _i64, C.c_void_p]
        L.orc_fmm2d_field.restype = C.c_int
        L.orc_fmm2d_field.argtypes = [_d, _d, _d, _u8, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double,
                                      C.c_int, _d, _d]
        L.orc_fmm2d_potential.restype = C.c_int
        L.orc_fmm2d_potential.argtypes = [_d, _d, _d, _u8, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_int, _d]
        L.orc_direct2d_field.argtypes = [_d, _d, _d, _u8, C.c_int64, _i64, C.c_int64, _d, _d]
        L.orc_fmm3d_velocity.restype = C.c_int
        L.orc_fmm3d_velocity.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_int64, C.c_int, C.c_double, C.c_double,
                                         _d, _d, _d]
        L.orc_fmm3d_velocity_at.restype = C.c_int
        L.orc_fmm3d_velocity_at.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_int64, C.c_int, C.c_double, C.c_double,
                                            _i64, C.c_int64, _d, _d, _d]
        L.orc_tree3d.restype = C.c_int64
        L.orc_tree3d.argtypes = [_d, _d, _d, _u8, C.c_int64, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_direct3d_velocity.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_int64, _i64, C.c_int64, _d, _d, _d]
        L.orc3_last_error.restype = C.c_char_p
        L.orc_treecell3d_tree.restype = C.c_int64
        L.orc_treecell3d_tree.argtypes = [_d, _d, _d, _u8, C.c_int64, C.c_int, C.c_int, C.c_double] + [C.c_void_p] * 5
        L.orc_treecell3d_velocity.restype = C.c_int
        L.orc_treecell3d_pairs.argtypes = [_i64]
        L.orc_treecell3d_velocity.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                              C.c_double, C.c_double, _d, _d, _d]

    def set_threads(self, n: int) -> None:
        self.lib.orc_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.lib.orc_max_threads())

    # ---- 2D ---------------------------------------------------------------
    def fmm2d_field(self, x, y, q, active, p=10, max_src=50, max_par=75, exp_pct=1.0, exact_binom=False):
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8a(active)
        ex = np.zeros(x.size)
        ey = np.zeros(x.size)
        rc = self.lib.orc_fmm2d_field(x, y, q, a, x.size, p, max_src, max_par, exp_pct, int(exact_binom), ex, ey)
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())
        return ex, ey

    def fmm2d_potential(self, x, y, q, active, p=10, max_src=50, max_par=75, exp_pct=1.0, exact_binom=False):
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8a(active)
        pot = np.zeros(x.size)
        rc = self.lib.orc_fmm2d_potential(x, y, q, a, x.size, p, max_src, max_par, exp_pct, int(exact_binom), pot)
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())
        return pot

    def direct2d_field(self, x, y, q, active, targets):
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8a(active)
        t = np.ascontiguousarray(targets, dtype=np.int64)
        ex = np.zeros(t.size)
        ey = np.zeros(t.size)
        self.lib.orc_direct2d_field(x, y, q, a, x.size, t, t.size, ex, ey)
        return ex, ey

    def tree2d(self, x, y, active, max_src=50, max_par=75, exp_pct=1.0) -> Tree2D:
        x, y, a = _f64(x), _f64(y), _u8a(active)
        h = self.lib.orc_tree2d_build(x, y, a, x.size, max_src, max_par, exp_pct)
        if not h:
            raise RuntimeError(self.lib.orc_last_error().decode())
        try:
            return self._dump(h, x.size)
        finally:
            self.lib.orc_tree2d_free(h)

    def _dump(self, h, n):
        L = self.lib
        nc, nl = L.orc_tree2d_ncells(h), L.orc_tree2d_nleaves(h)
        ids = np.zeros(nc, np.int64)
        ints = np.zeros((nc, 6), np.int32)
        cen = np.zeros((nc, 2))
        L.orc_tree2d_cells(h, ids, ints.reshape(-1), cen.reshape(-1))
        lid = np.zeros(nl, np.int64)
        loff = np.zeros(nl + 1, np.int64)
        lp = np.zeros(n, np.int32)
        L.orc_tree2d_leaves(h, lid, loff, lp)
        g = np.zeros(8)
        L.orc_tree2d_geom(h, g)
        return Tree2D(ids, ints, cen, lid, loff, lp, g)

    def lists2d(self, x, y, active, which, cell_ids, max_src=50, max_par=75, exp_pct=1.0):
        """CSR (offsets, ids) of list `which` (1..4) for the given cell IDs."""
        x, y, a = _f64(x), _f64(y), _u8a(active)
        h = self.lib.orc_tree2d_build(x, y, a, x.size, max_src, max_par, exp_pct)
        if not h:
            raise RuntimeError(self.lib.orc_last_error().decode())
        try:
            cid = np.ascontiguousarray(cell_ids, dtype=np.int64)
            offs = np.zeros(cid.size + 1, np.int64)
            self.lib.orc_tree2d_list(h, which, cid, cid.size, offs, None)
            out = np.zeros(int(offs[-1]), np.int64)
            self.lib.orc_tree2d_list(h, which, cid, cid.size, offs, out.ctypes.data_as(C.c_void_p))
            return offs, out
        finally:
            self.lib.orc_tree2d_free(h)

    # ---- 3D ---------------------------------------------------------------
    def fmm3d_velocity(self, x, y, z, ax, ay, az, active, leaf_cap=30, exp_pct=1.0, support=2.0):
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        a = _u8a(active)
        n = args[0].size
        u, v, w = np.zeros(n), np.zeros(n), np.zeros(n)
        rc = self.lib.orc_fmm3d_velocity(*args, a, n, leaf_cap, exp_pct, support, u, v, w)
        if rc != 0:
            raise RuntimeError(self.lib.orc3_last_error().decode())
        return u, v, w

    def fmm3d_velocity_at(self, x, y, z, ax, ay, az, active, targets, leaf_cap=30, exp_pct=1.0, support=2.0):
        """The treecode velocity at the sampled targets only (same tree, same per-target walk)."""
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        t = np.ascontiguousarray(targets, dtype=np.int64)
        u, v, w = np.zeros(t.size), np.zeros(t.size), np.zeros(t.size)
        rc = self.lib.orc_fmm3d_velocity_at(*args, _u8a(active), args[0].size, leaf_cap, exp_pct, support, t, t.size,
                                            u, v, w)
        if rc != 0:
            raise RuntimeError(self.lib.orc3_last_error().decode())
        return u, v, w

    def tree3d(self, x, y, z, active, leaf_cap=30, exp_pct=1.0):
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8a(active)
        nc = self.lib.orc_tree3d(x, y, z, a, x.size, leaf_cap, exp_pct, None, None)
        if nc < 0:
            raise RuntimeError(self.lib.orc3_last_error().decode())
        ints = np.zeros((nc, 6), np.int32)
        geom = np.zeros((nc, 4))
        self.lib.orc_tree3d(x, y, z, a, x.size, leaf_cap, exp_pct, ints.ctypes.data_as(C.c_void_p),
                            geom.ctypes.data_as(C.c_void_p))
        return ints, geom

    def treecell3d(self, x, y, z, active, max_src=30, max_par=50, exp_pct=1.0):
        """3D TreeCell (treeCell.cpp:1043-1243, DIM 3): (ids, ints, geom, leaf particle lists), by cell ID;
        ints = parNum, srcParNum, isLeaf, isActive, level, max_level (first row)."""
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8a(active)
        out = _treecell_dump(lambda *o: self.lib.orc_treecell3d_tree(x, y, z, a, x.size, max_src, max_par, exp_pct,
                                                                      *o))
        if out is None:
            raise RuntimeError(self.lib.orc3_last_error().decode())
        return out

    def treecell3d_velocity(self, x, y, z, ax, ay, az, active, target=None, max_src=30, max_par=50, exp_pct=1.0,
                            support=2.0):
        """fmm3D::calcVelocity (target None) or calcVelocityNearBody on the 3D TreeCell; far iff
        R > support x length (the reference's support factor is 2)."""
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        n = args[0].size
        t = None if target is None else _u8a(target)
        u, v, w = np.zeros(n), np.zeros(n), np.zeros(n)
        rc = self.lib.orc_treecell3d_velocity(*args, _u8a(active), None if t is None else _vp(t), n, max_src, max_par,
                                              exp_pct, support, u, v, w)
        if rc != 0:
            raise RuntimeError(self.lib.orc3_last_error().decode())
        return u, v, w

    def treecell3d_pairs(self):
        """(P2P pairs, M2P pairs) of the last treecell3d_velocity call."""
        out = np.zeros(2, np.int64)
        self.lib.orc_treecell3d_pairs(out)
        return int(out[0]), int(out[1])

    def direct3d_velocity(self, x, y, z, ax, ay, az, active, targets):
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        t = np.ascontiguousarray(targets, dtype=np.int64)
        u, v, w = np.zeros(t.size), np.zeros(t.size), np.zeros(t.size)
        self.lib.orc_direct3d_velocity(*args, _u8a(active), args[0].size, t, t.size, u, v, w)
        return u, v, w


class Reference:
    """The reference's own FMM, compiled from its sources (oracle/_ref)."""

    kind = "reference"

    def __init__(self):
        if not ref_available():
            raise FileNotFoundError("oracle/_ref not built (needs the reference sources at build time)")
        L2 = self.lib2 = C.CDLL(_REF2)
        L2.ref2d_last_error.restype = C.c_char_p
        L2.ref2d_set.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
        L2.ref2d_field.restype = C.c_int
        L2.ref2d_field.argtypes = [_d, _d, _d, _u8, C.c_int64, _d, _d]
        L2.ref2d_potential.restype = C.c_int
        L2.ref2d_potential.argtypes = [_d, _d, _d, _u8, C.c_int64, _d]
        L2.ref2d_tree_build.restype = C.c_void_p
        L2.ref2d_tree_build.argtypes = [_d, _d, _u8, C.c_int64]
        L2.ref2d_tree_free.argtypes = [C.c_void_p]
        L2.ref2d_tree_ncells.restype = C.c_int64
        L2.ref2d_tree_ncells.argtypes = [C.c_void_p]
        L2.ref2d_tree_nleaves.restype = C.c_int64
        L2.ref2d_tree_nleaves.argtypes = [C.c_void_p]
        L2.ref2d_tree_geom.argtypes = [C.c_void_p, _d]
        L2.ref2d_tree_cells.argtypes = [C.c_void_p, _i64, _i32, _d]
        L2.ref2d_tree_leaves.argtypes = [C.c_void_p, _i64, _i64, _i32]
        L2.ref2d_tree_list.restype = C.c_int
        L2.ref2d_tree_list.argtypes = [C.c_void_p, C.c_int, _i64, C.c_int64, _i64, C.c_void_p]
        L3 = self.lib3 = C.CDLL(_REF3)
        L3.ref3d_last_error.restype = C.c_char_p
        L3.ref3d_set.argtypes = [C.c_int, C.c_double]
        L3.ref3d_velocity.restype = C.c_int
        L3.ref3d_velocity.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_int64, _d, _d, _d]
        L3.ref3d_tree.restype = C.c_int64
        L3.ref3d_tree.argtypes = [_d, _d, _d, _u8, C.c_int64, C.c_void_p, C.c_void_p]
        L3.ref3d_tc_set.argtypes = [C.c_int, C.c_int, C.c_double]
        L3.ref3d_tc_velocity.restype = C.c_int
        L3.ref3d_tc_velocity.argtypes = [_d, _d, _d, _d, _d, _d, _u8, C.c_void_p, C.c_int64, _d, _d, _d]
        L3.ref3d_tc_tree.restype = C.c_int64
        L3.ref3d_tc_tree.argtypes = [_d, _d, _d, _u8, C.c_int64] + [C.c_void_p] * 5

    def fmm2d_field(self, x, y, q, active, p=10, max_src=50, max_par=75, exp_pct=1.0, exact_binom=False):
        if exact_binom:
            raise ValueError("the reference computes its own binomials")
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8a(active)
        self.lib2.ref2d_set(p, max_src, max_par, exp_pct)
        ex, ey = np.zeros(x.size), np.zeros(x.size)
        if self.lib2.ref2d_field(x, y, q, a, x.size, ex, ey) != 0:
            raise RuntimeError(self.lib2.ref2d_last_error().decode())
        return ex, ey

    def fmm2d_potential(self, x, y, q, active, p=10, max_src=50, max_par=75, exp_pct=1.0, exact_binom=False):
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8a(active)
        self.lib2.ref2d_set(p, max_src, max_par, exp_pct)
        pot = np.zeros(x.size)
        if self.lib2.ref2d_potential(x, y, q, a, x.size, pot) != 0:
            raise RuntimeError(self.lib2.ref2d_last_error().decode())
        return pot

    def tree2d(self, x, y, active, max_src=50, max_par=75, exp_pct=1.0) -> Tree2D:
        x, y, a = _f64(x), _f64(y), _u8a(active)
        self.lib2.ref2d_set(10, max_src, max_par, exp_pct)
        h = self.lib2.ref2d_tree_build(x, y, a, x.size)
        if not h:
            raise RuntimeError(self.lib2.ref2d_last_error().decode())
        try:
            L = self.lib2
            nc, nl = L.ref2d_tree_ncells(h), L.ref2d_tree_nleaves(h)
            ids = np.zeros(nc, np.int64)
            ints = np.zeros((nc, 6), np.int32)
            cen = np.zeros((nc, 2))
            L.ref2d_tree_cells(h, ids, ints.reshape(-1), cen.reshape(-1))
            lid = np.zeros(nl, np.int64)
            loff = np.zeros(nl + 1, np.int64)
            lp = np.zeros(x.size, np.int32)
            L.ref2d_tree_leaves(h, lid, loff, lp)
            g = np.zeros(8)
            L.ref2d_tree_geom(h, g)
            return Tree2D(ids, ints, cen, lid, loff, lp, g)
        finally:
            self.lib2.ref2d_tree_free(h)

    def lists2d(self, x, y, active, which, cell_ids, max_src=50, max_par=75, exp_pct=1.0):
        x, y, a = _f64(x), _f64(y), _u8a(active)
        self.lib2.ref2d_set(10, max_src, max_par, exp_pct)
        h = self.lib2.ref2d_tree_build(x, y, a, x.size)
        if not h:
            raise RuntimeError(self.lib2.ref2d_last_error().decode())
        try:
            cid = np.ascontiguousarray(cell_ids, dtype=np.int64)
            offs = np.zeros(cid.size + 1, np.int64)
            if self.lib2.ref2d_tree_list(h, which, cid, cid.size, offs, None) != 0:
                raise RuntimeError(self.lib2.ref2d_last_error().decode())
            out = np.zeros(int(offs[-1]), np.int64)
            self.lib2.ref2d_tree_list(h, which, cid, cid.size, offs, out.ctypes.data_as(C.c_void_p))
            return offs, out
        finally:
            self.lib2.ref2d_tree_free(h)

    def fmm3d_velocity(self, x, y, z, ax, ay, az, active, leaf_cap=30, exp_pct=1.0):
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        n = args[0].size
        self.lib3.ref3d_set(leaf_cap, exp_pct)
        u, v, w = np.zeros(n), np.zeros(n), np.zeros(n)
        if self.lib3.ref3d_velocity(*args, _u8a(active), n, u, v, w) != 0:
            raise RuntimeError(self.lib3.ref3d_last_error().decode())
        return u, v, w

    def tree3d(self, x, y, z, active, leaf_cap=30, exp_pct=1.0):
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8a(active)
        self.lib3.ref3d_set(leaf_cap, exp_pct)
        nc = self.lib3.ref3d_tree(x, y, z, a, x.size, None, None)
        if nc < 0:
            raise RuntimeError(self.lib3.ref3d_last_error().decode())
        ints = np.zeros((nc, 6), np.int32)
        geom = np.zeros((nc, 4))
        self.lib3.ref3d_tree(x, y, z, a, x.size, ints.ctypes.data_as(C.c_void_p), geom.ctypes.data_as(C.c_void_p))
        return ints, geom

    def treecell3d(self, x, y, z, active, max_src=30, max_par=50, exp_pct=1.0):
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8a(active)
        self.lib3.ref3d_tc_set(max_src, max_par, exp_pct)
        out = _treecell_dump(lambda *o: self.lib3.ref3d_tc_tree(x, y, z, a, x.size, *o))
        if out is None:
            raise RuntimeError(self.lib3.ref3d_last_error().decode())
        return out

    def treecell3d_velocity(self, x, y, z, ax, ay, az, active, target=None, max_src=30, max_par=50, exp_pct=1.0):
        args = [_f64(v) for v in (x, y, z, ax, ay, az)]
        n = args[0].size
        t = None if target is None else _u8a(target)
        self.lib3.ref3d_tc_set(max_src, max_par, exp_pct)
        u, v, w = np.zeros(n), np.zeros(n), np.zeros(n)
        if self.lib3.ref3d_tc_velocity(*args, _u8a(active), None if t is None else _vp(t), n, u, v, w) != 0:
            raise RuntimeError(self.lib3.ref3d_last_error().decode())
        return u, v, w
