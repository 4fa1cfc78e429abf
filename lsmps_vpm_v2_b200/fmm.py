"""Host-side front end of the B200 FMM velocity step.

``Context`` wraps one ``vpm_ctx`` (device buffers, stream). On top of it sit
mirrors of the reference's operator interface for this path, with the same
names, argument meaning and error behaviour (exceptions on failure):

* ``TreeCell``      — src/FMM/treeCell.hpp:83-195 (initializeTree, intList,
                      extList, leafList, min_level / max_level)
* ``fmm2D``         — src/FMM/fmm2D.hpp:15-68 (calcField, get_Field_x/y)
* ``Particle``, ``VelocityCalc`` — Utils.hpp:77-159 and
  src/velocity_calculation/velocity_calc.hpp:15-47 (get_velocity with the 2D
  FMM branch, velocity_calc.cpp:455-578)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import Params, Stats, VpmError, default_params, lib, treecell3d_params


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """One device context: buffers, stream and the last tree (for dumps)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().vpm_ctx_create(int(device), C.byref(self._h))
        if st != 0:
            raise VpmError(st, "vpm_ctx_create failed")
        self.device = device

    def close(self):
        if self._h:
            lib().vpm_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise VpmError(st, lib().vpm_last_error(self._h).decode())

    def set_stream(self, stream_ptr: int | None):
        self._check(lib().vpm_ctx_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def sync(self):
        self._check(lib().vpm_ctx_sync(self._h))

    # ---- 2D -----------------------------------------------------------------
    def field2d(self, x, y, q, active, params: Params | None = None, stats: bool = False):
        """(Ex, Ey) of the reference's fmm2D::calcField, host arrays in/out."""
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8(active)
        n = x.size
        ex, ey = np.empty(n), np.empty(n)
        p = params or default_params()
        s = Stats()
        self._check(lib().vpm_fmm2d_field(self._h, _ptr(x), _ptr(y), _ptr(q), _ptr(a), n, C.byref(p),
                                          _ptr(ex), _ptr(ey), C.byref(s) if stats else None))
        return (ex, ey, s) if stats else (ex, ey)

    def field2d_batched(self, solves, params: Params | None = None):
        """Independent 2D solves in one call. `solves` is a list of (x, y, q,
        active) tuples; returns a list of (ex, ey)."""
        sizes = [np.asarray(s[0]).size for s in solves]
        offs = np.zeros(len(solves) + 1, np.int64)
        offs[1:] = np.cumsum(sizes)
        cat = [np.ascontiguousarray(np.concatenate([np.asarray(s[k], dtype=np.float64) for s in solves]))
               for k in range(3)]
        act = np.ascontiguousarray(np.concatenate([np.asarray(s[3], dtype=np.uint8) for s in solves]))
        ex, ey = np.empty(int(offs[-1])), np.empty(int(offs[-1]))
        p = params or default_params()
        self._check(lib().vpm_fmm2d_field_batched(self._h, len(solves), _ptr(offs), _ptr(cat[0]), _ptr(cat[1]),
                                                  _ptr(cat[2]), _ptr(act), C.byref(p), _ptr(ex), _ptr(ey)))
        return [(ex[offs[i]:offs[i + 1]], ey[offs[i]:offs[i + 1]]) for i in range(len(solves))]

    def field2d_batched_device(self, offsets, x, y, q, active, ex, ey, params: Params | None = None):
        """Device-pointer batch (integers such as torch data_ptr()); offsets is
        a host int64 array of n_solves + 1 entries. Asynchronous."""
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        p = params or default_params()
        self._check(lib().vpm_fmm2d_field_batched_device(self._h, offs.size - 1, _ptr(offs), x, y, q, active,
                                                         C.byref(p), ex, ey))

    def batch_streams(self) -> int:
        """Streams the last batched call ran on (tuned on the first graph call of a layout)."""
        v = C.c_int32()
        self._check(lib().vpm_batch_streams(self._h, C.byref(v)))
        return int(v.value)

    def potential2d(self, x, y, q, active, params: Params | None = None, stats: bool = False):
        """phi_i = sum_j q_j log|x_i - x_j| by the 2D FMM (host arrays)."""
        x, y, q, a = _f64(x), _f64(y), _f64(q), _u8(active)
        phi = np.empty(x.size)
        p = params or default_params()
        st = Stats()
        self._check(lib().vpm_fmm2d_potential(self._h, _ptr(x), _ptr(y), _ptr(q), _ptr(a), x.size, C.byref(p),
                                              _ptr(phi), C.byref(st) if stats else None))
        return (phi, st) if stats else phi

    def field2d_device(self, x, y, q, active, ex, ey, params: Params | None = None):
        """Asynchronous field on device buffers (objects with .data_ptr(), e.g. torch CUDA tensors)."""
        p = params or default_params()
        n = int(x.numel())
        self._check(lib().vpm_fmm2d_field_device(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                 C.c_void_p(q.data_ptr()), C.c_void_p(active.data_ptr()), n,
                                                 C.byref(p), C.c_void_p(ex.data_ptr()), C.c_void_p(ey.data_ptr())))

    STAGES = ("keys_sort", "levels", "lists", "upward", "m2l", "l2l", "eval", "p2p")

    def stage_history(self, enable: bool = True, max_entries: int = 64):
        """Stage times (ms, one row per evaluation, columns STAGES) recorded
        since the last call; recording stays on if `enable`."""
        ms = np.zeros((max_entries, len(self.STAGES)), np.float32)
        cnt = C.c_int32()
        self._check(lib().vpm_stage_history(self._h, int(enable), max_entries, _ptr(ms), C.byref(cnt)))
        return ms[: cnt.value]

    def velocity2d(self, x, y, omega, s, active, u_inf=0.0, v_inf=0.0, params: Params | None = None,
                   stats: bool = False, out=None):
        """u = Ey + u_inf, v = -Ex + v_inf (host arrays). `out` = (u, v)
        preallocated float64 arrays (e.g. pinned) to write into."""
        x, y, w, sz, a = _f64(x), _f64(y), _f64(omega), _f64(s), _u8(active)
        n = x.size
        if out is not None:
            u, v = out
            assert u.dtype == np.float64 and v.dtype == np.float64 and u.flags.c_contiguous and v.flags.c_contiguous
        else:
            u, v = np.empty(n), np.empty(n)
        p = params or default_params()
        st = Stats()
        self._check(lib().vpm_velocity2d(self._h, _ptr(x), _ptr(y), _ptr(w), _ptr(sz), _ptr(a), n, C.byref(p),
                                         float(u_inf), float(v_inf), _ptr(u), _ptr(v),
                                         C.byref(st) if stats else None))
        return (u, v, st) if stats else (u, v)

    def velocity3d_alpha(self, x, y, z, ax, ay, az, active, params: Params | None = None, stats: bool = False):
        """u = sum_j alpha_j x r / |r|^3 by the octree treecode (host arrays)."""
        x, y, z = _f64(x), _f64(y), _f64(z)
        ax, ay, az, a = _f64(ax), _f64(ay), _f64(az), _u8(active)
        n = x.size
        u, v, w = np.empty(n), np.empty(n), np.empty(n)
        p = params or default_params()
        st = Stats()
        self._check(lib().vpm_fmm3d_velocity(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(ax), _ptr(ay), _ptr(az),
                                             _ptr(a), None, n, C.byref(p), _ptr(u), _ptr(v), _ptr(w),
                                             C.byref(st) if stats else None))
        return (u, v, w, st) if stats else (u, v, w)

    def velocity3d(self, x, y, z, wx, wy, wz, s, active, u_inf=0.0, v_inf=0.0, w_inf=0.0,
                   params: Params | None = None, stats: bool = False):
        """alpha = omega s^3 / (4 pi), then the treecode velocity plus the free stream."""
        x, y, z = _f64(x), _f64(y), _f64(z)
        wx, wy, wz, sz, a = _f64(wx), _f64(wy), _f64(wz), _f64(s), _u8(active)
        n = x.size
        u, v, w = np.empty(n), np.empty(n), np.empty(n)
        p = params or default_params()
        st = Stats()
        self._check(lib().vpm_velocity3d(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(wx), _ptr(wy), _ptr(wz), _ptr(sz),
                                         _ptr(a), n, C.byref(p), float(u_inf), float(v_inf), float(w_inf), _ptr(u),
                                         _ptr(v), _ptr(w), C.byref(st) if stats else None))
        return (u, v, w, st) if stats else (u, v, w)

    def velocity3d_device(self, n, x, y, z, ax, ay, az, active, u, v, w, params: Params | None = None):
        """Device-pointer form with an explicit particle count, asynchronous."""
        p = params or default_params()
        self._check(lib().vpm_fmm3d_velocity_device(self._h, x, y, z, ax, ay, az, active, int(n), C.byref(p),
                                                    u, v, w))

    def velocity3d_treecell(self, x, y, z, ax, ay, az, active, target=None, params: Params | None = None,
                            stats: bool = False):
        """u = sum_j alpha_j x r / |r|^3 by the treecode on the 3D TreeCell (host
        arrays); target flags select the evaluated particles (others zero)."""
        x, y, z = _f64(x), _f64(y), _f64(z)
        ax, ay, az, a = _f64(ax), _f64(ay), _f64(az), _u8(active)
        t = None if target is None else _u8(target)
        n = x.size
        u, v, w = np.empty(n), np.empty(n), np.empty(n)
        p = params or treecell3d_params()
        st = Stats()
        self._check(lib().vpm_fmm3d_velocity_treecell(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(ax), _ptr(ay),
                                                      _ptr(az), _ptr(a), None if t is None else _ptr(t), n,
                                                      C.byref(p), _ptr(u), _ptr(v), _ptr(w),
                                                      C.byref(st) if stats else None))
        return (u, v, w, st) if stats else (u, v, w)

    def velocity3d_treecell_device(self, n, x, y, z, ax, ay, az, active, target, u, v, w,
                                   params: Params | None = None):
        """Device-pointer form (target may be None), asynchronous."""
        p = params or treecell3d_params()
        self._check(lib().vpm_fmm3d_velocity_treecell_device(self._h, x, y, z, ax, ay, az, active, target, int(n),
                                                             C.byref(p), u, v, w))

    def build_treecell3d(self, x, y, z, active, params: Params | None = None) -> Stats:
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8(active)
        p = params or treecell3d_params()
        s = Stats()
        self._check(lib().vpm_treecell3d_build(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(a), x.size, C.byref(p),
                                               C.byref(s)))
        return s

    def tree3d_cell_ids(self) -> np.ndarray:
        """Reference cell IDs of the last 3D TreeCell, in library cell order."""
        nc, nl, depth = C.c_int64(), C.c_int64(), C.c_int32()
        self._check(lib().vpm_tree3d_counts(self._h, C.byref(nc), C.byref(nl), C.byref(depth)))
        ids = np.zeros(nc.value, np.int64)
        self._check(lib().vpm_tree3d_cell_ids(self._h, _ptr(ids)))
        return ids

    def build_tree3d(self, x, y, z, active, params: Params | None = None) -> Stats:
        x, y, z, a = _f64(x), _f64(y), _f64(z), _u8(active)
        p = params or default_params()
        s = Stats()
        self._check(lib().vpm_tree3d_build(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(a), x.size, C.byref(p),
                                           C.byref(s)))
        return s

    def dump_tree3d(self):
        """The last octree: per cell (library order) nPar, chdFlag, parent,
        isActive, level and geometry (xc, yc, zc, size), plus each leaf's
        particle IDs (CSR over cells)."""
        nc, nl, depth = C.c_int64(), C.c_int64(), C.c_int32()
        self._check(lib().vpm_tree3d_counts(self._h, C.byref(nc), C.byref(nl), C.byref(depth)))
        nc = nc.value
        ints = np.zeros((nc, 6), np.int32)
        geom = np.zeros((nc, 4))
        offs = np.zeros(nc + 1, np.int64)
        self._check(lib().vpm_tree3d_cells(self._h, _ptr(ints), _ptr(geom), _ptr(offs), None))
        pids = np.zeros(max(int(offs[-1]), 1), np.int32)
        self._check(lib().vpm_tree3d_cells(self._h, None, None, _ptr(offs), _ptr(pids)))
        return dict(npar=ints[:, 0], chd=ints[:, 1], parent=ints[:, 2], active=ints[:, 3].astype(bool),
                    level=ints[:, 4], depth=int(depth.value), n_leaves=int(nl.value), geom=geom, leaf_offs=offs,
                    leaf_pids=pids[: int(offs[-1])])

    def fma_peaks(self):
        """(FP64, FP32) FMA throughput of the device in TFLOP/s."""
        a, b = C.c_double(), C.c_double()
        self._check(lib().vpm_measure_fma_peaks(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def rcp_peak(self):
        """FP32 reciprocal (rcp.approx) throughput of the device in G/s."""
        a = C.c_double()
        self._check(lib().vpm_measure_rcp_peak(self._h, C.byref(a)))
        return a.value

    def last_stats(self) -> Stats:
        s = Stats()
        self._check(lib().vpm_last_stats(self._h, C.byref(s)))
        return s

    def build_tree2d(self, x, y, active, params: Params | None = None) -> Stats:
        x, y, a = _f64(x), _f64(y), _u8(active)
        p = params or default_params()
        s = Stats()
        self._check(lib().vpm_tree2d_build(self._h, _ptr(x), _ptr(y), _ptr(a), x.size, C.byref(p), C.byref(s)))
        return s

    def dump_tree2d(self):
        """The last 2D tree in the reference's vocabulary (see include/vpm_fmm.h)."""
        nc, nl = C.c_int64(), C.c_int64()
        ll = (C.c_int64 * 4)()
        self._check(lib().vpm_tree2d_counts(self._h, C.byref(nc), C.byref(nl), ll))
        nc, nl = nc.value, nl.value
        ids = np.zeros(nc, np.int64)
        ints = np.zeros((nc, 6), np.int32)
        cen = np.zeros((nc, 2))
        self._check(lib().vpm_tree2d_cells(self._h, _ptr(ids), _ptr(ints), _ptr(cen)))
        n = int(ints[0, 3]) if nc else 0
        lid = np.zeros(nl, np.int64)
        loff = np.zeros(nl + 1, np.int64)
        lp = np.zeros(max(n, 1), np.int32)
        self._check(lib().vpm_tree2d_leaves(self._h, _ptr(lid), _ptr(loff), _ptr(lp)))
        lists = {}
        for which in (1, 2, 3, 4):
            m = nl if which in (1, 3) else int(np.count_nonzero(ints[:, 0] >= 2))
            cid = np.zeros(m, np.int64)
            offs = np.zeros(m + 1, np.int64)
            out = np.zeros(max(int(ll[which - 1]), 1), np.int64)
            self._check(lib().vpm_tree2d_list(self._h, which, _ptr(cid), _ptr(offs), _ptr(out)))
            lists[which] = (cid, offs, out[: int(offs[-1])])
        return dict(ids=ids, level=ints[:, 0], ix=ints[:, 1], iy=ints[:, 2], par=ints[:, 3], src=ints[:, 4],
                    leaf=(ints[:, 5] & 1).astype(bool), active=(ints[:, 5] & 2).astype(bool), centers=cen,
                    leaf_ids=lid, leaf_offs=loff, leaf_pids=lp[:n], lists=lists)


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ---- mirrors of the reference's operator interface ---------------------------

class TreeCell:
    """Mirror of TreeCell (src/FMM/treeCell.hpp:83-195) backed by the GPU tree.

    Cells are addressed by the reference's cell ID; lists come from the GPU
    interaction lists."""

    def __init__(self, ctx: Context | None = None, params: Params | None = None):
        self.ctx = ctx or default_context()
        self.params = params or default_params()
        self.min_level = 2
        self.max_level = 2
        self.leafList: list[int] = []
        self.cellCount = 0
        self._dump = None

    def initializeTree(self, parPos, activeFlag):
        pos = np.asarray(parPos, dtype=np.float64)
        s = self.ctx.build_tree2d(pos[:, 0], pos[:, 1], np.asarray(activeFlag, dtype=np.uint8), self.params)
        self._dump = self.ctx.dump_tree2d()
        self.min_level, self.max_level = int(s.min_level), int(s.max_level)
        self.leafList = [int(v) for v in self._dump["leaf_ids"]]
        self.cellCount = int(s.n_cells)

    updateTree = initializeTree  # the reference rebuilds too (treeCell.cpp:1245-1249)

    def _list(self, which, cell_id):
        cid, offs, out = self._dump["lists"][which]
        k = int(np.searchsorted(cid, cell_id))
        if k >= cid.size or cid[k] != cell_id:
            raise IndexError(f"cell {cell_id} has no list {which}")
        return [int(v) for v in out[offs[k]:offs[k + 1]]]

    def intList(self, currID):
        """(list 1, list 3) of a leaf."""
        return self._list(1, currID), self._list(3, currID)

    def extList(self, currID):
        """(list 2, list 4) of a cell at level >= 2."""
        return self._list(2, currID), self._list(4, currID)


class fmm2D:
    """Mirror of fmm2D (src/FMM/fmm2D.hpp:15-68) on the GPU FMM."""

    def __init__(self, ctx: Context | None = None, params: Params | None = None):
        self.ctx = ctx or default_context()
        self.params = params or default_params()
        self._ex = self._ey = self._phi = None
        self.stats: Stats | None = None

    def calcField(self, _cellTree, parPos, activeFlag, srcVal):
        """The tree argument is accepted for interface parity; the GPU rebuilds
        it from the particles (the reference's tree is also a pure function of
        positions and marks)."""
        pos = np.asarray(parPos, dtype=np.float64)
        self._ex, self._ey, self.stats = self.ctx.field2d(pos[:, 0], pos[:, 1], srcVal, activeFlag, self.params,
                                                          stats=True)

    def get_Field_x(self):
        return self._ex

    def get_Field_y(self):
        return self._ey

    def calcPotential(self, _cellTree, parPos, activeMark, srcVal):
        """fmm2D::calcPotential (fmm2D.cpp:681-896) on the GPU FMM."""
        pos = np.asarray(parPos, dtype=np.float64)
        self._phi, self.stats = self.ctx.potential2d(pos[:, 0], pos[:, 1], srcVal, activeMark, self.params,
                                                     stats=True)

    def get_Potential(self):
        return self._phi


class fmm3D:
    """Mirror of fmm3D (src/FMM/fmm3D.hpp:106-138): the fast path
    calcVelocityFast, the TreeCell path calcVelocity / calcVelocityNearBody,
    and get_Field_x/y/z, on the GPU treecode."""

    def __init__(self, ctx: Context | None = None, params: Params | None = None):
        self.ctx = ctx or default_context()
        self.params = params or default_params()
        self._tc_params = params or treecell3d_params()
        self._u = self._v = self._w = None
        self.stats: Stats | None = None

    def calcVelocity(self, cellData, parPos, activeMark, alphaX, alphaY, alphaZ):
        """fmm3D::calcVelocity (fmm3D.cpp:1064-1405) on the 3D TreeCell of the
        same particles, built on the GPU in the same call; `cellData` is
        accepted for the reference's signature. Leaf caps: this object's params
        if given, else the reference's 3D 30/50."""
        self._treecell(parPos, activeMark, None, alphaX, alphaY, alphaZ)

    def calcVelocityNearBody(self, cellData, parPos, activeMark, targetFlag, alphaX, alphaY, alphaZ):
        """fmm3D::calcVelocityNearBody (fmm3D.cpp:1406-1606): only flagged
        targets are evaluated, the others get zero."""
        self._treecell(parPos, activeMark, targetFlag, alphaX, alphaY, alphaZ)

    def _treecell(self, parPos, activeMark, target, ax, ay, az):
        pos = np.asarray(parPos, dtype=np.float64)
        self._u, self._v, self._w, self.stats = self.ctx.velocity3d_treecell(
            pos[:, 0], pos[:, 1], pos[:, 2], ax, ay, az, activeMark, target, self._tc_params, stats=True)

    def calcVelocityFast(self, _parPos, _activeFlag, _targetFlag, _alphaX, _alphaY, _alphaZ):
        """The target flags are accepted and ignored, as the reference ignores them."""
        pos = np.asarray(_parPos, dtype=np.float64)
        self._u, self._v, self._w, self.stats = self.ctx.velocity3d_alpha(
            pos[:, 0], pos[:, 1], pos[:, 2], _alphaX, _alphaY, _alphaZ, _activeFlag, self.params, stats=True)

    def get_Field_x(self):
        return self._u

    def get_Field_y(self):
        return self._v

    def get_Field_z(self):
        return self._w


@dataclass
class Particle:
    """The fields of the reference's Particle (Utils.hpp:77-159) that the
    velocity step reads and writes."""
    x: np.ndarray
    y: np.ndarray
    s: np.ndarray
    vorticity: np.ndarray
    isActive: np.ndarray
    z: np.ndarray | None = None
    vortx: np.ndarray | None = None
    vorty: np.ndarray | None = None
    vortz: np.ndarray | None = None
    u: np.ndarray = field(default_factory=lambda: np.zeros(0))
    v: np.ndarray = field(default_factory=lambda: np.zeros(0))
    w: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @property
    def num(self) -> int:
        return int(np.asarray(self.x).size)


class VelocityCalc:
    """Mirror of VelocityCalc::get_velocity (velocity_calc.cpp:48-139) for the
    FMM branches: 2D (VELOCITY_2D_TYPE 2) u = Ey + u_inf, v = -Ex + v_inf;
    3D (VELOCITY_3D_TYPE 1, velocity_fmm_3d_fast) when the particles carry z,
    u = treecode velocity of alpha = omega s^3 / (4 pi) plus the free stream."""

    def __init__(self, ctx: Context | None = None, params: Params | None = None, u_inf: float = 0.0,
                 v_inf: float = 0.0, w_inf: float = 0.0):
        self.ctx = ctx or default_context()
        self.params = params or default_params()
        self.u_inf, self.v_inf, self.w_inf = u_inf, v_inf, w_inf
        self.stats: Stats | None = None

    def get_velocity(self, p: Particle, step: int = 0) -> None:
        if p.z is not None:
            u, v, w, self.stats = self.ctx.velocity3d(p.x, p.y, p.z, p.vortx, p.vorty, p.vortz, p.s, p.isActive,
                                                      self.u_inf, self.v_inf, self.w_inf, self.params, stats=True)
            p.u, p.v, p.w = u, v, w
            return
        u, v, self.stats = self.ctx.velocity2d(p.x, p.y, p.vorticity, p.s, p.isActive, self.u_inf, self.v_inf,
                                               self.params, stats=True)
        p.u, p.v = u, v
