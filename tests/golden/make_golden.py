"""Generate the golden fixtures from the reference's own FMM.

Runs here only (it needs oracle/_ref, built from the reference sources by
`make -C oracle ref`). Each fixture holds a seeded input set and the
reference's outputs: the tree dump (cells by ID, leafList, parIDList), lists
1-4, the field (calcField) and the potential (calcPotential) for 2D; the
treecode velocity and octree dump for 3D; for the 3D TreeCell path the cell
dump by ID and the velocities of calcVelocity and calcVelocityNearBody.

    python tests/golden/make_golden.py [case ...]   (all cases when none is named)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import Reference  # noqa: E402

import cases2d  # noqa: E402
from lsmps_vpm_v2_b200 import workloads  # noqa: E402

CASES_2D = [("lamb_small", 10, 50, 75), ("clustered", 10, 50, 75), ("partly_inactive", 10, 50, 75),
            ("aspect", 10, 50, 75), ("boundary_aligned", 16, 50, 75), ("clustered", 16, 20, 30),
            ("tiny300", 8, 50, 75), ("state500", 10, 50, 75)]


def main():
    ref = Reference()
    only = set(sys.argv[1:])
    for name, p, ms, mp in CASES_2D:
        if only and name not in only:
            continue
        d = cases2d.CASES[name]()
        x, y, q, a = d["x"], d["y"], d["q"], d["active"]
        t = ref.tree2d(x, y, a, max_src=ms, max_par=mp)
        out = dict(x=x, y=y, q=q, active=a, p=p, max_src=ms, max_par=mp, ids=t.ids,
                   ints=np.stack([t.level, t.ix, t.iy, t.par, t.src, t.leaf.astype(np.int32) | (t.active.astype(np.int32) << 1)], 1),
                   centers=t.centers, leaf_ids=t.leaf_ids, leaf_offs=t.leaf_offs, leaf_pids=t.leaf_pids, geom=t.geom)
        for which in (1, 2, 3, 4):
            cells = t.leaf_ids if which in (1, 3) else t.ids[t.level >= 2]
            offs, ids = ref.lists2d(x, y, a, which, cells, max_src=ms, max_par=mp)
            out[f"l{which}_cells"], out[f"l{which}_offs"], out[f"l{which}_ids"] = cells, offs, ids
        ex, ey = ref.fmm2d_field(x, y, q, a, p=p, max_src=ms, max_par=mp)
        pot = ref.fmm2d_potential(x, y, q, a, p=p, max_src=ms, max_par=mp)
        out.update(ex=ex, ey=ey, pot=pot)
        fn = os.path.join(HERE, f"fmm2d_{name}_p{p}_{ms}_{mp}.npz")
        np.savez_compressed(fn, **out)
        print(fn, x.size, t.ids.size)
    if not only or "treecell3d" in only:
        treecell3d(ref)
    if only and "ring3d" not in only:
        return
    # 3D treecode on a coarse ring.
    r = workloads.vortex_ring_3d(h=0.05)
    args = [r[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    u, v, w = ref.fmm3d_velocity(*args, r["active"], leaf_cap=30)
    ints, geom = ref.tree3d(r["x"], r["y"], r["z"], r["active"], leaf_cap=30)
    fn = os.path.join(HERE, "fmm3d_ring_h005.npz")
    np.savez_compressed(fn, x=r["x"], y=r["y"], z=r["z"], ax=r["ax"], ay=r["ay"], az=r["az"],
                        active=r["active"], u=u, v=v, w=w, ints=ints, geom=geom)
    print(fn, r["x"].size, ints.shape[0])



def treecell3d(ref):
    """3D TreeCell path on a coarse ring with every tenth particle inactive
    (inactive particles are P2P sources there) and every seventh a target."""
    r = workloads.vortex_ring_3d(h=0.05, seed=11)
    n = r["x"].size
    act = r["active"].copy()
    act[::10] = 0
    tgt = np.zeros(n, np.uint8)
    tgt[::7] = 1
    args = [r[k] for k in ("x", "y", "z", "ax", "ay", "az")]
    ids, ints, geom, leaves = ref.treecell3d(r["x"], r["y"], r["z"], act, max_src=30, max_par=50)
    offs = np.concatenate([[0], np.cumsum([len(v) for v in leaves])]).astype(np.int64)
    pids = np.concatenate(leaves).astype(np.int32)
    u, v, w = ref.treecell3d_velocity(*args, act, None, max_src=30, max_par=50)
    ub, vb, wb = ref.treecell3d_velocity(*args, act, tgt, max_src=30, max_par=50)
    fn = os.path.join(HERE, "treecell3d_ring_h005_30_50.npz")
    np.savez_compressed(fn, x=r["x"], y=r["y"], z=r["z"], ax=r["ax"], ay=r["ay"], az=r["az"], active=act,
                        target=tgt, ids=ids, ints=ints, geom=geom, leaf_offs=offs, leaf_pids=pids, u=u, v=v, w=w,
                        u_nb=ub, v_nb=vb, w_nb=wb)
    print(fn, n, ids.size)


if __name__ == "__main__":
    main()
