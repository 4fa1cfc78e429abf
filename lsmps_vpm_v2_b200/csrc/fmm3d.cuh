// Device data layout of one 3D evaluation: the octree treecode of the
// reference's default 3D velocity path (fmm3D::calcVelocityFast,
// src/FMM/fmm3D.cpp + src/FMM/fast3DFMM.cpp).
//
// Cells are level-major; within a level they are grouped by parent (in the
// parent order of the level above) and, under one parent, in octant order
// 0..7 (octant = [x > xc] + 2 [y > yc] + 4 [z > zc], fast3DFMM.hpp:17-22).
// The reference numbers cells in creation order instead (first particle to
// reach an octant); the cells themselves - centres, sizes, counts, flags -
// are identical, only their numbering differs. Particles are reordered so
// every leaf holds a contiguous range [lo, hi) in ascending original index
// (the reference's parID order); `perm` maps a sorted slot to the caller's
// index.
#pragma once

#include "prims.cuh"

namespace vpm {

constexpr int kMaxLevels3D = 60;     // octree depth limit (coincident particles)
constexpr int kWork3DCap = 512;      // union work list of one leaf's traversal, per level
constexpr int kEval3DWarps = 4;      // warps (leaves) per evaluation block
constexpr int kCoopMaxBlocks3D = 148 * 8;  // size of the per-block scan partials

// Geometry record of the bounding-box kernel (fast3DFMM.cpp:485-520 with the
// domain centre joined in, global.cpp:609-611).
struct Geom3D {
    double mn[3], mx[3];
    double cen[3];
    double root;
};

struct TreeInfo3D {
    int level_start[kMaxLevels3D + 2];  // first cell index of each level
    int n_cells;
    int n_leaves;
    int depth;            // deepest level holding a cell (reference max_level)
    int remaining;        // particles not yet settled in a leaf (build only)
    int scan_total;       // children created at the level being built
    int pad[3];
    unsigned long long p2p_pairs, m2p_pairs;
};

struct Tree3D {
    int n;
    int cap_cells;
    int leaf_cap;         // leaf iff particle count < leaf_cap
    Geom3D* geom;
    TreeInfo3D* info;
    // particles in leaf order
    uint32_t* perm;                   // sorted slot -> caller index
    double *px, *py, *pz, *ax, *ay, *az;
    uint8_t* pact;
    // per caller-index build state
    int32_t* pcell;                   // current cell of each particle
    uint8_t* settled;
    uint8_t* poct;                    // octant at the level being built
    // cells
    double *c_x, *c_y, *c_z, *c_size;
    int32_t *c_npar, *c_parent, *c_child0, *c_lo, *c_hi;
    uint32_t* c_chmask;               // child octants present (reference chdFlag)
    uint8_t *c_active, *c_level;
    double* mom;                      // [cap_cells][30]: moments of alpha_x, alpha_y, alpha_z
    int32_t* leaf_cells;              // leaves in cell order
    unsigned* gbar;                   // grid barrier words (2), zeroed per evaluation
    uint32_t* blk;                    // per-block scan partials [gridDim]
};

// Scratch of the 3D build (sort of particles by leaf).
struct Scratch3D {
    uint32_t *key_a, *key_b, *val_a, *val_b;
    SortScratch sort;
};

// Bounding box, octree, leaf order, P2M and M2M, all enqueued on `st`.
// center = the domain centre joined into the root box (Pars::xcenter etc.).
cudaError_t build_tree3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                         const double* az, const uint8_t* act, const double center[3], double exp_pct, Tree3D& t,
                         Scratch3D& s, double* bbox_partial, unsigned* err, cudaStream_t st, int* launches);

// Per-target traversal (M2P of far cells, P2P of near leaves) writing the
// velocity u = sum alpha x r / |r|^3 (+ free stream) in the caller's order.
// mixed: FP32 arithmetic for the P2P and M2P terms (FP64 geometry and
// decisions, FP64 accumulation per target).
cudaError_t eval3d(const Tree3D& t, bool mixed, double* u, double* v, double* w, double uinf, double vinf,
                   double winf, unsigned* err, cudaStream_t st, int* launches);

}  // namespace vpm
