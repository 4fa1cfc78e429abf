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
constexpr int kWork3DCap = 512;      // union work list of a warp's traversal per level, at support
                                     // factor 2 (eval3d scales it for larger factors)
constexpr int kEval3DWarps = 4;      // warps (leaves) per evaluation block
constexpr int kCoopMaxBlocks3D = 148 * 8;  // size of the per-block scan partials

// Geometry record of the bounding-box kernel (fast3DFMM.cpp:485-520 with the
// domain centre joined in, global.cpp:609-611).
struct Geom3D {
    double mn[3], mx[3];
    double cen[3];
    double root;
    double piv[3];        // TreeCell pivot (lower corner of the root box)
};

// Deepest level of the 3D TreeCell: its cell IDs (8^L - 1) / 7 + ix + iy 2^L +
// iz 4^L are 32-bit ints in the reference (treeCell.cpp:223-250) and overflow
// from level 11 on. Keys hold 3 bits per level.
constexpr int kTcLevels = 10;
constexpr int kTcTile = 1024;   // particles per tile of the level-count scan

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
    // mixed form: FP32 copies made once per evaluation (prep3d_f32)
    float4* ps32;                     // position minus its leaf's centre, active flag in .w
    float4* as32;                     // alpha
    float* mom32;                     // [cap_cells][30]
    int32_t* leaf_cells;              // leaves in cell order
    unsigned* gbar;                   // grid barrier words (2), zeroed per evaluation
    uint32_t* blk;                    // per-block scan partials [gridDim]
};

// Scratch of the 3D build (sort of particles by leaf; the TreeCell build's
// active-count scan, per-particle level record, per-tile level counts and
// per-cell Morton prefixes).
struct Scratch3D {
    uint32_t *key_a, *key_b, *val_a, *val_b;
    SortScratch sort;
    uint32_t *tc_act, *tc_scan, *tc_pinfo, *tc_tile, *tc_tot, *tc_code;
    ScanScratch scan;
    int tc_tiles;
};

// Bounding box, octree, leaf order, P2M and M2M, all enqueued on `st`.
// center = the domain centre joined into the root box (Pars::xcenter etc.).
cudaError_t build_tree3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                         const double* az, const uint8_t* act, const double center[3], double exp_pct, Tree3D& t,
                         Scratch3D& s, double* bbox_partial, unsigned* err, cudaStream_t st, int* launches);

// The same for the reference's 3D TreeCell (TreeCell::initializeTree with DIM
// 3, treeCell.cpp:1043-1243): the root box is the particle box alone, a cell is
// a leaf iff it holds at most max_src active and at most max_par particles,
// cells are the absolute-grid boxes of the pivot. The result uses the same
// Tree3D layout (level-major, Morton order within a level = parents in order
// and children in the reference's child order under a parent). Sets ERR_DEPTH
// past level 10 and ERR_LEAF1 when a level-1 cell of a deeper tree is a leaf.
cudaError_t build_treecell3d(const double* x, const double* y, const double* z, const double* ax,
                             const double* ay, const double* az, const uint8_t* act, int max_src, int max_par,
                             double exp_pct, Tree3D& t, Scratch3D& s, double* bbox_partial, unsigned* err,
                             cudaStream_t st, int* launches);

// FP32 copies for the mixed traversal: each particle's offset from its
// leaf's centre (formed in FP64, rounded once) with its active flag, its
// alpha, and every cell's moments.
cudaError_t prep3d_f32(const Tree3D& t, unsigned* err, cudaStream_t st, int* launches);

// Per-target traversal (M2P of far cells, P2P of near leaves) writing the
// velocity u = sum alpha x r / |r|^3 (+ free stream) in the caller's order.
// mixed: FP32 arithmetic for the P2P and M2P terms (FP64 geometry and
// decisions, FP64 accumulation per target). all_src: every particle of a near
// leaf is a P2P source (TreeCell path, fmm3D.cpp:1337-1352) instead of the
// active ones only (octree path). target (caller order, may be null): only
// flagged particles are evaluated, the others get zero (the free stream is
// not added to them). support: a child cell is far when R > support x its
// size (the reference's support factor 2).
cudaError_t eval3d(const Tree3D& t, bool mixed, bool all_src, const uint8_t* target, double support, double* u,
                   double* v, double* w, double uinf, double vinf, double winf, unsigned* err, cudaStream_t st,
                   int* launches);

}  // namespace vpm
