// ORACLE — test infrastructure only.
//
// C entry points around the reference's default 3D velocity path
// fmm3D::calcVelocityFast (src/FMM/fast3DFMM.cpp:32-92: FMMCell::generateTree,
// 10-term P2M/M2M, per-target traversal) and around its TreeCell path
// (TreeCell::initializeTree with DIM 3, fmm3D::calcVelocity and
// calcVelocityNearBody, src/FMM/fmm3D.cpp:585-1606), compiled by oracle/Makefile from a
// build-directory copy of the reference sources with DIM set to 3 (the
// reference fixes DIM with a #define in global.hpp:85). Output goes to
// oracle/_ref/libref3d.so only.
#include "src/FMM/fmm3D.hpp"
#include "src/FMM/fast3DFMM.hpp"
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

extern "C" void refpars_set(int p_max, double exp_tree, int par_max, int src_max);

namespace {
std::string g_err;
struct Quiet {
    int saved = -1;
    Quiet() {
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        if (dn >= 0) { dup2(dn, 1); close(dn); }
    }
    ~Quiet() {
        fflush(stdout);
        std::cout.flush();
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};
void pack(const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
          std::vector<std::vector<double>>& pos, std::vector<bool>& mark) {
    pos.assign(n, std::vector<double>(3, 0.0));
    mark.assign(n, false);
    for (int64_t i = 0; i < n; ++i) { pos[i][0] = x[i]; pos[i][1] = y[i]; pos[i][2] = z[i]; mark[i] = act[i] != 0; }
}
}  // namespace

extern "C" {

const char* ref3d_last_error() { return g_err.c_str(); }

void ref3d_set(int leaf_cap, double exp_pct) { refpars_set(12, exp_pct, 50, leaf_cap); }

int ref3d_velocity(const double* x, const double* y, const double* z,
                   const double* ax, const double* ay, const double* az, const uint8_t* act, int64_t n,
                   double* u, double* v, double* w) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark, target(n, true);
        pack(x, y, z, act, n, pos, mark);
        std::vector<double> sx(ax, ax + n), sy(ay, ay + n), sz(az, az + n);
        fmm3D f;
        f.calcVelocityFast(pos, mark, target, sx, sy, sz);
        std::vector<double> fx = f.get_Field_x(), fy = f.get_Field_y(), fz = f.get_Field_z();
        std::memcpy(u, fx.data(), sizeof(double) * n);
        std::memcpy(v, fy.data(), sizeof(double) * n);
        std::memcpy(w, fz.data(), sizeof(double) * n);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

// Octree dump in the reference's cell order (creation order). ints per cell:
// nPar, chdFlag, parentID, isActive, level, max_level(first cell only);
// geom per cell: xc, yc, zc, size. Returns the cell count; call with
// null outputs first to size them.
int64_t ref3d_tree(const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
                   int32_t* ints, double* geom) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, z, act, n, pos, mark);
        FMMCell t;
        t.generateTree(pos, mark);
        if (ints && geom) {
            for (int c = 0; c < t.cellNum; ++c) {
                int32_t* r = ints + 6 * c;
                r[0] = t.nPar[c]; r[1] = t.chdFlag[c]; r[2] = t.parentID[c]; r[3] = t.isActive[c] ? 1 : 0;
                r[4] = t.getCellLevel(t.size[c]); r[5] = (c == 0) ? t.maxLevel : 0;
                geom[4 * c] = t.xc[c]; geom[4 * c + 1] = t.yc[c]; geom[4 * c + 2] = t.zc[c]; geom[4 * c + 3] = t.size[c];
            }
        }
        return t.cellNum;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// TreeCell leaf caps (read by the TreeCell constructor) and root expansion.
void ref3d_tc_set(int max_src, int max_par, double exp_pct) { refpars_set(12, exp_pct, max_par, max_src); }

// fmm3D::calcVelocity (target null) or calcVelocityNearBody (target flags)
// on a TreeCell built from the same particles.
int ref3d_tc_velocity(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                      const double* az, const uint8_t* act, const uint8_t* target, int64_t n, double* u, double* v,
                      double* w) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, z, act, n, pos, mark);
        std::vector<double> sx(ax, ax + n), sy(ay, ay + n), sz(az, az + n);
        TreeCell t;
        t.initializeTree(pos, mark);
        fmm3D f;
        if (target) {
            std::vector<bool> tg(n, false);
            for (int64_t i = 0; i < n; ++i) tg[i] = target[i] != 0;
            f.calcVelocityNearBody(t, pos, mark, tg, sx, sy, sz);
        } else {
            f.calcVelocity(t, pos, mark, sx, sy, sz);
        }
        std::vector<double> fx = f.get_Field_x(), fy = f.get_Field_y(), fz = f.get_Field_z();
        std::memcpy(u, fx.data(), sizeof(double) * n);
        std::memcpy(v, fy.data(), sizeof(double) * n);
        std::memcpy(w, fz.data(), sizeof(double) * n);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

// TreeCell dump in ascending cell ID: ids; ints per cell = parNum, srcParNum,
// isLeaf, isActive, level, max_level (first cell only); geom = centre,
// length; leaf parIDList as CSR. Returns the cell count; call with null
// outputs first to size them.
int64_t ref3d_tc_tree(const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
                      int64_t* ids, int32_t* ints, double* geom, int64_t* leaf_offs, int32_t* pids) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, z, act, n, pos, mark);
        TreeCell t;
        t.initializeTree(pos, mark);
        std::vector<int> keys;
        for (const auto& kv : t.treeData) keys.push_back(kv.first);
        std::sort(keys.begin(), keys.end());
        int64_t off = 0;
        for (size_t k = 0; k < keys.size(); ++k) {
            const Cell* c = t.treeData.at(keys[k]);
            if (ids) ids[k] = c->ID;
            if (ints) {
                int32_t* r = ints + 6 * k;
                r[0] = c->parNum; r[1] = c->srcParNum; r[2] = c->isLeaf ? 1 : 0; r[3] = c->isActive ? 1 : 0;
                r[4] = c->level; r[5] = k == 0 ? t.max_level : 0;
            }
            if (geom)
                for (int d = 0; d < 3; ++d) geom[4 * k + d] = c->centerPos[d];
            if (geom) geom[4 * k + 3] = c->length;
            if (leaf_offs) leaf_offs[k] = off;
            for (int pid : c->parIDList) {
                if (pids) pids[off] = pid;
                ++off;
            }
        }
        if (leaf_offs) leaf_offs[keys.size()] = off;
        return (int64_t)keys.size();
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
