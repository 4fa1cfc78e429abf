// ORACLE — test infrastructure only.
//
// C entry points around the reference's own 2D FMM (TreeCell::initializeTree,
// intList/extList and fmm2D::calcField/calcPotential), compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libref2d.so. Used by
// tests/golden/make_golden.py to generate fixtures, by the oracle-vs-reference
// tests, and by bench.py as the timed CPU baseline. Reference files:
// src/FMM/treeCell.{hpp,cpp}, src/FMM/fmm2D.{hpp,cpp}.
#include "src/FMM/treeCell.hpp"
#include "src/FMM/fmm2D.hpp"
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

extern "C" void refpars_set(int p_max, double exp_tree, int par_max, int src_max);

namespace {
std::string g_err;

// The reference prints per-stage timings to stdout; keep them off the caller's
// stdout (bench.py prints exactly one JSON line).
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

void pack(const double* x, const double* y, const uint8_t* act, int64_t n,
          std::vector<std::vector<double>>& pos, std::vector<bool>& mark) {
    pos.assign(n, std::vector<double>(2, 0.0));
    mark.assign(n, false);
    for (int64_t i = 0; i < n; ++i) { pos[i][0] = x[i]; pos[i][1] = y[i]; mark[i] = act[i] != 0; }
}
}  // namespace

extern "C" {

const char* ref2d_last_error() { return g_err.c_str(); }

void ref2d_set(int p, int max_src, int max_par, double exp_pct) { refpars_set(p, exp_pct, max_par, max_src); }

int ref2d_field(const double* x, const double* y, const double* q, const uint8_t* act, int64_t n,
                double* ex, double* ey) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, act, n, pos, mark);
        std::vector<double> src(q, q + n);
        TreeCell tree;
        tree.initializeTree(pos, mark);
        fmm2D f;
        f.calcField(tree, pos, mark, src);
        std::vector<double> fx = f.get_Field_x(), fy = f.get_Field_y();
        std::memcpy(ex, fx.data(), sizeof(double) * n);
        std::memcpy(ey, fy.data(), sizeof(double) * n);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

int ref2d_potential(const double* x, const double* y, const double* q, const uint8_t* act, int64_t n,
                    double* pot) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, act, n, pos, mark);
        std::vector<double> src(q, q + n);
        TreeCell tree;
        tree.initializeTree(pos, mark);
        fmm2D f;
        f.calcPotential(tree, pos, mark, src);
        std::vector<double> p = f.get_Potential();
        std::memcpy(pot, p.data(), sizeof(double) * n);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

void* ref2d_tree_build(const double* x, const double* y, const uint8_t* act, int64_t n) {
    try {
        Quiet quiet;
        std::vector<std::vector<double>> pos;
        std::vector<bool> mark;
        pack(x, y, act, n, pos, mark);
        TreeCell* t = new TreeCell();
        t->initializeTree(pos, mark);
        return t;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref2d_tree_free(void* h) { delete (TreeCell*)h; }
int64_t ref2d_tree_ncells(void* h) { return (int64_t)((TreeCell*)h)->treeData.size(); }
int64_t ref2d_tree_nleaves(void* h) { return (int64_t)((TreeCell*)h)->leafList.size(); }

void ref2d_tree_geom(void* h, double* g) {
    TreeCell* t = (TreeCell*)h;
    g[0] = t->minDomain[0]; g[1] = t->maxDomain[0]; g[2] = t->minDomain[1]; g[3] = t->maxDomain[1];
    g[4] = t->rootLength; g[5] = t->pivotCoord[0]; g[6] = t->pivotCoord[1];
    g[7] = (double)(t->min_level | (t->max_level << 16));
}

void ref2d_tree_cells(void* h, int64_t* ids, int32_t* ints, double* centers) {
    TreeCell* t = (TreeCell*)h;
    std::vector<int> keys;
    for (const auto& kv : t->treeData) keys.push_back(kv.first);
    std::sort(keys.begin(), keys.end());
    for (size_t k = 0; k < keys.size(); ++k) {
        const Cell* c = t->treeData.at(keys[k]);
        ids[k] = c->ID;
        int32_t* r = ints + 6 * k;
        r[0] = c->level; r[1] = c->index[0]; r[2] = c->index[1]; r[3] = c->parNum; r[4] = c->srcParNum;
        r[5] = (c->isLeaf ? 1 : 0) | (c->isActive ? 2 : 0);
        centers[2 * k] = c->centerPos[0];
        centers[2 * k + 1] = c->centerPos[1];
    }
}

void ref2d_tree_leaves(void* h, int64_t* leaf_ids, int64_t* offs, int32_t* pids) {
    TreeCell* t = (TreeCell*)h;
    int64_t o = 0;
    for (size_t k = 0; k < t->leafList.size(); ++k) {
        leaf_ids[k] = t->leafList[k];
        offs[k] = o;
        for (int p : t->treeData.at(t->leafList[k])->parIDList) pids[o++] = p;
    }
    offs[t->leafList.size()] = o;
}

int ref2d_tree_list(void* h, int which, const int64_t* cell_ids, int64_t m, int64_t* offs, int64_t* out_ids) {
    TreeCell* t = (TreeCell*)h;
    try {
        Quiet quiet;
        int64_t o = 0;
        std::vector<int> la, lb;
        for (int64_t k = 0; k < m; ++k) {
            offs[k] = o;
            int id = (int)cell_ids[k];
            if (which == 1 || which == 3) t->intList(id, la, lb);
            else t->extList(id, la, lb);
            const std::vector<int>& v = (which == 1 || which == 2) ? la : lb;
            if (out_ids) for (size_t e = 0; e < v.size(); ++e) out_ids[o + (int64_t)e] = v[e];
            o += (int64_t)v.size();
        }
        offs[m] = o;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

}  // extern "C"
