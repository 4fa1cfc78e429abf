// ORACLE — test infrastructure only.
//
// CPU restatement of the reference's default 3D velocity path
// (VELOCITY_3D_TYPE 1: fmm3D::calcVelocityFast), used by tests/, smoke() and
// bench.py's cpu_baseline leg as the checker; never part of the product.
//
//   * octree                  src/FMM/fast3DFMM.cpp:485-745 (FMMCell::generateTree)
//   * octant rule             src/FMM/fast3DFMM.hpp:17-22
//   * 10-term P2M / M2M       src/FMM/fmm3D.cpp:84-132, fast3DFMM.cpp:164-302
//   * M2P multipliers         src/FMM/fmm3D.cpp:147-200
//   * per-target traversal    src/FMM/fast3DFMM.cpp:318-472 (far iff R^2 > (2 size)^2; the
//                             factor 2 is the reference's support factor, a parameter here)
// the alternative 3D path on the shared TreeCell (VELOCITY_3D_TYPE 2: TreeCell
// with DIM 3, fmm3D::calcVelocity / calcVelocityNearBody; section below), and
// the FP64 direct Biot-Savart sum u_i = sum_j (a_j x r_ij) / |r_ij|^3.
//
// Geometry decisions (octant comparisons, R^2 against (2 size)^2) use separate
// IEEE operations in the reference's order; build without -march.

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Oct {
    std::vector<int> npar, chd_flag, parent;
    std::vector<double> xc, yc, zc, size;
    std::vector<char> active;
    std::vector<std::vector<int>> pids;
    std::vector<std::array<int, 8>> chd;
    std::vector<int> level_start;
    int max_level = 0;
    int cap = 30;
    double root = 0;
    int ncell() const { return (int)npar.size(); }
    bool leaf(int c) const { return npar[c] < cap; }
};

thread_local std::string g_err3;

// fast3DFMM.cpp:485-745. The root box is the particle box joined with the
// domain centre (0,0,0) (global.cpp:609-611), side = max extent * (1+exp/100).
bool build_oct(Oct& t, const double* x, const double* y, const double* z, const uint8_t* act,
               int64_t n, int cap, double exp_pct) {
    t.cap = cap;
    double mn[3] = {0.0, 0.0, 0.0}, mx[3] = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < n; ++i) {
        const double p[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d) {
            if (p[d] < mn[d]) mn[d] = p[d];
            if (p[d] > mx[d]) mx[d] = p[d];
        }
    }
    double cen[3];
    t.root = 0.0;
    for (int d = 0; d < 3; ++d) {
        double len = mx[d] - mn[d];
        t.root = std::max(len, t.root);
        cen[d] = 0.5 * (mx[d] + mn[d]);
    }
    t.root *= (1 + (exp_pct / 100));
    auto add_cell = [&](int parent, double cx, double cy, double cz, double sz) {
        t.npar.push_back(0); t.chd_flag.push_back(0); t.parent.push_back(parent);
        t.xc.push_back(cx); t.yc.push_back(cy); t.zc.push_back(cz); t.size.push_back(sz);
        t.active.push_back(0); t.pids.emplace_back();
        std::array<int, 8> z8; z8.fill(0); t.chd.push_back(z8);
        return t.ncell() - 1;
    };
    add_cell(-1, cen[0], cen[1], cen[2], t.root);
    t.npar[0] = (int)n;
    t.active[0] = 1;
    t.level_start.assign(1, 0);

    std::vector<char> settled(n, 0);
    std::vector<int> cell_of(n, 0);
    int64_t remaining = n;
    int L = 0;
    while (remaining > 0) {
        ++L;
        if (L > 60) { g_err3 = "octree deeper than 60 levels (coincident particles)"; return false; }
        t.level_start.push_back(t.ncell());
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i]) continue;
            int c = cell_of[i];
            int oct = (x[i] > t.xc[c]) * 1 + (y[i] > t.yc[c]) * 2 + (z[i] > t.zc[c]) * 4;
            if (((t.chd_flag[c] >> oct) & 1) == 0) {
                double h = t.size[c] / 2.0;
                double cx = t.xc[c] + h * (((oct >> 0) & 1) - 0.5);
                double cy = t.yc[c] + h * (((oct >> 1) & 1) - 0.5);
                double cz = t.zc[c] + h * (((oct >> 2) & 1) - 0.5);
                int k = add_cell(c, cx, cy, cz, h);
                t.chd[c][oct] = k;
                t.chd_flag[c] |= (1 << oct);
            }
            int k = t.chd[c][oct];
            cell_of[i] = k;
            t.npar[k]++;
        }
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i]) continue;
            int c = cell_of[i];
            if (t.npar[c] < cap) {
                t.pids[c].push_back((int)i);
                if (act[i]) t.active[c] = 1;
                settled[i] = 1;
                --remaining;
            }
        }
    }
    t.max_level = L;
    t.level_start.push_back(t.ncell());
    for (int lv = t.max_level - 1; lv > 0; --lv) {
        for (int c = t.level_start[lv]; c < t.level_start[lv + 1]; ++c) {
            if (t.leaf(c)) continue;
            for (int o = 0; o < 8; ++o) {
                if (((t.chd_flag[c] >> o) & 1) == 0) continue;
                if (t.active[t.chd[c][o]]) { t.active[c] = 1; break; }
            }
        }
    }
    return true;
}

// Moments (q, q d, q d^2/2, cross terms) with d = centre - particle
// (fmm3D.cpp:84-103) and their shift to the parent (fmm3D.cpp:114-132).
inline void p2m(double* m, double s, double dx, double dy, double dz) {
    m[0] += s;
    m[1] += s * dx; m[2] += s * dy; m[3] += s * dz;
    m[4] += s * dx * dx * 0.5; m[5] += s * dy * dy * 0.5; m[6] += s * dz * dz * 0.5;
    m[7] += s * dx * dy; m[8] += s * dy * dz; m[9] += s * dx * dz;
}

inline void m2m(double* m, const double* c, double dx, double dy, double dz) {
    m[0] += c[0];
    m[1] += c[1] + c[0] * dx;
    m[2] += c[2] + c[0] * dy;
    m[3] += c[3] + c[0] * dz;
    m[4] += c[4] + (c[0] * dx * dx * 0.5) + (c[1] * dx);
    m[5] += c[5] + (c[0] * dy * dy * 0.5) + (c[2] * dy);
    m[6] += c[6] + (c[0] * dz * dz * 0.5) + (c[3] * dz);
    m[7] += c[7] + (c[0] * dx * dy) + (c[1] * dy) + (c[2] * dx);
    m[8] += c[8] + (c[0] * dy * dz) + (c[2] * dz) + (c[3] * dy);
    m[9] += c[9] + (c[0] * dx * dz) + (c[1] * dz) + (c[3] * dx);
}

// Derivatives of r/|r|^3 paired with the 10 moments (fmm3D.cpp:147-200).
inline void m2p_mul(double R2, double dx, double dy, double dz, double* gx, double* gy, double* gz) {
    double R = std::sqrt(R2), R3 = R * R2, R5 = R3 * R2, R7 = R5 * R2;
    gx[0] = dx / R3;
    gx[1] = -(3 * dx * dx / R5) + (1 / R3);
    gx[2] = -(3 * dx * dy / R5);
    gx[3] = -(3 * dx * dz / R5);
    gx[4] = (15 * dx * dx * dx / R7) - (9 * dx / R5);
    gx[5] = (15 * dx * dy * dy / R7) - (3 * dx / R5);
    gx[6] = (15 * dx * dz * dz / R7) - (3 * dx / R5);
    gx[7] = (15 * dx * dx * dy / R7) - (3 * dy / R5);
    gx[8] = (15 * dx * dy * dz / R7);
    gx[9] = (15 * dx * dx * dz / R7) - (3 * dz / R5);
    gy[0] = dy / R3;
    gy[1] = -(3 * dy * dx / R5);
    gy[2] = -(3 * dy * dy / R5) + (1 / R3);
    gy[3] = -(3 * dy * dz / R5);
    gy[4] = (15 * dy * dx * dx / R7) - (3 * dy / R5);
    gy[5] = (15 * dy * dy * dy / R7) - (9 * dy / R5);
    gy[6] = (15 * dy * dz * dz / R7) - (3 * dy / R5);
    gy[7] = (15 * dy * dx * dy / R7) - (3 * dx / R5);
    gy[8] = (15 * dy * dy * dz / R7) - (3 * dz / R5);
    gy[9] = (15 * dy * dx * dz / R7);
    gz[0] = dz / R3;
    gz[1] = -(3 * dz * dx / R5);
    gz[2] = -(3 * dz * dy / R5);
    gz[3] = -(3 * dz * dz / R5) + (1 / R3);
    gz[4] = (15 * dz * dx * dx / R7) - (3 * dz / R5);
    gz[5] = (15 * dz * dy * dy / R7) - (3 * dz / R5);
    gz[6] = (15 * dz * dz * dz / R7) - (9 * dz / R5);
    gz[7] = (15 * dz * dx * dy / R7);
    gz[8] = (15 * dz * dy * dz / R7) - (3 * dy / R5);
    gz[9] = (15 * dz * dx * dz / R7) - (3 * dx / R5);
}

// ---------------------------------------------------------------------------
// 3D TreeCell path (VELOCITY_3D_TYPE 2, VELOCITY_CALCULATION_TYPE 2):
//   tree        TreeCell::initializeTree with DIM 3   src/FMM/treeCell.cpp:1043-1243
//   cell IDs    start(L) = (8^L - 1) / 7, ID = start + ix + iy 2^L + iz 4^L
//               (treeCell.cpp:114-148, 223-250); index = (int)((c - pivot) / size_L),
//               size_L = root / 2^L (treeCell.cpp:101-105, 290-300); children in the
//               order ix + ((i >> 0) & 1), iy + ((i >> 1) & 1), iz + ((i >> 2) & 1)
//               (treeCell.cpp:395-417)
//   P2M, M2M    fmm3D::setupVelocityFMM                src/FMM/fmm3D.cpp:585-784
//   traversal   fmm3D::calcVelocity / calcVelocityNearBody  fmm3D.cpp:1064-1606:
//               from the level-1 cells, far iff R^2 > (2 length)^2 (fmm3D.cpp:3),
//               near leaves by direct sum over ALL their particles (inactive ones
//               included), j != i.
// ---------------------------------------------------------------------------
constexpr int kTcMaxLevel = 10;   // deeper cells overflow the reference's int cell IDs
int64_t g_tc_pairs[2] = {0, 0};   // P2P (target, source) and M2P (target, cell) pairs of the last evaluation

struct TC3 {
    double root = 0, piv[3] = {0, 0, 0};
    std::vector<int64_t> id;
    std::vector<int> level, npar, nsrc, ix, iy, iz;
    std::vector<char> leaf, active;
    std::vector<double> xc, yc, zc, len;
    std::vector<std::vector<int>> pids;
    std::vector<int> level_start;       // cells level-major, creation order within a level
    std::unordered_map<int64_t, int> at;  // cell ID -> index
    int max_level = 0;
    int ncell() const { return (int)id.size(); }
    int find(int64_t cid) const {
        auto it = at.find(cid);
        return it == at.end() ? -1 : it->second;
    }
};

inline int64_t tc_start(int L) { return ((int64_t)1 << (3 * L)) / 7; }   // (8^L - 1) / 7
inline int64_t tc_id(int L, int ix, int iy, int iz) {
    return tc_start(L) + ix + ((int64_t)iy << L) + ((int64_t)iz << (2 * L));
}

bool build_tc3(TC3& t, const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
               int max_src, int max_par, double exp_pct) {
    const double* p[3] = {x, y, z};
    double mn[3], mx[3];
    for (int d = 0; d < 3; ++d) mn[d] = mx[d] = p[d][0];
    for (int64_t i = 1; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            if (mn[d] > p[d][i]) mn[d] = p[d][i];
            if (mx[d] < p[d][i]) mx[d] = p[d][i];
        }
    t.root = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double ext = std::abs(mx[d] - mn[d]);
        if (ext > t.root) t.root = ext;
    }
    t.root *= 1.0 + (exp_pct / 100.0);
    for (int d = 0; d < 3; ++d) t.piv[d] = (mx[d] + mn[d] - t.root) / 2.0;
    auto add = [&](int64_t cid, int L, int a, int b, int c, double l) {
        t.at[cid] = t.ncell();
        t.id.push_back(cid);
        t.level.push_back(L);
        t.npar.push_back(0);
        t.nsrc.push_back(0);
        t.ix.push_back(a);
        t.iy.push_back(b);
        t.iz.push_back(c);
        t.leaf.push_back(0);
        t.active.push_back(0);
        t.len.push_back(l);
        t.xc.push_back(t.piv[0] + ((0.5 + a) * l));
        t.yc.push_back(t.piv[1] + ((0.5 + b) * l));
        t.zc.push_back(t.piv[2] + ((0.5 + c) * l));
        t.pids.emplace_back();
    };
    add(0, 0, 0, 0, 0, t.root);
    t.npar[0] = (int)n;
    for (int64_t i = 0; i < n; ++i) t.nsrc[0] += act[i] ? 1 : 0;
    t.active[0] = t.nsrc[0] != 0;
    t.level_start.assign(1, 0);
    std::vector<char> settled(n, 0);
    std::vector<int> pcell(n, 0);
    int64_t unsettled = n;
    int L = 0;
    while (unsettled > 0) {
        ++L;
        if (L > kTcMaxLevel) {
            g_err3 = "TreeCell deeper than level 10: the reference's 32-bit cell IDs overflow";
            return false;
        }
        t.level_start.push_back(t.ncell());
        const double size = t.root / std::pow(2.0, L);
        const int count = 1 << L;
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i]) continue;
            int idx[3];
            for (int d = 0; d < 3; ++d) idx[d] = (int)((p[d][i] - t.piv[d]) / size);
            for (int d = 0; d < 3; ++d)
                if (idx[d] < 0 || idx[d] >= count) {
                    g_err3 = "particle outside the root box";
                    return false;
                }
            const int64_t cid = tc_id(L, idx[0], idx[1], idx[2]);
            int c = t.find(cid);
            if (c < 0) {
                c = t.ncell();
                add(cid, L, idx[0], idx[1], idx[2], size);
            }
            pcell[i] = c;
            t.npar[c] += 1;
            if (act[i]) t.nsrc[c] += 1;
        }
        for (int c = t.level_start[L]; c < t.ncell(); ++c) {
            if (t.nsrc[c] <= max_src && t.npar[c] <= max_par) t.leaf[c] = 1;
            if (t.nsrc[c] != 0) t.active[c] = 1;
        }
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i] || !t.leaf[pcell[i]]) continue;
            t.pids[pcell[i]].push_back((int)i);
            settled[i] = 1;
            --unsettled;
        }
        t.max_level = L;   // the last leaf created lies on the deepest level
    }
    t.level_start.push_back(t.ncell());
    return true;
}

}  // namespace

extern "C" {

const char* orc3_last_error() { return g_err3.c_str(); }

// TreeCell dump, cells level-major in creation order: ids = reference cell
// IDs; ints per cell = nPar, srcParNum, isLeaf, isActive, level, (max_level
// on cell 0); geom = xc, yc, zc, length; leaf particle IDs (ascending) as
// CSR leaf_offs[c]..leaf_offs[c+1]. Returns the cell count (-1 on error);
// call with null outputs first to size them.
int64_t orc_treecell3d_tree(const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
                            int max_src, int max_par, double exp_pct, int64_t* ids, int32_t* ints, double* geom,
                            int64_t* leaf_offs, int32_t* pids) {
    TC3 t;
    if (n < 1 || !build_tc3(t, x, y, z, act, n, max_src, max_par, exp_pct)) return -1;
    int64_t off = 0;
    for (int c = 0; c < t.ncell(); ++c) {
        if (ids) ids[c] = t.id[c];
        if (ints) {
            int32_t* r = ints + 6 * (size_t)c;
            r[0] = t.npar[c]; r[1] = t.nsrc[c]; r[2] = t.leaf[c]; r[3] = t.active[c]; r[4] = t.level[c];
            r[5] = c == 0 ? t.max_level : 0;
        }
        if (geom) {
            geom[4 * (size_t)c] = t.xc[c]; geom[4 * (size_t)c + 1] = t.yc[c];
            geom[4 * (size_t)c + 2] = t.zc[c]; geom[4 * (size_t)c + 3] = t.len[c];
        }
        if (leaf_offs) leaf_offs[c] = off;
        for (int i : t.pids[c]) {
            if (pids) pids[off] = i;
            ++off;
        }
    }
    if (leaf_offs) leaf_offs[t.ncell()] = off;
    return t.ncell();
}

// TreeCell treecode velocity: every particle a target (calcVelocity) when
// target is null, else only flagged ones (calcVelocityNearBody; the others
// get zero). Returns -1 with the reference's failure when a level-1 cell is
// a leaf of a deeper tree (its traversal asks for that leaf's children).
int orc_treecell3d_velocity(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                            const double* az, const uint8_t* act, const uint8_t* target, int64_t n, int max_src,
                            int max_par, double exp_pct, double support, double* u, double* v, double* w) {
    TC3 t;
    if (n < 1 || !build_tc3(t, x, y, z, act, n, max_src, max_par, exp_pct)) return -1;
    const int nc = t.ncell();
    for (int c = t.level_start[1]; c < t.level_start[2] && t.max_level > 1; ++c)
        if (t.leaf[c]) {
            g_err3 = "a level-1 cell is a leaf: the reference's traversal cannot take its children";
            return -1;
        }
    std::vector<double> mx((size_t)nc * 10, 0.0), my((size_t)nc * 10, 0.0), mz((size_t)nc * 10, 0.0);
    for (int c = 0; c < nc; ++c) {
        if (!t.leaf[c] || !t.active[c]) continue;
        for (int i : t.pids[c]) {
            if (!act[i]) continue;
            double dx = t.xc[c] - x[i], dy = t.yc[c] - y[i], dz = t.zc[c] - z[i];
            p2m(&mx[(size_t)c * 10], ax[i], dx, dy, dz);
            p2m(&my[(size_t)c * 10], ay[i], dx, dy, dz);
            p2m(&mz[(size_t)c * 10], az[i], dx, dy, dz);
        }
    }
    // children of a non-leaf cell in the reference's order (-1 where absent)
    auto children = [&](int c, int ch[8]) {
        const int L = t.level[c] + 1;
        for (int o = 0; o < 8; ++o)
            ch[o] = t.find(tc_id(L, 2 * t.ix[c] + (o & 1), 2 * t.iy[c] + ((o >> 1) & 1), 2 * t.iz[c] + ((o >> 2) & 1)));
    };
    for (int lv = t.max_level - 1; lv > 0; --lv) {
        for (int c = t.level_start[lv]; c < t.level_start[lv + 1]; ++c) {
            if (t.leaf[c] || !t.active[c]) continue;
            int ch[8];
            children(c, ch);
            for (int o = 0; o < 8; ++o) {
                const int k = ch[o];
                if (k < 0) continue;
                double dx = t.xc[c] - t.xc[k], dy = t.yc[c] - t.yc[k], dz = t.zc[c] - t.zc[k];
                m2m(&mx[(size_t)c * 10], &mx[(size_t)k * 10], dx, dy, dz);
                m2m(&my[(size_t)c * 10], &my[(size_t)k * 10], dx, dy, dz);
                m2m(&mz[(size_t)c * 10], &mz[(size_t)k * 10], dx, dy, dz);
            }
        }
    }
    std::vector<int> first;   // the level-1 cells that exist, in ID order
    for (int o = 0; o < 8; ++o) {
        const int c = t.find(1 + o);
        if (c >= 0) first.push_back(c);
    }
    int64_t n_p2p = 0, n_m2p = 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(+ : n_p2p, n_m2p)
    for (int64_t i = 0; i < n; ++i) {
        double vx = 0, vy = 0, vz = 0;
        if (target == nullptr || target[i]) {
            const double xp = x[i], yp = y[i], zp = z[i];
            std::vector<int> cur(first), nxt;
            double gx[10], gy[10], gz[10];
            for (int lv = 1; lv < t.max_level; ++lv) {
                nxt.clear();
                for (int c : cur) {
                    int ch[8];
                    children(c, ch);
                    for (int o = 0; o < 8; ++o) {
                        const int k = ch[o];
                        if (k < 0 || !t.active[k]) continue;
                        double dx = xp - t.xc[k], dy = yp - t.yc[k], dz = zp - t.zc[k];
                        double R2 = dx * dx + dy * dy + dz * dz;
                        double Rc = t.len[k] * support;
                        if (R2 > Rc * Rc) {
                            ++n_m2p;
                            m2p_mul(R2, dx, dy, dz, gx, gy, gz);
                            const double* Mx = &mx[(size_t)k * 10];
                            const double* My = &my[(size_t)k * 10];
                            const double* Mz = &mz[(size_t)k * 10];
                            for (int m = 0; m < 10; ++m) {
                                vx += My[m] * gz[m] - Mz[m] * gy[m];
                                vy += Mz[m] * gx[m] - Mx[m] * gz[m];
                                vz += Mx[m] * gy[m] - My[m] * gx[m];
                            }
                        } else if (!t.leaf[k]) {
                            nxt.push_back(k);
                        } else {
                            for (int j : t.pids[k]) {
                                if (j == i) continue;
                                ++n_p2p;
                                double ex = xp - x[j], ey = yp - y[j], ez = zp - z[j];
                                double r2 = ex * ex + ey * ey + ez * ez;
                                double r3 = std::sqrt(r2) * r2;
                                vx += (ay[j] * ez - az[j] * ey) / r3;
                                vy += (az[j] * ex - ax[j] * ez) / r3;
                                vz += (ax[j] * ey - ay[j] * ex) / r3;
                            }
                        }
                    }
                }
                cur.swap(nxt);
            }
        }
        u[i] = vx; v[i] = vy; w[i] = vz;
    }
    g_tc_pairs[0] = n_p2p;
    g_tc_pairs[1] = n_m2p;
    return 0;
}

// Pair counts of the last orc_treecell3d_velocity call: out[0] = P2P
// (target, source) pairs, j != i; out[1] = M2P (target, far cell) pairs.
void orc_treecell3d_pairs(int64_t* out) {
    out[0] = g_tc_pairs[0];
    out[1] = g_tc_pairs[1];
}

}  // extern "C"

namespace {

// Octree plus the 10-term moments of every active cell (fast3DFMM.cpp:164-302).
struct OctMoments {
    Oct t;
    std::vector<double> mx, my, mz;
};

bool build_moments(OctMoments& om, const double* x, const double* y, const double* z, const double* ax,
                   const double* ay, const double* az, const uint8_t* act, int64_t n, int leaf_cap,
                   double exp_pct) {
    Oct& t = om.t;
    if (!build_oct(t, x, y, z, act, n, leaf_cap, exp_pct)) return false;
    const int nc = t.ncell();
    om.mx.assign((size_t)nc * 10, 0.0);
    om.my.assign((size_t)nc * 10, 0.0);
    om.mz.assign((size_t)nc * 10, 0.0);
    #pragma omp parallel for schedule(dynamic, 16)
    for (int c = 0; c < nc; ++c) {
        if (!t.leaf(c) || !t.active[c]) continue;
        for (int i : t.pids[c]) {
            if (!act[i]) continue;
            double dx = t.xc[c] - x[i], dy = t.yc[c] - y[i], dz = t.zc[c] - z[i];
            p2m(&om.mx[(size_t)c * 10], ax[i], dx, dy, dz);
            p2m(&om.my[(size_t)c * 10], ay[i], dx, dy, dz);
            p2m(&om.mz[(size_t)c * 10], az[i], dx, dy, dz);
        }
    }
    for (int lv = t.max_level - 1; lv > 0; --lv) {
        for (int c = t.level_start[lv]; c < t.level_start[lv + 1]; ++c) {
            if (!t.active[c] || t.leaf(c)) continue;
            for (int o = 0; o < 8; ++o) {
                if (((t.chd_flag[c] >> o) & 1) == 0) continue;
                int k = t.chd[c][o];
                double dx = t.xc[c] - t.xc[k], dy = t.yc[c] - t.yc[k], dz = t.zc[c] - t.zc[k];
                m2m(&om.mx[(size_t)c * 10], &om.mx[(size_t)k * 10], dx, dy, dz);
                m2m(&om.my[(size_t)c * 10], &om.my[(size_t)k * 10], dx, dy, dz);
                m2m(&om.mz[(size_t)c * 10], &om.mz[(size_t)k * 10], dx, dy, dz);
            }
        }
    }
    return true;
}

// One target's walk (fast3DFMM.cpp:340-470): from the root's children, far
// children (R^2 > (support size)^2; the reference's support factor is 2,
// fast3DFMM.cpp:4) through their moments, near leaves directly.
void eval_target(const OctMoments& om, const double* x, const double* y, const double* z, const double* ax,
                 const double* ay, const double* az, const uint8_t* act, int64_t i, double support, double* out) {
    const Oct& t = om.t;
    const double xp = x[i], yp = y[i], zp = z[i];
    double vx = 0, vy = 0, vz = 0;
    std::vector<int> cur, nxt;
    for (int o = 0; o < 8; ++o)
        if ((t.chd_flag[0] >> o) & 1) cur.push_back(t.chd[0][o]);
    double gx[10], gy[10], gz[10];
    for (int lv = 1; lv < t.max_level; ++lv) {
        nxt.clear();
        for (int c : cur) {
            for (int o = 0; o < 8; ++o) {
                if (((t.chd_flag[c] >> o) & 1) == 0) continue;
                int k = t.chd[c][o];
                if (!t.active[k]) continue;
                double dx = xp - t.xc[k], dy = yp - t.yc[k], dz = zp - t.zc[k];
                double R2 = dx * dx + dy * dy + dz * dz;
                double Rc = t.size[k] * support;
                if (R2 > Rc * Rc) {
                    m2p_mul(R2, dx, dy, dz, gx, gy, gz);
                    const double* Mx = &om.mx[(size_t)k * 10];
                    const double* My = &om.my[(size_t)k * 10];
                    const double* Mz = &om.mz[(size_t)k * 10];
                    for (int m = 0; m < 10; ++m) {
                        vx += My[m] * gz[m] - Mz[m] * gy[m];
                        vy += Mz[m] * gx[m] - Mx[m] * gz[m];
                        vz += Mx[m] * gy[m] - My[m] * gx[m];
                    }
                } else if (t.chd_flag[k] != 0) {
                    nxt.push_back(k);
                } else {
                    for (int j : t.pids[k]) {
                        if (!act[j] || j == i) continue;
                        double ex = xp - x[j], ey = yp - y[j], ez = zp - z[j];
                        double r2 = ex * ex + ey * ey + ez * ez;
                        double r3 = std::sqrt(r2) * r2;
                        vx += (ay[j] * ez - az[j] * ey) / r3;
                        vy += (az[j] * ex - ax[j] * ez) / r3;
                        vz += (ax[j] * ey - ay[j] * ex) / r3;
                    }
                }
            }
        }
        cur.swap(nxt);
    }
    out[0] = vx; out[1] = vy; out[2] = vz;
}

}  // namespace

extern "C" {

// Treecode velocity (reference calcVelocityFast with every particle a target).
int orc_fmm3d_velocity(const double* x, const double* y, const double* z,
                       const double* ax, const double* ay, const double* az, const uint8_t* act,
                       int64_t n, int leaf_cap, double exp_pct, double support, double* u, double* v, double* w) {
    OctMoments om;
    if (!build_moments(om, x, y, z, ax, ay, az, act, n, leaf_cap, exp_pct)) return -1;
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        double o[3];
        eval_target(om, x, y, z, ax, ay, az, act, i, support, o);
        u[i] = o[0]; v[i] = o[1]; w[i] = o[2];
    }
    return 0;
}

// The same treecode evaluated only at the m targets tgt[0..m-1] (the
// reference's traversal is per target, fast3DFMM.cpp:340-470, so a sample of
// targets gives exactly those targets' velocities).
int orc_fmm3d_velocity_at(const double* x, const double* y, const double* z,
                          const double* ax, const double* ay, const double* az, const uint8_t* act,
                          int64_t n, int leaf_cap, double exp_pct, double support, const int64_t* tgt, int64_t m,
                          double* u, double* v, double* w) {
    OctMoments om;
    if (!build_moments(om, x, y, z, ax, ay, az, act, n, leaf_cap, exp_pct)) return -1;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t k = 0; k < m; ++k) {
        double o[3];
        eval_target(om, x, y, z, ax, ay, az, act, tgt[k], support, o);
        u[k] = o[0]; v[k] = o[1]; w[k] = o[2];
    }
    return 0;
}

// Octree dump in creation order: ints per cell = nPar, chdFlag, parent,
// active, level, (max_level on cell 0); geom = xc, yc, zc, size.
int64_t orc_tree3d(const double* x, const double* y, const double* z, const uint8_t* act, int64_t n,
                   int leaf_cap, double exp_pct, int32_t* ints, double* geom) {
    Oct t;
    if (!build_oct(t, x, y, z, act, n, leaf_cap, exp_pct)) return -1;
    if (ints && geom) {
        for (int lv = 0; lv <= t.max_level; ++lv) {
            for (int c = t.level_start[lv]; c < t.level_start[lv + 1]; ++c) {
                int32_t* r = ints + 6 * c;
                r[0] = t.npar[c]; r[1] = t.chd_flag[c]; r[2] = t.parent[c]; r[3] = t.active[c];
                r[4] = lv; r[5] = (c == 0) ? t.max_level : 0;
                geom[4 * c] = t.xc[c]; geom[4 * c + 1] = t.yc[c]; geom[4 * c + 2] = t.zc[c]; geom[4 * c + 3] = t.size[c];
            }
        }
    }
    return t.ncell();
}

// FP64 direct velocity at m sampled targets from all active sources.
void orc_direct3d_velocity(const double* x, const double* y, const double* z,
                           const double* ax, const double* ay, const double* az, const uint8_t* act,
                           int64_t n, const int64_t* tgt, int64_t m, double* u, double* v, double* w) {
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < m; ++k) {
        int64_t i = tgt[k];
        double vx = 0, vy = 0, vz = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i || !act[j]) continue;
            double ex = x[i] - x[j], ey = y[i] - y[j], ez = z[i] - z[j];
            double r2 = ex * ex + ey * ey + ez * ez;
            double r3 = std::sqrt(r2) * r2;
            vx += (ay[j] * ez - az[j] * ey) / r3;
            vy += (az[j] * ex - ax[j] * ez) / r3;
            vz += (ax[j] * ey - ay[j] * ex) / r3;
        }
        u[k] = vx; v[k] = vy; w[k] = vz;
    }
}

}  // extern "C"
