// ORACLE — test infrastructure only.
//
// CPU restatement of the reference's 2D FMM velocity step, used by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
// It is never linked into, loaded by, or called from the product library.
//
// What it restates (reference anggarapangestu/LSMPS_VPM_v2):
//   * adaptive quadtree         src/FMM/treeCell.cpp:1043-1243 (initializeTree)
//   * cell index arithmetic     src/FMM/treeCell.cpp:114-148, 223-318, 336-417
//   * same-level neighbours     src/FMM/treeCell.cpp:562-625 (findNghLvl)
//   * lists 1 and 3             src/FMM/treeCell.cpp:636-804 (intList)
//   * lists 2 and 4             src/FMM/treeCell.cpp:818-1032 (extList)
//   * P2M/M2M/M2L/L2L           src/FMM/fmm2D.cpp:192-663 (setupFMM)
//   * P2P/M2P/L2P field         src/FMM/fmm2D.cpp:135-179, 907-1123 (calcField)
//   * P2P/M2P/L2P potential     src/FMM/fmm2D.cpp:77-122, 681-896 (calcPotential)
// plus an FP64 direct O(N*M) Biot-Savart sum on sampled targets, the accuracy
// yardstick for the chosen (mixed / tuned) forms.
//
// Every floating-point step that decides an integer (cell index, adjacency,
// separation) is written as separate IEEE operations in the same order as the
// reference; build without -march so the compiler emits no FMA contraction.
// Series arithmetic (expansions) uses power tables instead of std::pow; it is
// equal to the reference up to rounding (checked to 1e-12 against the compiled
// reference in tests/test_oracle_ref.py).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

const double kTol = 10e-10;  // EPSILON_TOLERANCE, treeCell.cpp:5 (= 1e-9)

inline int64_t start_id(int L) { return (((int64_t)1 << (2 * L)) - 1) / 3; }
inline int64_t cell_id(int L, int64_t ix, int64_t iy) { return start_id(L) + ix + (iy << L); }

struct Cell {
    int64_t id;
    int level;
    int ix, iy;
    double len, cx, cy;
    int par, src;
    bool leaf, active;
    std::vector<int> pids;  // particle IDs (leaf only), ascending
};

struct Tree {
    std::vector<Cell> cells;                   // creation order
    std::unordered_map<int64_t, int> where;    // id -> index in cells
    std::vector<int64_t> leaf_list;            // creation order (reference leafList)
    double minD[2], maxD[2], root, pivot[2];
    int min_level, max_level, max_src, max_par;
    std::string err;

    const Cell* find(int64_t id) const {
        auto it = where.find(id);
        return it == where.end() ? nullptr : &cells[it->second];
    }
};

// Level of a (possibly non-existing) cell from its ID: the reference uses a
// log formula with a fix-up (treeCell.cpp:21-79); the exact integer search
// below gives the same level for every ID whose level is <= 30.
inline int level_of(int64_t id) {
    int L = 0;
    while (start_id(L + 1) <= id) ++L;
    return L;
}

inline void index_of(int64_t id, int L, int64_t& ix, int64_t& iy) {
    int64_t loc = id - start_id(L);
    int64_t cnt = (int64_t)1 << L;
    ix = loc % cnt;
    iy = (loc / cnt) % cnt;
}

inline int64_t parent_id(int64_t id) {
    int L = level_of(id);
    int64_t ix, iy;
    index_of(id, L, ix, iy);
    return cell_id(L - 1, ix / 2, iy / 2);
}

// treeCell.cpp:1043-1243. Returns false (err set) where the reference would
// throw or never terminate.
bool build_tree(Tree& t, const double* x, const double* y, const uint8_t* act, int64_t n,
                int max_src, int max_par, double exp_pct) {
    t.max_src = max_src;
    t.max_par = max_par;
    if (n <= 0) { t.err = "empty input"; return false; }
    t.minD[0] = t.maxD[0] = x[0];
    t.minD[1] = t.maxD[1] = y[0];
    for (int64_t i = 1; i < n; ++i) {
        if (t.minD[0] > x[i]) t.minD[0] = x[i];
        if (t.maxD[0] < x[i]) t.maxD[0] = x[i];
        if (t.minD[1] > y[i]) t.minD[1] = y[i];
        if (t.maxD[1] < y[i]) t.maxD[1] = y[i];
    }
    t.root = 0.0;
    for (int d = 0; d < 2; ++d) {
        double s = std::fabs(t.maxD[d] - t.minD[d]);
        if (s > t.root) t.root = s;
    }
    double expansion = 1.0 + (exp_pct / 100.0);
    t.root *= expansion;
    for (int d = 0; d < 2; ++d) t.pivot[d] = (t.maxD[d] + t.minD[d] - t.root) / 2.0;
    if (!(t.root > 0.0) || !std::isfinite(t.root)) { t.err = "degenerate domain"; return false; }

    Cell rc;
    rc.id = 0; rc.level = 0; rc.ix = rc.iy = 0; rc.len = t.root;
    rc.cx = t.pivot[0] + (0.5 * t.root);
    rc.cy = t.pivot[1] + (0.5 * t.root);
    rc.par = (int)n;
    rc.src = 0;
    for (int64_t i = 0; i < n; ++i) rc.src += act[i] ? 1 : 0;
    rc.active = rc.src != 0;
    rc.leaf = false;
    t.cells.push_back(rc);
    t.where[0] = 0;

    std::vector<char> settled(n, 0);
    std::vector<int> cell_of(n, 0);
    int64_t remaining = n;
    int L = 0;
    while (remaining > 0) {
        ++L;
        if (L > 30) { t.err = "tree deeper than 30 levels (coincident particles)"; return false; }
        double size = t.root / std::pow(2.0, L);
        int64_t cnt = (int64_t)1 << L;
        std::vector<int> created;
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i]) continue;
            int64_t ix = (int64_t)((x[i] - t.pivot[0]) / size);
            int64_t iy = (int64_t)((y[i] - t.pivot[1]) / size);
            if (ix < 0 || ix >= cnt || iy < 0 || iy >= cnt) { t.err = "cell index out of range"; return false; }
            int64_t id = cell_id(L, ix, iy);
            auto it = t.where.find(id);
            int ci;
            if (it == t.where.end()) {
                Cell c;
                c.id = id; c.level = L; c.ix = (int)ix; c.iy = (int)iy; c.len = size;
                c.cx = t.pivot[0] + ((0.5 + (double)ix) * size);
                c.cy = t.pivot[1] + ((0.5 + (double)iy) * size);
                c.par = 0; c.src = 0; c.leaf = false; c.active = false;
                ci = (int)t.cells.size();
                t.cells.push_back(c);
                t.where[id] = ci;
                created.push_back(ci);
            } else {
                ci = it->second;
            }
            cell_of[i] = ci;
            t.cells[ci].par++;
            if (act[i]) t.cells[ci].src++;
        }
        for (int ci : created) {
            Cell& c = t.cells[ci];
            if (c.src <= max_src && c.par <= max_par) {
                c.leaf = true;
                t.leaf_list.push_back(c.id);
            }
            if (c.src != 0) c.active = true;
        }
        for (int64_t i = 0; i < n; ++i) {
            if (settled[i]) continue;
            Cell& c = t.cells[cell_of[i]];
            if (c.leaf) {
                c.pids.push_back((int)i);
                settled[i] = 1;
                --remaining;
            }
        }
    }
    t.min_level = t.find(t.leaf_list.front())->level;
    t.max_level = t.find(t.leaf_list.back())->level;
    return true;
}

// Same-level 3x3 block including the cell itself, in-range only
// (treeCell.cpp:562-625); order: x fastest, from (-1,-1) to (+1,+1).
void same_level_block(const Tree& t, const Cell* c, std::vector<int64_t>& out) {
    out.clear();
    int64_t cnt = (int64_t)1 << c->level;
    for (int k = 0; k < 9; ++k) {
        int dx = k % 3 - 1, dy = (k / 3) % 3 - 1;
        int64_t jx = c->ix + dx, jy = c->iy + dy;
        if (jx < 0 || jx >= cnt || jy < 0 || jy >= cnt) continue;
        out.push_back(cell_id(c->level, jx, jy));
    }
}

void child_ids(const Cell* c, int64_t out[4]) {
    for (int i = 0; i < 4; ++i)
        out[i] = cell_id(c->level + 1, 2 * (int64_t)c->ix + (i & 1), 2 * (int64_t)c->iy + ((i >> 1) & 1));
}

// Lists 1 and 3 of a leaf (treeCell.cpp:636-804).
void int_list(const Tree& t, int64_t cur_id, std::vector<int64_t>& l1, std::vector<int64_t>& l3) {
    l1.clear(); l3.clear();
    const Cell* cur = t.find(cur_id);
    std::vector<int64_t> queue;
    same_level_block(t, cur, queue);
    std::unordered_map<int64_t, char> seen, from_parent;
    for (int64_t q : queue) seen[q] = 1;
    for (size_t i = 0; i < queue.size(); ++i) {
        int64_t nid = queue[i];
        const Cell* nc = t.find(nid);
        if (!nc) {
            int64_t pid = parent_id(nid);
            if (!seen.count(pid)) { queue.push_back(pid); seen[pid] = 1; from_parent[pid] = 1; }
            continue;
        }
        if (!nc->active) continue;
        if (nc->leaf) { l1.push_back(nid); continue; }
        if (from_parent.count(nid)) continue;
        int64_t ch[4];
        child_ids(nc, ch);
        double adj = ((cur->len + (nc->len / 2.0)) / 2.0) + kTol;
        for (int k = 0; k < 4; ++k) {
            const Cell* cc = t.find(ch[k]);
            if (!cc || !cc->active) continue;
            bool adjacent = !(std::fabs(cc->cx - cur->cx) > adj) && !(std::fabs(cc->cy - cur->cy) > adj);
            if (adjacent) {
                if (!seen.count(ch[k])) { queue.push_back(ch[k]); seen[ch[k]] = 1; }
            } else {
                l3.push_back(ch[k]);
            }
        }
    }
}

// Lists 2 and 4 of any cell at level >= 2 (treeCell.cpp:818-1032).
void ext_list(const Tree& t, int64_t cur_id, std::vector<int64_t>& l2, std::vector<int64_t>& l4) {
    l2.clear(); l4.clear();
    const Cell* cur = t.find(cur_id);
    int64_t pid = parent_id(cur_id);
    const Cell* par = t.find(pid);
    std::vector<int64_t> blk, q4;
    std::unordered_map<int64_t, char> seen4;
    same_level_block(t, par, blk);
    for (int64_t nid : blk) {
        if (nid == pid) continue;
        const Cell* nc = t.find(nid);
        if (!nc) {
            int64_t gp = parent_id(nid);
            if (!seen4.count(gp)) { q4.push_back(gp); seen4[gp] = 1; }
            continue;
        }
        if (!nc->active) continue;
        if (nc->leaf) { q4.push_back(nid); seen4[nid] = 1; continue; }
        int64_t ch[4];
        child_ids(nc, ch);
        double min_dist = cur->len + kTol;
        for (int k = 0; k < 4; ++k) {
            const Cell* cc = t.find(ch[k]);
            if (!cc || !cc->active) continue;
            bool sep = (std::fabs(cc->cx - cur->cx) > min_dist) || (std::fabs(cc->cy - cur->cy) > min_dist);
            if (sep) l2.push_back(ch[k]);
        }
    }
    for (size_t i = 0; i < q4.size(); ++i) {
        int64_t nid = q4[i];
        const Cell* nc = t.find(nid);
        if (!nc) {
            int64_t gp = parent_id(nid);
            if (!seen4.count(gp)) { q4.push_back(gp); seen4[gp] = 1; }
            continue;
        }
        if (!nc->active || !nc->leaf) continue;
        double min_dist = ((nc->len + cur->len) / 2.0) + kTol;
        bool sep = (std::fabs(nc->cx - cur->cx) > min_dist) || (std::fabs(nc->cy - cur->cy) > min_dist);
        if (sep) l4.push_back(nid);
    }
}

// Binomial coefficient as the reference computes it (fmm2D.cpp:28-58): the
// product n!/max(k,n-k)! is formed in 32-bit int and wraps for the largest
// M2L orders (e.g. C(18,9) and C(19,9), used at p=10), then is divided by
// min(k,n-k)! with truncation. exact=true gives the true value instead.
int64_t binom(int n, int k, bool exact) {
    if (k > n) return 0;
    if (exact) {
        int64_t c = 1;
        for (int i = 1; i <= k; ++i) c = c * (n - k + i) / i;
        return c;
    }
    int inv = n - k;
    int mx = inv > k ? inv : k;
    int mn = inv > k ? k : inv;
    int32_t c = 1;
    for (int i = n; i > mx; --i) c = (int32_t)((uint32_t)c * (uint32_t)i);
    for (int i = mn; i > 1; --i) c /= i;
    return c;
}

// Expansions of every cell (fmm2D.cpp:192-663). a, b indexed by cell index.
void setup_fmm(const Tree& t, const double* x, const double* y, const uint8_t* act, const double* q,
               int P, std::vector<cplx>& a, std::vector<cplx>& b, bool want_b0, bool exact) {
    const int nc = (int)t.cells.size();
    const int W = P + 1;
    a.assign((size_t)nc * W, cplx(0, 0));
    b.assign((size_t)nc * W, cplx(0, 0));

    // P2M over active leaves, active particles (fmm2D.cpp:237-284).
    #pragma omp parallel for schedule(dynamic, 16)
    for (int ci = 0; ci < nc; ++ci) {
        const Cell& c = t.cells[ci];
        if (!c.leaf || !c.active) continue;
        cplx z0(c.cx, c.cy);
        cplx* ac = &a[(size_t)ci * W];
        for (int pidx : c.pids) {
            if (!act[pidx]) continue;
            cplx w = cplx(x[pidx], y[pidx]) - z0;
            ac[0] += q[pidx];
            cplx wp(1, 0);
            for (int p = 1; p <= P; ++p) { wp *= w; ac[p] += q[pidx] * wp; }
        }
    }

    // Cells by level, for the level sweeps.
    std::vector<std::vector<int>> by_level(64);
    for (int ci = 0; ci < nc; ++ci) by_level[t.cells[ci].level].push_back(ci);

    // M2M, levels max-1 .. 1, active non-leaf parents (fmm2D.cpp:309-379).
    for (int L = t.max_level - 1; L > 0; --L) {
        const std::vector<int>& cl = by_level[L];
        #pragma omp parallel for schedule(dynamic, 16)
        for (int ii = 0; ii < (int)cl.size(); ++ii) {
            const Cell& c = t.cells[cl[ii]];
            if (c.leaf || !c.active) continue;
            cplx z0(c.cx, c.cy);
            cplx* ap = &a[(size_t)cl[ii] * W];
            int64_t ch[4];
            child_ids(&c, ch);
            std::vector<cplx> tp(W);
            for (int k = 0; k < 4; ++k) {
                auto it = t.where.find(ch[k]);
                if (it == t.where.end()) continue;
                const Cell& cc = t.cells[it->second];
                const cplx* acd = &a[(size_t)it->second * W];
                cplx tt = cplx(cc.cx, cc.cy) - z0;
                tp[0] = 1;
                for (int m = 1; m <= P; ++m) tp[m] = tp[m - 1] * tt;
                ap[0] += acd[0];
                for (int p = 1; p <= P; ++p) {
                    cplx s = acd[0] * tp[p];
                    for (int kk = 1; kk <= p; ++kk)
                        s += (double)binom(p - 1, kk - 1, exact) * ((double)p / (double)kk) * acd[kk] * tp[p - kk];
                    ap[p] += s;
                }
            }
        }
    }

    // M2L from lists 2 and 4, every cell at level >= 2 (fmm2D.cpp:396-556).
    #pragma omp parallel for schedule(dynamic, 16)
    for (int ci = 0; ci < nc; ++ci) {
        const Cell& c = t.cells[ci];
        if (c.level < 2) continue;
        std::vector<int64_t> l2, l4;
        ext_list(t, c.id, l2, l4);
        cplx z0(c.cx, c.cy);
        cplx* bc = &b[(size_t)ci * W];
        std::vector<cplx> ip(2 * P + 2);
        for (int pass = 0; pass < 2; ++pass) {
            const std::vector<int64_t>& lst = pass == 0 ? l2 : l4;
            for (int64_t sid : lst) {
                int si = t.where.at(sid);
                const Cell& s = t.cells[si];
                const cplx* as = &a[(size_t)si * W];
                cplx z1(s.cx, s.cy);
                cplx tinv = 1.0 / (z1 - z0);
                ip[0] = 1;
                for (int m = 1; m <= 2 * P; ++m) ip[m] = ip[m - 1] * tinv;
                if (want_b0) {
                    cplx s0 = as[0] * std::log(z0 - z1);
                    for (int k = 1; k <= P; ++k) s0 -= as[k] / (double)k * (double)((k & 1) ? -1 : 1) * ip[k];
                    bc[0] += s0;
                }
                for (int p = 1; p <= P; ++p) {
                    cplx s1 = (as[0] / (double)p) * ip[p];
                    for (int k = 1; k <= P; ++k)
                        s1 += (double)binom(p + k - 1, k - 1, exact) * (double)((k & 1) ? -1 : 1) / (double)k * as[k] * ip[p + k];
                    bc[p] -= s1;
                }
            }
        }
    }

    // L2L, parent levels 2 .. max-1, non-leaf parents (fmm2D.cpp:587-651).
    for (int L = 2; L < t.max_level; ++L) {
        const std::vector<int>& cl = by_level[L];
        #pragma omp parallel for schedule(dynamic, 16)
        for (int ii = 0; ii < (int)cl.size(); ++ii) {
            const Cell& c = t.cells[cl[ii]];
            if (c.leaf) continue;
            cplx z1(c.cx, c.cy);
            const cplx* bp = &b[(size_t)cl[ii] * W];
            int64_t ch[4];
            child_ids(&c, ch);
            std::vector<cplx> tp(W);
            for (int k = 0; k < 4; ++k) {
                auto it = t.where.find(ch[k]);
                if (it == t.where.end()) continue;
                const Cell& cc = t.cells[it->second];
                cplx* bcd = &b[(size_t)it->second * W];
                cplx tt = cplx(cc.cx, cc.cy) - z1;
                tp[0] = 1;
                for (int m = 1; m <= P; ++m) tp[m] = tp[m - 1] * tt;
                for (int p = want_b0 ? 0 : 1; p <= P; ++p) {
                    cplx s = 0;
                    for (int kk = p; kk <= P; ++kk) s += (double)binom(kk, p, exact) * bp[kk] * tp[kk - p];
                    bcd[p] += s;
                }
            }
        }
    }
}

// Field evaluation at the particles of every leaf (fmm2D.cpp:907-1123) or the
// potential (fmm2D.cpp:681-896).
void evaluate(const Tree& t, const double* x, const double* y, const double* q, int P,
              const std::vector<cplx>& a, const std::vector<cplx>& b,
              double* ex, double* ey, double* pot) {
    const int W = P + 1;
    const int nl = (int)t.leaf_list.size();
    #pragma omp parallel for schedule(dynamic, 8)
    for (int li = 0; li < nl; ++li) {
        int ci = t.where.at(t.leaf_list[li]);
        const Cell& c = t.cells[ci];
        std::vector<int64_t> l1, l3;
        int_list(t, c.id, l1, l3);
        // P2P over list 1 (all particles of those cells, j != i).
        for (int64_t sid : l1) {
            const Cell& s = *t.find(sid);
            for (int j : s.pids) {
                for (int i : c.pids) {
                    if (i == j) continue;
                    double dx = x[i] - x[j], dy = y[i] - y[j];
                    double r2 = dx * dx + dy * dy;
                    if (pot) {
                        pot[i] += q[j] * std::log(r2) / 2.0;
                    } else {
                        ex[i] += q[j] * dx / r2;
                        ey[i] += q[j] * dy / r2;
                    }
                }
            }
        }
        const cplx* bc = &b[(size_t)ci * W];
        cplx z0(c.cx, c.cy);
        for (int i : c.pids) {
            cplx z(x[i], y[i]);
            // M2P over list 3.
            for (int64_t sid : l3) {
                int si = t.where.at(sid);
                const Cell& s = t.cells[si];
                const cplx* as = &a[(size_t)si * W];
                cplx w = z - cplx(s.cx, s.cy);
                if (pot) {
                    cplx f = as[0] * std::log(w);
                    cplx winv = 1.0 / w, wp = winv;
                    for (int p = 1; p <= P; ++p) { f -= as[p] / (double)p * wp; wp *= winv; }
                    pot[i] += f.real();
                } else {
                    cplx winv = 1.0 / w, wp = winv, f = 0;
                    for (int p = 0; p <= P; ++p) { f += as[p] * wp; wp *= winv; }
                    ex[i] += f.real();
                    ey[i] -= f.imag();
                }
            }
            // L2P.
            cplx w = z - z0;
            if (pot) {
                cplx f = 0, wp = 1;
                for (int p = 0; p <= P; ++p) { f += bc[p] * wp; wp *= w; }
                pot[i] += f.real();
            } else {
                cplx f = 0, wp = 1;
                for (int p = 1; p <= P; ++p) { f += (double)p * bc[p] * wp; wp *= w; }
                ex[i] += f.real();
                ey[i] -= f.imag();
            }
        }
    }
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Opaque 2D tree handle for dumps.
void* orc_tree2d_build(const double* x, const double* y, const uint8_t* act, int64_t n,
                       int max_src, int max_par, double exp_pct) {
    Tree* t = new Tree();
    if (!build_tree(*t, x, y, act, n, max_src, max_par, exp_pct)) {
        g_err = t->err;
        delete t;
        return nullptr;
    }
    return t;
}

void orc_tree2d_free(void* h) { delete (Tree*)h; }

int64_t orc_tree2d_ncells(void* h) { return (int64_t)((Tree*)h)->cells.size(); }
int64_t orc_tree2d_nleaves(void* h) { return (int64_t)((Tree*)h)->leaf_list.size(); }

// geom[0..7] = minx, maxx, miny, maxy, root, pivot_x, pivot_y, (min_level | max_level << 16)
void orc_tree2d_geom(void* h, double* geom) {
    Tree* t = (Tree*)h;
    geom[0] = t->minD[0]; geom[1] = t->maxD[0]; geom[2] = t->minD[1]; geom[3] = t->maxD[1];
    geom[4] = t->root; geom[5] = t->pivot[0]; geom[6] = t->pivot[1];
    geom[7] = (double)(t->min_level | (t->max_level << 16));
}

// Cells sorted by ID. ints[i*6..]: level, ix, iy, par, src, flags(leaf|active<<1)
void orc_tree2d_cells(void* h, int64_t* ids, int32_t* ints, double* centers) {
    Tree* t = (Tree*)h;
    std::vector<int> order(t->cells.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return t->cells[a].id < t->cells[b].id; });
    for (size_t k = 0; k < order.size(); ++k) {
        const Cell& c = t->cells[order[k]];
        ids[k] = c.id;
        int32_t* r = ints + 6 * k;
        r[0] = c.level; r[1] = c.ix; r[2] = c.iy; r[3] = c.par; r[4] = c.src;
        r[5] = (c.leaf ? 1 : 0) | (c.active ? 2 : 0);
        centers[2 * k] = c.cx;
        centers[2 * k + 1] = c.cy;
    }
}

// Leaf IDs in reference leafList order, and each leaf's particle IDs (CSR).
void orc_tree2d_leaves(void* h, int64_t* leaf_ids, int64_t* offs, int32_t* pids) {
    Tree* t = (Tree*)h;
    int64_t o = 0;
    for (size_t k = 0; k < t->leaf_list.size(); ++k) {
        leaf_ids[k] = t->leaf_list[k];
        offs[k] = o;
        const Cell* c = t->find(t->leaf_list[k]);
        for (int p : c->pids) pids[o++] = p;
    }
    offs[t->leaf_list.size()] = o;
}

// Interaction list `which` (1..4) for the given cell IDs, CSR. With
// out_ids == nullptr only offsets are filled (count pass).
void orc_tree2d_list(void* h, int which, const int64_t* cell_ids, int64_t m, int64_t* offs, int64_t* out_ids) {
    Tree* t = (Tree*)h;
    int64_t o = 0;
    std::vector<int64_t> la, lb;
    for (int64_t k = 0; k < m; ++k) {
        offs[k] = o;
        if (which == 1 || which == 3) int_list(*t, cell_ids[k], la, lb);
        else ext_list(*t, cell_ids[k], la, lb);
        const std::vector<int64_t>& v = (which == 1 || which == 2) ? la : lb;
        if (out_ids) for (size_t e = 0; e < v.size(); ++e) out_ids[o + (int64_t)e] = v[e];
        o += (int64_t)v.size();
    }
    offs[m] = o;
}

// Full FMM field (reference calcField): ex, ey are the reference's Ex, Ey.
int orc_fmm2d_field(const double* x, const double* y, const double* q, const uint8_t* act, int64_t n,
                    int P, int max_src, int max_par, double exp_pct, int exact_binom, double* ex, double* ey) {
    Tree t;
    if (!build_tree(t, x, y, act, n, max_src, max_par, exp_pct)) { g_err = t.err; return -1; }
    std::vector<cplx> a, b;
    setup_fmm(t, x, y, act, q, P, a, b, false, exact_binom != 0);
    std::memset(ex, 0, sizeof(double) * n);
    std::memset(ey, 0, sizeof(double) * n);
    evaluate(t, x, y, q, P, a, b, ex, ey, nullptr);
    return 0;
}

// Full FMM potential (reference calcPotential).
int orc_fmm2d_potential(const double* x, const double* y, const double* q, const uint8_t* act, int64_t n,
                        int P, int max_src, int max_par, double exp_pct, int exact_binom, double* pot) {
    Tree t;
    if (!build_tree(t, x, y, act, n, max_src, max_par, exp_pct)) { g_err = t.err; return -1; }
    std::vector<cplx> a, b;
    setup_fmm(t, x, y, act, q, P, a, b, true, exact_binom != 0);
    std::memset(pot, 0, sizeof(double) * n);
    evaluate(t, x, y, q, P, a, b, nullptr, nullptr, pot);
    return 0;
}

// FP64 direct field at m sampled targets from all active sources (j != i):
// E = sum q_j (x_i - x_j) / r^2. The FMM approximates this sum when every
// particle is active.
void orc_direct2d_field(const double* x, const double* y, const double* q, const uint8_t* act, int64_t n,
                        const int64_t* tgt, int64_t m, double* ex, double* ey) {
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < m; ++k) {
        int64_t i = tgt[k];
        double sx = 0, sy = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i || !act[j]) continue;
            double dx = x[i] - x[j], dy = y[i] - y[j];
            double r2 = dx * dx + dy * dy;
            sx += q[j] * dx / r2;
            sy += q[j] * dy / r2;
        }
        ex[k] = sx;
        ey[k] = sy;
    }
}

}  // extern "C"
