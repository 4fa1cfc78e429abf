// Interaction lists of the reference's adaptive quadtree, one GPU thread per
// cell:
//   list 1 / list 3 of every leaf     TreeCell::intList   src/FMM/treeCell.cpp:636-804
//   list 2 / list 4 of every cell L>=2 TreeCell::extList  src/FMM/treeCell.cpp:818-1032
// with the same queue rules: a missing neighbour is replaced by its parent
// (flagged, and only ever taken as a leaf), non-leaf neighbours are opened
// one level, the 1e-9 distance tolerance, active-only membership. Cells are
// addressed by (level, ix, iy); an existing cell is found by binary search of
// its Morton code inside its level. Compiled with --fmad=false so the
// adjacency and separation tests round exactly as the reference's.
#include "fmm2d.cuh"

namespace vpm {

namespace {

struct TreeView {
    Tree2D t;
    double root;
    int depth, n_cells;
    __device__ TreeView(const Tree2D& tt) : t(tt), root(tt.geom->root), depth(tt.info->depth), n_cells(tt.info->n_cells) {}
    __device__ __forceinline__ double len(int L) const { return xdiv(root, ldexp(1.0, L)); }
    // Index of the cell (L, ix, iy) or -1 when it does not exist: one load
    // from the dense grid (validated against the cell's own level and index,
    // since the grid is never cleared) or a binary search of the level's
    // Morton codes.
    __device__ int find(int L, int ix, int iy) const {
        if (L < 0 || L > depth) return -1;
        const long long cnt = 1ll << L;
        if (ix < 0 || iy < 0 || ix >= cnt || iy >= cnt) return -1;
        if (t.dense && L <= t.dense_levels) {
            const int e = t.dense[start_id2(L) + ix + ((int64_t)iy << L)];
            if (e >= 0 && e < n_cells && t.c_level[e] == L && t.c_ix[e] == ix && t.c_iy[e] == iy) return e;
            return -1;
        }
        int lo = t.info->level_start[L], hi = t.info->level_start[L + 1];
        const uint64_t code = morton2((uint32_t)ix, (uint32_t)iy);
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (t.c_code[mid] < code) lo = mid + 1;
            else hi = mid;
        }
        if (lo < t.info->level_start[L + 1] && t.c_code[lo] == code) return lo;
        return -1;
    }
};

struct Queue {
    int lv[kQueueCap], ix[kQueueCap], iy[kQueueCap], cell[kQueueCap];
    uint8_t par[kQueueCap];
    int n = 0;
    __device__ bool seen(int L, int x, int y) const {
        for (int k = 0; k < n; ++k)
            if (lv[k] == L && ix[k] == x && iy[k] == y) return true;
        return false;
    }
    __device__ bool push(int L, int x, int y, int c, uint8_t fp, unsigned* err) {
        if (n >= kQueueCap) { set_err(err, ERR_QUEUE); return false; }
        lv[n] = L; ix[n] = x; iy[n] = y; cell[n] = c; par[n] = fp;
        ++n;
        return true;
    }
};

// intList of leaf `c`. mode 0: count; mode 1: fill at the given offsets.
__device__ void int_list(const TreeView& v, int c, double eps, int mode, uint32_t* n1, uint32_t* n3,
                         int32_t* out1, int32_t* out3, long long cap1, long long cap3, uint32_t off1,
                         uint32_t off3, unsigned* err) {
    const Tree2D& t = v.t;
    Queue q;
    const int L = t.c_level[c], cx = t.c_ix[c], cy = t.c_iy[c];
    const double cur_len = v.len(L), ccx = t.c_cx[c], ccy = t.c_cy[c];
    const long long cnt = 1ll << L;
    for (int k = 0; k < 9; ++k) {
        int jx = cx + k % 3 - 1, jy = cy + k / 3 - 1;
        if (jx < 0 || jy < 0 || jx >= cnt || jy >= cnt) continue;
        q.push(L, jx, jy, v.find(L, jx, jy), 0, err);
    }
    uint32_t k1 = 0, k3 = 0;
    for (int h = 0; h < q.n; ++h) {
        const int e = q.cell[h];
        if (e < 0) {
            int pl = q.lv[h] - 1, px = q.ix[h] >> 1, py = q.iy[h] >> 1;
            if (!q.seen(pl, px, py)) q.push(pl, px, py, v.find(pl, px, py), 1, err);
            continue;
        }
        const uint8_t f = t.c_flags[e];
        if (!(f & CELL_ACTIVE)) continue;
        if (f & CELL_LEAF) {
            if (mode == 1) {
                if ((long long)off1 + k1 < cap1) out1[off1 + k1] = e;
                else set_err(err, ERR_LIST_CAP);
            } else if (mode == 2 && (long long)k1 < cap1) {
                out1[k1] = e;
            }
            ++k1;
            continue;
        }
        if (q.par[h]) continue;
        const double adj = xadd(xdiv(xadd(cur_len, xdiv(v.len(q.lv[h]), 2.0)), 2.0), eps);
        const int c0 = t.c_child0[e];
        const unsigned m = t.c_chmask[e];
        int r = 0;
        for (int d = 0; d < 4; ++d) {
            if (!(m & (1u << d))) continue;
            const int ch = c0 + r++;
            if (!(t.c_flags[ch] & CELL_ACTIVE)) continue;
            const bool adjacent = !(fabs(xsub(t.c_cx[ch], ccx)) > adj) && !(fabs(xsub(t.c_cy[ch], ccy)) > adj);
            if (adjacent) {
                const int chl = q.lv[h] + 1, chx = 2 * q.ix[h] + (d & 1), chy = 2 * q.iy[h] + (d >> 1);
                if (!q.seen(chl, chx, chy)) q.push(chl, chx, chy, ch, 0, err);
            } else {
                if (mode == 1) {
                    if ((long long)off3 + k3 < cap3) out3[off3 + k3] = ch;
                    else set_err(err, ERR_LIST_CAP);
                } else if (mode == 2 && (long long)k3 < cap3) {
                    out3[k3] = ch;
                }
                ++k3;
            }
        }
    }
    *n1 = k1;
    *n3 = k3;
}

// Counts and the first kListSlot1 / kListSlot3 entries of lists 1 and 3 of
// every leaf into fixed slots, in one pass.
__global__ void int_list_slots(Tree2D t, double eps, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    TreeView v(t);
    const int nl = t.info->n_leaves;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.cap_leaves; i += gridDim.x * blockDim.x) {
        if (i >= nl) {
            l.l1_cnt[i] = 0;
            l.l3_cnt[i] = 0;
            continue;
        }
        uint32_t n1, n3;
        int_list(v, t.leaf_cells[i], eps, 2, &n1, &n3, l.l1_slot + (size_t)i * kListSlot1,
                 l.l3_slot + (size_t)i * kListSlot3, kListSlot1, kListSlot3, 0, 0, err);
        l.l1_cnt[i] = n1;
        l.l3_cnt[i] = n3;
    }
}

// Slots to CSR, one warp per leaf; a leaf whose list outgrew its slots is
// filled again by int_list_overflow.
__global__ void int_list_compact(Tree2D t, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nl; i += warps) {
        const uint32_t n1 = l.l1_cnt[i], n3 = l.l3_cnt[i];
        const uint32_t o1 = l.l1_off[i], o3 = l.l3_off[i];
        if (n1 <= kListSlot1 && (long long)o1 + n1 <= l.cap_l1) {
            for (uint32_t k = lane; k < n1; k += 32) l.l1_src[o1 + k] = l.l1_slot[(size_t)i * kListSlot1 + k];
        }
        if (n3 <= kListSlot3 && (long long)o3 + n3 <= l.cap_l3) {
            for (uint32_t k = lane; k < n3; k += 32) l.l3_src[o3 + k] = l.l3_slot[(size_t)i * kListSlot3 + k];
        }
    }
}

__global__ void int_list_overflow(Tree2D t, double eps, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    TreeView v(t);
    const int nl = t.info->n_leaves;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
        const uint32_t n1 = l.l1_cnt[i], n3 = l.l3_cnt[i];
        const bool big1 = n1 > kListSlot1 || (long long)l.l1_off[i] + n1 > l.cap_l1;
        const bool big3 = n3 > kListSlot3 || (long long)l.l3_off[i] + n3 > l.cap_l3;
        if (!big1 && !big3) continue;
        uint32_t m1, m3;
        int_list(v, t.leaf_cells[i], eps, 1, &m1, &m3, l.l1_src, l.l3_src, l.cap_l1, l.cap_l3, l.l1_off[i],
                 l.l3_off[i], err);
    }
}

__global__ void int_list_kernel(Tree2D t, double eps, int mode, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    TreeView v(t);
    const int nl = t.info->n_leaves;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.cap_leaves; i += gridDim.x * blockDim.x) {
        if (i >= nl) {
            if (mode == 0) { l.l1_cnt[i] = 0; l.l3_cnt[i] = 0; }
            continue;
        }
        uint32_t n1, n3;
        const int c = t.leaf_cells[i];
        if (mode == 0) {
            int_list(v, c, eps, 0, &n1, &n3, nullptr, nullptr, 0, 0, 0, 0, err);
            l.l1_cnt[i] = n1;
            l.l3_cnt[i] = n3;
        } else {
            int_list(v, c, eps, 1, &n1, &n3, l.l1_src, l.l3_src, l.cap_l1, l.cap_l3, l.l1_off[i], l.l3_off[i], err);
        }
    }
}

// extList of cell `c` (level >= 2).
__device__ void ext_list(const TreeView& v, int c, double eps, int32_t* l2, uint8_t* slot, uint8_t* n2,
                         int32_t* l4, uint8_t* n4, unsigned* err) {
    const Tree2D& t = v.t;
    const int L = t.c_level[c], cx = t.c_ix[c], cy = t.c_iy[c];
    const double cur_len = v.len(L), ccx = t.c_cx[c], ccy = t.c_cy[c];
    const int p = t.c_parent[c];
    const int PL = L - 1, px = t.c_ix[p], py = t.c_iy[p];
    const long long cnt = 1ll << PL;
    Queue q;  // list-4 candidates
    int k2 = 0;
    const double min2 = xadd(cur_len, eps);
    for (int k = 0; k < 9; ++k) {
        int jx = px + k % 3 - 1, jy = py + k / 3 - 1;
        if (jx < 0 || jy < 0 || jx >= cnt || jy >= cnt) continue;
        if (jx == px && jy == py) continue;
        const int e = v.find(PL, jx, jy);
        if (e < 0) {
            int gl = PL - 1, gx = jx >> 1, gy = jy >> 1;
            if (!q.seen(gl, gx, gy)) q.push(gl, gx, gy, v.find(gl, gx, gy), 0, err);
            continue;
        }
        const uint8_t f = t.c_flags[e];
        if (!(f & CELL_ACTIVE)) continue;
        if (f & CELL_LEAF) {
            q.push(PL, jx, jy, e, 0, err);
            continue;
        }
        const int c0 = t.c_child0[e];
        const unsigned m = t.c_chmask[e];
        int r = 0;
        for (int d = 0; d < 4; ++d) {
            if (!(m & (1u << d))) continue;
            const int ch = c0 + r++;
            if (!(t.c_flags[ch] & CELL_ACTIVE)) continue;
            const bool sep = (fabs(xsub(t.c_cx[ch], ccx)) > min2) || (fabs(xsub(t.c_cy[ch], ccy)) > min2);
            if (!sep) continue;
            if (k2 < kList2Cap) {
                const int dx = 2 * jx + (d & 1) - cx, dy = 2 * jy + (d >> 1) - cy;
                l2[k2] = ch;
                slot[k2] = (uint8_t)((dy + 3) * 7 + (dx + 3));
            } else {
                set_err(err, ERR_LIST2);
            }
            ++k2;
        }
    }
    int k4 = 0;
    for (int h = 0; h < q.n; ++h) {
        const int e = q.cell[h];
        if (e < 0) {
            int gl = q.lv[h] - 1, gx = q.ix[h] >> 1, gy = q.iy[h] >> 1;
            if (!q.seen(gl, gx, gy)) q.push(gl, gx, gy, v.find(gl, gx, gy), 0, err);
            continue;
        }
        const uint8_t f = t.c_flags[e];
        if (!(f & CELL_ACTIVE) || !(f & CELL_LEAF)) continue;
        const double md = xadd(xdiv(xadd(v.len(q.lv[h]), cur_len), 2.0), eps);
        const bool sep = (fabs(xsub(t.c_cx[e], ccx)) > md) || (fabs(xsub(t.c_cy[e], ccy)) > md);
        if (!sep) continue;
        if (k4 < kList4Cap) l4[k4] = e;
        else set_err(err, ERR_LIST4);
        ++k4;
    }
    *n2 = (uint8_t)min(k2, kList2Cap);
    *n4 = (uint8_t)min(k4, kList4Cap);
}

__global__ void ext_list_kernel(Tree2D t, double eps, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    TreeView v(t);
    const int c0 = t.info->level_start[2], c1 = t.info->n_cells;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.cap_cells; i += gridDim.x * blockDim.x) {
        if (i < c0 || i >= c1) {
            if (i < t.cap_cells) { l.l2_n[i] = 0; l.l4_n[i] = 0; }
            continue;
        }
        ext_list(v, i, eps, l.l2_src + (size_t)i * kList2Cap, l.l2_slot + (size_t)i * kList2Cap, &l.l2_n[i],
                 l.l4_src + (size_t)i * kList4Cap, &l.l4_n[i], err);
    }
}

// Interaction totals for the statistics.
__global__ void list_totals(Tree2D t, Lists2D l, unsigned* err) {
    if (fatal(err)) return;
    TreeInfo2D* info = t.info;
    const int nl = info->n_leaves;
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        info->list1_len = l.l1_off[nl];
        info->list3_len = l.l3_off[nl];
    }
}

}  // namespace

cudaError_t build_ext_lists2d(const Tree2D& t, Lists2D& l, double eps, unsigned* err, cudaStream_t st,
                              int* launches) {
    const int gc = std::max(1, std::min(148 * 4, ceil_div(t.cap_cells, 128)));
    ext_list_kernel<<<gc, 128, 0, st>>>(t, eps, l, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t build_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                          cudaStream_t st, int* launches) {
    cudaError_t e = build_ext_lists2d(t, l, eps, err, st, launches);
    if (e != cudaSuccess) return e;
    return build_int_lists2d(t, l, scan, eps, err, st, launches);
}

cudaError_t build_int_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                              cudaStream_t st, int* launches) {
    const int gl = std::max(1, std::min(148 * 4, ceil_div(l.cap_leaves, 128)));
    if (l.l1_slot && l.l3_slot) {
        int_list_slots<<<gl, 128, 0, st>>>(t, eps, l, err);
        cudaError_t e = scan_exclusive(l.l1_cnt, l.l1_off, l.cap_leaves, l.l1_off + l.cap_leaves, scan, err, st);
        if (e != cudaSuccess) return e;
        e = scan_exclusive(l.l3_cnt, l.l3_off, l.cap_leaves, l.l3_off + l.cap_leaves, scan, err, st);
        if (e != cudaSuccess) return e;
        int_list_compact<<<148 * 8, 256, 0, st>>>(t, l, err);
        int_list_overflow<<<gl, 128, 0, st>>>(t, eps, l, err);
        list_totals<<<1, 32, 0, st>>>(t, l, err);
        *launches += 6;
        return cudaGetLastError();
    }
    int_list_kernel<<<gl, 128, 0, st>>>(t, eps, 0, l, err);
    *launches += 1;
    cudaError_t e = scan_exclusive(l.l1_cnt, l.l1_off, l.cap_leaves, l.l1_off + l.cap_leaves, scan, err, st);
    if (e != cudaSuccess) return e;
    e = scan_exclusive(l.l3_cnt, l.l3_off, l.cap_leaves, l.l3_off + l.cap_leaves, scan, err, st);
    if (e != cudaSuccess) return e;
    int_list_kernel<<<gl, 128, 0, st>>>(t, eps, 1, l, err);
    list_totals<<<1, 32, 0, st>>>(t, l, err);
    *launches += 4;
    return cudaGetLastError();
}

}  // namespace vpm
