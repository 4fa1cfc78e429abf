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
    // since the grid is never cleared); below the dense levels, the dense
    // ancestor's children are followed down (one child mask and first child
    // per level); without a dense grid, a binary search of the level's Morton
    // codes.
    __device__ int find(int L, int ix, int iy) const {
        if (L < 0 || L > depth) return -1;
        const long long cnt = 1ll << L;
        if (ix < 0 || iy < 0 || ix >= cnt || iy >= cnt) return -1;
        if (t.dense) {
            const int D = L < t.dense_levels ? L : t.dense_levels;
            const int ax = ix >> (L - D), ay = iy >> (L - D);
            int e = t.dense[start_id2(D) + ax + ((int64_t)ay << D)];
            if (!(e >= 0 && e < n_cells && t.c_level[e] == D && t.c_ix[e] == ax && t.c_iy[e] == ay)) return -1;
            for (int lv = D + 1; lv <= L; ++lv) {
                const unsigned m = t.c_chmask[e];
                const int d = ((ix >> (L - lv)) & 1) | (((iy >> (L - lv)) & 1) << 1);
                if (!(m & (1u << d))) return -1;
                e = t.c_child0[e] + __popc(m & ((1u << d) - 1u));
            }
            return e;
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
    const int L = t.c_level[c], cx = t.c_ix[c], cy = t.c_iy[c];
    const long long cnt = 1ll << L;
    // The nine same-level neighbours (-2: outside the box). When each one
    // exists and is a leaf or inactive, the queue below would take exactly the
    // active ones in this order and open nothing: list 1 is those, list 3 is
    // empty.
    int nb[9];
    bool simple = true;
    #pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int jx = cx + k % 3 - 1, jy = cy + k / 3 - 1;
        nb[k] = (jx < 0 || jy < 0 || jx >= cnt || jy >= cnt) ? -2 : v.find(L, jx, jy);
    }
    uint8_t nf[9];
    #pragma unroll
    for (int k = 0; k < 9; ++k) {
        nf[k] = nb[k] >= 0 ? t.c_flags[nb[k]] : 0;
        if (nb[k] == -1 || (nb[k] >= 0 && (nf[k] & CELL_ACTIVE) && !(nf[k] & CELL_LEAF))) simple = false;
    }
    if (simple) {
        uint32_t k1 = 0;
        #pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (nb[k] < 0 || !(nf[k] & CELL_ACTIVE)) continue;
            if (mode == 1) {
                if ((long long)off1 + k1 < cap1) out1[off1 + k1] = nb[k];
                else set_err(err, ERR_LIST_CAP);
            } else if (mode == 2 && (long long)k1 < cap1) {
                out1[k1] = nb[k];
            }
            ++k1;
        }
        *n1 = k1;
        *n3 = 0;
        return;
    }
    Queue q;
    const double cur_len = v.len(L), ccx = t.c_cx[c], ccy = t.c_cy[c];
    for (int k = 0; k < 9; ++k)
        if (nb[k] != -2) q.push(L, cx + k % 3 - 1, cy + k / 3 - 1, nb[k], 0, err);
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

// intList of leaf `c` by one warp. The reference's FIFO queue is run in
// rounds: the entries queued before a round are processed by one lane each
// (32 at a time, in queue order), and their list-1/list-3 outputs and new
// queue entries are placed by warp prefix sums in (entry, child) order, so
// the lists and the queue come out exactly as the sequential queue makes
// them. A new entry is dropped when the same cell is already queued or was
// proposed by an earlier entry of the same group (the reference's `seen`).
// Leaves whose nine neighbours all exist and are leaves or inactive skip the
// queue. Outputs as int_list (mode 1: CSR at off1/off3; mode 2: slots);
// returns the list lengths in lane 0's *n1 / *n3.
struct WarpQueue {
    long long key[kQueueCap];   // start_id2(level) + ix + iy 2^level
    int cell[kQueueCap];
    uint8_t par[kQueueCap];
    long long cand[4 * 32];     // proposals of the current group, in order
};

__device__ __forceinline__ long long cell_key(int L, int x, int y) {
    return (long long)start_id2(L) + x + ((long long)y << L);
}
__device__ __forceinline__ void key_cell(long long k, int& L, int& x, int& y) {
    int lv = 0;
    while (lv < 31 && (long long)start_id2(lv + 1) <= k) ++lv;
    const long long r = k - (long long)start_id2(lv);
    L = lv;
    x = (int)(r & ((1ll << lv) - 1));
    y = (int)(r >> lv);
}

__device__ void int_list_warp(const TreeView& v, int c, double eps, int mode, uint32_t* n1o, uint32_t* n3o,
                              int32_t* out1, int32_t* out3, long long cap1, long long cap3, uint32_t off1,
                              uint32_t off3, WarpQueue& q, unsigned* err) {
    const Tree2D& t = v.t;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int L = t.c_level[c], cx = t.c_ix[c], cy = t.c_iy[c];
    const long long cnt = 1ll << L;
    const int jx = cx + lane % 3 - 1, jy = cy + lane / 3 - 1;
    const bool inr = lane < 9 && !(jx < 0 || jy < 0 || jx >= cnt || jy >= cnt);
    const int e0 = inr ? v.find(L, jx, jy) : -2;
    const uint8_t f0 = e0 >= 0 ? t.c_flags[e0] : 0;
    uint32_t k1 = 0, k3 = 0;
    auto put1 = [&](uint32_t pos, int val) {
        if (mode == 1) {
            if ((long long)off1 + pos < cap1) out1[off1 + pos] = val;
            else set_err(err, ERR_LIST_CAP);
        } else if (mode == 2 && (long long)pos < cap1) {
            out1[pos] = val;
        }
    };
    auto put3 = [&](uint32_t pos, int val) {
        if (mode == 1) {
            if ((long long)off3 + pos < cap3) out3[off3 + pos] = val;
            else set_err(err, ERR_LIST_CAP);
        } else if (mode == 2 && (long long)pos < cap3) {
            out3[pos] = val;
        }
    };
    const bool open0 = inr && (e0 == -1 || (e0 >= 0 && (f0 & CELL_ACTIVE) && !(f0 & CELL_LEAF)));
    if (!__any_sync(0xffffffffu, open0)) {
        const bool take = e0 >= 0 && (f0 & CELL_ACTIVE);
        const unsigned b = __ballot_sync(0xffffffffu, take);
        if (take) put1(__popc(b & lt), e0);
        *n1o = __popc(b);
        *n3o = 0;
        return;
    }
    const double cur_len = v.len(L), ccx = t.c_cx[c], ccy = t.c_cy[c];
    // queue: the in-range neighbours in order
    {
        const unsigned b = __ballot_sync(0xffffffffu, inr);
        if (inr) {
            const int pos = __popc(b & lt);
            q.key[pos] = cell_key(L, jx, jy);
            q.cell[pos] = e0;
            q.par[pos] = 0;
        }
        __syncwarp();
    }
    int tail = __popc(__ballot_sync(0xffffffffu, inr));
    int head = 0;
    while (head < tail) {
        const int end = tail;   // this round: entries [head, end)
        for (int base = head; base < end; base += 32) {
            const int h = base + lane;
            const bool has = h < end;
            int hl = 0, hx = 0, hy = 0, he = -2;
            uint8_t hp = 0, hf = 0;
            if (has) {
                key_cell(q.key[h], hl, hx, hy);
                he = q.cell[h];
                hp = q.par[h];
                if (he >= 0) hf = t.c_flags[he];
            }
            const bool active = he >= 0 && (hf & CELL_ACTIVE);
            // list 1
            const bool is1 = active && (hf & CELL_LEAF);
            const unsigned b1 = __ballot_sync(0xffffffffu, is1);
            if (is1) put1(k1 + __popc(b1 & lt), he);
            k1 += __popc(b1);
            // proposals (in d order) and list-3 children
            long long prop[4];
            int np = 0, n3 = 0, l3c[4];
            if (has && he < 0) {
                prop[np++] = cell_key(hl - 1, hx >> 1, hy >> 1);
            } else if (active && !(hf & CELL_LEAF) && !hp) {
                const double adj = xadd(xdiv(xadd(cur_len, xdiv(v.len(hl), 2.0)), 2.0), eps);
                const int c0 = t.c_child0[he];
                const unsigned m = t.c_chmask[he];
                int r = 0;
                for (int d = 0; d < 4; ++d) {
                    if (!(m & (1u << d))) continue;
                    const int ch = c0 + r++;
                    if (!(t.c_flags[ch] & CELL_ACTIVE)) continue;
                    const bool adjacent =
                        !(fabs(xsub(t.c_cx[ch], ccx)) > adj) && !(fabs(xsub(t.c_cy[ch], ccy)) > adj);
                    if (adjacent) prop[np++] = cell_key(hl + 1, 2 * hx + (d & 1), 2 * hy + (d >> 1));
                    else l3c[n3++] = ch;
                }
            }
            // list 3 in (entry, child) order
            {
                int x = n3;
                #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                const int tot = __shfl_sync(0xffffffffu, x, 31);
                for (int i = 0; i < n3; ++i) put3(k3 + (x - n3) + i, l3c[i]);
                k3 += tot;
            }
            // stage the proposals in order, then keep those not yet queued nor proposed before
            int x = np;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            const int ntot = __shfl_sync(0xffffffffu, x, 31);
            const int p0 = x - np;
            for (int i = 0; i < np; ++i) q.cand[p0 + i] = prop[i];
            __syncwarp();
            int keep = 0;
            bool kept[4] = {false, false, false, false};
            for (int i = 0; i < np; ++i) {
                const long long kk = prop[i];
                bool dup = false;
                for (int j = 0; j < tail && !dup; ++j) dup = q.key[j] == kk;
                for (int j = 0; j < p0 + i && !dup; ++j) dup = q.cand[j] == kk;
                kept[i] = !dup;
                keep += !dup;
            }
            int y = keep;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            const int ktot = __shfl_sync(0xffffffffu, y, 31);
            __syncwarp();
            int w = tail + (y - keep);
            for (int i = 0; i < np; ++i) {
                if (!kept[i]) continue;
                if (w < kQueueCap) {
                    int pl, px, py;
                    key_cell(prop[i], pl, px, py);
                    q.key[w] = prop[i];
                    q.cell[w] = v.find(pl, px, py);
                    q.par[w] = he < 0 ? 1 : 0;
                } else {
                    set_err(err, ERR_QUEUE);
                }
                ++w;
            }
            (void)ntot;
            tail = min(kQueueCap, tail + ktot);
            __syncwarp();
        }
        head = end;
    }
    *n1o = k1;
    *n3o = k3;
}

// Counts and the first kListSlot1 / kListSlot3 entries of lists 1 and 3 of
// every leaf into fixed slots, in one pass; one warp per leaf.
__global__ void __launch_bounds__(128) int_list_slots(Tree2D t, double eps, Lists2D l, unsigned* err) {
    __shared__ WarpQueue s_q[4];
    if (fatal(err)) return;
    TreeView v(t);
    const int nl = t.info->n_leaves;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int i = nl + blockIdx.x * blockDim.x + threadIdx.x; i < l.cap_leaves; i += gridDim.x * blockDim.x) {
        l.l1_cnt[i] = 0;
        l.l3_cnt[i] = 0;
    }
    for (int i = blockIdx.x * 4 + wib; i < nl; i += gridDim.x * 4) {
        uint32_t n1, n3;
        int_list_warp(v, t.leaf_cells[i], eps, 2, &n1, &n3, l.l1_slot + (size_t)i * kListSlot1,
                      l.l3_slot + (size_t)i * kListSlot3, kListSlot1, kListSlot3, 0, 0, s_q[wib], err);
        if (lane == 0) {
            l.l1_cnt[i] = n1;
            l.l3_cnt[i] = n3;
        }
        __syncwarp();
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

// extList of cell `c` (level >= 2), one warp per cell. Lane (k, d) takes
// child d of the k-th of the parent's eight neighbours (the reference's
// neighbour order with the parent itself skipped): list 2 is the ballot of
// the active children separated from c, in (k, d) order as the reference
// appends them. Neighbours that are missing or leaves seed the list-4 queue,
// which lane 0 then runs exactly as the reference does (it is empty for most
// cells).
__device__ void ext_list_warp(const TreeView& v, int c, double eps, int32_t* l2, uint8_t* slot, uint8_t* n2,
                              int32_t* l4, uint8_t* n4, int32_t* blk, int* s_e, unsigned* err) {
    const Tree2D& t = v.t;
    const int lane = threadIdx.x & 31;
    const int L = t.c_level[c], cx = t.c_ix[c], cy = t.c_iy[c];
    const double cur_len = v.len(L), ccx = t.c_cx[c], ccy = t.c_cy[c];
    const int p = t.c_parent[c];
    const int PL = L - 1, px = t.c_ix[p], py = t.c_iy[p];
    const long long cnt = 1ll << PL;
    const int k8 = lane >> 2, d = lane & 3;
    const int k = k8 < 4 ? k8 : k8 + 1;   // neighbour index 0..8 without the centre
    const int jx = px + k % 3 - 1, jy = py + k / 3 - 1;
    const bool inr = !(jx < 0 || jy < 0 || jx >= cnt || jy >= cnt);
    int e = -2;   // -2: outside the box
    if (d == 0 && inr) e = v.find(PL, jx, jy);
    e = __shfl_sync(0xffffffffu, e, lane & ~3);
    const uint8_t f = e >= 0 ? t.c_flags[e] : 0;
    const bool open = e >= 0 && (f & CELL_ACTIVE) && !(f & CELL_LEAF);
    // list 2: child d of an open neighbour, active and separated from c
    bool take = false;
    int ch = -1, cand = -1;
    if (open) {
        const unsigned m = t.c_chmask[e];
        if (m & (1u << d)) {
            ch = t.c_child0[e] + __popc(m & ((1u << d) - 1u));
            if (t.c_flags[ch] & CELL_ACTIVE) {
                cand = ch;
                const double min2 = xadd(cur_len, eps);
                take = (fabs(xsub(t.c_cx[ch], ccx)) > min2) || (fabs(xsub(t.c_cy[ch], ccy)) > min2);
            }
        }
    }
    // the candidates of the parent's children, once per parent (by its first child)
    if (blk && c == t.c_child0[p]) blk[(size_t)p * 32 + lane] = cand;
    // The per-parent M2L of the mixed form takes list 2 to be the candidates
    // at an integer offset of 2 or more on some axis; flag a tree where the
    // tolerance of the separation test decides otherwise.
    {
        const int ox = 2 * jx + (d & 1) - cx, oy = 2 * jy + (d >> 1) - cy;
        const bool far = ox <= -2 || ox >= 2 || oy <= -2 || oy >= 2;
        if (__any_sync(0xffffffffu, cand >= 0 && take != far) && lane == 0) atomicOr(&t.info->l2_irregular, 1);
    }
    const unsigned tb = __ballot_sync(0xffffffffu, take);
    if (take) {
        const int pos = __popc(tb & ((1u << lane) - 1u));
        if (pos < kList2Cap) {
            const int dx = 2 * jx + (d & 1) - cx, dy = 2 * jy + (d >> 1) - cy;
            l2[pos] = ch;
            slot[pos] = (uint8_t)((dy + 3) * 7 + (dx + 3));
        }
    }
    // list-4 seeds: a missing neighbour (its parent) or an active leaf one
    const bool seed = d == 0 && inr && (e == -1 || (e >= 0 && (f & CELL_ACTIVE) && (f & CELL_LEAF)));
    const unsigned sb = __ballot_sync(0xffffffffu, seed);
    if (d == 0) s_e[k8] = e;
    __syncwarp();
    int k4 = 0;
    if (sb && lane == 0) {
        Queue q;
        for (int kk = 0; kk < 8; ++kk) {
            if (!(sb & (1u << (4 * kk)))) continue;
            const int nk = kk < 4 ? kk : kk + 1;
            const int qx = px + nk % 3 - 1, qy = py + nk / 3 - 1;
            const int ee = s_e[kk];
            if (ee < 0) {
                const int gl = PL - 1, gx = qx >> 1, gy = qy >> 1;
                if (!q.seen(gl, gx, gy)) q.push(gl, gx, gy, v.find(gl, gx, gy), 0, err);
            } else {
                q.push(PL, qx, qy, ee, 0, err);
            }
        }
        for (int h = 0; h < q.n; ++h) {
            const int ee = q.cell[h];
            if (ee < 0) {
                int gl = q.lv[h] - 1, gx = q.ix[h] >> 1, gy = q.iy[h] >> 1;
                if (!q.seen(gl, gx, gy)) q.push(gl, gx, gy, v.find(gl, gx, gy), 0, err);
                continue;
            }
            const uint8_t ff = t.c_flags[ee];
            if (!(ff & CELL_ACTIVE) || !(ff & CELL_LEAF)) continue;
            const double md = xadd(xdiv(xadd(v.len(q.lv[h]), cur_len), 2.0), eps);
            const bool sep = (fabs(xsub(t.c_cx[ee], ccx)) > md) || (fabs(xsub(t.c_cy[ee], ccy)) > md);
            if (!sep) continue;
            if (k4 < kList4Cap) l4[k4] = ee;
            else set_err(err, ERR_LIST4);
            ++k4;
        }
    }
    if (lane == 0) {
        const int k2 = __popc(tb);
        if (k2 > kList2Cap) set_err(err, ERR_LIST2);
        *n2 = (uint8_t)min(k2, kList2Cap);
        *n4 = (uint8_t)min(k4, kList4Cap);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(128) ext_list_kernel(Tree2D t, double eps, Lists2D l, unsigned* err) {
    __shared__ int s_e[4][8];
    if (fatal(err)) return;
    TreeView v(t);
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int c0 = t.info->level_start[2], c1 = t.info->n_cells;
    const int warps = gridDim.x * 4;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.cap_cells; i += gridDim.x * blockDim.x)
        if (i < c0 || i >= c1) {
            l.l2_n[i] = 0;
            l.l4_n[i] = 0;
        }
    for (int i = c0 + blockIdx.x * 4 + wib; i < c1; i += warps)
        ext_list_warp(v, i, eps, l.l2_src + (size_t)i * kList2Cap, l.l2_slot + (size_t)i * kList2Cap, &l.l2_n[i],
                      l.l4_src + (size_t)i * kList4Cap, &l.l4_n[i], l.l2_blk, s_e[wib], err);
    (void)lane;
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
    ext_list_kernel<<<148 * 16, 128, 0, st>>>(t, eps, l, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t build_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                          cudaStream_t st, int* launches) {
    cudaError_t e = build_ext_lists2d(t, l, eps, err, st, launches);
    if (e != cudaSuccess) return e;
    return build_int_lists2d(t, l, scan, eps, err, st, launches);
}

bool int_lists_slotted(const Lists2D& l) { return l.l1_slot && l.l3_slot; }

cudaError_t build_int_slots2d(const Tree2D& t, Lists2D& l, double eps, unsigned* err, cudaStream_t st, int* launches) {
    if (!int_lists_slotted(l)) return cudaErrorInvalidValue;
    int_list_slots<<<148 * 16, 128, 0, st>>>(t, eps, l, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t build_int_csr2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                            cudaStream_t st, int* launches) {
    if (!int_lists_slotted(l)) return cudaErrorInvalidValue;
    const int gl = std::max(1, std::min(148 * 4, ceil_div(l.cap_leaves, 128)));
    cudaError_t e = scan_exclusive(l.l1_cnt, l.l1_off, l.cap_leaves, l.l1_off + l.cap_leaves, scan, err, st);
    if (e != cudaSuccess) return e;
    e = scan_exclusive(l.l3_cnt, l.l3_off, l.cap_leaves, l.l3_off + l.cap_leaves, scan, err, st);
    if (e != cudaSuccess) return e;
    int_list_compact<<<148 * 8, 256, 0, st>>>(t, l, err);
    int_list_overflow<<<gl, 128, 0, st>>>(t, eps, l, err);
    list_totals<<<1, 32, 0, st>>>(t, l, err);
    *launches += 5;
    return cudaGetLastError();
}

cudaError_t build_int_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                              cudaStream_t st, int* launches) {
    const int gl = std::max(1, std::min(148 * 4, ceil_div(l.cap_leaves, 128)));
    if (int_lists_slotted(l)) {
        cudaError_t e = build_int_slots2d(t, l, eps, err, st, launches);
        if (e != cudaSuccess) return e;
        return build_int_csr2d(t, l, scan, eps, err, st, launches);
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
