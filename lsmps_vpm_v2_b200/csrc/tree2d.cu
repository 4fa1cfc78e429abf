// Adaptive quadtree of the reference (TreeCell::initializeTree,
// src/FMM/treeCell.cpp:1043-1243), rebuilt for the GPU.
//
// The reference bins the unsettled particles level by level with
//   index_L = (int)((x - pivot) / (rootLength / 2^L))       treeCell.cpp:290-303
// and makes a cell a leaf when srcParNum <= max_src && parNum <= max_par
// (treeCell.cpp:1195-1196). Dividing by 2^L is exact in binary floating point,
// so RN(d / size_L) = RN(d / size_K) / 2^(K-L) and index_L is the top L bits of
// index_K. One Morton key at level K therefore determines the cell of every
// particle at every level: one stable radix sort of the keys, then each level's
// cells are the distinct key prefixes inside the non-leaf cells of the level
// above. A leaf at level L covers a contiguous range of the sorted particles.
//
// This file is compiled with --fmad=false: every geometric value (root box,
// pivot, index, cell centre) is formed by separate IEEE operations in the
// reference's order.
#include "fmm2d.cuh"

namespace vpm {

namespace {

constexpr int kLvlWarps = 8;                 // parents per tile, one warp each
constexpr int kLvlThreads = 32 * kLvlWarps;
constexpr uint64_t kLvA = 1ull << 62;
constexpr uint64_t kLvP = 2ull << 62;
constexpr uint64_t kLvMask = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bounding box and root geometry (treeCell.cpp:1061-1092).
__global__ void __launch_bounds__(256)
bbox2d(const double* __restrict__ x, const double* __restrict__ y, int n, double exp_pct, int key_levels,
       Geom2D* g, double* partial, unsigned* done, unsigned* err) {
    double mnx = x[0], mxx = x[0], mny = y[0], mxy = y[0];
    bool bad = false;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double a = x[i], b = y[i];
        bad |= !isfinite(a) || !isfinite(b);
        mnx = fmin(mnx, a); mxx = fmax(mxx, a);
        mny = fmin(mny, b); mxy = fmax(mxy, b);
    }
    if (bad) set_err(err, ERR_NONFINITE);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    __shared__ double sh[4][8];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sh[0][warp] = mnx; sh[1][warp] = mxx; sh[2][warp] = mny; sh[3][warp] = mxy; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mnx = fmin(mnx, sh[0][w]); mxx = fmax(mxx, sh[1][w]);
            mny = fmin(mny, sh[2][w]); mxy = fmax(mxy, sh[3][w]);
        }
        double* p = partial + 4 * blockIdx.x;
        p[0] = mnx; p[1] = mxx; p[2] = mny; p[3] = mxy;
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // The last block reduces the per-block partials, all threads in parallel.
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double* p = partial + 4 * b;
        mnx = fmin(mnx, __ldcg(p)); mxx = fmax(mxx, __ldcg(p + 1));
        mny = fmin(mny, __ldcg(p + 2)); mxy = fmax(mxy, __ldcg(p + 3));
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    __syncthreads();
    if (lane == 0) { sh[0][warp] = mnx; sh[1][warp] = mxx; sh[2][warp] = mny; sh[3][warp] = mxy; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        mnx = fmin(mnx, sh[0][w]); mxx = fmax(mxx, sh[1][w]);
        mny = fmin(mny, sh[2][w]); mxy = fmax(mxy, sh[3][w]);
    }
    double root = 0.0;
    double ex = fabs(xsub(mxx, mnx)), ey = fabs(xsub(mxy, mny));
    if (ex > root) root = ex;
    if (ey > root) root = ey;
    double expansion = xadd(1.0, xdiv(exp_pct, 100.0));
    root = xmul(root, expansion);
    g->minx = mnx; g->maxx = mxx; g->miny = mny; g->maxy = mxy;
    g->root = root;
    g->pivx = xdiv(xsub(xadd(mxx, mnx), root), 2.0);
    g->pivy = xdiv(xsub(xadd(mxy, mny), root), 2.0);
    g->size_k = xdiv(root, ldexp(1.0, key_levels));
    if (!(root > 0.0) || !isfinite(root)) set_err(err, ERR_NONFINITE);
    *done = 0;
}

// Morton key of each particle at the key level (treeCell.cpp:290-303).
// Key type KT: 32-bit when 2 * key_levels <= 32 (halves the sort's traffic).
template <typename KT>
__global__ void keys2d(const double* __restrict__ x, const double* __restrict__ y, int n, const Geom2D* g,
                       int key_levels, KT* key, uint32_t* idx, unsigned* err) {
    const double pivx = g->pivx, pivy = g->pivy, s = g->size_k;
    const double lim = ldexp(1.0, key_levels);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double tx = xdiv(xsub(x[i], pivx), s);
        double ty = xdiv(xsub(y[i], pivy), s);
        uint32_t ix = 0, iy = 0;
        if (tx >= 0.0 && tx < lim && ty >= 0.0 && ty < lim) {
            ix = (uint32_t)__double2ull_rz(tx);
            iy = (uint32_t)__double2ull_rz(ty);
        } else {
            set_err(err, ERR_RANGE);
        }
        key[i] = (KT)morton2(ix, iy);
        idx[i] = (uint32_t)i;
    }
}

// Sorted copies of the particle data and the active flags as 0/1 words; the
// sorted keys (from whichever buffer the sort ended in, 32- or 64-bit) and
// permutation land in the tree's own arrays.
template <typename KT>
__global__ void gather2d(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ q,
                         const uint8_t* __restrict__ act, const KT* __restrict__ skey,
                         const uint32_t* __restrict__ sperm, int n, uint64_t* key, uint32_t* perm, double* px,
                         double* py, double* pq, uint8_t* pact, uint32_t* act_u32, unsigned* err) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t j = sperm[i];
        if ((const void*)skey != (const void*)key) key[i] = (uint64_t)skey[i];
        if (sperm != perm) perm[i] = j;
        if (j >= (uint32_t)n) {
            set_err(err, ERR_INDEX);
            continue;
        }
        px[i] = x[j];
        py[i] = y[j];
        pq[i] = q[j];
        uint8_t a = act[j] ? 1 : 0;
        pact[i] = a;
        act_u32[i] = a;
    }
}

// Root cell (treeCell.cpp:1117-1133): never a leaf.
__global__ void tree_root2d(Tree2D t) {
    const Geom2D* g = t.geom;
    TreeInfo2D* info = t.info;
    t.c_lo[0] = 0;
    t.c_hi[0] = t.n;
    int src = (int)t.actscan[t.n];
    t.c_src[0] = src;
    t.c_flags[0] = src != 0 ? CELL_ACTIVE : 0;
    t.c_parent[0] = -1;
    t.c_child0[0] = -1;
    t.c_chmask[0] = 0;
    t.c_level[0] = 0;
    t.c_ix[0] = 0;
    t.c_iy[0] = 0;
    t.c_code[0] = 0;
    t.c_leafidx[0] = -1;
    t.c_cx[0] = xadd(g->pivx, xmul(0.5, g->root));
    t.c_cy[0] = xadd(g->pivy, xmul(0.5, g->root));
    if (t.dense) t.dense[0] = 0;
    for (int L = 0; L < kMaxLevels2D + 3; ++L) {
        info->level_start[L] = L == 0 ? 0 : 1;
        info->leaf_start[L] = 0;
    }
    info->n_cells = 1;
    info->n_leaves = 0;
    info->depth = 0;
}

// The three inner child boundaries of a parent range [lo, hi): the first
// index whose level code (key >> shift) is >= v+1, v+2 and v+3. The three
// 33-ary searches run interleaved, each lane issuing up to three independent
// loads per round, so the warp waits on one chain of dependent loads instead
// of three; the first round's probes are shared. Results are warp-uniform.
__device__ __forceinline__ void warp_split3(const uint64_t* __restrict__ key, int lo, int hi, int shift, uint64_t v,
                                            int lane, int& r1, int& r2, int& r3) {
    int a[3] = {lo, lo, lo}, b[3] = {hi, hi, hi};
    if (hi - lo > 32) {
        const long long len = hi - lo;
        const uint64_t kv = key[lo + (int)(((long long)(lane + 1) * len) / 33)] >> shift;
        #pragma unroll
        for (int t = 0; t < 3; ++t) {
            const unsigned m = __ballot_sync(0xffffffffu, kv >= v + 1 + t);
            if (m == 0) {
                a[t] = lo + (int)((32ll * len) / 33) + 1;
            } else {
                const int f = __ffs(m) - 1;
                b[t] = lo + (int)(((long long)(f + 1) * len) / 33);
                if (f > 0) a[t] = lo + (int)(((long long)f * len) / 33) + 1;
            }
        }
    }
    for (;;) {
        bool more = false;
        uint64_t kv[3];
        #pragma unroll
        for (int t = 0; t < 3; ++t) {
            const long long len = b[t] - a[t];
            kv[t] = 0;
            if (len > 32) {
                more = true;
                kv[t] = key[a[t] + (int)(((long long)(lane + 1) * len) / 33)] >> shift;
            }
        }
        if (!more) break;
        #pragma unroll
        for (int t = 0; t < 3; ++t) {
            const long long len = b[t] - a[t];
            if (len <= 32) continue;
            const unsigned m = __ballot_sync(0xffffffffu, kv[t] >= v + 1 + t);
            const int a0 = a[t];
            if (m == 0) {
                a[t] = a0 + (int)((32ll * len) / 33) + 1;
            } else {
                const int f = __ffs(m) - 1;
                b[t] = a0 + (int)(((long long)(f + 1) * len) / 33);
                if (f > 0) a[t] = a0 + (int)(((long long)f * len) / 33) + 1;
            }
        }
    }
    int r[3];
    uint64_t kv[3];
    #pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int pos = a[t] + lane;
        kv[t] = pos < b[t] ? key[pos] >> shift : 0;
    }
    #pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int pos = a[t] + lane;
        const unsigned m = __ballot_sync(0xffffffffu, pos < b[t] && kv[t] >= v + 1 + t);
        r[t] = m ? a[t] + __ffs(m) - 1 : b[t];
    }
    r1 = r[0];
    r2 = r[1];
    r3 = r[2];
}

__device__ __forceinline__ int sel4(int i, int v0, int v1, int v2, int v3) {
    return i == 0 ? v0 : i == 1 ? v1 : i == 2 ? v2 : v3;
}

// Cells of level L from the non-leaf cells of level L-1, one warp per parent,
// kLvlWarps parents per tile. Tiles take ordered tickets and combine their
// packed (cells, leaves) counts by decoupled look-back, so children are
// emitted in parent order, i.e. Morton order within the level. Each new cell
// also lands in the dense lookup grid (indexed by the reference's cell ID)
// when its level is covered by it.
//
// Everything this step reads that an earlier level wrote (level starts,
// parent cells) is loaded through L2 (ld.cg): in the cooperative kernel all
// levels run in one launch and L1 is not coherent across blocks.
__device__ void level_step(const Tree2D& t, int L, int max_src, int max_par, int* dense, int dense_levels,
                           uint64_t* status, unsigned* ticket, unsigned* err) {
    __shared__ unsigned s_tile;
    __shared__ uint64_t s_prefix;
    __shared__ int s_cnt[kLvlWarps], s_lf[kLvlWarps], s_xc[kLvlWarps], s_xl[kLvlWarps];
    __shared__ unsigned s_stop;
    TreeInfo2D* info = t.info;
    // One read of the error word per block, so the whole block takes the same exit.
    if (threadIdx.x == 0) s_stop = *(volatile const unsigned*)err & (ERR_CELL_CAP | ERR_TIMEOUT | ERR_NONFINITE);
    __syncthreads();
    if (s_stop) return;
    const int p0 = __ldcg(&info->level_start[L - 1]);
    const int np = __ldcg(&info->level_start[L]) - p0;
    const int ntiles = np > 0 ? ceil_div(np, kLvlWarps) : 1;
    const int base_cell = __ldcg(&info->level_start[L]);
    const int base_leaf = __ldcg(&info->leaf_start[L]);
    const int shift = 2 * (t.key_levels - L);
    const double len = xdiv(t.geom->root, ldexp(1.0, L));
    const double pivx = t.geom->pivx, pivy = t.geom->pivy;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
        __syncthreads();
        const int tile = (int)s_tile;
        if (tile >= ntiles) return;
        const int pi = tile * kLvlWarps + warp;
        const int p = p0 + pi;
        const bool nonleaf = pi < np && !(__ldcg(&t.c_flags[p]) & CELL_LEAF);   // warp-uniform
        int b0 = 0, b1 = 0, b2 = 0, b3 = 0, b4 = 0;
        bool has = false, leaf = false;
        unsigned mask = 0, lmask = 0;
        int clo = 0, chi = 0, src = 0;
        if (nonleaf) {
            b0 = __ldcg(&t.c_lo[p]);
            b4 = __ldcg(&t.c_hi[p]);
            const uint64_t pc = __ldcg(&t.c_code[p]) << 2;
            warp_split3(t.key, b0, b4, shift, pc, lane, b1, b2, b3);
            clo = sel4(lane, b0, b1, b2, b3);
            chi = sel4(lane, b1, b2, b3, b4);
            has = lane < 4 && chi > clo;
            if (has) {
                src = (int)(t.actscan[chi] - t.actscan[clo]);
                leaf = src <= max_src && (chi - clo) <= max_par;
            }
            mask = __ballot_sync(0xffffffffu, has);
            lmask = __ballot_sync(0xffffffffu, leaf);
        }
        if (lane == 0) {
            s_cnt[warp] = __popc(mask);
            s_lf[warp] = __popc(lmask);
        }
        __syncthreads();
        if (warp == 0) {
            int c = lane < kLvlWarps ? s_cnt[lane] : 0, lf = lane < kLvlWarps ? s_lf[lane] : 0;
            int ic = c, il = lf;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int yc = __shfl_up_sync(0xffffffffu, ic, o), yl = __shfl_up_sync(0xffffffffu, il, o);
                if (lane >= o) { ic += yc; il += yl; }
            }
            if (lane < kLvlWarps) { s_xc[lane] = ic - c; s_xl[lane] = il - lf; }
            const uint64_t agg = (uint64_t)__shfl_sync(0xffffffffu, ic, 31) |
                                 ((uint64_t)__shfl_sync(0xffffffffu, il, 31) << 31);
            uint64_t prefix = 0;
            if (tile == 0) {
                if (lane == 0) st_relaxed(&status[0], kLvP | agg);
            } else {
                if (lane == 0) st_relaxed(&status[tile], kLvA | agg);
                prefix = warp_lookback<kLvP, kLvMask>(status, tile, err);
                if (lane == 0) st_relaxed(&status[tile], kLvP | (prefix + agg));
            }
            if (lane == 0) {
                s_prefix = prefix;
                if (tile == ntiles - 1) {
                    const uint64_t tot = prefix + agg;
                    const int ncell = (int)(tot & 0x7FFFFFFFull), nlf = (int)(tot >> 31);
                    for (int k2 = L + 1; k2 < kMaxLevels2D + 3; ++k2) {
                        info->level_start[k2] = base_cell + ncell;
                        info->leaf_start[k2] = base_leaf + nlf;
                    }
                    info->n_cells = base_cell + ncell;
                    info->n_leaves = base_leaf + nlf;
                    if (ncell > 0) info->depth = L;
                    if (base_cell + ncell > t.cap_cells) set_err(err, ERR_CELL_CAP);
                }
            }
        }
        __syncthreads();
        if (nonleaf) {
            const int nchild = __popc(mask);
            const int ci0 = base_cell + (int)(s_prefix & 0x7FFFFFFFull) + s_xc[warp];
            const int li0 = base_leaf + (int)(s_prefix >> 31) + s_xl[warp];
            if (lane == 0) {
                const bool fits = ci0 + nchild <= t.cap_cells;
                t.c_child0[p] = fits ? ci0 : -1;
                t.c_chmask[p] = fits ? (uint8_t)mask : 0;
            }
            if (has) {
                const unsigned below = (1u << lane) - 1u;
                const int ci = ci0 + __popc(mask & below);
                if (ci >= t.cap_cells) {
                    set_err(err, ERR_CELL_CAP);
                } else {
                    const int ix = 2 * __ldcg(&t.c_ix[p]) + (lane & 1), iy = 2 * __ldcg(&t.c_iy[p]) + (lane >> 1);
                    t.c_lo[ci] = clo;
                    t.c_hi[ci] = chi;
                    t.c_src[ci] = src;
                    t.c_flags[ci] = (leaf ? CELL_LEAF : 0) | (src != 0 ? CELL_ACTIVE : 0);
                    t.c_parent[ci] = p;
                    t.c_child0[ci] = -1;
                    t.c_chmask[ci] = 0;
                    t.c_level[ci] = (uint8_t)L;
                    t.c_ix[ci] = ix;
                    t.c_iy[ci] = iy;
                    t.c_code[ci] = (__ldcg(&t.c_code[p]) << 2) + lane;
                    t.c_cx[ci] = xadd(pivx, xmul(xadd(0.5, (double)ix), len));
                    t.c_cy[ci] = xadd(pivy, xmul(xadd(0.5, (double)iy), len));
                    if (dense && L <= dense_levels) dense[start_id2(L) + ix + ((int64_t)iy << L)] = ci;
                    if (leaf) {
                        const int li = li0 + __popc(lmask & below);
                        t.c_leafidx[ci] = li;
                        t.leaf_cells[li] = ci;
                    } else {
                        t.c_leafidx[ci] = -1;
                        if (L == t.key_levels) set_err(err, ERR_DEPTH);
                    }
                }
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kLvlThreads)
tree_level2d(Tree2D t, int L, int max_src, int max_par, int* dense, int dense_levels, uint64_t* status,
             unsigned* ticket, unsigned* err) {
    level_step(t, L, max_src, max_par, dense, dense_levels, status, ticket, err);
}

// All levels in one cooperative launch: a grid barrier between levels, and a
// stop as soon as a level creates no cells (that test reads a value written
// before the barrier, so every block takes the same decision).
__global__ void __launch_bounds__(kLvlThreads)
tree_levels_coop(Tree2D t, int max_src, int max_par, int* dense, int dense_levels, uint64_t* status, int stride,
                 unsigned* tickets, unsigned* bar, unsigned* err) {
    for (int L = 1; L <= t.key_levels; ++L) {
        level_step(t, L, max_src, max_par, dense, dense_levels, status + (size_t)L * stride, tickets + L, err);
        grid_sync(bar, err);
        const int created = __ldcg(&t.info->level_start[L + 1]) - __ldcg(&t.info->level_start[L]);
        if (created == 0) break;
    }
}

// Leaf level range (TreeCell::min_level / max_level, treeCell.cpp:1236-1240).
__global__ void tree_finish2d(TreeInfo2D* info) {
    int mn = -1, mx = -1;
    for (int L = 0; L <= kMaxLevels2D; ++L) {
        if (info->leaf_start[L + 1] > info->leaf_start[L]) {
            if (mn < 0) mn = L;
            mx = L;
        }
    }
    info->min_leaf_level = mn;
    info->max_leaf_level = mx;
}

}  // namespace

cudaError_t keys_sort2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                        TreeScratch2D& s, double exp_pct, unsigned* err, cudaStream_t st, int* launches) {
    const int n = t.n;
    const int K = t.key_levels;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    unsigned* done = s.lvl_ticket + kMaxLevels2D + 1;
    const int bb_blocks = std::max(1, std::min(kBBoxBlocks, ceil_div(n, 256)));
    cudaError_t e = cudaMemsetAsync(s.lvl_ticket, 0, sizeof(unsigned) * kTicketWords, st);
    if (e != cudaSuccess) return e;
    bbox2d<<<bb_blocks, 256, 0, st>>>(x, y, n, exp_pct, K, t.geom, s.bbox_partial, done, err);
    *launches += 2;
    uint32_t* vals = t.perm;
    if (2 * K <= 32) {
        // 32-bit keys in the two halves of key_alt
        uint32_t* k32 = reinterpret_cast<uint32_t*>(s.key_alt);
        keys2d<uint32_t><<<gridN, 256, 0, st>>>(x, y, n, t.geom, K, k32, t.perm, err);
        e = radix_sort_pairs(&k32, &vals, k32 + n, s.val_alt, n, 2 * K, s.sort, err, st, launches);
        if (e != cudaSuccess) return e;
        gather2d<uint32_t><<<gridN, 256, 0, st>>>(x, y, q, act, k32, vals, n, t.key, t.perm, t.px, t.py, t.pq,
                                                  t.pact, s.act_u32, err);
    } else {
        uint64_t* keys = t.key;
        keys2d<uint64_t><<<gridN, 256, 0, st>>>(x, y, n, t.geom, K, t.key, t.perm, err);
        e = radix_sort_pairs(&keys, &vals, s.key_alt, s.val_alt, n, 2 * K, s.sort, err, st, launches);
        if (e != cudaSuccess) return e;
        gather2d<uint64_t><<<gridN, 256, 0, st>>>(x, y, q, act, keys, vals, n, t.key, t.perm, t.px, t.py, t.pq,
                                                  t.pact, s.act_u32, err);
    }
    *launches += 1;
    e = scan_exclusive(s.act_u32, t.actscan, n, t.actscan + n, s.scan, err, st);
    if (e != cudaSuccess) return e;
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t levels2d(Tree2D& t, TreeScratch2D& s, int max_src, int max_par, unsigned* err, cudaStream_t st,
                     int* launches) {
    const int K = t.key_levels;
    cudaError_t e = cudaMemsetAsync(s.lvl_status, 0, sizeof(uint64_t) * (size_t)(K + 1) * s.lvl_max_tiles, st);
    if (e != cudaSuccess) return e;
    tree_root2d<<<1, 1, 0, st>>>(t);
    *launches += 1;
    if (t.gbar) {
        int grid = 0;
        e = launch_coop(tree_levels_coop, kLvlThreads, 0, st, 8, &grid, t, max_src, max_par, t.dense, t.dense_levels,
                        s.lvl_status, s.lvl_max_tiles, s.lvl_ticket, t.gbar, err);
        if (e == cudaSuccess) {
            *launches += 1;
            tree_finish2d<<<1, 1, 0, st>>>(t.info);
            *launches += 1;
            return cudaGetLastError();
        }
        (void)cudaGetLastError();  // cooperative launch refused: one launch per level instead
    }
    for (int L = 1; L <= K; ++L) {
        long long bound = std::min<long long>(t.cap_cells, 1ll << std::min(2 * (L - 1), 40));
        int tiles = std::max(1, ceil_div(bound, kLvlWarps));
        if (tiles > s.lvl_max_tiles) return cudaErrorInvalidValue;
        int grid = std::min(tiles, 148 * 8);
        tree_level2d<<<grid, kLvlThreads, 0, st>>>(t, L, max_src, max_par, t.dense, t.dense_levels,
                                                   s.lvl_status + (size_t)L * s.lvl_max_tiles, s.lvl_ticket + L, err);
        *launches += 1;
    }
    tree_finish2d<<<1, 1, 0, st>>>(t.info);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t build_tree2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                         TreeScratch2D& s, int max_src, int max_par, double exp_pct, unsigned* err, cudaStream_t st,
                         int* launches) {
    cudaError_t e = keys_sort2d(x, y, q, act, t, s, exp_pct, err, st, launches);
    if (e != cudaSuccess) return e;
    return levels2d(t, s, max_src, max_par, err, st, launches);
}

}  // namespace vpm
