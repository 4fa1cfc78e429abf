// Octree of the reference's default 3D velocity path and its upward pass:
//   root box                FMMCell::generateTree   src/FMM/fast3DFMM.cpp:499-538
//   level-by-level binning  fast3DFMM.cpp:620-705   (octant rule fast3DFMM.hpp:17-22)
//   active flags            fast3DFMM.cpp:711-741
//   P2M                     fast3DFMM.cpp:164-214, fmm3D.cpp:84-103
//   M2M                     fast3DFMM.cpp:230-302, fmm3D.cpp:114-132
// Compiled with --fmad=false: cell centres, octant tests and the moment sums
// round exactly as the reference's scalar code, in the same order.
#include "fmm3d.cuh"

#include <algorithm>

namespace vpm {

namespace {

constexpr int kT3Threads = 256;
constexpr int kBBox3Blocks = 296;

// Min/max of the particle box joined with the domain centre, root length and
// centre (fast3DFMM.cpp:506-528). Each block reduces its share; the last
// block to finish combines the partials and writes the geometry.
// treecell: the particle box alone (start from the empty box), then the
// TreeCell root length and pivot (treeCell.cpp:1058-1090).
__global__ void __launch_bounds__(256)
bbox3d(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z, int n,
       double cx0, double cy0, double cz0, double exp_pct, bool treecell, Geom3D* g, double* partial,
       unsigned* done, unsigned* err) {
    __shared__ double s_v[6][256];
    __shared__ bool s_last;
    const double lo0[3] = {treecell ? HUGE_VAL : cx0, treecell ? HUGE_VAL : cy0, treecell ? HUGE_VAL : cz0};
    const double hi0[3] = {treecell ? -HUGE_VAL : cx0, treecell ? -HUGE_VAL : cy0, treecell ? -HUGE_VAL : cz0};
    double mn[3] = {lo0[0], lo0[1], lo0[2]}, mx[3] = {hi0[0], hi0[1], hi0[2]};
    const double* p[3] = {x, y, z};
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double v = p[d][i];
            if (!isfinite(v)) bad = true;
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
        }
    }
    if (bad) set_err(err, ERR_NONFINITE);
    #pragma unroll
    for (int d = 0; d < 3; ++d) {
        s_v[d][threadIdx.x] = mn[d];
        s_v[3 + d][threadIdx.x] = mx[d];
    }
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                s_v[d][threadIdx.x] = fmin(s_v[d][threadIdx.x], s_v[d][threadIdx.x + o]);
                s_v[3 + d][threadIdx.x] = fmax(s_v[3 + d][threadIdx.x], s_v[3 + d][threadIdx.x + o]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[blockIdx.x * 6 + threadIdx.x] = s_v[threadIdx.x][0];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: combine the partials
    double a[6] = {lo0[0], lo0[1], lo0[2], hi0[0], hi0[1], hi0[2]};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            a[d] = fmin(a[d], __ldcg(&partial[b * 6 + d]));
            a[3 + d] = fmax(a[3 + d], __ldcg(&partial[b * 6 + 3 + d]));
        }
    }
    #pragma unroll
    for (int d = 0; d < 6; ++d) s_v[d][threadIdx.x] = a[d];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                s_v[d][threadIdx.x] = fmin(s_v[d][threadIdx.x], s_v[d][threadIdx.x + o]);
                s_v[3 + d][threadIdx.x] = fmax(s_v[3 + d][threadIdx.x], s_v[3 + d][threadIdx.x + o]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double root = 0.0;
        for (int d = 0; d < 3; ++d) {
            g->mn[d] = s_v[d][0];
            g->mx[d] = s_v[3 + d][0];
            const double len = xsub(g->mx[d], g->mn[d]);
            root = len > root ? len : root;   // std::max(domLen[d], rootLength)
            g->cen[d] = xmul(0.5, xadd(g->mx[d], g->mn[d]));
        }
        g->root = xmul(root, xadd(1.0, xdiv(exp_pct, 100.0)));
        if (!(g->root > 0.0)) set_err(err, ERR_RANGE);   // all particles at the domain centre
        for (int d = 0; d < 3; ++d) g->piv[d] = xdiv(xsub(xadd(g->mx[d], g->mn[d]), g->root), 2.0);
        *done = 0;
    }
}

// Root cell and the per-particle build state (fast3DFMM.cpp:533-550, 620-625).
__global__ void root3d(Tree3D t) {
    const int n = t.n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        t.pcell[i] = 0;
        t.settled[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const Geom3D* g = t.geom;
        t.c_x[0] = g->cen[0];
        t.c_y[0] = g->cen[1];
        t.c_z[0] = g->cen[2];
        t.c_size[0] = g->root;
        t.c_npar[0] = n;
        t.c_parent[0] = -1;
        t.c_child0[0] = -1;
        t.c_chmask[0] = 0;
        t.c_active[0] = 1;
        t.c_level[0] = 0;
        TreeInfo3D* info = t.info;
        for (int L = 0; L < kMaxLevels3D + 2; ++L) info->level_start[L] = L == 0 ? 0 : 1;
        info->n_cells = 1;
        info->n_leaves = 0;
        info->depth = 0;
        info->remaining = n;
        info->scan_total = 0;
        info->p2p_pairs = 0;
        info->m2p_pairs = 0;
    }
}

__device__ __forceinline__ int block_sum_int(int v, int* s_red) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    int tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_red[w];
    return tot;
}

// Exclusive scan of one int per thread over the block (blockDim = 256).
__device__ __forceinline__ int block_excl_int(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    int base = 0, tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        if (w < warp) base += s_warp[w];
        tot += s_warp[w];
    }
    *total = tot;
    return base + x - v;
}

// All levels of the octree in one cooperative launch (fast3DFMM.cpp:620-705).
// Per level: (1) every unsettled particle finds its octant in its current
// cell and flags that child; (2) the children of the level's cells are
// numbered, parents in order and octants 0..7 under each parent, and their
// centres computed as the reference does (size/2, centre + len (bit - 0.5));
// (3) particles move to their child and count themselves in it; (4) those in
// cells with fewer than leaf_cap particles settle, marking the leaf and its
// ancestors active when the particle is active (equivalent to the reference's
// bottom-up pass, fast3DFMM.cpp:711-741). Grid barriers separate the steps;
// data written by other blocks is read through L2. A particle is always
// handled by the same thread, so its own state needs no barrier.
__global__ void __launch_bounds__(kT3Threads)
octree_levels3d(Tree3D t, const double* __restrict__ x, const double* __restrict__ y,
                const double* __restrict__ z, const uint8_t* __restrict__ act, int max_blocks, unsigned* err) {
    __shared__ int s_red[kT3Threads / 32];
    __shared__ int s_warp[kT3Threads / 32];
    __shared__ int s_carry;
    if ((int)gridDim.x > max_blocks) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_err(err, ERR_INDEX);
        return;  // uniform: every block sees the same gridDim
    }
    TreeInfo3D* info = t.info;
    const int n = t.n, cap = t.leaf_cap;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    for (int L = 1; L <= kMaxLevels3D; ++L) {
        if (__ldcg(&info->remaining) <= 0) break;  // written before the last barrier: uniform
        const bool skip = block_fatal(err);  // per block; barriers are still taken by everyone
        const int p0 = __ldcg(&info->level_start[L - 1]), p1 = __ldcg(&info->level_start[L]);
        // (1) octants
        if (!skip) {
            for (int i = gtid; i < n; i += gstride) {
                if (t.settled[i]) continue;
                const int c = t.pcell[i];
                const int oct = (x[i] > __ldcg(&t.c_x[c])) * 1 + (y[i] > __ldcg(&t.c_y[c])) * 2 +
                                (z[i] > __ldcg(&t.c_z[c])) * 4;
                t.poct[i] = (uint8_t)oct;
                atomicOr(&t.c_chmask[c], 1u << oct);
            }
        }
        grid_sync(t.gbar, err);
        // (2) number the children of cells p0..p1-1: block b owns a contiguous chunk
        const int np = skip ? 0 : max(0, min(p1, t.cap_cells) - p0);
        const int per = ceil_div(np, (int)gridDim.x);
        const int b0 = p0 + min(np, (int)blockIdx.x * per), b1 = p0 + min(np, ((int)blockIdx.x + 1) * per);
        int mine = 0;
        for (int c = b0 + threadIdx.x; c < b1; c += blockDim.x) mine += __popc(__ldcg(&t.c_chmask[c]));
        const int bsum = block_sum_int(mine, s_red);
        if (threadIdx.x == 0) t.blk[blockIdx.x] = (uint32_t)bsum;
        grid_sync(t.gbar, err);
        int before = 0, all = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
            const int v = (int)__ldcg(&t.blk[b]);
            all += v;
            if (b < (int)blockIdx.x) before += v;
        }
        before = block_sum_int(before, s_red);
        all = block_sum_int(all, s_red);
        const int base = p1 + before;  // first child index of this block's parents
        if (threadIdx.x == 0) s_carry = 0;
        __syncthreads();
        for (int c0 = b0; c0 < b1; c0 += blockDim.x) {
            const int c = c0 + threadIdx.x;
            const unsigned m = c < b1 ? __ldcg(&t.c_chmask[c]) : 0u;
            int tot;
            const int off = block_excl_int(__popc(m), s_warp, &tot) + s_carry;
            if (m) {
                const int k0 = base + off;
                t.c_child0[c] = k0;
                const double len = xdiv(__ldcg(&t.c_size[c]), 2.0);
                const double px = __ldcg(&t.c_x[c]), py = __ldcg(&t.c_y[c]), pz = __ldcg(&t.c_z[c]);
                int r = 0;
                for (int o = 0; o < 8; ++o) {
                    if (!((m >> o) & 1u)) continue;
                    const int k = k0 + r++;
                    if (k >= t.cap_cells) {
                        set_err(err, ERR_CELL_CAP);
                        continue;
                    }
                    t.c_x[k] = xadd(px, xmul(len, (double)((o >> 0) & 1) - 0.5));
                    t.c_y[k] = xadd(py, xmul(len, (double)((o >> 1) & 1) - 0.5));
                    t.c_z[k] = xadd(pz, xmul(len, (double)((o >> 2) & 1) - 0.5));
                    t.c_size[k] = len;
                    t.c_parent[k] = c;
                    t.c_child0[k] = -1;
                    t.c_chmask[k] = 0;
                    t.c_npar[k] = 0;
                    t.c_active[k] = 0;
                    t.c_level[k] = (uint8_t)L;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_carry += tot;
            __syncthreads();
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int k2 = L + 1; k2 < kMaxLevels3D + 2; ++k2) info->level_start[k2] = p1 + all;
            info->n_cells = p1 + all;
            if (all > 0) info->depth = L;
            if (p1 + all > t.cap_cells) set_err(err, ERR_CELL_CAP);
        }
        grid_sync(t.gbar, err);
        // (3) move particles to their child
        const bool skip3 = block_fatal(err);
        if (!skip3) {
            for (int i = gtid; i < n; i += gstride) {
                if (t.settled[i]) continue;
                const int c = t.pcell[i];
                const unsigned m = __ldcg(&t.c_chmask[c]);
                const int k = __ldcg(&t.c_child0[c]) + __popc(m & ((1u << t.poct[i]) - 1u));
                if (k < 0 || k >= t.cap_cells) {
                    set_err(err, ERR_INDEX);
                    continue;
                }
                t.pcell[i] = k;
                atomicAdd(&t.c_npar[k], 1);
            }
        }
        grid_sync(t.gbar, err);
        // (4) settle particles whose cell is a leaf
        int settled_now = 0;
        if (!skip3) {
            for (int i = gtid; i < n; i += gstride) {
                if (t.settled[i]) continue;
                const int k = t.pcell[i];
                if (__ldcg(&t.c_npar[k]) < cap) {
                    t.settled[i] = 1;
                    ++settled_now;
                    if (act[i]) {
                        for (int c = k; c > 0 && !__ldcg(&t.c_active[c]); c = __ldcg(&t.c_parent[c])) t.c_active[c] = 1;
                    }
                }
            }
        }
        settled_now = block_sum_int(settled_now, s_red);
        if (threadIdx.x == 0 && settled_now) atomicSub(&info->remaining, settled_now);
        if (skip3 && blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&info->remaining, 0);
        grid_sync(t.gbar, err);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && __ldcg(&info->remaining) > 0) set_err(err, ERR_DEPTH);
}

// Leaf ranges after the particles were sorted by leaf: key[j] = leaf of the
// particle in sorted slot j; gathers the particle data into leaf order.
__global__ void leaf_ranges3d(Tree3D t, const uint32_t* __restrict__ key, const uint32_t* __restrict__ idx,
                              const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, const double* __restrict__ ax,
                              const double* __restrict__ ay, const double* __restrict__ az,
                              const uint8_t* __restrict__ act, unsigned* err) {
    const int n = t.n;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t k = key[j], i = idx[j];
        if (k >= (uint32_t)t.cap_cells || i >= (uint32_t)n) {
            set_err(err, ERR_INDEX);
            continue;
        }
        if (j == 0 || key[j - 1] != k) t.c_lo[k] = j;
        if (j == n - 1 || key[j + 1] != k) t.c_hi[k] = j + 1;
        t.perm[j] = i;
        t.px[j] = x[i];
        t.py[j] = y[i];
        t.pz[j] = z[i];
        t.ax[j] = ax[i];
        t.ay[j] = ay[i];
        t.az[j] = az[i];
        t.pact[j] = act[i] ? 1 : 0;
    }
}

// Sort keys: the leaf of every particle, values its index.
__global__ void leaf_keys3d(Tree3D t, uint32_t* key, uint32_t* idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.n; i += gridDim.x * blockDim.x) {
        key[i] = (uint32_t)t.pcell[i];
        idx[i] = (uint32_t)i;
    }
}

__device__ __forceinline__ void p2m_term(double& m, int j, double s, double dx, double dy, double dz) {
    // fmm3D.cpp:84-103, one of the ten moments
    switch (j) {
        case 0: m += s; break;
        case 1: m += s * dx; break;
        case 2: m += s * dy; break;
        case 3: m += s * dz; break;
        case 4: m += s * dx * dx * 0.5; break;
        case 5: m += s * dy * dy * 0.5; break;
        case 6: m += s * dz * dz * 0.5; break;
        case 7: m += s * dx * dy; break;
        case 8: m += s * dy * dz; break;
        default: m += s * dx * dz; break;
    }
}

// P2M of every active leaf, one warp per cell: lane 10 a + j sums moment j of
// source component a over the leaf's active particles in ascending index
// order, d = centre - particle (fast3DFMM.cpp:164-214). Non-leaf moments
// start at zero.
__global__ void __launch_bounds__(128)
p2m3d(Tree3D t, unsigned* err) {
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31;
    const int nc = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int a = lane / 10, j = lane - 10 * (lane / 10);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nc; c += warps) {
        double m = 0.0;
        if (t.c_chmask[c] == 0 && t.c_active[c] && lane < 30) {
            const double xc = t.c_x[c], yc = t.c_y[c], zc = t.c_z[c];
            const double* src = a == 0 ? t.ax : a == 1 ? t.ay : t.az;
            for (int s = t.c_lo[c]; s < t.c_hi[c]; ++s) {
                if (!t.pact[s]) continue;
                p2m_term(m, j, src[s], xc - t.px[s], yc - t.py[s], zc - t.pz[s]);
            }
        }
        if (lane < 30) t.mom[(size_t)c * 30 + lane] = m;
    }
}

// M2M into the active non-leaf cells of one level from their children in
// octant order (fmm3D.cpp:114-132), d = parent centre - child centre; lane
// 10 a + j forms moment j of component a.
__device__ __forceinline__ void m2m3d_level(const Tree3D& t, int L) {
    const int lane = threadIdx.x & 31;
    const int a = lane / 10, j = lane - 10 * (lane / 10);
    const int c0 = t.info->level_start[L], c1 = t.info->level_start[L + 1];
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c0 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < c1; c += warps) {
        const unsigned mask = t.c_chmask[c];
        if (mask == 0 || !t.c_active[c] || lane >= 30) continue;
        const int k0 = t.c_child0[c];
        const double xc = t.c_x[c], yc = t.c_y[c], zc = t.c_z[c];
        double m = 0.0;
        int r = 0;
        for (int o = 0; o < 8; ++o) {
            if (!((mask >> o) & 1u)) continue;
            const int k = k0 + r++;
            const double dx = xc - t.c_x[k], dy = yc - t.c_y[k], dz = zc - t.c_z[k];
            const double* ch = &t.mom[(size_t)k * 30 + 10 * a];
            const double c_0 = __ldcg(&ch[0]), c_1 = __ldcg(&ch[1]), c_2 = __ldcg(&ch[2]), c_3 = __ldcg(&ch[3]);
            const double cj = __ldcg(&ch[j]);
            switch (j) {
                case 0: m += cj; break;
                case 1: m += cj + c_0 * dx; break;
                case 2: m += cj + c_0 * dy; break;
                case 3: m += cj + c_0 * dz; break;
                case 4: m += cj + (c_0 * dx * dx * 0.5) + (c_1 * dx); break;
                case 5: m += cj + (c_0 * dy * dy * 0.5) + (c_2 * dy); break;
                case 6: m += cj + (c_0 * dz * dz * 0.5) + (c_3 * dz); break;
                case 7: m += cj + (c_0 * dx * dy) + (c_1 * dy) + (c_2 * dx); break;
                case 8: m += cj + (c_0 * dy * dz) + (c_2 * dz) + (c_3 * dy); break;
                default: m += cj + (c_0 * dx * dz) + (c_1 * dz) + (c_3 * dx); break;
            }
        }
        t.mom[(size_t)c * 30 + lane] = m;
    }
}

// M2M of levels depth-1 .. 1 in one cooperative launch.
__global__ void __launch_bounds__(128)
m2m3d_coop(Tree3D t, unsigned* err) {
    const int depth = t.info->depth;
    for (int L = depth - 1; L >= 1; --L) {
        if (!block_fatal(err)) m2m3d_level(t, L);
        grid_sync(t.gbar + 2, err);
    }
}

__global__ void __launch_bounds__(128)
m2m3d_one(Tree3D t, int L, unsigned* err) {
    if (block_fatal(err)) return;
    if (L < t.info->depth) m2m3d_level(t, L);
}

__global__ void count_leaves3d(Tree3D t) {
    __shared__ int s_red[8];
    const int nc = t.info->n_cells;
    int k = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) k += t.c_chmask[c] == 0;
    k = block_sum_int(k, s_red);
    if (threadIdx.x == 0 && k) atomicAdd(&t.info->n_leaves, k);
}

// ---------------------------------------------------------------------------
// 3D TreeCell (TreeCell::initializeTree with DIM 3, treeCell.cpp:1043-1243).
//
// The reference bins every unsettled particle at level L by
// index = (int)((c - pivot) / size_L), size_L = root / 2^L (treeCell.cpp:101-105,
// 290-300). size_L is root / 2^L exactly, and rounding commutes with scaling
// by a power of two, so RN(d / size_L) = RN(d / size_10) / 2^(10-L) and the
// level-L index is the level-10 index shifted right by 10 - L. Particles are
// therefore sorted once by their level-10 Morton key (x in bit 0 of every
// 3-bit digit, the reference's child order ix + ((i >> 0) & 1), iy + ((i >> 1)
// & 1), iz + ((i >> 2) & 1), treeCell.cpp:395-417), and the cells of level L
// are the runs of equal level-L prefixes whose parent run is split. A run is
// split when it holds more than max_par particles or more than max_src active
// ones (treeCell.cpp:1170-1215); a split run's parent is split too, so a run is
// a cell exactly when its parent run is split, and every level is built at
// once from per-particle records.
// ---------------------------------------------------------------------------

// Equal leading 3-bit digits (levels) of two level-10 keys (30 bits).
__device__ __forceinline__ int tc_lcp(uint32_t a, uint32_t b) {
    const uint32_t d = a ^ b;
    return d == 0 ? kTcLevels : (__clz(d) - 2) / 3;
}

__device__ __forceinline__ uint32_t tc_spread(uint32_t v) {   // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ int tc_compact(uint32_t v) {       // inverse of tc_spread
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x3ffu;
    return (int)v;
}

// Level-10 key and index of every particle; the grid index of an axis is
// (int)((c - pivot) / (root / 1024)), which must lie in [0, 1024).
__global__ void tc_keys3d(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                          int n, const Geom3D* __restrict__ g, uint32_t* __restrict__ key, uint32_t* __restrict__ idx,
                          unsigned* err) {
    const double size = xdiv(g->root, 1024.0);
    const double pv[3] = {g->piv[0], g->piv[1], g->piv[2]};
    const double* p[3] = {x, y, z};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        bool bad = false;
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double q = xdiv(xsub(p[d][i], pv[d]), size);
            bad |= !(q > -1.0 && q < 1024.0);
            const int ix = bad ? 0 : (int)q;
            k |= tc_spread((uint32_t)ix) << d;
        }
        if (bad) set_err(err, ERR_RANGE);
        key[i] = k;
        idx[i] = (uint32_t)i;
    }
}

// Active flags in key order, for the active-count scan.
__global__ void tc_act3d(const uint8_t* __restrict__ act, const uint32_t* __restrict__ idx, int n,
                         uint32_t* __restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) out[j] = act[idx[j]] ? 1u : 0u;
}

// First m in [lo, hi) with as[m] >= target (as non-decreasing), galloping up from lo.
__device__ __forceinline__ int tc_gallop_ge(const uint32_t* __restrict__ as, int lo, int hi, uint32_t target) {
    int L = lo, R = hi, step = 1;
    while (L + step < R && as[L + step] < target) {
        L += step;
        step <<= 1;
    }
    R = min(R, L + step);
    while (L < R) {
        const int mid = (L + R) >> 1;
        if (as[mid] < target) L = mid + 1;
        else R = mid;
    }
    return L;
}

// First j' <= j whose key has the same prefix (key >> sh) as particle j.
__device__ __forceinline__ int tc_group_start(const uint32_t* __restrict__ key, int j, int sh) {
    const uint32_t v = key[j] >> sh;
    int L = 0, R = j;
    for (int step = 1; R - step >= L; step <<= 1) {
        if ((key[R - step] >> sh) == v) {
            R -= step;
        } else {
            L = R - step + 1;
            break;
        }
    }
    while (L < R) {
        const int mid = (L + R) >> 1;
        if ((key[mid] >> sh) == v) R = mid;
        else L = mid + 1;
    }
    return L;
}

// One past the last j' in [lo, cap) with the prefix of particle lo.
__device__ __forceinline__ int tc_group_end(const uint32_t* __restrict__ key, int lo, int cap, int sh) {
    const uint32_t v = key[lo] >> sh;
    int L = lo + 1, R = cap;
    while (L < R) {
        const int mid = (L + R) >> 1;
        if ((key[mid] >> sh) == v) L = mid + 1;
        else R = mid;
    }
    return L;
}

// pinfo[j] = lvl | (big + 1) << 8: lvl = the first level at which particle j
// starts a run (kTcLevels + 1 for a key equal to its predecessor's), big =
// the deepest level at which that run is split (-1: none). The run of level
// L >= lvl starting at j holds more than max_par particles iff particle
// j + max_par shares its prefix, more than max_src active ones iff the
// (max_src + 1)-th active particle from j does.
__global__ void tc_bigl3d(const uint32_t* __restrict__ key, const uint32_t* __restrict__ as, int n, int max_src,
                          int max_par, uint32_t* __restrict__ pinfo) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t kj = key[j];
        const int lvl = j == 0 ? 1 : tc_lcp(key[j - 1], kj) + 1;
        int big = -1;
        if ((long long)j + max_par < n) big = tc_lcp(kj, key[j + max_par]);
        const uint32_t target = as[j] + (uint32_t)max_src + 1u;   // as[] < 2^30, max_src < 2^31: no wrap
        if (as[n] >= target) {
            const int from = (int)min((long long)n, (long long)j + max_src + 1);
            const int m = tc_gallop_ge(as, from, n + 1, target);   // particle m-1 is that one
            big = max(big, tc_lcp(kj, key[m - 1]));
        }
        pinfo[j] = (uint32_t)lvl | ((uint32_t)(big + 1) << 8);
    }
}

// The levels of the cells particle j starts (first..last, 0 = none; bits
// 16..23 and 24..31 of pinfo) and the per-tile counts of cells and leaves of
// every level: rows 0..10 cells, rows 11..21 leaves, tiles columns.
__global__ void __launch_bounds__(kTcTile)
tc_cells3d(const uint32_t* __restrict__ key, uint32_t* __restrict__ pinfo, int n, uint32_t* __restrict__ tile_cnt,
           int tiles, unsigned* err) {
    __shared__ unsigned s_c[kTcLevels + 1], s_l[kTcLevels + 1];
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        if (threadIdx.x <= kTcLevels) s_c[threadIdx.x] = s_l[threadIdx.x] = 0;
        __syncthreads();
        const int j = tile * kTcTile + threadIdx.x;
        if (j < n) {
            const uint32_t w = pinfo[j];
            const int lvl = (int)(w & 0xff), big = (int)((w >> 8) & 0xff) - 1;
            int first = 0, last = 0;
            if (lvl <= kTcLevels) {
                bool exists = lvl == 1;   // the root is always split
                if (!exists) {
                    const int sp = tc_group_start(key, j, 3 * (kTcLevels - (lvl - 1)));
                    exists = (int)((pinfo[sp] >> 8) & 0xff) - 1 >= lvl - 1;
                }
                if (exists) {
                    first = lvl;
                    last = min(kTcLevels, max(lvl, big + 1));
                    if (big >= kTcLevels) set_err(err, ERR_DEPTH);   // a level-10 cell would need splitting
                    for (int L = first; L <= last; ++L) atomicAdd(&s_c[L], 1u);
                    if (big < last) atomicAdd(&s_l[last], 1u);
                }
            }
            pinfo[j] = (w & 0xffffu) | ((uint32_t)first << 16) | ((uint32_t)last << 24);
        }
        __syncthreads();
        if (threadIdx.x <= kTcLevels) {
            tile_cnt[(size_t)threadIdx.x * tiles + tile] = s_c[threadIdx.x];
            tile_cnt[(size_t)(kTcLevels + 1 + threadIdx.x) * tiles + tile] = s_l[threadIdx.x];
        }
        __syncthreads();
    }
}

// One block per row of tile counts: exclusive scan in place, row total.
__global__ void __launch_bounds__(1024)
tc_scan_rows3d(uint32_t* __restrict__ tile_cnt, int tiles, uint32_t* __restrict__ row_tot) {
    __shared__ uint32_t s_w[32];
    __shared__ uint32_t s_carry;
    uint32_t* row = tile_cnt + (size_t)blockIdx.x * tiles;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = 0; b < tiles; b += blockDim.x) {
        const int k = b + threadIdx.x;
        const uint32_t v = k < tiles ? row[k] : 0u;
        uint32_t incl = v;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        uint32_t before = 0, all = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            before += w < warp ? s_w[w] : 0u;
            all += s_w[w];
        }
        const uint32_t carry = s_carry;
        if (k < tiles) row[k] = carry + before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + all;
        __syncthreads();
    }
    if (threadIdx.x == 0) row_tot[blockIdx.x] = s_carry;
}

// Level starts, depth and the root cell (treeCell.cpp:1117-1133); ERR_LEAF1
// when a level-1 cell is a leaf and the tree goes deeper: the reference's
// traversal asks for that leaf's children and throws (fmm3D.cpp:1286).
__global__ void tc_totals3d(Tree3D t, const uint32_t* __restrict__ row_tot, const uint32_t* __restrict__ as,
                            unsigned* err) {
    TreeInfo3D* info = t.info;
    int cells = 1, depth = 0;
    info->level_start[0] = 0;
    for (int L = 1; L < kMaxLevels3D + 2; ++L) {
        info->level_start[L] = cells;
        if (L <= kTcLevels) {
            const int c = (int)row_tot[L];
            if (c > 0) depth = L;
            cells += c;
        }
    }
    info->n_cells = cells;
    info->n_leaves = 0;   // counted after the leaf sort
    info->depth = depth;
    info->remaining = 0;
    info->scan_total = 0;
    info->p2p_pairs = 0;
    info->m2p_pairs = 0;
    if (cells > t.cap_cells) set_err(err, ERR_CELL_CAP);
    if (depth > 1 && row_tot[kTcLevels + 1 + 1] > 0) set_err(err, ERR_LEAF1);
    const Geom3D* g = t.geom;
    t.c_x[0] = xadd(g->piv[0], xmul(0.5, g->root));
    t.c_y[0] = xadd(g->piv[1], xmul(0.5, g->root));
    t.c_z[0] = xadd(g->piv[2], xmul(0.5, g->root));
    t.c_size[0] = g->root;
    t.c_npar[0] = t.n;
    t.c_parent[0] = -1;
    t.c_child0[0] = -1;   // lowered by tc_link3d (unsigned minimum: -1 = none)
    t.c_chmask[0] = 0;
    t.c_active[0] = as[t.n] != 0 ? 1 : 0;
    t.c_level[0] = 0;
    t.c_lo[0] = 0;
    t.c_hi[0] = t.n;
}

// Cell records of every particle's cell levels; cell index = level start +
// scanned tile count + rank of the particle among the tile's emitters of that
// level (warp ballots). code[c] = level-L Morton prefix | leaf << 31.
__global__ void __launch_bounds__(kTcTile)
tc_emit3d(Tree3D t, const uint32_t* __restrict__ key, const uint32_t* __restrict__ pinfo,
          const uint32_t* __restrict__ tile_cnt, int tiles, uint32_t* __restrict__ code_out, unsigned* err) {
    __shared__ int s_wc[kTcLevels + 1][kTcTile / 32];
    if (block_fatal(err)) return;
    const int n = t.n;
    const TreeInfo3D* info = t.info;
    const Geom3D* g = t.geom;
    const double root = g->root;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int j = tile * kTcTile + threadIdx.x;
        const uint32_t w = j < n ? pinfo[j] : 0u;
        const int first = (int)((w >> 16) & 0xff), last = (int)(w >> 24), big = (int)((w >> 8) & 0xff) - 1;
        if (lane <= kTcLevels) s_wc[lane][warp] = 0;
        __syncwarp();
        for (int L = 1; L <= kTcLevels; ++L) {
            const unsigned m = __ballot_sync(0xffffffffu, first && first <= L && L <= last);
            if (lane == 0) s_wc[L][warp] = __popc(m);
        }
        __syncthreads();
        for (int L = 1; L <= kTcLevels; ++L) {
            const bool has = first && first <= L && L <= last;
            const unsigned m = __ballot_sync(0xffffffffu, has);
            if (!has) continue;
            int before = 0;
            for (int k = 0; k < warp; ++k) before += s_wc[L][k];
            const int ci = info->level_start[L] + (int)tile_cnt[(size_t)L * tiles + tile] + before + __popc(m & below);
            if (ci >= t.cap_cells) {
                set_err(err, ERR_CELL_CAP);
                continue;
            }
            const bool leaf = L == last && big < last;
            const uint32_t pre = key[j] >> (3 * (kTcLevels - L));
            const int ix = tc_compact(pre), iy = tc_compact(pre >> 1), iz = tc_compact(pre >> 2);
            const double len = xdiv(root, ldexp(1.0, L));
            t.c_x[ci] = xadd(g->piv[0], xmul(xadd(0.5, (double)ix), len));
            t.c_y[ci] = xadd(g->piv[1], xmul(xadd(0.5, (double)iy), len));
            t.c_z[ci] = xadd(g->piv[2], xmul(xadd(0.5, (double)iz), len));
            t.c_size[ci] = len;
            t.c_lo[ci] = j;
            t.c_child0[ci] = -1;
            t.c_chmask[ci] = 0;
            t.c_level[ci] = (uint8_t)L;
            code_out[ci] = pre | (leaf ? 0x80000000u : 0u);
        }
        __syncthreads();
    }
}

// Range, counts and activity of every cell (one search per cell), its parent
// (the level L-1 cell of its prefix >> 3, by bisection over that level's
// prefixes), the parent's child mask and first child; every leaf records
// itself as the cell of its particles.
__global__ void tc_link3d(Tree3D t, const uint32_t* __restrict__ key, const uint32_t* __restrict__ idx,
                          const uint32_t* __restrict__ as, const uint32_t* __restrict__ code, int max_par,
                          unsigned* err) {
    if (fatal(err)) return;
    const int nc = t.info->n_cells, n = t.n;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x + 1; c < nc; c += gridDim.x * blockDim.x) {
        const int L = t.c_level[c];
        const uint32_t cw = code[c];
        const bool leaf = (cw >> 31) != 0;
        const uint32_t pre = cw & 0x7fffffffu;
        const int lo = t.c_lo[c];
        const int cap = leaf ? (int)min((long long)n, (long long)lo + max_par) : n;
        const int hi = tc_group_end(key, lo, cap, 3 * (kTcLevels - L));
        t.c_hi[c] = hi;
        t.c_npar[c] = hi - lo;
        t.c_active[c] = as[hi] != as[lo] ? 1 : 0;
        int p = 0;
        if (L >= 2) {
            int a = t.info->level_start[L - 1], b = t.info->level_start[L];
            const uint32_t want = pre >> 3;
            while (a < b) {
                const int mid = (a + b) >> 1;
                if ((code[mid] & 0x7fffffffu) < want) a = mid + 1;
                else b = mid;
            }
            p = a;
            if (p >= t.info->level_start[L] || (code[p] & 0x7fffffffu) != want) {
                set_err(err, ERR_INDEX);
                continue;
            }
        }
        t.c_parent[c] = p;
        atomicOr(&t.c_chmask[p], 1u << (pre & 7u));
        atomicMin(reinterpret_cast<unsigned*>(&t.c_child0[p]), (unsigned)c);
        if (leaf)
            for (int k = lo; k < hi; ++k) t.pcell[idx[k]] = c;
    }
}

}  // namespace

static cudaError_t leaves_upward3d(const double* x, const double* y, const double* z, const double* ax,
                                   const double* ay, const double* az, const uint8_t* act, Tree3D& t, Scratch3D& s,
                                   unsigned* err, cudaStream_t st, int* launches);

// Tree build (bounding box, levels, leaf order) and upward pass, enqueued on st.
cudaError_t build_tree3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                         const double* az, const uint8_t* act, const double center[3], double exp_pct, Tree3D& t,
                         Scratch3D& s, double* bbox_partial, unsigned* err, cudaStream_t st, int* launches) {
    const int n = t.n;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    cudaError_t e = cudaMemsetAsync(t.gbar, 0, sizeof(unsigned) * 8, st);
    if (e != cudaSuccess) return e;
    const int bb = std::max(1, std::min(kBBox3Blocks, ceil_div(n, 256)));
    bbox3d<<<bb, 256, 0, st>>>(x, y, z, n, center[0], center[1], center[2], exp_pct, false, t.geom, bbox_partial,
                                t.gbar + 6, err);
    root3d<<<gridN, 256, 0, st>>>(t);
    *launches += 2;
    int grid = 0;
    e = launch_coop(octree_levels3d, kT3Threads, 0, st, 4, &grid, t, x, y, z, act, kCoopMaxBlocks3D, err);
    if (e != cudaSuccess) return e;
    *launches += 1;
    return leaves_upward3d(x, y, z, ax, ay, az, act, t, s, err, st, launches);
}

// Particles in leaf order (stable: ascending index within a leaf, the
// reference's parIDList order), leaf ranges, P2M and the M2M levels.
static cudaError_t leaves_upward3d(const double* x, const double* y, const double* z, const double* ax,
                                   const double* ay, const double* az, const uint8_t* act, Tree3D& t, Scratch3D& s,
                                   unsigned* err, cudaStream_t st, int* launches) {
    const int n = t.n;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    cudaError_t e = cudaSuccess;
    int grid = 0;
    leaf_keys3d<<<gridN, 256, 0, st>>>(t, s.key_a, s.val_a);
    *launches += 1;
    int bits = 1;
    while ((1ll << bits) < (long long)t.cap_cells) ++bits;
    uint32_t* keys = s.key_a;
    uint32_t* vals = s.val_a;
    e = radix_sort_pairs(&keys, &vals, s.key_b, s.val_b, n, bits, s.sort, err, st, launches);
    if (e != cudaSuccess) return e;
    leaf_ranges3d<<<gridN, 256, 0, st>>>(t, keys, vals, x, y, z, ax, ay, az, act, err);
    count_leaves3d<<<148, 256, 0, st>>>(t);
    p2m3d<<<148 * 8, 128, 0, st>>>(t, err);
    *launches += 3;
    e = launch_coop(m2m3d_coop, 128, 0, st, 8, &grid, t, err);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        for (int L = kMaxLevels3D - 1; L >= 1; --L) {
            m2m3d_one<<<148 * 4, 128, 0, st>>>(t, L, err);
            *launches += 1;
        }
        return cudaGetLastError();
    }
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t build_treecell3d(const double* x, const double* y, const double* z, const double* ax,
                             const double* ay, const double* az, const uint8_t* act, int max_src, int max_par,
                             double exp_pct, Tree3D& t, Scratch3D& s, double* bbox_partial, unsigned* err,
                             cudaStream_t st, int* launches) {
    const int n = t.n;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    const int tiles = ceil_div(n, kTcTile);
    if (tiles > s.tc_tiles) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(t.gbar, 0, sizeof(unsigned) * 8, st);
    if (e != cudaSuccess) return e;
    const int bb = std::max(1, std::min(kBBox3Blocks, ceil_div(n, 256)));
    bbox3d<<<bb, 256, 0, st>>>(x, y, z, n, 0.0, 0.0, 0.0, exp_pct, true, t.geom, bbox_partial, t.gbar + 6, err);
    tc_keys3d<<<gridN, 256, 0, st>>>(x, y, z, n, t.geom, s.key_a, s.val_a, err);
    *launches += 2;
    uint32_t* keys = s.key_a;
    uint32_t* vals = s.val_a;
    e = radix_sort_pairs(&keys, &vals, s.key_b, s.val_b, n, 3 * kTcLevels, s.sort, err, st, launches);
    if (e != cudaSuccess) return e;
    tc_act3d<<<gridN, 256, 0, st>>>(act, vals, n, s.tc_act);
    *launches += 1;
    e = scan_exclusive(s.tc_act, s.tc_scan, n, s.tc_scan + n, s.scan, err, st);
    if (e != cudaSuccess) return e;
    *launches += 1;
    const int gt = std::max(1, std::min(tiles, 148 * 2));
    tc_bigl3d<<<gridN, 256, 0, st>>>(keys, s.tc_scan, n, max_src, max_par, s.tc_pinfo);
    tc_cells3d<<<gt, kTcTile, 0, st>>>(keys, s.tc_pinfo, n, s.tc_tile, tiles, err);
    tc_scan_rows3d<<<2 * (kTcLevels + 1), 1024, 0, st>>>(s.tc_tile, tiles, s.tc_tot);
    tc_totals3d<<<1, 1, 0, st>>>(t, s.tc_tot, s.tc_scan, err);
    tc_emit3d<<<gt, kTcTile, 0, st>>>(t, keys, s.tc_pinfo, s.tc_tile, tiles, s.tc_code, err);
    const int gc = std::max(1, std::min(148 * 8, ceil_div(t.cap_cells, 256)));
    tc_link3d<<<gc, 256, 0, st>>>(t, keys, vals, s.tc_scan, s.tc_code, max_par, err);
    *launches += 6;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return leaves_upward3d(x, y, z, ax, ay, az, act, t, s, err, st, launches);
}

}  // namespace vpm
