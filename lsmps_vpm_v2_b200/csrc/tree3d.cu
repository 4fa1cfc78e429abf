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
__global__ void __launch_bounds__(256)
bbox3d(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z, int n,
       double cx0, double cy0, double cz0, double exp_pct, Geom3D* g, double* partial, unsigned* done,
       unsigned* err) {
    __shared__ double s_v[6][256];
    __shared__ bool s_last;
    double mn[3] = {cx0, cy0, cz0}, mx[3] = {cx0, cy0, cz0};
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
    double a[6] = {cx0, cy0, cz0, cx0, cy0, cz0};
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

}  // namespace

// Tree build (bounding box, levels, leaf order) and upward pass, enqueued on st.
cudaError_t build_tree3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                         const double* az, const uint8_t* act, const double center[3], double exp_pct, Tree3D& t,
                         Scratch3D& s, double* bbox_partial, unsigned* err, cudaStream_t st, int* launches) {
    const int n = t.n;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    cudaError_t e = cudaMemsetAsync(t.gbar, 0, sizeof(unsigned) * 8, st);
    if (e != cudaSuccess) return e;
    const int bb = std::max(1, std::min(kBBox3Blocks, ceil_div(n, 256)));
    bbox3d<<<bb, 256, 0, st>>>(x, y, z, n, center[0], center[1], center[2], exp_pct, t.geom, bbox_partial,
                                t.gbar + 6, err);
    root3d<<<gridN, 256, 0, st>>>(t);
    *launches += 2;
    int grid = 0;
    e = launch_coop(octree_levels3d, kT3Threads, 0, st, 4, &grid, t, x, y, z, act, kCoopMaxBlocks3D, err);
    if (e != cudaSuccess) return e;
    *launches += 1;
    // particles in leaf order (stable: ascending index within a leaf)
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

}  // namespace vpm
