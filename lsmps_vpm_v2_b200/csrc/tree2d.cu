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

// Root cell of the box [mnx, mxx] x [mny, mxy] (treeCell.cpp:1061-1092).
__device__ void root_geometry(double mnx, double mxx, double mny, double mxy, double exp_pct, int key_levels,
                              Geom2D& g, unsigned* err) {
    double root = 0.0;
    double ex = fabs(xsub(mxx, mnx)), ey = fabs(xsub(mxy, mny));
    if (ex > root) root = ex;
    if (ey > root) root = ey;
    double expansion = xadd(1.0, xdiv(exp_pct, 100.0));
    root = xmul(root, expansion);
    g.minx = mnx; g.maxx = mxx; g.miny = mny; g.maxy = mxy;
    g.root = root;
    g.pivx = xdiv(xsub(xadd(mxx, mnx), root), 2.0);
    g.pivy = xdiv(xsub(xadd(mxy, mny), root), 2.0);
    g.size_k = xdiv(root, ldexp(1.0, key_levels));
    if (err && (!(root > 0.0) || !isfinite(root))) set_err(err, ERR_NONFINITE);
}

// Morton key of one particle at the key level (treeCell.cpp:290-303).
__device__ __forceinline__ uint64_t particle_key(double x, double y, double pivx, double pivy, double s, double lim,
                                                 unsigned* err) {
    double tx = xdiv(xsub(x, pivx), s);
    double ty = xdiv(xsub(y, pivy), s);
    uint32_t ix = 0, iy = 0;
    if (tx >= 0.0 && tx < lim && ty >= 0.0 && ty < lim) {
        ix = (uint32_t)__double2ull_rz(tx);
        iy = (uint32_t)__double2ull_rz(ty);
    } else {
        set_err(err, ERR_RANGE);
    }
    return morton2(ix, iy);
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
    Geom2D gg;
    root_geometry(mnx, mxx, mny, mxy, exp_pct, key_levels, gg, err);
    *g = gg;
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
        key[i] = (KT)particle_key(x[i], y[i], pivx, pivy, s, lim, err);
        idx[i] = (uint32_t)i;
    }
}

// Sorted copies of the particle data and the active flags as 0/1 words; the
// sorted keys (from whichever buffer the sort ended in, 32- or 64-bit) and
// permutation land in the tree's own arrays. q may be null: the strengths are
// then gathered later (gather_strengths2d).
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
        if (q) pq[i] = q[j];
        uint8_t a = act[j] ? 1 : 0;
        pact[i] = a;
        act_u32[i] = a;
    }
}

// ---- the sorted particle order in one cooperative launch ------------------------
//
// With 32-bit keys and at most kCoopSortMaxChunk particles per block, one
// launch of one 1024-thread block per SM replaces bbox2d, keys2d, the radix
// sort, gather2d and the active-count scan (ten launches, most of them
// latency-bound at these sizes). Block b owns the contiguous range
// [b C, (b+1) C) of every pass's input. A pass ranks the block's items by
// digit warp by warp in index order (so the sort is stable), publishes the
// block's 256 digit counts, meets the grid at a barrier, takes each digit's
// output base from the column sums of the count table (the blocks before it
// plus the digit's global start), reorders its items by digit in shared
// memory and writes each digit's run contiguously. Results are identical to
// the multi-kernel path: the same keys, the same stable order.
constexpr int kCoopSortThreads = 1024;
constexpr int kCoopSortWarps = kCoopSortThreads / 32;
constexpr int kCoopBarrierWord = 6;
constexpr int kCoopRounds = 6;        // rounds of 32 items per warp loaded together
constexpr int kCoopActRun = 16;       // sorted flags per thread in the active scan (kCoopSortMaxChunk / 1024)   // grid-barrier words 6, 7 of Tree2D::gbar

// Exclusive scan over the 1024 threads of the block; *total = the block sum.
// Every thread must call it (it holds three block barriers).
__device__ __forceinline__ uint32_t coop_block_scan(uint32_t v, uint32_t* s_ws, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = s_ws[lane];
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_ws[lane] = w;
    }
    __syncthreads();
    const uint32_t base = warp ? s_ws[warp - 1] : 0u;
    *total = s_ws[kCoopSortWarps - 1];
    __syncthreads();
    return base + x - v;
}

// Word offsets in the count tables of sort2d_coop (GM = kCoopSortGridMax):
// per-block digit counts [256][GM] and active counts [256][GM] (column d
// holds the blocks' counts of digit d), their exclusive prefixes over blocks
// [GM][256] (row b is what block b reads) and the per-digit totals.
constexpr int kCwCount = 0;
constexpr int kCwActCount = 256 * kCoopSortGridMax;
constexpr int kCwPrefix = 512 * kCoopSortGridMax;
constexpr int kCwActPrefix = 768 * kCoopSortGridMax;
constexpr int kCwTotal = 1024 * kCoopSortGridMax;
constexpr int kCwActTotal = kCwTotal + 256;
constexpr int kCwFlag = kCwActTotal + 256;   // set when the shallow attempt must be redone
static_assert(kCwFlag + 1 <= kCoopSortWords, "count tables of the cooperative sort");

// kb0/kb1: 32-bit key ping-pong buffers (pass 0's keys are computed into
// kb0); vb0/vb1: index ping-pong buffers, vb1 may alias t.perm (the last
// pass reads vb0). An index carries its particle's active flag in bit 31.
// The last pass gathers x, y and q by index (from L2: the bounding box has
// just read them) and also produces the active-count scan: a block's
// sorted items form one run per digit, so the count before an item is the
// digit's global start, the runs of that digit in earlier blocks, and the
// item's place in its own run.
//
// Shallow attempt (shallow_cap > 0, four passes needed): the lowest digit
// (levels K-3 .. K) is left out and the keys are stored with it cleared, so
// particles are ordered by their level-(K-4) cells, ties in input order. The
// tree built from those keys is the tree of the full keys whenever no
// level-(K-4) cell needs splitting; that holds when no shallow_cap + 1
// consecutive particles share a cell (shallow_cap = min(max_src, max_par)),
// which the kernel checks after the three passes. Otherwise it sorts again
// with all four passes.
__global__ void __launch_bounds__(kCoopSortThreads, 1)
sort2d_coop(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ q,
            const uint8_t* __restrict__ act, double exp_pct, int passes, int shallow_cap, Tree2D t, double* partial,
            uint32_t* kb0, uint32_t* kb1, uint32_t* vb0, uint32_t* vb1, uint32_t* words, int chunk_cap,
            unsigned* err) {
    extern __shared__ __align__(16) unsigned char cs_sm[];
    __shared__ uint32_t s_wh[kCoopSortWarps][256];   // per-warp digit counts, then warp-exclusive prefixes
    __shared__ uint32_t s_local[256];                // tile-local start of each digit
    __shared__ uint32_t s_base[256];                 // output index minus tile-local index, per digit
    __shared__ uint32_t s_wa[256];                   // last pass: the block's active count per digit
    __shared__ uint32_t s_abase[256];                // last pass: active count before the digit's run, minus local
    __shared__ uint32_t s_ws[32];
    __shared__ double s_red[4][kCoopSortWarps];
    __shared__ double s_geo[3];
    const int n = t.n;
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int chunk = (n + G - 1) / G;
    if (chunk > chunk_cap || G > kCoopSortGridMax) {   // uniform over the grid: no block reaches a barrier
        if (b == 0 && tid == 0) set_err(err, ERR_INDEX);
        return;
    }
    unsigned* bar = t.gbar + kCoopBarrierWord;
    uint32_t* s_key = (uint32_t*)cs_sm;                  // [chunk_cap]
    uint32_t* s_val = s_key + chunk_cap;                 // [chunk_cap]
    uint16_t* s_rank = (uint16_t*)(s_val + chunk_cap);   // [chunk_cap]
    const int c0 = min(n, b * chunk), c1 = min(n, c0 + chunk);
    const int S = (chunk + kCoopSortWarps - 1) / kCoopSortWarps;   // items per warp
    const int w0 = min(c1, c0 + warp * S), w1 = min(c1, w0 + S);

    // 1. bounding box (block partials, barrier, every block reduces all of
    //    them)
    {
        double mnx = x[0], mxx = x[0], mny = y[0], mxy = y[0];
        bool bad = false;
        #pragma unroll 6
        for (int i = c0 + tid; i < c1; i += kCoopSortThreads) {
            const double a = x[i], c = y[i];
            bad |= !isfinite(a) || !isfinite(c);
            mnx = fmin(mnx, a); mxx = fmax(mxx, a);
            mny = fmin(mny, c); mxy = fmax(mxy, c);
        }
        if (bad) set_err(err, ERR_NONFINITE);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        if (lane == 0) { s_red[0][warp] = mnx; s_red[1][warp] = mxx; s_red[2][warp] = mny; s_red[3][warp] = mxy; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < kCoopSortWarps; ++w) {
                mnx = fmin(mnx, s_red[0][w]); mxx = fmax(mxx, s_red[1][w]);
                mny = fmin(mny, s_red[2][w]); mxy = fmax(mxy, s_red[3][w]);
            }
            double* pp = partial + 4 * b;
            pp[0] = mnx; pp[1] = mxx; pp[2] = mny; pp[3] = mxy;
        }
        grid_sync_counter(bar, err);
        if (warp == 0) {
            mnx = __ldcg(partial); mxx = __ldcg(partial + 1); mny = __ldcg(partial + 2); mxy = __ldcg(partial + 3);
            #pragma unroll 5
            for (int bb = lane; bb < G; bb += 32) {
                const double* pp = partial + 4 * bb;
                mnx = fmin(mnx, __ldcg(pp)); mxx = fmax(mxx, __ldcg(pp + 1));
                mny = fmin(mny, __ldcg(pp + 2)); mxy = fmax(mxy, __ldcg(pp + 3));
            }
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
                mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
                mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
                mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
            }
            if (lane == 0) {
                Geom2D gg;
                root_geometry(mnx, mxx, mny, mxy, exp_pct, t.key_levels, gg, b == 0 ? err : nullptr);
                s_geo[0] = gg.pivx;
                s_geo[1] = gg.pivy;
                s_geo[2] = gg.size_k;
                if (b == 0) *t.geom = gg;
            }
        }
        __syncthreads();
    }
    const double pivx = s_geo[0], pivy = s_geo[1], size_k = s_geo[2];
    const double lim = ldexp(1.0, t.key_levels);

    // 2. LSD passes of 8 bits
    const unsigned lt = (1u << lane) - 1u;
    if (b == 0 && tid == 0) words[kCwFlag] = 0u;
    const bool try_shallow = passes == 4 && shallow_cap > 0;
    for (int attempt = try_shallow ? 0 : 1; attempt < 2; ++attempt) {
    const int np = attempt == 0 ? 3 : passes;
    const int skip = passes - np;                               // low digits left out
    const uint32_t kmask = skip ? ~((1u << (8 * skip)) - 1u) : ~0u;
    for (int p = 0; p < np; ++p) {
        const int shift = 8 * (p + skip);
        const bool last = p == np - 1;
        const uint32_t* kin = (p & 1) ? kb1 : kb0;
        uint32_t* kout = (p & 1) ? kb0 : kb1;
        const uint32_t* vin = ((np - 1 - p) & 1) ? vb1 : vb0;
        uint32_t* vout = ((np - 2 - p) & 1) ? vb1 : vb0;
        for (int i = tid; i < kCoopSortWarps * 256; i += kCoopSortThreads) (&s_wh[0][0])[i] = 0u;
        if (tid < 256) s_wa[tid] = 0u;
        __syncthreads();
        // rank of each item among the warp's items of its digit, in index order
        for (int i0 = w0; i0 < w1; i0 += 32 * kCoopRounds) {
            // kCoopRounds rounds of 32 items: loads first (independent), then the ranking
            uint32_t kr[kCoopRounds], fr[kCoopRounds];
            #pragma unroll
            for (int r = 0; r < kCoopRounds; ++r) {
                const int i = i0 + r * 32 + lane;
                kr[r] = 0u;
                fr[r] = 0u;
                if (i < w1) {
                    if (p == 0) {
                        kr[r] = (uint32_t)particle_key(x[i], y[i], pivx, pivy, size_k, lim, err);
                        kb0[i] = kr[r];
                        if (last) fr[r] = act[i] ? 1u : 0u;
                    } else {
                        kr[r] = __ldcg(kin + i);
                        if (last) fr[r] = __ldcg(vin + i) >> 31;
                    }
                }
            }
            #pragma unroll
            for (int r = 0; r < kCoopRounds; ++r) {
                const int i = i0 + r * 32 + lane;
                const bool ok = i < w1;
                const int d = (int)((kr[r] >> shift) & 255u);
                // lanes holding the same digit: one ballot per digit bit
                unsigned m = __ballot_sync(0xffffffffu, ok);
                #pragma unroll
                for (int bit = 0; bit < 8; ++bit) {
                    const bool bs = (d >> bit) & 1;
                    const unsigned bv = __ballot_sync(0xffffffffu, bs);
                    m &= bs ? bv : ~bv;
                }
                uint32_t prior = 0;
                if (ok) prior = s_wh[warp][d];
                __syncwarp();
                if (ok && (m & lt) == 0) s_wh[warp][d] = prior + __popc(m);
                __syncwarp();
                if (ok) {
                    s_rank[i - c0] = (uint16_t)(prior + __popc(m & lt));
                    if (fr[r]) atomicAdd(&s_wa[d], 1u);
                }
            }
        }
        __syncthreads();
        uint32_t run = 0, tot = 0;
        if (tid < 256) {
            for (int w = 0; w < kCoopSortWarps; ++w) {
                const uint32_t c = s_wh[w][tid];
                s_wh[w][tid] = run;
                run += c;
            }
            words[kCwCount + (size_t)tid * kCoopSortGridMax + b] = run;
            if (last) words[kCwActCount + (size_t)tid * kCoopSortGridMax + b] = s_wa[tid];
        }
        const uint32_t loc = coop_block_scan(tid < 256 ? run : 0u, s_ws, &tot);
        if (tid < 256) s_local[tid] = loc;
        uint32_t aloc = 0;
        if (last) aloc = coop_block_scan(tid < 256 ? s_wa[tid] : 0u, s_ws, &tot);
        grid_sync_counter(bar, err);
        // prefixes over blocks, one digit column per warp: block b takes
        // digits b + (warp + 32 m) G; lane l holds blocks 5l .. 5l+4
        for (int d = b + warp * G; d < 256; d += kCoopSortWarps * G) {
            #pragma unroll 1
            for (int tb = 0; tb < (last ? 2 : 1); ++tb) {
                const uint32_t* col = words + (tb ? kCwActCount : kCwCount) + (size_t)d * kCoopSortGridMax;
                uint32_t v[5], sum = 0;
                #pragma unroll
                for (int u = 0; u < 5; ++u) {
                    const int bb = 5 * lane + u;
                    v[u] = bb < G ? __ldcg(col + bb) : 0u;
                    sum += v[u];
                }
                uint32_t incl = sum;
                #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t yv = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += yv;
                }
                uint32_t ex = incl - sum;
                uint32_t* pre = words + (tb ? kCwActPrefix : kCwPrefix);
                #pragma unroll
                for (int u = 0; u < 5; ++u) {
                    const int bb = 5 * lane + u;
                    if (bb < G) pre[(size_t)bb * 256 + d] = ex;
                    ex += v[u];
                }
                if (lane == 31) words[(tb ? kCwActTotal : kCwTotal) + d] = incl;
            }
        }
        grid_sync_counter(bar, err);
        {
            const uint32_t before = tid < 256 ? __ldcg(words + kCwPrefix + (size_t)b * 256 + tid) : 0u;
            const uint32_t all = tid < 256 ? __ldcg(words + kCwTotal + tid) : 0u;
            const uint32_t start = coop_block_scan(all, s_ws, &tot);
            if (tid < 256) s_base[tid] = start + before - s_local[tid];   // modulo 2^32
            if (last) {
                const uint32_t abefore = tid < 256 ? __ldcg(words + kCwActPrefix + (size_t)b * 256 + tid) : 0u;
                const uint32_t aall = tid < 256 ? __ldcg(words + kCwActTotal + tid) : 0u;
                uint32_t atot = 0;
                const uint32_t astart = coop_block_scan(aall, s_ws, &atot);
                if (tid < 256) s_abase[tid] = astart + abefore - aloc;
                if (b == 0 && tid == 0) t.actscan[n] = atot;
            }
        }
        __syncthreads();
        // reorder by digit in shared memory
        for (int i0 = w0; i0 < w1; i0 += 32 * kCoopRounds) {
            uint32_t kr[kCoopRounds], vr[kCoopRounds];
            #pragma unroll
            for (int r = 0; r < kCoopRounds; ++r) {
                const int i = i0 + r * 32 + lane;
                kr[r] = 0u;
                vr[r] = 0u;
                if (i < w1) {
                    if (p == 0) {
                        kr[r] = kb0[i];
                        vr[r] = (uint32_t)i | (act[i] ? 0x80000000u : 0u);
                    } else {
                        kr[r] = __ldcg(kin + i);
                        vr[r] = __ldcg(vin + i);
                    }
                }
            }
            #pragma unroll
            for (int r = 0; r < kCoopRounds; ++r) {
                const int i = i0 + r * 32 + lane;
                if (i < w1) {
                    const int d = (int)((kr[r] >> shift) & 255u);
                    const uint32_t lp = s_local[d] + s_wh[warp][d] + s_rank[i - c0];
                    s_key[lp] = kr[r];
                    s_val[lp] = vr[r];
                }
            }
        }
        __syncthreads();
        const int cnt = c1 - c0;
        if (last) {
            // active flags before each staged item (thread tid: a contiguous run), into s_rank
            const int a0 = tid * kCoopActRun;
            uint32_t fl[kCoopActRun], na = 0;
            #pragma unroll
            for (int u = 0; u < kCoopActRun; ++u) {
                fl[u] = a0 + u < cnt ? s_val[a0 + u] >> 31 : 0u;
                na += fl[u];
            }
            uint32_t ra = coop_block_scan(na, s_ws, &tot);
            #pragma unroll
            for (int u = 0; u < kCoopActRun; ++u) {
                if (a0 + u < cnt) s_rank[a0 + u] = (uint16_t)ra;
                ra += fl[u];
            }
            __syncthreads();
        }
        #pragma unroll 4
        for (int j = tid; j < cnt; j += kCoopSortThreads) {
            const uint32_t key = s_key[j], vf = s_val[j];
            const uint32_t val = vf & 0x7fffffffu;
            const uint32_t d = (key >> shift) & 255u;
            const uint32_t pos = s_base[d] + (uint32_t)j;
            if (pos >= (uint32_t)n || val >= (uint32_t)n) {
                set_err(err, ERR_INDEX);
                continue;
            }
            if (!last) {
                kout[pos] = key;
                vout[pos] = vf;
            } else {
                const double px = x[val], py = y[val], pq = q ? q[val] : 0.0;
                t.key[pos] = key & kmask;
                t.perm[pos] = val;
                t.px[pos] = px;
                t.py[pos] = py;
                if (q) t.pq[pos] = pq;
                t.pact[pos] = (uint8_t)(vf >> 31);
                t.actscan[pos] = s_abase[d] + s_rank[j];
            }
        }
        if (!last) grid_sync_counter(bar, err);
    }
    if (attempt == 1) break;
    // is any level-(K-4) cell holding more than shallow_cap particles?
    grid_sync_counter(bar, err);
    {
        bool over = false;
        for (int i = c0 + tid; i < c1; i += kCoopSortThreads) {
            const int j = i + shallow_cap;
            if (j < n && __ldcg(t.key + i) == __ldcg(t.key + j)) over = true;
        }
        if (__syncthreads_or(over) && tid == 0) atomicOr(&words[kCwFlag], 1u);
    }
    grid_sync_counter(bar, err);
    if (__ldcg(&words[kCwFlag]) == 0u) break;
    }
}

// ---- flat build: every level at once ------------------------------------------
//
// With the particles sorted by their level-K Morton key, the cells of level L
// are the runs ("groups") of equal level-L key prefixes whose parent group is
// split, and a group is split ("big") when it holds more than max_par
// particles or more than max_src active ones (treeCell.cpp:1170-1215). A big
// group's parent is big too (it contains it), so a group is a cell exactly
// when its parent is big, which needs no level-by-level sweep:
//   lvl(i)   the first level at which particle i starts a group
//            (1 + shared leading key digits of particles i-1 and i);
//   bigL(i)  the deepest level at which the group starting at i is big: the
//            group holds particle i + max_par, or the (max_src+1)-th active
//            particle from i, iff the keys share that many leading digits;
//   cells    particle i starts the cells at levels lvl(i) .. min(K,
//            max(lvl(i), bigL(i) + 1)) when the parent group of its first
//            one (the level lvl(i)-1 group containing i: it starts at the
//            last particle before i with lvl <= lvl(i)-1) is big; the
//            deepest of them is a leaf unless it is big.
// Cell and leaf indices then come from per-tile, per-level counts (scan over
// tiles, in tile order = Morton order within each level); so do parents (the
// last cell of the level above starting at or before a cell's particle).
// Range ends follow from the children partitioning their parent: a cell ends
// where the next sibling of its nearest ancestor-or-self that has one starts.
// Kernels: flat_bigl (lvl, bigL), flat_cells (cell levels, tile counts),
// flat_scan (scanned counts, level totals), flat_emit (cell records, parents,
// first children), flat_link (range ends, counts, activity, child masks).

__device__ __forceinline__ int lcp_levels(uint64_t a, uint64_t b, int K) {
    const uint64_t x = a ^ b;
    if (x == 0) return K;
    const int m = 63 - __clzll((long long)x);
    return (2 * K - 1 - m) >> 1;
}

// Smallest m in [lo, hi] with a[m] >= target, or hi + 1 (a nondecreasing):
// galloping from lo, then bisection.
__device__ __forceinline__ int gallop_ge(const uint32_t* __restrict__ a, int lo, int hi, uint32_t target) {
    if (lo > hi) return hi + 1;
    if (a[lo] >= target) return lo;
    int prev = lo, step = 1;
    int cur = lo + 1;
    while (cur <= hi && a[cur] < target) {
        prev = cur;
        step <<= 1;
        cur = lo + step;
    }
    int L = prev + 1, R = min(cur, hi + 1);  // answer in [L, R]
    while (L < R) {
        const int mid = (L + R) >> 1;
        if (a[mid] >= target) R = mid;
        else L = mid + 1;
    }
    return L;
}

// First j <= i with the same key prefix (>> sh) as particle i, with the whole
// warp on one query (i and sh the same in every lane): 32 probes per round,
// galloping back from i by 1, 2, 4, ... 2^30, then 32-way splits of the
// bracket, so a group of d particles takes about 1 + log_31(d) rounds of loads
// instead of 2 log_2(d) dependent ones for one thread alone.
__device__ __forceinline__ int group_start_warp(const uint64_t* __restrict__ key, int i, int sh) {
    const int lane = threadIdx.x & 31;
    const uint64_t v = key[i] >> sh;
    const int p0 = lane < 31 ? max(0, i - (1 << lane)) : 0;
    const unsigned in0 = __ballot_sync(0xffffffffu, (key[p0] >> sh) == v);
    if (in0 == 0xffffffffu) return 0;                  // the group reaches particle 0
    const int t0 = __ffs(~in0) - 1;                     // first probe outside the group
    int lo = __shfl_sync(0xffffffffu, p0, t0) + 1;
    int hi = t0 == 0 ? i : __shfl_sync(0xffffffffu, p0, t0 - 1);
    while (lo < hi) {                                   // the answer is in [lo, hi]; hi is in the group
        const int step = (hi - lo + 30) / 31;
        const int q = min(hi, lo + step * lane);
        const unsigned in = __ballot_sync(0xffffffffu, (key[q] >> sh) == v);
        const int t = __ffs(in) - 1;                    // lane 31 probes hi: t >= 0
        if (t == 0) return lo;
        const int qt = __shfl_sync(0xffffffffu, q, t), qp = __shfl_sync(0xffffffffu, q, t - 1);
        lo = qp + 1;
        hi = qt;
    }
    return lo;
}

__device__ __forceinline__ uint32_t compact2(uint64_t x) {
    x &= 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
    return (uint32_t)x;
}

// pinfo[i] = lvl | (bigL + 1) << 8
__global__ void __launch_bounds__(kFlatTile)
flat_bigl(Tree2D t, int max_src, int max_par, uint32_t* __restrict__ pinfo, unsigned* err) {
    const int n = t.n, K = t.key_levels;
    const uint64_t* __restrict__ key = t.key;
    const uint32_t* __restrict__ as = t.actscan;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t ki = key[i];
        const int lvl = i == 0 ? 1 : lcp_levels(key[i - 1], ki, K) + 1;   // K + 1: equal keys
        int big = -1;
        if (i + max_par < n) big = lcp_levels(ki, key[i + max_par], K);
        const uint32_t target = as[i] + (uint32_t)max_src + 1u;
        if (as[n] >= target) {
            // as[m] - as[i] <= m - i, so m >= i + max_src + 1: start the search there
            const int m = gallop_ge(as, min(n, i + max_src + 1), n, target);  // particle m-1 is that active one
            big = max(big, lcp_levels(ki, key[m - 1], K));
        }
        pinfo[i] = (uint32_t)lvl | ((uint32_t)(big + 1) << 8);
    }
}

// The cell levels of every particle (pinfo bits 16..23 first, 24..31 last; 0 =
// none) and the per-tile counts of cells and leaves of every level. A particle
// starting a group at level lvl starts cells only if the parent group (level
// lvl-1) is big; that group starts at the last particle before it that starts
// a group at level <= lvl-1, found from per-warp ballots of the tile (most
// parents start in the same tile) and otherwise by a search of the keys back
// from the tile's first particle.
__global__ void __launch_bounds__(kFlatTile)
flat_cells(Tree2D t, uint32_t* __restrict__ pinfo, uint32_t* __restrict__ tile_cnt, int tiles, unsigned* err) {
    __shared__ unsigned s_c[kMaxLevels2D + 1], s_l[kMaxLevels2D + 1];
    __shared__ uint32_t s_pi[kFlatTile];                          // the tile's pinfo words
    __shared__ unsigned s_mk[kMaxLevels2D + 1][kFlatTile / 32];   // per warp: lanes starting a group at level <= m
    const int n = t.n, K = t.key_levels;
    const uint64_t* __restrict__ key = t.key;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        for (int k = threadIdx.x; k <= K; k += blockDim.x) s_c[k] = s_l[k] = 0;
        const int tb = tile * kFlatTile;
        const int i = tb + threadIdx.x;
        const uint32_t w = i < n ? pinfo[i] : 0xffu;   // past the end: no group start
        const int lvl = (int)(w & 0xff);
        s_pi[threadIdx.x] = w;
        for (int m = 1; m <= K; ++m) {
            const unsigned mk = __ballot_sync(0xffffffffu, lvl <= m);
            if (lane == 0) s_mk[m][warp] = mk;
        }
        __syncthreads();
        // pinfo word of the parent group's first particle (only bits 0..15,
        // lvl and big, are read: they are not rewritten below)
        const bool starts = lvl <= K;   // implies i < n
        const int m = lvl - 1;
        uint32_t wp = 0;
        bool need = false;
        if (starts && lvl > 1) {
            unsigned mk = s_mk[m][warp] & ((1u << lane) - 1u);
            int wq = warp;
            while (!mk && wq > 0) mk = s_mk[m][--wq];
            if (mk) wp = s_pi[wq * 32 + 31 - __clz(mk)];
            else need = true;
        }
        // parents starting before the tile: one cooperative search per level
        for (unsigned qm = __ballot_sync(0xffffffffu, need); qm;) {
            const int mq = __shfl_sync(0xffffffffu, m, __ffs(qm) - 1);
            const uint32_t wg = pinfo[group_start_warp(key, tb, 2 * (K - mq))];
            if (need && m == mq) wp = wg;
            qm &= ~__ballot_sync(0xffffffffu, need && m == mq);
        }
        if (i < n) {
            const int big = (int)((w >> 8) & 0xff) - 1;
            int first = 0, last = 0;
            if (starts) {
                const bool exists = lvl == 1 || (int)((wp >> 8) & 0xff) - 1 >= m;
                if (exists) {
                    first = lvl;
                    last = min(K, max(lvl, big + 1));
                    if (big >= K) set_err(err, ERR_DEPTH);  // a group of level K cannot be split
                    for (int L = first; L <= last; ++L) atomicAdd(&s_c[L], 1u);
                    if (big < last) atomicAdd(&s_l[last], 1u);
                }
            }
            pinfo[i] = (w & 0xffffu) | ((uint32_t)first << 16) | ((uint32_t)last << 24);
        }
        __syncthreads();
        for (int k = threadIdx.x; k <= K; k += blockDim.x) {
            tile_cnt[(size_t)k * tiles + tile] = s_c[k];
            tile_cnt[(size_t)(kMaxLevels2D + 1 + k) * tiles + tile] = s_l[k];
        }
        __syncthreads();
    }
}

// Level starts, totals and the root cell (treeCell.cpp:1117-1133), from the
// row totals of flat_scan: one warp, lane l for level l + 1 (K <= 31).
__device__ void flat_totals(Tree2D t, const uint32_t* __restrict__ level_tot, unsigned* err) {
    const int K = t.key_levels, lane = threadIdx.x & 31, L = lane + 1;
    TreeInfo2D* info = t.info;
    const int c = L <= K ? (int)__ldcg(level_tot + L) : 0;
    const int lf = L <= K ? (int)__ldcg(level_tot + kMaxLevels2D + 1 + L) : 0;
    int ci = c, li = lf;   // inclusive sums over levels 1..L
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int yc = __shfl_up_sync(0xffffffffu, ci, o), yl = __shfl_up_sync(0xffffffffu, li, o);
        if (lane >= o) {
            ci += yc;
            li += yl;
        }
    }
    const int cells = 1 + __shfl_sync(0xffffffffu, ci, 31), leaves = __shfl_sync(0xffffffffu, li, 31);
    // first cell / leaf of each level: the root, then the levels below it
    info->level_start[L] = 1 + ci - c;
    info->leaf_start[L] = li - lf;
    const int depth = (int)__reduce_max_sync(0xffffffffu, c > 0 ? (unsigned)L : 0u);
    // leaf level range (TreeCell::min_level / max_level, treeCell.cpp:1236-1240)
    const unsigned mn = __reduce_min_sync(0xffffffffu, lf > 0 ? (unsigned)L : 255u);
    const unsigned mx = __reduce_max_sync(0xffffffffu, lf > 0 ? (unsigned)L : 0u);
    if (lane != 0) return;
    info->level_start[0] = 0;
    info->leaf_start[0] = 0;
    for (int k = 33; k < kMaxLevels2D + 3; ++k) {
        info->level_start[k] = cells;
        info->leaf_start[k] = leaves;
    }
    info->n_cells = cells;
    info->n_leaves = leaves;
    info->depth = depth;
    info->l2_irregular = 0;
    info->min_leaf_level = mn == 255u ? -1 : (int)mn;
    info->max_leaf_level = mx == 0u ? -1 : (int)mx;
    if (cells > t.cap_cells) set_err(err, ERR_CELL_CAP);
    const Geom2D* g = t.geom;
    t.c_lo[0] = 0;
    t.c_hi[0] = t.n;
    const int src = (int)t.actscan[t.n];
    t.c_src[0] = src;
    t.c_flags[0] = src != 0 ? CELL_ACTIVE : 0;
    t.c_parent[0] = -1;
    t.c_child0[0] = -1;   // set by flat_emit (the first level-1 cell)
    t.c_chmask[0] = 0;
    t.c_level[0] = 0;
    t.c_ix[0] = 0;
    t.c_iy[0] = 0;
    t.c_code[0] = 0;
    t.c_leafidx[0] = -1;
    t.c_cx[0] = xadd(g->pivx, xmul(0.5, g->root));
    t.c_cy[0] = xadd(g->pivy, xmul(0.5, g->root));
    if (t.dense) t.dense[0] = 0;
    if (t.nonleaf && cells > 1) t.nonleaf[0] = 0;
}

// One block per (kind, level) row of levels 0..K: exclusive scan of the tile
// counts in place (kScanPer consecutive counts per thread and round) and the
// row total; the last block to finish then sets the level starts, totals and
// root cell (flat_totals). ticket: zero on entry.
constexpr int kScanPer = 4;

__global__ void __launch_bounds__(1024)
flat_scan(Tree2D t, uint32_t* __restrict__ tile_cnt, int tiles, uint32_t* __restrict__ level_tot, unsigned* ticket,
          unsigned* err) {
    __shared__ uint32_t s_w[32];
    __shared__ bool s_last;
    const int K = t.key_levels;
    const int r = blockIdx.x <= K ? (int)blockIdx.x : kMaxLevels2D + 1 + ((int)blockIdx.x - K - 1);
    uint32_t* row = tile_cnt + (size_t)r * tiles;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < tiles; b0 += 1024 * kScanPer) {
        const int k0 = b0 + threadIdx.x * kScanPer;
        uint32_t v[kScanPer], sum = 0;
        #pragma unroll
        for (int u = 0; u < kScanPer; ++u) {
            v[u] = k0 + u < tiles ? row[k0 + u] : 0u;
            sum += v[u];
        }
        uint32_t x = sum;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t y = s_w[lane];
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            s_w[lane] = y;   // inclusive over warps
        }
        __syncthreads();
        uint32_t e = carry + (warp ? s_w[warp - 1] : 0u) + x - sum;
        #pragma unroll
        for (int u = 0; u < kScanPer; ++u) {
            if (k0 + u < tiles) row[k0 + u] = e;
            e += v[u];
        }
        carry += s_w[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        level_tot[r] = carry;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && warp == 0) {
        __threadfence();
        flat_totals(t, level_tot, err);
    }
}

// Cell records (and leaf entries) of every particle's cell levels, indices
// from the scanned tile counts plus the rank inside the tile. The parent of a
// level-L cell starting at particle i is the last level-(L-1) cell starting
// at or before i (cells of a level are disjoint and in particle order), so it
// too is a count; a split cell's first child starts at the same particle and
// sets the parent's child0 (the only writer: leaves set their own -1). Range
// ends: flat_link. A warp's (particle, level) cells are spread over its lanes,
// one per lane and round, so a particle starting many levels does not hold
// the block at its barrier.
__global__ void __launch_bounds__(kFlatTile, 8)
flat_emit(Tree2D t, const uint32_t* __restrict__ pinfo, const uint32_t* __restrict__ tile_cnt, int tiles,
          int max_par, unsigned* err) {
    constexpr int NW = kFlatTile / 32;
    __shared__ unsigned s_mc[kMaxLevels2D + 1][NW], s_ml[kMaxLevels2D + 1][NW];   // lanes with a cell / leaf at L
    __shared__ int s_c0[kMaxLevels2D + 1], s_l0[kMaxLevels2D + 1];   // the tile's first cell / leaf of each level
    __shared__ double s_len[kMaxLevels2D + 1];                        // cell size of each level
    if (block_fatal(err)) return;
    const int n = t.n, K = t.key_levels;
    const TreeInfo2D* info = t.info;
    const double root = t.geom->root, pivx = t.geom->pivx, pivy = t.geom->pivy;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k <= K; k += blockDim.x) s_len[k] = xdiv(root, ldexp(1.0, k));
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int tb = tile * kFlatTile;
        const int i = tb + threadIdx.x;
        const uint32_t w = i < n ? pinfo[i] : 0u;
        const uint64_t ki = i < n ? t.key[i] : 0ull;
        for (int k = threadIdx.x; k <= K; k += blockDim.x) {
            s_c0[k] = info->level_start[k] + (int)tile_cnt[(size_t)k * tiles + tile];
            s_l0[k] = info->leaf_start[k] + (int)tile_cnt[(size_t)(kMaxLevels2D + 1 + k) * tiles + tile];
        }
        const int first = (int)((w >> 16) & 0xff), last = (int)(w >> 24), big = (int)((w >> 8) & 0xff) - 1;
        const int ncell = first ? last - first + 1 : 0;
        // lane masks of every level (zero outside the warp's range), then one barrier
        const int Llo = (int)__reduce_min_sync(0xffffffffu, first ? (unsigned)first : 255u);
        const int Lhi = (int)__reduce_max_sync(0xffffffffu, first ? (unsigned)last : 0u);
        if (lane <= K) {
            s_mc[lane][warp] = 0u;
            s_ml[lane][warp] = 0u;
        }
        __syncwarp();
        for (int L = Llo; L <= Lhi; ++L) {
            const bool has = first && first <= L && L <= last;
            const bool lf = has && L == last && big < last;
            const unsigned mc = __ballot_sync(0xffffffffu, has), ml = __ballot_sync(0xffffffffu, lf);
            if (lane == 0) {
                s_mc[L][warp] = mc;
                s_ml[L][warp] = ml;
            }
        }
        __syncthreads();
        // the warp's cells in (lane, level) order, 32 per round
        int incl = ncell;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int r0 = 0; r0 < total; r0 += 32) {
            const int q = r0 + lane;
            // owner lane of cell q: the number of lanes whose inclusive count is <= q
            int ol = 0;
            #pragma unroll
            for (int step = 16; step >= 1; step >>= 1)
                if (__shfl_sync(0xffffffffu, incl, ol + step - 1) <= q) ol += step;
            ol = min(ol, 31);
            const int ofirst = __shfl_sync(0xffffffffu, first, ol), olast = __shfl_sync(0xffffffffu, last, ol);
            const int obig = __shfl_sync(0xffffffffu, big, ol);
            const int oexcl = __shfl_sync(0xffffffffu, incl - ncell, ol);
            const uint64_t okey = __shfl_sync(0xffffffffu, ki, ol);
            if (q >= total) continue;
            const int L = ofirst + (q - oexcl);
            const bool lf = L == olast && obig < olast;
            const unsigned lt = (1u << ol) - 1u;
            int bc = 0, bl = 0, bp = 0;
            for (int k = 0; k < warp; ++k) {
                bc += __popc(s_mc[L][k]);
                bl += __popc(s_ml[L][k]);
                bp += __popc(s_mc[L - 1][k]);
            }
            const int ci = s_c0[L] + bc + __popc(s_mc[L][warp] & lt);
            if (ci >= t.cap_cells) {
                set_err(err, ERR_CELL_CAP);
                continue;
            }
            const int io = tb + warp * 32 + ol;   // the particle starting the cell
            // parent: level-(L-1) cells starting at or before particle io, minus one
            const int p = L == 1 ? 0 : s_c0[L - 1] + bp + __popc(s_mc[L - 1][warp] & (lt | (1u << ol))) - 1;
            const int sh = 2 * (K - L);
            const uint64_t code = okey >> sh;
            const int ix = (int)compact2(code), iy = (int)compact2(code >> 1);
            const double len = s_len[L];
            t.c_lo[ci] = io;
            t.c_parent[ci] = p;
            t.c_flags[ci] = lf ? CELL_LEAF : 0;   // counts and activity: flat_link
            if (L == olast) t.c_child0[ci] = -1;  // no child (split cells: set by their first child)
            if (L > ofirst || io == 0) t.c_child0[p] = ci;   // the parent starts at this particle too
            t.c_chmask[ci] = 0;
            t.c_level[ci] = (uint8_t)L;
            t.c_ix[ci] = ix;
            t.c_iy[ci] = iy;
            t.c_code[ci] = code;
            t.c_cx[ci] = xadd(pivx, xmul(xadd(0.5, (double)ix), len));
            t.c_cy[ci] = xadd(pivy, xmul(xadd(0.5, (double)iy), len));
            if (t.dense && L <= t.dense_levels) t.dense[start_id2(L) + ix + ((int64_t)iy << L)] = ci;
            // leaves before this cell: of the lower levels, then of this level
            const int li = s_l0[L] + bl + __popc(s_ml[L][warp] & lt);
            if (lf) {
                t.c_leafidx[ci] = li;
                t.leaf_cells[li] = ci;
            } else {
                t.c_leafidx[ci] = -1;
                if (t.nonleaf) t.nonleaf[ci - li] = ci;   // the cells before it that are not leaves
            }
        }
        __syncthreads();
    }
}

// Range end, source count and activity of every cell, and the parent's child
// mask. The children of a split cell partition its range, so a cell's range
// ends where the next sibling of its nearest ancestor-or-self that has one
// starts (a walk up the parent links, one level per step; most cells stop at
// their own next sibling), or at n.
__global__ void flat_link(Tree2D t, int max_par, unsigned* err) {
    if (fatal(err)) return;
    const int nc = t.info->n_cells, n = t.n;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x + 1; c < nc; c += gridDim.x * blockDim.x) {
        const int L = t.c_level[c];
        const uint64_t code = t.c_code[c];
        const uint8_t fl = t.c_flags[c];
        const int lo = t.c_lo[c], p = t.c_parent[c];
        int hi = n;
        {
            int a = c, ap = p, aL = L;
            uint64_t acode = code;
            while (aL >= 1) {
                const int s = a + 1;
                if (s < nc && t.c_level[s] == aL && (t.c_code[s] >> 2) == (acode >> 2)) {
                    hi = t.c_lo[s];
                    break;
                }
                if (ap <= 0) break;   // the parent is the root: the range runs to n
                a = ap;
                ap = t.c_parent[a];
                aL -= 1;
                acode >>= 2;
            }
        }
        if (hi <= lo || hi > n || p < 0 || p >= nc || t.c_level[p] != L - 1 || t.c_code[p] != (code >> 2)) {
            set_err(err, ERR_INDEX);
            continue;
        }
        const int src = (int)(t.actscan[hi] - t.actscan[lo]);
        t.c_hi[c] = hi;
        t.c_src[c] = src;
        if (src != 0) t.c_flags[c] = fl | CELL_ACTIVE;
        unsigned* word = reinterpret_cast<unsigned*>(reinterpret_cast<uintptr_t>(&t.c_chmask[p]) & ~(uintptr_t)3);
        const unsigned shift = 8u * (unsigned)(reinterpret_cast<uintptr_t>(&t.c_chmask[p]) & 3);
        atomicOr(word, (1u << (unsigned)(code & 3)) << shift);
    }
}

}  // namespace

// Grid and per-block share of the cooperative sort for n particles (about
// `items` per block, at most one block per SM), or false when it does not
// apply (share above kCoopSortMaxChunk, or fewer than one resident block per
// SM).
bool coop_sort_shape(int n, int items, int* grid, int* chunk) {
    static int sms = 0, smem_set = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return false;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
    }
    const int g = std::max(std::max(1, ceil_div(n, kCoopSortMaxChunk)),
                           std::min(std::min(sms, kCoopSortGridMax), ceil_div(n, items)));
    const int c = ceil_div(n, g);
    if (c > kCoopSortMaxChunk) return false;
    if (smem_set == 0) {
        if (cudaFuncSetAttribute(sort2d_coop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kCoopSortMaxChunk * 10) != cudaSuccess)
            return false;
        smem_set = 1;
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sort2d_coop, kCoopSortThreads, (size_t)c * 10) !=
            cudaSuccess ||
        occ < 1)
        return false;
    *grid = g;
    *chunk = c;
    return true;
}

cudaError_t keys_sort2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                        TreeScratch2D& s, double exp_pct, unsigned* err, cudaStream_t st, int* launches,
                        int shallow_cap, int items_per_block) {
    const int n = t.n;
    const int K = t.key_levels;
    const int gridN = std::max(1, std::min(148 * 8, ceil_div(n, 256)));
    unsigned* done = s.lvl_ticket + kMaxLevels2D + 1;
    const int bb_blocks = std::max(1, std::min(kBBoxBlocks, ceil_div(n, 256)));
    cudaError_t e = cudaMemsetAsync(s.lvl_ticket, 0, sizeof(unsigned) * kTicketWords, st);
    if (e != cudaSuccess) return e;
    *launches += 1;
    int coop_grid = 0, coop_chunk = 0;
    if (2 * K <= 32 && s.coop_words && coop_sort_shape(n, items_per_block, &coop_grid, &coop_chunk)) {
        uint32_t* k32 = reinterpret_cast<uint32_t*>(s.key_alt);
        const size_t smem = (size_t)coop_chunk * 10;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(coop_grid);
        cfg.blockDim = dim3(kCoopSortThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, sort2d_coop, x, y, q, act, exp_pct, (2 * K + 7) / 8, shallow_cap, t,
                               s.bbox_partial,
                               k32, k32 + n, s.val_alt, t.perm, s.coop_words, coop_chunk,
                               err);
        if (e != cudaSuccess) return e;
        *launches += 1;
        return cudaGetLastError();
    }
    bbox2d<<<bb_blocks, 256, 0, st>>>(x, y, n, exp_pct, K, t.geom, s.bbox_partial, done, err);
    *launches += 1;
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

namespace {
// pq[i] = q[perm[i]]: the strengths in tree order, for a sort that ran
// without them (keys_sort2d with q = null).
__global__ void __launch_bounds__(256) gather_strengths2d(const uint32_t* __restrict__ perm,
                                                          const double* __restrict__ q, double* __restrict__ pq, int n,
                                                          unsigned* err) {
    if (fatal(err)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t j = __ldg(perm + i);
        if (j >= (uint32_t)n) {
            set_err(err, ERR_INDEX);
            continue;
        }
        pq[i] = __ldg(q + j);
    }
}
}  // namespace

cudaError_t gather_strengths2d(const Tree2D& t, const double* q, unsigned* err, cudaStream_t st, int* launches) {
    gather_strengths2d<<<std::max(1, std::min(148 * 8, ceil_div(t.n, 256))), 256, 0, st>>>(t.perm, q, t.pq, t.n, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t levels2d_flat(Tree2D& t, TreeScratch2D& s, int max_src, int max_par, unsigned* err, cudaStream_t st,
                          int* launches) {
    const int n = t.n;
    const int tiles = ceil_div(n, kFlatTile);
    if (tiles > s.flat_tiles) return cudaErrorInvalidValue;
    const int grid = std::max(1, std::min(tiles, 148 * 8));
    flat_bigl<<<grid, kFlatTile, 0, st>>>(t, max_src, max_par, s.pinfo, err);
    flat_cells<<<grid, kFlatTile, 0, st>>>(t, s.pinfo, s.tile_cnt, tiles, err);
    // lvl_ticket[0]: zeroed with the other tickets before the sort
    flat_scan<<<2 * (t.key_levels + 1), 1024, 0, st>>>(t, s.tile_cnt, tiles, s.level_tot, s.lvl_ticket, err);
    flat_emit<<<grid, kFlatTile, 0, st>>>(t, s.pinfo, s.tile_cnt, tiles, max_par, err);
    const int gc = std::max(1, std::min(148 * 8, ceil_div(t.cap_cells, 256)));
    flat_link<<<gc, 256, 0, st>>>(t, max_par, err);
    *launches += 5;
    return cudaGetLastError();
}

cudaError_t levels2d(Tree2D& t, TreeScratch2D& s, int max_src, int max_par, unsigned* err, cudaStream_t st,
                     int* launches) {
    return levels2d_flat(t, s, max_src, max_par, err, st, launches);
}


cudaError_t build_tree2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                         TreeScratch2D& s, int max_src, int max_par, double exp_pct, unsigned* err, cudaStream_t st,
                         int* launches) {
    cudaError_t e = keys_sort2d(x, y, q, act, t, s, exp_pct, err, st, launches, std::min(max_src, max_par));
    if (e != cudaSuccess) return e;
    return levels2d(t, s, max_src, max_par, err, st, launches);
}

}  // namespace vpm
