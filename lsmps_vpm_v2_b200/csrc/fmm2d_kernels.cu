// FP64 (plain form) translation and evaluation kernels of the 2D Laurent FMM
// (reference src/FMM/fmm2D.cpp). Expansions are complex: multipole
//   a_k = sum_j q_j (z_j - z_c)^k                      (P2M, fmm2D.cpp:237-284)
// and local coefficients b_p, with the field at z taken as
//   E_x = Re F, E_y = -Im F,  F = sum of q/(z - z_j) terms.
//
// Stage map:
//   fmm2d_upward_direct  moments of every cell of at most 1024 particles
//                 straight from its particles (upward_direct2d), then M2M of
//                 the larger cells level by level in one cooperative launch
//                 (m2m_big_levels_coop), with an optional event between the
//                 two; fmm2D.cpp:237-284, 309-379.
//   fmm2d_upward  P2M of every active leaf, then M2M over all levels (p2m2d,
//                 m2m_levels_coop), for orders the direct form does not cover.
//   fmm2d_m2l_only  lists 2 and 4 of every cell at level >= 2 in FP64 with the
//                 49 precomputed list-2 operators (m2l2d_op, fmm2D.cpp:396-556);
//                 the mixed forms' per-parent list-2 M2L is in m2l_tc.cu.
//   fmm2d_l2l_leaves, fmm2d_l2l  every leaf's local expansion from its
//                 ancestors' M2L parts, or the level loop (fmm2D.cpp:587-651).
//   fmm2d_eval, fmm2d_m2p, fmm2d_eval_combine  M2P over list 3
//                 (fmm2D.cpp:1040-1066) and L2P (fmm2D.cpp:1076-1093), warp per
//                 leaf; the combine pass adds the near field and writes the
//                 output in the caller's order.
//   fmm2d_p2p_f64_tma, fmm2d_p2p_f32  near field over list 1, j != i
//                 (fmm2D.cpp:135-179): FP64 warp kernel for the plain form,
//                 packed FP32 tiles for the mixed forms.
#include "fmm2d.cuh"

#include <complex>
#include <vector>

namespace vpm {

namespace {

constexpr int W = kMaxP + 1;

int64_t binom_host(int n, int k, bool exact) {
    if (k > n) return 0;
    if (exact) {
        int64_t c = 1;
        for (int i = 1; i <= k; ++i) c = c * (n - k + i) / i;
        return c;
    }
    // The reference's binComb: n!/max(k,n-k)! in 32-bit int (wrapping), then
    // truncating divisions by min(k,n-k)!.
    int inv = n - k;
    int mx = inv > k ? inv : k, mn = inv > k ? k : inv;
    int32_t c = 1;
    for (int i = n; i > mx; --i) c = (int32_t)((uint32_t)c * (uint32_t)i);
    for (int i = mn; i > 1; --i) c /= i;
    return c;
}

// 1 / a for the FP64 near field: the hardware seed (about 23 correct bits)
// refined by one third-order step, y (1 + e + e^2) with e = 1 - a y, which
// leaves a relative error of order e^3 (below the double's own rounding), in
// three FMAs where two Newton steps take four.
__device__ __forceinline__ double rcp_nr(double a) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    const double e = fma(-a, y, 1.0);
    return fma(y, fma(e, e, e), y);
}


// ---- upward pass -----------------------------------------------------------

constexpr int kP2MWarps = 2;
constexpr int kAccPad = 33;  // padded lane stride of the P2M accumulators

// P2M, one warp per leaf: lane j takes particles j, j+32, ... and adds
// q (z - z_c)^k into its own shared-memory accumulator column k; the columns
// are then summed in a fixed order (deterministic).
__global__ void __launch_bounds__(32 * kP2MWarps)
p2m2d(Tree2D t, double2* __restrict__ a, int P, unsigned* err) {
    extern __shared__ double2 acc_sm[];
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double2* acc = acc_sm + (size_t)wib * (P + 1) * kAccPad;
    const int nl = t.info->n_leaves;
    const int warps = gridDim.x * kP2MWarps;
    for (int li = blockIdx.x * kP2MWarps + wib; li < nl; li += warps) {
        const int c = t.leaf_cells[li];
        if (!(t.c_flags[c] & CELL_ACTIVE)) continue;
        for (int k = 0; k <= P; ++k) acc[k * kAccPad + lane] = make_double2(0.0, 0.0);
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        for (int j = lo + lane; j < hi; j += 32) {
            if (!t.pact[j]) continue;
            const double2 w = make_double2(t.px[j] - zx, t.py[j] - zy);
            double2 wk = make_double2(t.pq[j], 0.0);
            for (int k = 0; k <= P; ++k) {
                double2* ak = &acc[k * kAccPad + lane];
                *ak = cadd(*ak, wk);
                wk = cmul(wk, w);
            }
        }
        __syncwarp();
        if (lane <= P) {
            double2 sum = make_double2(0.0, 0.0);
            for (int l = 0; l < 32; ++l) sum = cadd(sum, acc[lane * kAccPad + l]);
            a[(size_t)c * (P + 1) + lane] = sum;
        }
        __syncwarp();
    }
}

// Warps per block of the level kernels (M2M, L2L): the cooperative loops run
// one 256-thread block per SM, so a grid barrier has 148 arrivals.
constexpr int kLevelWarps = 8;

// M2M into the active non-leaf cells of level L (fmm2D.cpp:309-379). A warp
// holds G = 32/(P+1) cells, lane (g, p) computing a_p of cell g by Horner's
// rule in t = z_child - z_parent for all children at once (independent
// chains), then summing the children in order:
//   a_p += a0 t^p + sum_{k=1..p} m2m[p][k] a_k t^(p-k).
// Child expansions are read through L2 (ld.cg): in the cooperative kernel the
// level below was written by other blocks of the same launch.
__device__ __forceinline__ void m2m_level_body(const Tree2D& t, double2* __restrict__ a,
                                               const double* __restrict__ coef, int P, int L, int min_count = -1) {
    __shared__ double2 s_child[kLevelWarps][4][32];  // [warp][child][g * (P+1) + k]
    __shared__ double2 s_tt[kLevelWarps][4][16];     // [warp][child][g]
    const double* g_m2m = coef + kCoefM2M;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int Q = P + 1, G = 32 / Q, g = lane / Q, k = lane - g * Q;
    const int c0 = t.info->level_start[L], c1 = t.info->level_start[L + 1];
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
    for (int cb = c0 + gw * G; cb < c1; cb += warps * G) {
        const int c = cb + g;
        bool ok = g < G && c < c1;
        if (ok) {
            const uint8_t f = t.c_flags[c];
            ok = !(f & CELL_LEAF) && (f & CELL_ACTIVE) && t.c_hi[c] - t.c_lo[c] > min_count;
        }
        unsigned m = 0;
        int ch0 = -1;
        if (ok) {
            m = t.c_chmask[c];
            ch0 = t.c_child0[c];
            ok = ch0 >= 0;
        }
        const int nch = ok ? __popc(m) : 0;
        #pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r < nch) s_child[wib][r][lane] = __ldcg(&a[(size_t)(ch0 + r) * Q + k]);
        if (k < nch) s_tt[wib][k][g] = make_double2(t.c_cx[ch0 + k] - t.c_cx[c], t.c_cy[ch0 + k] - t.c_cy[c]);
        __syncwarp();
        if (ok) {
            double2 acc = make_double2(0.0, 0.0);
            if (k == 0) {
                for (int r = 0; r < nch; ++r) acc = cadd(acc, s_child[wib][r][g * Q]);
            } else {
                double2 S[4], tt[4];
                #pragma unroll
                for (int r = 0; r < 4; ++r) {
                    S[r] = s_child[wib][r][g * Q];
                    tt[r] = s_tt[wib][r][g];
                }
                for (int j = k - 1; j >= 0; --j) {
                    const int kk = k - j;
                    const double cf = g_m2m[k * W + kk];
                    #pragma unroll
                    for (int r = 0; r < 4; ++r)
                        if (r < nch) S[r] = cfma(S[r], tt[r], cscale(s_child[wib][r][g * Q + kk], cf));
                }
                #pragma unroll
                for (int r = 0; r < 4; ++r)
                    if (r < nch) acc = cadd(acc, S[r]);
            }
            a[(size_t)c * Q + k] = acc;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(128)
m2m_level2d(Tree2D t, double2* __restrict__ a, const double* __restrict__ coef, int P, int L, unsigned* err) {
    if (block_fatal(err)) return;
    m2m_level_body(t, a, coef, P, L);
}

// All M2M levels (depth-1 down to 1) in one cooperative launch, a grid
// barrier between levels (barrier word: zeroed before every evaluation, used
// by this kernel only).
__global__ void __launch_bounds__(32 * kLevelWarps)
m2m_levels_coop(Tree2D t, double2* __restrict__ a, const double* __restrict__ coef, int P, unsigned* bar,
                unsigned* err) {
    const int depth = t.info->depth;
    for (int L = depth - 1; L >= 1; --L) {
        if (!block_fatal(err)) m2m_level_body(t, a, coef, P, L);
        grid_sync_counter(bar, err);
    }
}

// The same level loop over the cells of more than min_count particles only
// (the others are final already), from the deepest level holding one
// (*top_level, written by upward_direct2d) up to level 1.
__global__ void __launch_bounds__(32 * kLevelWarps)
m2m_big_levels_coop(Tree2D t, double2* __restrict__ a, const double* __restrict__ coef, int P, int min_count,
                    const unsigned* top_level, unsigned* bar, unsigned* err) {
    const int top = (int)*top_level;
    for (int L = top; L >= 1; --L) {
        if (!block_fatal(err)) m2m_level_body(t, a, coef, P, L, min_count);
        grid_sync_counter(bar, err);
    }
}

// L2L pull into every cell of level L >= 3 from its parent (fmm2D.cpp:587-651,
// where each non-leaf parent at levels 2..max-1 pushes into its children):
//   b_p(c) += sum_{k=p..P} l2l[p][k] b_k(parent) t^(k-p),  t = z_c - z_parent.
// A warp holds G = 32/(P+1) cells, lane (g, p) computing b_p of cell g. The
// parent's expansion is final because level L-1 is complete (previous launch,
// or before the grid barrier in the cooperative kernel); it is read through
// L2 (ld.cg).
__device__ __forceinline__ void l2l_level_body(const Tree2D& t, double2* __restrict__ b,
                                               const double* __restrict__ coef, int P, int L) {
    __shared__ double2 s_par[kLevelWarps][32];
    const double* g_l2l = coef + kCoefL2L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int Q = P + 1, G = 32 / Q, g = lane / Q, k = lane - g * Q;
    const int c0 = t.info->level_start[L], c1 = t.info->level_start[L + 1];
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
    for (int cb = c0 + gw * G; cb < c1; cb += warps * G) {
        const int c = cb + g;
        const bool ok = g < G && c < c1;
        const int par = ok ? t.c_parent[c] : 0;
        if (ok) s_par[wib][lane] = __ldcg(&b[(size_t)par * Q + k]);
        __syncwarp();
        if (ok) {
            const double2 tt = make_double2(t.c_cx[c] - t.c_cx[par], t.c_cy[c] - t.c_cy[par]);
            const double* cf = g_l2l + k * W;
            const double2* sp = &s_par[wib][g * Q];
            double2 S = cscale(sp[P], cf[P]);
            for (int kk = P - 1; kk >= k; --kk) S = cfma(S, tt, cscale(sp[kk], cf[kk]));
            double2* bc = &b[(size_t)c * Q + k];
            *bc = cadd(__ldcg(bc), S);
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(128)
l2l_level2d(Tree2D t, double2* __restrict__ b, const double* __restrict__ coef, int P, int L, unsigned* err) {
    if (block_fatal(err)) return;
    l2l_level_body(t, b, coef, P, L);
}

// All L2L levels (3 down to the depth) in one cooperative launch.
__global__ void __launch_bounds__(32 * kLevelWarps)
l2l_levels_coop(Tree2D t, double2* __restrict__ b, const double* __restrict__ coef, int P, unsigned* bar,
                unsigned* err) {
    const int depth = t.info->depth;
    for (int L = 3; L <= depth; ++L) {
        if (!block_fatal(err)) l2l_level_body(t, b, coef, P, L);
        grid_sync_counter(bar, err);
    }
}

// ---- M2L -------------------------------------------------------------------

// One warp per target cell. The warp is split into G = 32/P groups of P lanes;
// lane (g, p-1) accumulates b_p over the sources g, g+G, ... of list 2 then
// list 4. Powers w^m = (z_src - z_tgt)^(-m), m = 1..2P, go through shared
// memory per group.
__global__ void __launch_bounds__(128)
m2l2d(Tree2D t, Lists2D l, const double2* __restrict__ a, double2* __restrict__ b, const double* __restrict__ coef,
      int P, unsigned* err) {
    const double* g_m2l = coef + kCoefM2L;
    extern __shared__ double2 sm[];
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int G = 32 / P;
    const int g = lane / P, p = lane % P + 1;
    const bool on = g < G;
    // per warp: pw[G][2P+1], as[G][P+1], part[G][P+1]
    double2* pw = sm + (size_t)wib * (G * (2 * P + 1) + 2 * G * (P + 1));
    double2* as = pw + G * (2 * P + 1);
    double2* part = as + G * (P + 1);
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c_begin + blockIdx.x * (blockDim.x >> 5) + wib; c < c_end; c += warps) {
        const int n2 = l.l2_n[c], n4 = l.l4_n[c];
        const int ns = n2 + n4;
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        double2 acc = make_double2(0.0, 0.0);
        for (int s0 = 0; s0 < ns; s0 += G) {
            const int si = s0 + g;
            const bool has = on && si < ns;
            int src = -1;
            if (has) src = si < n2 ? l.l2_src[(size_t)c * kList2Cap + si] : l.l4_src[(size_t)c * kList4Cap + (si - n2)];
            double2 w = make_double2(0.0, 0.0);
            if (has) w = cinv(make_double2(t.c_cx[src] - zx, t.c_cy[src] - zy));
            // w^p by binary powering, then w^(p+P) = w^p * w^P.
            double2 wp = make_double2(1.0, 0.0), base = w;
            for (int e = p; e > 0; e >>= 1) {
                if (e & 1) wp = cmul(wp, base);
                base = cmul(base, base);
            }
            const double2 wP = make_double2(__shfl_sync(0xffffffffu, wp.x, on ? g * P + P - 1 : lane),
                                            __shfl_sync(0xffffffffu, wp.y, on ? g * P + P - 1 : lane));
            if (has) {
                pw[g * (2 * P + 1) + p] = wp;
                pw[g * (2 * P + 1) + p + P] = cmul(wp, wP);
                as[g * (P + 1) + p] = a[(size_t)src * (P + 1) + p];
                if (p == 1) as[g * (P + 1)] = a[(size_t)src * (P + 1)];
            }
            __syncwarp();
            if (has) {
                const double2* A = as + g * (P + 1);
                const double2* Wg = pw + g * (2 * P + 1);
                double2 s = cscale(cmul(A[0], Wg[p]), 1.0 / (double)p);
                const double* cf = g_m2l + p * W;
                for (int k = 1; k <= P; ++k) s = cfma(cscale(A[k], cf[k]), Wg[p + k], s);
                acc = csub(acc, s);
            }
            __syncwarp();
        }
        if (on) part[g * (P + 1) + p] = acc;
        __syncwarp();
        if (lane < P) {
            double2 tot = make_double2(0.0, 0.0);
            for (int gg = 0; gg < G; ++gg) tot = cadd(tot, part[gg * (P + 1) + lane + 1]);
            b[(size_t)c * (P + 1) + lane + 1] = tot;
        }
        if (lane == 0) b[(size_t)c * (P + 1)] = make_double2(0.0, 0.0);
        __syncwarp();
    }
}

// M2L with precomputed list-2 operators. For a list-2 pair the source sits
// at the integer offset tau = (dx, dy) in {-3..3}^2 cell lengths r, and with
// scaled expansions a~_k = a_k / r^k, b~_p = r^p b_p the translation
//   b~_p = sum_{k=0..P} T_tau[p][k] a~_k,
//   T_tau[p][0] = -(1/p) tau^-p,  T_tau[p][k] = -m2l[p][k] tau^-(p+k)
// does not depend on the level (the same algebra as fmm2D.cpp:471-481). The
// 49 operators (stored [slot][k][p], p fastest) replace the per-pair powers.
// List-4 sources (coarser leaves, arbitrary offsets) use the direct formula.
// One warp per target cell, split into G = 32/P groups of P lanes.
__global__ void __launch_bounds__(128)
m2l2d_op(Tree2D t, Lists2D l, const double2* __restrict__ a, double2* __restrict__ b,
         const double2* __restrict__ op, const double* __restrict__ coef, int P, unsigned* err) {
    extern __shared__ double2 sm[];
    if (fatal(err)) return;
    const double* g_m2l = coef + kCoefM2L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int G = 32 / P;
    const int g = lane / P, p = lane % P + 1;
    const bool on = g < G;
    // per warp: as[G][P+1] (scaled sources), pw[G][2P+1] (list-4 powers), part[G][P+1]
    double2* as = sm + (size_t)wib * (G * (P + 1) * 2 + G * (2 * P + 1));
    double2* part = as + G * (P + 1);
    double2* pw = part + G * (P + 1);
    const double root = t.geom->root;
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c_begin + blockIdx.x * (blockDim.x >> 5) + wib; c < c_end; c += warps) {
        const int n2 = l.l2_n[c], n4 = l.l4_n[c];
        const double rinv = ldexp(1.0, (int)t.c_level[c]) / root;  // 1 / cell length
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        double2 acc_s = make_double2(0.0, 0.0);  // scaled (list 2)
        double2 acc = make_double2(0.0, 0.0);    // unscaled (list 4)
        // rinv^k for the lanes' k = p (and k = 0 handled by p == 1 lanes)
        double rk = 1.0;
        for (int e = 0; e < p; ++e) rk *= rinv;  // rinv^p
        for (int s0 = 0; s0 < n2; s0 += G) {
            const int si = s0 + g;
            const bool has = on && si < n2;
            int src = 0, slot = 0;
            if (has) {
                src = l.l2_src[(size_t)c * kList2Cap + si];
                slot = l.l2_slot[(size_t)c * kList2Cap + si];
                as[g * (P + 1) + p] = cscale(a[(size_t)src * (P + 1) + p], rk);
                if (p == 1) as[g * (P + 1)] = a[(size_t)src * (P + 1)];
            }
            __syncwarp();
            if (has) {
                const double2* A = as + g * (P + 1);
                const double2* T = op + (size_t)slot * (P + 1) * P + (p - 1);
                double2 sacc = acc_s;
                for (int k = 0; k <= P; ++k) sacc = cfma(T[(size_t)k * P], A[k], sacc);
                acc_s = sacc;
            }
            __syncwarp();
        }
        for (int s0 = 0; s0 < n4; s0 += G) {
            const int si = s0 + g;
            const bool has = on && si < n4;
            int src = 0;
            if (has) src = l.l4_src[(size_t)c * kList4Cap + si];
            double2 w = make_double2(0.0, 0.0);
            if (has) w = cinv(make_double2(t.c_cx[src] - zx, t.c_cy[src] - zy));
            double2 wp = make_double2(1.0, 0.0), base = w;
            for (int e = p; e > 0; e >>= 1) {
                if (e & 1) wp = cmul(wp, base);
                base = cmul(base, base);
            }
            const double2 wP = make_double2(__shfl_sync(0xffffffffu, wp.x, on ? g * P + P - 1 : lane),
                                            __shfl_sync(0xffffffffu, wp.y, on ? g * P + P - 1 : lane));
            double2* Wg = pw + g * (2 * P + 1);
            if (has) {
                Wg[p] = wp;
                Wg[p + P] = cmul(wp, wP);
                as[g * (P + 1) + p] = a[(size_t)src * (P + 1) + p];
                if (p == 1) as[g * (P + 1)] = a[(size_t)src * (P + 1)];
            }
            __syncwarp();
            if (has) {
                const double2* A = as + g * (P + 1);
                double2 sv = cscale(cmul(A[0], Wg[p]), 1.0 / (double)p);
                const double* cf = g_m2l + p * W;
                for (int k = 1; k <= P; ++k) sv = cfma(cscale(A[k], cf[k]), Wg[p + k], sv);
                acc = csub(acc, sv);
            }
            __syncwarp();
        }
        if (on) part[g * (P + 1) + p] = cadd(cscale(acc_s, rk), acc);
        __syncwarp();
        if (lane < P) {
            double2 tot = make_double2(0.0, 0.0);
            for (int gg = 0; gg < G; ++gg) tot = cadd(tot, part[gg * (P + 1) + lane + 1]);
            b[(size_t)c * (P + 1) + lane + 1] = tot;
        }
        if (lane == 0) b[(size_t)c * (P + 1)] = make_double2(0.0, 0.0);
        __syncwarp();
    }
}

// ---- leaf evaluation: M2P (list 3), L2P --------------------------------------

// Far field of targets i of a leaf, lane-owned: M2P over list 3
// (fmm2D.cpp:1040-1066) and L2P of the leaf's complete local expansion
// (fmm2D.cpp:1076-1093). With TWO, each lane takes a second target and both
// run through the list-3 sources together (one load of every source's
// coefficients serves both, and the two chains are independent). Each
// target's sums run in the same order either way. MODE kEvalFull does both;
// kEvalM2P writes the list-3 sums alone to fx/fy; kEvalL2P starts from those
// sums (the same value the full mode reaches after its list-3 loop) and adds
// L2P, so the split gives the same bits as one pass.
constexpr int kEvalFull = 0, kEvalM2P = 1, kEvalL2P = 2;
template <bool TWO, int MODE>
__device__ __forceinline__ void eval_targets(const Tree2D& t, const Lists2D& l, const double2* __restrict__ a,
                                             const double2* s_b, int P, int i0, int i1, bool h0, bool h1, double zx,
                                             double zy, const int32_t* src3, uint32_t n3, double* fx, double* fy,
                                             const double* nx, const double* ny, double* out0, double* out1,
                                             int velocity, double u_inf, double v_inf, unsigned* err) {
    double x[2], y[2], ex[2] = {0.0, 0.0}, ey[2] = {0.0, 0.0};
    bool h[2] = {h0, h1};
    const int ii[2] = {i0, i1};
    #pragma unroll
    for (int u = 0; u < (TWO ? 2 : 1); ++u) {
        x[u] = h[u] ? t.px[ii[u]] : zx + 1.0;
        y[u] = h[u] ? t.py[ii[u]] : zy;
    }
    if (MODE == kEvalL2P) {
        #pragma unroll
        for (int u = 0; u < (TWO ? 2 : 1); ++u)
            if (h[u]) {
                ex[u] = fx[ii[u]];
                ey[u] = fy[ii[u]];
            }
        n3 = 0;
    }
    for (uint32_t k = 0; k < n3; ++k) {
        const int s = src3[k];
        const double sx = t.c_cx[s], sy = t.c_cy[s];
        const double2* A = a + (size_t)s * (P + 1);
        double2 w[2], S[2];
        #pragma unroll
        for (int u = 0; u < (TWO ? 2 : 1); ++u) {
            w[u] = cinv(make_double2(x[u] - sx, y[u] - sy));
            S[u] = A[P];
        }
        for (int pp = P - 1; pp >= 0; --pp) {
            const double2 Ap = A[pp];
            #pragma unroll
            for (int u = 0; u < (TWO ? 2 : 1); ++u) S[u] = cfma(S[u], w[u], Ap);
        }
        #pragma unroll
        for (int u = 0; u < (TWO ? 2 : 1); ++u) {
            S[u] = cmul(S[u], w[u]);
            ex[u] += S[u].x;
            ey[u] -= S[u].y;
        }
    }
    if (MODE == kEvalM2P) {
        #pragma unroll
        for (int u = 0; u < (TWO ? 2 : 1); ++u)
            if (h[u]) {
                fx[ii[u]] = ex[u];
                fy[ii[u]] = ey[u];
            }
        return;
    }
    #pragma unroll
    for (int u = 0; u < (TWO ? 2 : 1); ++u) {
        const double2 w = make_double2(x[u] - zx, y[u] - zy);
        double2 S = cscale(s_b[P], (double)P);
        for (int pp = P - 1; pp >= 1; --pp) S = cfma(S, w, cscale(s_b[pp], (double)pp));
        double fxv = ex[u] + S.x, fyv = ey[u] - S.y;
        if (!h[u]) continue;
        const int i = ii[u];
        if (nx) {
            // near field already computed: write the total in the caller's order
            fxv = nx[i] + fxv;
            fyv = ny[i] + fyv;
            const uint32_t orig = t.perm[i];
            if (orig >= (uint32_t)t.n) {
                set_err(err, ERR_INDEX);
            } else if (velocity) {
                out0[orig] = fyv + u_inf;
                out1[orig] = -fxv + v_inf;
            } else {
                out0[orig] = fxv;
                out1[orig] = fyv;
            }
        } else {
            fx[i] = fxv;
            fy[i] = fyv;
        }
    }
}

constexpr int kEvalWarps = 4;   // one warp per leaf
constexpr int kEvalThreads = 32 * kEvalWarps;

// Far field of every particle of a leaf (eval_targets), one warp per leaf,
// 64 targets per pass (two per lane). Cells above level 2 carry no local
// expansion (M2L starts at level 2).
template <int MODE>
__global__ void __launch_bounds__(kEvalThreads)
eval2d(Tree2D t, Lists2D l, const double2* __restrict__ a, const double2* __restrict__ b, double* __restrict__ fx,
       double* __restrict__ fy, int P, const double* __restrict__ nx, const double* __restrict__ ny,
       double* __restrict__ out0, double* __restrict__ out1, int velocity, double u_inf, double v_inf, int lists,
       unsigned* err) {
    __shared__ double2 s_bw[kEvalWarps][W];
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double2* s_b = s_bw[wib];
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x * kEvalWarps + wib; li < nl; li += gridDim.x * kEvalWarps) {
        const int c = t.leaf_cells[li];
        const int L = t.c_level[c];
        if (MODE != kEvalM2P)
            for (int k = lane; k <= P; k += 32)
                s_b[k] = L >= 2 ? b[(size_t)c * (P + 1) + k] : make_double2(0.0, 0.0);
        __syncwarp();
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        // list 3 of the leaf: the CSR, or (M2P) the fixed slots of
        // int_list_slots, the leaves whose list outgrew them coming in a
        // second pass from the CSR
        const int32_t* src3 = nullptr;
        uint32_t n3 = 0;
        if (MODE != kEvalL2P) {
            bool csr = lists == kP2PListCsr;
            if (!csr) {
                const uint32_t cnt = l.l3_cnt[li];
                const bool spill = cnt > (uint32_t)kListSlot3;
                if (spill != (lists == kP2PListSpill)) continue;   // the other pass takes this leaf
                csr = spill;
                if (!spill) {
                    src3 = l.l3_slot + (size_t)li * kListSlot3;
                    n3 = cnt;
                }
            }
            if (csr) {
                const uint32_t o3 = l.l3_off[li];
                src3 = l.l3_src + o3;
                n3 = l.l3_off[li + 1] - o3;
            }
        }
        for (int i0 = lo; i0 < hi; i0 += 64) {
            const int ia = i0 + lane, ib = i0 + 32 + lane;
            if (i0 + 32 < hi)   // warp-uniform
                eval_targets<true, MODE>(t, l, a, s_b, P, ia, ib, ia < hi, ib < hi, zx, zy, src3, n3, fx, fy, nx, ny,
                                         out0, out1, velocity, u_inf, v_inf, err);
            else
                eval_targets<false, MODE>(t, l, a, s_b, P, ia, ib, ia < hi, false, zx, zy, src3, n3, fx, fy, nx, ny,
                                          out0, out1, velocity, u_inf, v_inf, err);
        }
        __syncwarp();
    }
}

// ---- P2P over list 1 --------------------------------------------------------

constexpr int kP2PThreads = 128;

// Writes one target's total field (near + far) in the caller's order; with
// fx == nullptr (near field computed concurrently with the far field) the
// near field alone, in tree order, into out0/out1.
__device__ __forceinline__ void p2p_store(const Tree2D& t, int ti, double ex, double ey, const double* fx,
                                          const double* fy, double* out0, double* out1, int velocity, double u_inf,
                                          double v_inf, unsigned* err) {
    if (!fx) {
        out0[ti] = ex;
        out1[ti] = ey;
        return;
    }
    ex += fx[ti];
    ey += fy[ti];
    const uint32_t orig = t.perm[ti];
    if (orig >= (uint32_t)t.n) {
        set_err(err, ERR_INDEX);
    } else if (velocity) {
        out0[orig] = ey + u_inf;
        out1[orig] = -ex + v_inf;
    } else {
        out0[orig] = ex;
        out1[orig] = ey;
    }
}

// One block per leaf (grid-stride). With H = ceil(T/2), thread (t, split)
// owns targets t and t + H and the sources split, split + ns, ... of every
// list-1 cell (ns = 128 / H), so each source load serves two targets. Sources
// come straight from global memory (L1-resident, nearly warp-uniform
// addresses); the j == i exclusion is only tested inside the target's own
// leaf. Partial sums are combined in a fixed order.
__global__ void __launch_bounds__(kP2PThreads)
p2p2d(Tree2D t, Lists2D l, const double* __restrict__ fx, const double* __restrict__ fy, double* __restrict__ out0,
      double* __restrict__ out1, int velocity, double u_inf, double v_inf, unsigned* err) {
    __shared__ double s_px[2][kP2PThreads], s_py[2][kP2PThreads];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    const double* __restrict__ px = t.px;
    const double* __restrict__ py = t.py;
    const double* __restrict__ pq = t.pq;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        for (int tb = lo; tb < hi; tb += 2 * kP2PThreads) {
            const int T = min(2 * kP2PThreads, hi - tb);
            const int H = (T + 1) >> 1;
            const int ns = kP2PThreads / H;
            const int tt = threadIdx.x % H, split = threadIdx.x / H;
            const bool on = split < ns;
            const int ta = tb + tt, tbb = tb + tt + H;
            const bool hasb = tt + H < T;
            const double xa = px[ta], ya = py[ta];
            const double xb = hasb ? px[tbb] : xa, yb = hasb ? py[tbb] : ya;
            double exa = 0.0, eya = 0.0, exb = 0.0, eyb = 0.0;
            if (on) {
                for (uint32_t k = o1; k < e1; ++k) {
                    const int sc = l.l1_src[k];
                    const int s_hi = t.c_hi[sc];
                    if (sc != c) {
                        for (int j = t.c_lo[sc] + split; j < s_hi; j += ns) {
                            const double sx = __ldg(px + j), sy = __ldg(py + j), sq = __ldg(pq + j);
                            const double dxa = xa - sx, dya = ya - sy, dxb = xb - sx, dyb = yb - sy;
                            const double fa = sq * rcp_nr(fma(dxa, dxa, dya * dya));
                            const double fb = sq * rcp_nr(fma(dxb, dxb, dyb * dyb));
                            exa = fma(fa, dxa, exa);
                            eya = fma(fa, dya, eya);
                            exb = fma(fb, dxb, exb);
                            eyb = fma(fb, dyb, eyb);
                        }
                    } else {
                        for (int j = t.c_lo[sc] + split; j < s_hi; j += ns) {
                            const double sx = __ldg(px + j), sy = __ldg(py + j), sq = __ldg(pq + j);
                            const double dxa = xa - sx, dya = ya - sy, dxb = xb - sx, dyb = yb - sy;
                            const double fa = (j == ta) ? 0.0 : sq * rcp_nr(fma(dxa, dxa, dya * dya));
                            const double fb = (j == tbb) ? 0.0 : sq * rcp_nr(fma(dxb, dxb, dyb * dyb));
                            exa = fma(fa, dxa, exa);
                            eya = fma(fa, dya, eya);
                            exb = fma(fb, dxb, exb);
                            eyb = fma(fb, dyb, eyb);
                        }
                    }
                }
            }
            if (on && split > 0) {
                s_px[0][threadIdx.x] = exa; s_py[0][threadIdx.x] = eya;
                s_px[1][threadIdx.x] = exb; s_py[1][threadIdx.x] = eyb;
            }
            __syncthreads();
            if (split == 0) {
                for (int s = 1; s < ns; ++s) {
                    exa += s_px[0][s * H + tt]; eya += s_py[0][s * H + tt];
                    exb += s_px[1][s * H + tt]; eyb += s_py[1][s * H + tt];
                }
                p2p_store(t, ta, exa, eya, fx, fy, out0, out1, velocity, u_inf, v_inf, err);
                if (hasb) p2p_store(t, tbb, exb, eyb, fx, fy, out0, out1, velocity, u_inf, v_inf, err);
            }
            __syncthreads();
        }
    }
}

// ---- mixed form: FP32 near field ---------------------------------------------

// FP32 reciprocal (hardware approximation, ~1 ulp) of the mixed near field.
__device__ __forceinline__ float rcp_approx(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}


// ---- TMA-staged P2P (bulk copies into shared memory) ------------------------------

constexpr int kStageCells = 64;  // list-1 cells of one leaf held in the stage descriptor

struct StageCell {
    int start, end;  // staged slots [start, end)
    float ox, oy;    // c_src - c_tgt (FP64 difference rounded once)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait on the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// One bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, size a multiple of 16 (float4 elements).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Per-precision pieces of the TMA-staged P2P.
struct P2PF64 {
    using Elem = double4;  // (x, y, q, -) in FP64, absolute coordinates
    using Acc = double;
    static __device__ __forceinline__ void shift(Elem&, float, float) {}
    static __device__ __forceinline__ double inv(double r2) { return rcp_nr(r2); }
    static constexpr int kWarps = 4;
    static constexpr int kMinBlocks = 5;   // <= 102 registers
};

// Stage the list-1 sources of leaf `li` into `buf` with one bulk copy per
// source cell (one thread). Returns the staged slot count, or -1 when the
// leaf does not fit (the barrier is still armed, with zero bytes, so its
// phase completes); cells[k] receives each cell's slot range and its centre
// offset relative to the target leaf (FP64 difference rounded once).
template <class Elem>
__device__ int stage_leaf(const Tree2D& t, const Lists2D& l, const Elem* src, int li, Elem* buf, int cap,
                          StageCell* cells, uint64_t* bar) {
    const int c = t.leaf_cells[li];
    const double ccx = t.c_cx[c], ccy = t.c_cy[c];
    const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
    int total = 0;
    bool fits = (int)(e1 - o1) <= kStageCells;
    if (fits) {
        for (uint32_t k = o1; k < e1; ++k) {
            const int sc = l.l1_src[k];
            total += t.c_hi[sc] - t.c_lo[sc];
        }
        fits = total <= cap;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, fits ? (unsigned)(total * sizeof(Elem)) : 0u);
    if (!fits) return -1;
    int pos = 0, kk = 0;
    for (uint32_t k = o1; k < e1; ++k, ++kk) {
        const int sc = l.l1_src[k];
        const int lo = t.c_lo[sc], hi = t.c_hi[sc];
        cells[kk].start = pos;
        cells[kk].end = pos + (hi - lo);
        cells[kk].ox = (float)(t.c_cx[sc] - ccx);
        cells[kk].oy = (float)(t.c_cy[sc] - ccy);
        bulk_g2s(buf + pos, src + lo, (unsigned)((hi - lo) * sizeof(Elem)), bar);
        pos += hi - lo;
    }
    return total;
}

constexpr int kTPT = 4;  // targets per thread in the TMA P2P

// Pair loop of one thread over source slots [j0, j1) (step ns) for kTPT
// targets; slot self[k] is excluded for target k (-1: none). FP32 sums are
// flushed into the FP64 accumulators every 64 sources.
template <class Tr>
__device__ __forceinline__ void pair_loop4(const typename Tr::Elem* __restrict__ buf, int j0, int j1, int ns,
                                           const double* tx, const double* ty, const int* self, double* ex,
                                           double* ey) {
    using A = typename Tr::Acc;
    A x[kTPT], y[kTPT];
    #pragma unroll
    for (int k = 0; k < kTPT; ++k) { x[k] = (A)tx[k]; y[k] = (A)ty[k]; }
    const bool has_self = self[0] >= 0 || self[1] >= 0 || self[2] >= 0 || self[3] >= 0;
    for (int jb = j0; jb < j1; jb += 64 * ns) {
        const int je = min(j1, jb + 64 * ns);
        A px[kTPT], py[kTPT];
        #pragma unroll
        for (int k = 0; k < kTPT; ++k) { px[k] = 0; py[k] = 0; }
        if (!has_self) {
            // the next source is loaded while this one is computed
            typename Tr::Elem nv = jb < je ? buf[jb] : typename Tr::Elem{};
            for (int j = jb; j < je; j += ns) {
                const typename Tr::Elem sv = nv;
                if (j + ns < je) nv = buf[j + ns];
                const A sx = (A)sv.x, sy = (A)sv.y, sq = (A)sv.z;
                #pragma unroll
                for (int k = 0; k < kTPT; ++k) {
                    const A dx = x[k] - sx, dy = y[k] - sy;
                    const A f = sq * Tr::inv(dx * dx + dy * dy);
                    px[k] += f * dx;
                    py[k] += f * dy;
                }
            }
        } else {
            for (int j = jb; j < je; j += ns) {
                const typename Tr::Elem sv = buf[j];
                const A sx = (A)sv.x, sy = (A)sv.y, sq = (A)sv.z;
                #pragma unroll
                for (int k = 0; k < kTPT; ++k) {
                    const A dx = x[k] - sx, dy = y[k] - sy;
                    A f = sq * Tr::inv(dx * dx + dy * dy);
                    if (j == self[k]) f = 0;
                    px[k] += f * dx;
                    py[k] += f * dy;
                }
            }
        }
        #pragma unroll
        for (int k = 0; k < kTPT; ++k) { ex[k] += (double)px[k]; ey[k] += (double)py[k]; }
    }
}

// TMA-staged P2P. Each block walks its leaves (grid-stride) with two stage
// buffers: while the block computes leaf i from one buffer, thread 0 has bulk
// copies of leaf i+1's list-1 sources in flight into the other (one mbarrier
// per buffer, bounded waits). After a stage lands the block adds each source
// cell's centre offset (FP32 form: sources then share the target leaf's
// frame), so the pair loop is one flat loop over the staged slots. Thread
// (t, split) owns targets t and t + H (H = ceil(T/2)) and slots split,
// split + ns, ... A leaf whose sources do not fit is computed from global
// memory cell by cell.
template <class Tr>
__global__ void __launch_bounds__(kP2PThreads)
p2p2d_tma(Tree2D t, Lists2D l, const typename Tr::Elem* __restrict__ src, const double* __restrict__ fx,
          const double* __restrict__ fy, double* __restrict__ out0, double* __restrict__ out1, int velocity,
          double u_inf, double v_inf, int cap, unsigned* err) {
    using Elem = typename Tr::Elem;
    extern __shared__ __align__(16) unsigned char p2p_sm[];
    Elem* bufs = (Elem*)p2p_sm;                                        // [2][cap]
    StageCell* scells = (StageCell*)(bufs + 2 * (size_t)cap);          // [2][kStageCells]
    uint64_t* bars = (uint64_t*)(scells + 2 * kStageCells);            // [2]
    int* s_count = (int*)(bars + 2);                                   // [2]
    __shared__ double s_px[kTPT][kP2PThreads], s_py[kTPT][kP2PThreads];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    if ((int)blockIdx.x >= nl) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_count[0] = stage_leaf<Elem>(t, l, src, blockIdx.x, bufs, cap, scells, &bars[0]);
    }
    __syncthreads();
    int iter = 0;
    for (int li = blockIdx.x; li < nl; li += gridDim.x, ++iter) {
        const int b = iter & 1;
        const int nxt = li + gridDim.x;
        if (threadIdx.x == 0 && nxt < nl)
            s_count[b ^ 1] = stage_leaf<Elem>(t, l, src, nxt, bufs + (size_t)(b ^ 1) * cap, cap,
                                              scells + (b ^ 1) * kStageCells, &bars[b ^ 1]);
        const bool ok = mbar_wait(&bars[b], (iter >> 1) & 1);
        if (!ok) set_err(err, ERR_TIMEOUT);
        const int staged = s_count[b];
        Elem* buf = bufs + (size_t)b * cap;
        const StageCell* cells = scells + b * kStageCells;
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double ccx = t.c_cx[c], ccy = t.c_cy[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        const int ncell = (int)(e1 - o1);
        // Own-leaf slot range, and the frame shift of the staged sources.
        int own0 = -1;
        if (staged >= 0 && ok) {
            for (int kk = 0; kk < ncell; ++kk) {
                const StageCell ci = cells[kk];
                if (l.l1_src[o1 + kk] == c) own0 = ci.start;
                for (int j = ci.start + threadIdx.x; j < ci.end; j += blockDim.x) Tr::shift(buf[j], ci.ox, ci.oy);
            }
        }
        __syncthreads();
        for (int tb = lo; tb < hi; tb += kTPT * kP2PThreads) {
            const int T = min(kTPT * kP2PThreads, hi - tb);
            const int H = (T + kTPT - 1) / kTPT;
            const int ns = kP2PThreads / H;
            const int tt = threadIdx.x % H, split = threadIdx.x / H;
            const bool on = split < ns && ok;
            int ti[kTPT];
            double tx[kTPT], ty[kTPT], ex[kTPT], ey[kTPT];
            #pragma unroll
            for (int k = 0; k < kTPT; ++k) {
                const int off = tt + k * H;
                ti[k] = off < T ? tb + off : -1;
                const Elem g = src[ti[k] >= 0 ? ti[k] : tb + tt];
                tx[k] = g.x;
                ty[k] = g.y;
                ex[k] = 0.0;
                ey[k] = 0.0;
            }
            if (on) {
                if (staged >= 0) {
                    int self[kTPT];
                    #pragma unroll
                    for (int k = 0; k < kTPT; ++k) self[k] = (own0 >= 0 && ti[k] >= 0) ? own0 + (ti[k] - lo) : -1;
                    // Slots of the own leaf need the j == i test; the others do not.
                    if (own0 >= 0) {
                        const int own1 = own0 + (hi - lo);
                        const int none[kTPT] = {-1, -1, -1, -1};
                        pair_loop4<Tr>(buf, split, own0, ns, tx, ty, none, ex, ey);
                        const int j0 = own0 + ((split - own0) % ns + ns) % ns;
                        pair_loop4<Tr>(buf, j0, own1, ns, tx, ty, self, ex, ey);
                        const int j2 = own1 + ((split - own1) % ns + ns) % ns;
                        pair_loop4<Tr>(buf, j2, staged, ns, tx, ty, none, ex, ey);
                    } else {
                        pair_loop4<Tr>(buf, split, staged, ns, tx, ty, self, ex, ey);
                    }
                } else {
                    for (int kk = 0; kk < ncell; ++kk) {
                        const int sc = l.l1_src[o1 + kk];
                        const int slo = t.c_lo[sc], shi = t.c_hi[sc];
                        double sx = 0.0, sy = 0.0;
                        if (sizeof(Elem) == sizeof(float4)) {
                            sx = (double)(float)(t.c_cx[sc] - ccx);
                            sy = (double)(float)(t.c_cy[sc] - ccy);
                        }
                        double tx2[kTPT], ty2[kTPT];
                        int self[kTPT];
                        #pragma unroll
                        for (int k = 0; k < kTPT; ++k) {
                            tx2[k] = tx[k] - sx;
                            ty2[k] = ty[k] - sy;
                            self[k] = (sc == c) ? ti[k] : -1;
                        }
                        pair_loop4<Tr>(src, slo + split, shi, ns, tx2, ty2, self, ex, ey);
                    }
                }
            }
            if (on && split > 0) {
                #pragma unroll
                for (int k = 0; k < kTPT; ++k) { s_px[k][threadIdx.x] = ex[k]; s_py[k][threadIdx.x] = ey[k]; }
            }
            __syncthreads();
            if (split == 0 && ok) {
                for (int s2 = 1; s2 < ns; ++s2) {
                    #pragma unroll
                    for (int k = 0; k < kTPT; ++k) { ex[k] += s_px[k][s2 * H + tt]; ey[k] += s_py[k][s2 * H + tt]; }
                }
                #pragma unroll
                for (int k = 0; k < kTPT; ++k)
                    if (ti[k] >= 0) p2p_store(t, ti[k], ex[k], ey[k], fx, fy, out0, out1, velocity, u_inf, v_inf, err);
            }
            __syncthreads();
        }
    }
    // Copies are only issued for leaves this block then waits on; after a
    // timed-out wait, wait once more (bounded) so no copy lands in freed
    // shared memory.
    if (threadIdx.x == 0 && iter > 0) {
        const int last = iter - 1;
        (void)mbar_wait(&bars[last & 1], (last >> 1) & 1);
    }
}

// Warp-per-leaf P2P (the plain FP64 form's near field). Each warp owns one
// leaf at a time (grid-stride over leaves), so no block-wide barrier sits in
// the loop.
// With H = ceil(T/4) lanes per split, lane (t, split) owns targets t, t+H,
// t+2H, t+3H and the sources split, split + ns, ... (ns = 32/H) of every
// list-1 cell, read straight from global memory (nearly warp-uniform
// addresses, L1-resident). Split partials are summed in a fixed order through
// a per-warp shared-memory tile.
constexpr int kP2PMeta = 64;   // list-1 cells staged per leaf (longer lists read them directly)

template <class Tr>
__global__ void __launch_bounds__(32 * Tr::kWarps, Tr::kMinBlocks)
p2p2d_warp(Tree2D t, Lists2D l, const typename Tr::Elem* __restrict__ src, const double* __restrict__ fx,
           const double* __restrict__ fy, double* __restrict__ out0, double* __restrict__ out1, int velocity,
           double u_inf, double v_inf, unsigned* err) {
    using Elem = typename Tr::Elem;
    __shared__ double s_red[Tr::kWarps][2 * kTPT][32];
    // list-1 cells of the warp's leaf: first/last slot, FP32-rounded centre
    // offset, loaded by the whole warp at once (one round of latency)
    __shared__ int4 s_meta[Tr::kWarps][kP2PMeta];
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nl = t.info->n_leaves;
    const bool rel = sizeof(Elem) == sizeof(float4);
    for (int li = blockIdx.x * Tr::kWarps + wib; li < nl; li += gridDim.x * Tr::kWarps) {
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double ccx = t.c_cx[c], ccy = t.c_cy[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        const int n1 = (int)(e1 - o1);
        const bool meta = n1 <= kP2PMeta;
        if (meta) {
            for (int k = lane; k < n1; k += 32) {
                const int sc = l.l1_src[o1 + k];
                float ox = 0.f, oy = 0.f;
                if (rel) {
                    ox = (float)(t.c_cx[sc] - ccx);
                    oy = (float)(t.c_cy[sc] - ccy);
                }
                s_meta[wib][k] = make_int4(t.c_lo[sc], sc == c ? -t.c_hi[sc] - 1 : t.c_hi[sc], __float_as_int(ox),
                                           __float_as_int(oy));
            }
            __syncwarp();
        }
        for (int tb = lo; tb < hi; tb += kTPT * 32) {
            const int T = min(kTPT * 32, hi - tb);
            const int H = (T + kTPT - 1) / kTPT;
            const int ns = 32 / H;
            const int tt = lane % H, split = lane / H;
            const bool on = split < ns;
            int ti[kTPT];
            double tx[kTPT], ty[kTPT], ex[kTPT], ey[kTPT];
            #pragma unroll
            for (int k = 0; k < kTPT; ++k) {
                const int off = tt + k * H;
                ti[k] = off < T ? tb + off : -1;
                const Elem g = src[ti[k] >= 0 ? ti[k] : tb];
                tx[k] = g.x;
                ty[k] = g.y;
                ex[k] = 0.0;
                ey[k] = 0.0;
            }
            if (on) {
                for (uint32_t kk = o1; kk < e1; ++kk) {
                    int slo, shi;
                    bool own;
                    double sx = 0.0, sy = 0.0;
                    if (meta) {
                        const int4 m = s_meta[wib][kk - o1];
                        slo = m.x;
                        own = m.y < 0;
                        shi = own ? -m.y - 1 : m.y;
                        sx = (double)__int_as_float(m.z);
                        sy = (double)__int_as_float(m.w);
                    } else {
                        const int sc = l.l1_src[kk];
                        slo = t.c_lo[sc];
                        shi = t.c_hi[sc];
                        own = sc == c;
                        if (rel) {
                            sx = (double)(float)(t.c_cx[sc] - ccx);
                            sy = (double)(float)(t.c_cy[sc] - ccy);
                        }
                    }
                    double tx2[kTPT], ty2[kTPT];
                    int self[kTPT];
                    #pragma unroll
                    for (int k = 0; k < kTPT; ++k) {
                        tx2[k] = tx[k] - sx;
                        ty2[k] = ty[k] - sy;
                        self[k] = own ? ti[k] : -1;
                    }
                    pair_loop4<Tr>(src, slo + split, shi, ns, tx2, ty2, self, ex, ey);
                }
            }
            // sum the splits of each target: lanes tt, tt + H, ... hold its parts
            #pragma unroll
            for (int k = 0; k < kTPT; ++k) {
                s_red[wib][2 * k][lane] = on ? ex[k] : 0.0;
                s_red[wib][2 * k + 1][lane] = on ? ey[k] : 0.0;
            }
            __syncwarp();
            if (split == 0) {
                #pragma unroll
                for (int k = 0; k < kTPT; ++k) {
                    double sx2 = 0.0, sy2 = 0.0;
                    for (int s2 = 0; s2 < ns; ++s2) {
                        sx2 += s_red[wib][2 * k][s2 * H + tt];
                        sy2 += s_red[wib][2 * k + 1][s2 * H + tt];
                    }
                    if (ti[k] >= 0) p2p_store(t, ti[k], sx2, sy2, fx, fy, out0, out1, velocity, u_inf, v_inf, err);
                }
            }
            __syncwarp();
        }
    }
}

// Warp-per-leaf FP32 near field (the mixed form's default). A chunk of
// T <= 192 targets of the warp's leaf is spread over H lanes (the smallest
// power of two with M = ceil(T/H) <= 12 targets per lane), so all 32 lanes
// are busy and at most H - 1 target slots idle. The leaf's list-1 cells form
// one flat sequence of sources; every step the warp stages the next
// kTileStage of them in shared memory (loads issued a step ahead, moved into
// the target leaf's frame: scaled by the exact power of two between the two
// leaves' sizes plus the FP32 cell offset; stored with x, y and q duplicated
// so that they feed packed FP32x2 instructions directly), and
// lane group ("split") s of the ns = 32/H groups applies staged sources
// s, s + ns, ... to its M targets. Every kTileFlush sources the per-lane FP32
// sums are reduced over the splits with shuffles into FP64 accumulators in
// shared memory (target k is kept by split k mod ns); the sums are in units
// of the leaf size and are scaled back on the store.
//
// i == j needs no test: r^2 is formed as dx dx + dy dy + kTileEps, and a
// particle of the leaf meets itself at dx = dy = 0 exactly (the own cell's
// offset is zero, its scale one), so q / kTileEps multiplies zero offsets.
// In leaf units, the smallest non-zero FP32 offset squared is about 1e-15,
// so kTileEps changes no other pair, and q / kTileEps stays finite for
// |q| < 3e14.
constexpr int kTileWarps = 8;
constexpr int kTileFlush = 128;
constexpr int kTileMaxM = 6;
constexpr int kTileChunk = 16 * kTileMaxM;      // targets per chunk (H <= 16, so ns >= 2)
constexpr int kTileSlots = kTileMaxM / 2;       // FP64 target slots per lane (ns >= 2)
constexpr int kTileStage = 64;                  // sources staged per step (two per lane)
constexpr float kTileEps = 1e-24f;

struct TileShared {
    float4 xy[kTileWarps][kTileStage];             // (x, x, y, y) of the staged sources
    float2 qq[kTileWarps][kTileStage];             // (q, q)
    int2 meta[kTileWarps][kP2PMeta];               // (lo, size) per list-1 cell
    int cs[kTileWarps][kP2PMeta + 1];              // flat start of each cell, then the total
    double acc[kTileWarps][2 * kTileSlots][32];    // FP64 accumulators: row 2i x, 2i+1 y of slot i
};

// Two targets (packed: low half the first) against one source, on the
// packed FP32x2 instructions: d = -t + s, r2 = d.d + eps, f = q rcp(r2),
// p += f d.
__device__ __forceinline__ void tile_pair2(uint64_t nx, uint64_t ny, uint64_t sx, uint64_t sy, uint64_t sq,
                                           uint64_t eps, uint64_t& px, uint64_t& py) {
    asm("{\n\t"
        ".reg .b64 dx, dy, r2, rr, fq;\n\t"
        ".reg .f32 a, b;\n\t"
        "add.rn.f32x2 dx, %2, %4;\n\t"
        "add.rn.f32x2 dy, %3, %5;\n\t"
        "fma.rn.f32x2 r2, dx, dx, %7;\n\t"
        "fma.rn.f32x2 r2, dy, dy, r2;\n\t"
        "mov.b64 {a, b}, r2;\n\t"
        "rcp.approx.ftz.f32 a, a;\n\t"
        "rcp.approx.ftz.f32 b, b;\n\t"
        "mov.b64 rr, {a, b};\n\t"
        "mul.rn.f32x2 fq, %6, rr;\n\t"
        "fma.rn.f32x2 %0, fq, dx, %0;\n\t"
        "fma.rn.f32x2 %1, fq, dy, %1;\n\t"
        "}"
        : "+l"(px), "+l"(py)
        : "l"(nx), "l"(ny), "l"(sx), "l"(sy), "l"(sq), "l"(eps));
}

__device__ __forceinline__ uint64_t pack2(float lo, float hi) {
    return ((uint64_t)__float_as_uint(hi) << 32) | (uint64_t)__float_as_uint(lo);
}
__device__ __forceinline__ float lo2(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float hi2(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }

// Staged sources split, split + NS, ... below cnt applied to the lane's M
// targets: a loop with constant bounds and strides (NS = 32 >> HS), so no
// index arithmetic is left between the pair updates.
template <int M, int HS>
__device__ __forceinline__ void tile_pairs(const ulonglong2* xy, const uint64_t* qq, int split, int cnt,
                                           const uint64_t* nx, const uint64_t* ny, float nxo, float nyo, uint64_t* px,
                                           uint64_t* py, float& pxo, float& pyo) {
    constexpr int MP = M / 2, NS = 32 >> HS, PER = kTileStage / NS;
    constexpr bool ODD = (M & 1) != 0;
    const uint64_t eps = pack2(kTileEps, kTileEps);
    const ulonglong2* xs = xy + split;
    const uint64_t* qs = qq + split;
    const int nrun = (cnt - split + NS - 1) / NS;   // sources of this split in the stage
    #pragma unroll
    for (int u = 0; u < PER; ++u) {
        if (u >= nrun) break;
        const ulonglong2 sv = xs[u * NS];   // (x, x), (y, y)
        const uint64_t sq = qs[u * NS];     // (q, q)
        #pragma unroll
        for (int h = 0; h < MP; ++h) tile_pair2(nx[h], ny[h], sv.x, sv.y, sq, eps, px[h], py[h]);
        if (ODD) {
            const float dx = nxo + lo2(sv.x), dy = nyo + lo2(sv.y);
            const float fq = lo2(sq) * rcp_approx(fmaf(dy, dy, fmaf(dx, dx, kTileEps)));
            pxo = fmaf(fq, dx, pxo);
            pyo = fmaf(fq, dy, pyo);
        }
    }
}

// Coordinate of a particle in the target leaf's frame, in units of its size:
// formed in FP64 and rounded once (a particle of the leaf gets the same value
// as a target and as a source).
__device__ __forceinline__ float leaf_unit(double x, double c, double ih) { return (float)((x - c) * ih); }

template <int M, int HS>
__device__ __forceinline__ void tile_chunk(TileShared& sm, const Tree2D& t, const int32_t* __restrict__ src1, int c,
                                           double ccx, double ccy, double ih, int n1, int tb, int T,
                                           const double* fx, const double* fy, double* out0, double* out1,
                                           int velocity, double u_inf, double v_inf, unsigned* err) {
    constexpr int MP = M / 2;
    constexpr int NP = MP > 0 ? MP : 1;
    constexpr int hs = HS, H = 1 << HS, ns = 32 >> HS;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int tt = lane & (H - 1), split = lane >> hs;
    // negated target coordinates (leaf frame); target k of this lane is chunk slot tt + k H
    uint64_t nx[NP], ny[NP], px[NP], py[NP];
    float nxo = 0.f, nyo = 0.f, pxo = 0.f, pyo = 0.f;
    #pragma unroll
    for (int h = 0; h < MP; ++h) {
        const int i0 = tt + ((2 * h) << hs), i1 = tt + ((2 * h + 1) << hs);
        const int j0 = tb + (i0 < T ? i0 : 0), j1 = tb + (i1 < T ? i1 : 0);
        nx[h] = pack2(-leaf_unit(t.px[j0], ccx, ih), -leaf_unit(t.px[j1], ccx, ih));
        ny[h] = pack2(-leaf_unit(t.py[j0], ccy, ih), -leaf_unit(t.py[j1], ccy, ih));
        px[h] = py[h] = 0ull;
    }
    if (M & 1) {
        const int i0 = tt + ((M - 1) << hs);
        const int j0 = tb + (i0 < T ? i0 : 0);
        nxo = -leaf_unit(t.px[j0], ccx, ih);
        nyo = -leaf_unit(t.py[j0], ccy, ih);
    }
    double* acc = &sm.acc[wib][0][lane];
    #pragma unroll
    for (int i = 0; i < 2 * kTileSlots; ++i) acc[32 * i] = 0.0;
    // reduce the FP32 partials over the splits into the FP64 slots
    auto flush = [&]() {
        #pragma unroll
        for (int k = 0; k < M; ++k) {
            float vx = (k < 2 * MP) ? ((k & 1) ? hi2(px[k >> 1]) : lo2(px[k >> 1])) : pxo;
            float vy = (k < 2 * MP) ? ((k & 1) ? hi2(py[k >> 1]) : lo2(py[k >> 1])) : pyo;
            for (int o = H; o < 32; o <<= 1) {
                vx += __shfl_xor_sync(0xffffffffu, vx, o);
                vy += __shfl_xor_sync(0xffffffffu, vy, o);
            }
            if ((k & (ns - 1)) == split) {
                const int slot = k >> (5 - hs);
                acc[32 * (2 * slot)] -= (double)vx;
                acc[32 * (2 * slot + 1)] -= (double)vy;
            }
        }
        #pragma unroll
        for (int h = 0; h < MP; ++h) px[h] = py[h] = 0ull;
        pxo = pyo = 0.f;
    };
    int steps = 0;   // staged sources since the last flush (each lane applied steps / ns of them)
    for (int seg = 0; seg < n1; seg += kP2PMeta) {
        const int nseg = min(kP2PMeta, n1 - seg);
        __syncwarp();
        // metadata and flat prefix of the segment
        {
            int sz[2] = {0, 0};
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = lane + 32 * h;
                if (k < nseg) {
                    const int sc = src1[seg + k];
                    const int slo = t.c_lo[sc];
                    sz[h] = t.c_hi[sc] - slo;
                    sm.meta[wib][k] = make_int2(slo, sz[h]);
                }
            }
            int inc0 = sz[0], inc1 = sz[1];
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int a0 = __shfl_up_sync(0xffffffffu, inc0, o), a1 = __shfl_up_sync(0xffffffffu, inc1, o);
                if (lane >= o) {
                    inc0 += a0;
                    inc1 += a1;
                }
            }
            const int tot0 = __shfl_sync(0xffffffffu, inc0, 31);
            const int tot1 = __shfl_sync(0xffffffffu, inc1, 31);
            if (lane < nseg) sm.cs[wib][lane] = inc0 - sz[0];
            if (lane + 32 < nseg) sm.cs[wib][lane + 32] = tot0 + inc1 - sz[1];
            if (lane == 0) sm.cs[wib][nseg] = tot0 + tot1;
        }
        __syncwarp();
        const int total = sm.cs[wib][nseg];
        // per-lane walkers over the flat sequence: the lane stages flat sources
        // cb + lane and cb + 32 + lane of step cb
        int k0 = 0, q0 = lane, k1 = 0, q1 = lane + 32;
        while (k0 < nseg && q0 >= sm.meta[wib][k0].y) {
            q0 -= sm.meta[wib][k0].y;
            ++k0;
        }
        while (k1 < nseg && q1 >= sm.meta[wib][k1].y) {
            q1 -= sm.meta[wib][k1].y;
            ++k1;
        }
        auto fetch = [&](int k, int o) -> float4 {
            if (k >= nseg) return make_float4(0.f, 0.f, 0.f, 0.f);
            const int j = sm.meta[wib][k].x + o;
            return make_float4(leaf_unit(t.px[j], ccx, ih), leaf_unit(t.py[j], ccy, ih), (float)t.pq[j], 0.f);
        };
        auto advance = [&](int& k, int& o) {
            o += kTileStage;
            while (k < nseg && o >= sm.meta[wib][k].y) {
                o -= sm.meta[wib][k].y;
                ++k;
            }
        };
        float4 pv0 = fetch(k0, q0), pv1 = fetch(k1, q1);
        for (int cb = 0; cb < total; cb += kTileStage) {
            sm.xy[wib][lane] = make_float4(pv0.x, pv0.x, pv0.y, pv0.y);
            sm.qq[wib][lane] = make_float2(pv0.z, pv0.z);
            sm.xy[wib][lane + 32] = make_float4(pv1.x, pv1.x, pv1.y, pv1.y);
            sm.qq[wib][lane + 32] = make_float2(pv1.z, pv1.z);
            __syncwarp();
            advance(k0, q0);
            advance(k1, q1);
            pv0 = fetch(k0, q0);
            pv1 = fetch(k1, q1);
            tile_pairs<M, HS>(reinterpret_cast<const ulonglong2*>(sm.xy[wib]),
                              reinterpret_cast<const uint64_t*>(sm.qq[wib]), split, min(kTileStage, total - cb), nx,
                              ny, nxo, nyo, px, py, pxo, pyo);
            __syncwarp();
            steps += kTileStage;
            if (steps >= kTileFlush * ns) {
                flush();
                steps = 0;
            }
        }
    }
    flush();
    __syncwarp();
    #pragma unroll
    for (int i = 0; i < kTileSlots; ++i) {
        const int kk = split + (i << (5 - hs));
        const int ti = tt + (kk << hs);
        if (kk < M && ti < T)
            p2p_store(t, tb + ti, acc[32 * (2 * i)] * ih, acc[32 * (2 * i + 1)] * ih, fx, fy, out0, out1, velocity, u_inf,
                      v_inf, err);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kTileWarps, 3)
p2p2d_tile_f32(Tree2D t, Lists2D l, const double* __restrict__ fx,
               const double* __restrict__ fy, double* __restrict__ out0, double* __restrict__ out1, int velocity,
               double u_inf, double v_inf, int lists, unsigned* err) {
    __shared__ TileShared sm;
    if (fatal(err)) return;
    const int wib = threadIdx.x >> 5;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x * kTileWarps + wib; li < nl; li += gridDim.x * kTileWarps) {
        // list 1 of the leaf: CSR, or the fixed slots of int_list_slots (the
        // leaves whose list outgrew them come in a second pass, from the CSR)
        const int32_t* src1;
        int n1;
        if (lists == kP2PListCsr) {
            src1 = l.l1_src + l.l1_off[li];
            n1 = (int)(l.l1_off[li + 1] - l.l1_off[li]);
        } else {
            const uint32_t cnt = l.l1_cnt[li];
            const bool spill = cnt > (uint32_t)kListSlot1;
            if (spill != (lists == kP2PListSpill)) continue;
            src1 = spill ? l.l1_src + l.l1_off[li] : l.l1_slot + (size_t)li * kListSlot1;
            n1 = spill ? (int)(l.l1_off[li + 1] - l.l1_off[li]) : (int)cnt;
        }
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double ccx = t.c_cx[c], ccy = t.c_cy[c];
        const int lev = t.c_level[c];
        const double ih = ldexp(1.0, lev) / t.geom->root;   // 1 / leaf size
        for (int tb = lo; tb < hi; tb += kTileChunk) {
            const int T = min(kTileChunk, hi - tb);
            int hs = 0;   // the smallest H = 2^hs with ceil(T / H) <= kTileMaxM (H <= 16)
            while (((T + (1 << hs) - 1) >> hs) > kTileMaxM) ++hs;
            const int M = (T + (1 << hs) - 1) >> hs;
            switch ((hs << 4) | M) {
#define VPM_TILE_CASE(HH, MM)                                                                                       \
    case (HH << 4) | MM:                                                                                            \
        tile_chunk<MM, HH>(sm, t, src1, c, ccx, ccy, ih, n1, tb, T, fx, fy, out0, out1, velocity, u_inf, v_inf, err); \
        break;
#define VPM_TILE_ROW(HH) VPM_TILE_CASE(HH, 1) VPM_TILE_CASE(HH, 2) VPM_TILE_CASE(HH, 3) VPM_TILE_CASE(HH, 4)         \
    VPM_TILE_CASE(HH, 5) VPM_TILE_CASE(HH, 6)
                VPM_TILE_ROW(0) VPM_TILE_ROW(1) VPM_TILE_ROW(2) VPM_TILE_ROW(3) VPM_TILE_ROW(4)
#undef VPM_TILE_ROW
#undef VPM_TILE_CASE
                default: break;
            }
        }
    }
}

// AoS (x, y, q) copy of the sorted particles for the FP64 TMA P2P (bulk
// copies need 16-byte aligned ranges).
__global__ void particles_aos(Tree2D t, double4* __restrict__ aos, unsigned* err) {
    if (fatal(err)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.n; i += gridDim.x * blockDim.x)
        aos[i] = make_double4(t.px[i], t.py[i], t.pq[i], 0.0);
}

template <class Tr>
cudaError_t launch_p2p_tma(const Tree2D& t, const Lists2D& l, const typename Tr::Elem* src, const Expansions2D& e,
                           double* out0, double* out1, int velocity, double u_inf, double v_inf, unsigned* err,
                           cudaStream_t st, int max_par) {
    // Room for twelve full leaves: the nine neighbours at the leaf's level plus finer ones.
    const int cap = std::min(4096, std::max(512, 12 * max_par));
    const size_t smem = 2 * (size_t)cap * sizeof(typename Tr::Elem) + 2 * kStageCells * sizeof(StageCell) + 64;
    static size_t smem_set = 0;
    if (smem > smem_set) {
        cudaError_t r = cudaFuncSetAttribute(p2p2d_tma<Tr>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        smem_set = smem;
    }
    p2p2d_tma<Tr><<<148 * 8, kP2PThreads, smem, st>>>(t, l, src, e.fx, e.fy, out0, out1, velocity, u_inf, v_inf, cap,
                                                      err);
    return cudaGetLastError();
}

}  // namespace

cudaError_t set_coefficients2d(int P, bool exact, double* dst, cudaStream_t st) {
    std::vector<double> tab(3 * W * W, 0.0);
    double* m2m = tab.data() + kCoefM2M;
    double* m2l = tab.data() + kCoefM2L;
    double* l2l = tab.data() + kCoefL2L;
    for (int p = 0; p <= P; ++p) {
        for (int k = 1; k <= p; ++k) m2m[p * W + k] = (double)binom_host(p - 1, k - 1, exact) * ((double)p / (double)k);
        for (int k = 1; k <= P; ++k)
            m2l[p * W + k] = (double)binom_host(p + k - 1, k - 1, exact) * ((k & 1) ? -1.0 : 1.0) / (double)k;
        for (int k = p; k <= P; ++k) l2l[p * W + k] = (double)binom_host(k, p, exact);
    }
    cudaError_t e = cudaMemcpyAsync(dst, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    // The host vectors go out of scope: wait for the copies.
    return cudaStreamSynchronize(st);
}

// ---- upward pass in two launches ----------------------------------------------
//
// The multipole of any cell is a_k = sum of q_j (z_j - z_c)^k over the active
// particles of its subtree (P2M at a leaf, fmm2D.cpp:237-284), and M2M
// (fmm2D.cpp:309-379) shifts the children's moments with the binomial
// coefficients C(p, k) = C(p-1, k-1) p / k, which gives the same moments
// whenever those coefficients are exact (orders up to 18 with the reference's
// 32-bit binComb, any order with exact binomials). Every cell covers a
// contiguous range of the sorted particles, so a cell of at most kDirectMax
// particles takes its moments straight from that range (upward_direct2d: one
// warp per cell, all levels at once, no ordering between cells). The larger
// cells (the top of the tree, about n / kDirectMax per level) follow by M2M
// from their children in the cooperative level loop m2m_big_levels_coop,
// from the deepest level holding one. Sums run in a fixed order (lane order
// over the particles, then lanes in order; children in child order). A large
// cell without active particles gets zero moments from the first launch, so
// every cell's moments are written in every evaluation.
constexpr int kUpWarps = 8;
constexpr int kDirectMax = 1024;
constexpr int kUpMaxP = 18;

template <int P>
__global__ void __launch_bounds__(32 * kUpWarps)
upward_direct2d(Tree2D t, double2* __restrict__ a, unsigned* __restrict__ top_level, unsigned* err) {
    constexpr int Q = P + 1, CS = 2 * Q + 1;   // components per lane, padded row stride
    extern __shared__ double up_sm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* red = up_sm + (size_t)wib * 32 * CS;   // [lane][component]
    if (fatal(err)) return;
    const int c_begin = t.info->level_start[1], c_end = t.info->n_cells;
    const int nw = gridDim.x * kUpWarps;
    for (int c = c_begin + blockIdx.x * kUpWarps + wib; c < c_end; c += nw) {
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const uint8_t f = t.c_flags[c];
        if (hi - lo > kDirectMax && !(f & CELL_LEAF)) {
            if (f & CELL_ACTIVE) {   // by M2M afterwards (m2m_big_levels_coop)
                if (lane == 0) atomicMax(top_level, (unsigned)t.c_level[c]);
            } else {                 // no active particle: zero moments (its parent's M2M reads them)
                for (int comp = lane; comp < 2 * Q; comp += 32) reinterpret_cast<double*>(a + (size_t)c * Q)[comp] = 0.0;
            }
            continue;
        }
        double re[Q], im[Q];
        #pragma unroll
        for (int k = 0; k < Q; ++k) re[k] = im[k] = 0.0;
        if (f & CELL_ACTIVE) {
            const double zx = t.c_cx[c], zy = t.c_cy[c];
            for (int j = lo + lane; j < hi; j += 32) {
                if (!t.pact[j]) continue;
                const double wx = t.px[j] - zx, wy = t.py[j] - zy;
                double pr = t.pq[j], pi = 0.0;
                re[0] += pr;
                #pragma unroll
                for (int k = 1; k < Q; ++k) {
                    const double nr = pr * wx - pi * wy, ni = pr * wy + pi * wx;
                    pr = nr;
                    pi = ni;
                    re[k] += pr;
                    im[k] += pi;
                }
            }
        }
        #pragma unroll
        for (int k = 0; k < Q; ++k) {
            red[lane * CS + 2 * k] = re[k];
            red[lane * CS + 2 * k + 1] = im[k];
        }
        __syncwarp();
        for (int comp = lane; comp < 2 * Q; comp += 32) {
            double sum = 0.0;
            for (int l = 0; l < 32; ++l) sum += red[l * CS + comp];
            reinterpret_cast<double*>(a + (size_t)c * Q)[comp] = sum;
        }
        __syncwarp();
    }
}

bool upward_direct_ok(int P, bool exact) { return P >= 1 && P <= kUpMaxP && (exact || P <= 18); }
static_assert(kUpMaxP <= 18, "the reference's 32-bit M2M binomials wrap from order 19");

template <int P>
cudaError_t launch_upward_direct(const Tree2D& t, Expansions2D& e, unsigned* err, cudaStream_t st, cudaEvent_t mid) {
    const size_t smem = sizeof(double) * kUpWarps * 32 * (2 * (P + 1) + 1);
    cudaError_t r = cudaFuncSetAttribute(upward_direct2d<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    upward_direct2d<P><<<148 * 4, 32 * kUpWarps, smem, st>>>(t, e.a, t.gbar + 3, err);
    if (mid) {
        r = cudaEventRecord(mid, st);
        if (r != cudaSuccess) return r;
    }
    // A small grid: the large cells are a few hundred per level, and the
    // blocks of this loop wait at its barriers most of the time while the
    // near field runs beside it on the other streams, so every block it does
    // not hold is SM room for that (16 blocks: mixed step 0.442 -> 0.430 ms
    // at 778k against one block per SM).
    int grid = 0;
    r = launch_coop_max(m2m_big_levels_coop, 32 * kLevelWarps, 0, st, 1, std::max(16, t.n >> 16), &grid, t, e.a,
                        (const double*)e.coef, P, kDirectMax, (const unsigned*)(t.gbar + 3), t.gbar + 2, err);
    return r != cudaSuccess ? r : cudaGetLastError();
}

// Upward pass of orders the direct form covers (upward_direct_ok): one launch.
// Otherwise the P2M + M2M level loop below.
cudaError_t fmm2d_upward_direct(const Tree2D& t, Expansions2D& e, int P, bool exact, unsigned* err, cudaStream_t st,
                                int* launches, cudaEvent_t mid) {
    // the level loop over all cells: every moment is final only at its end
    auto full = [&]() -> cudaError_t {
        cudaError_t r = fmm2d_upward(t, e, P, err, st, launches);
        if (r == cudaSuccess && mid) r = cudaEventRecord(mid, st);
        return r;
    };
    if (!upward_direct_ok(P, exact) || !t.gbar) return full();
    cudaError_t r;
    switch (P) {
#define VPM_UP_CASE(PP) \
    case PP: r = launch_upward_direct<PP>(t, e, err, st, mid); break;
        VPM_UP_CASE(1) VPM_UP_CASE(2) VPM_UP_CASE(3) VPM_UP_CASE(4) VPM_UP_CASE(5) VPM_UP_CASE(6)
        VPM_UP_CASE(7) VPM_UP_CASE(8) VPM_UP_CASE(9) VPM_UP_CASE(10) VPM_UP_CASE(11) VPM_UP_CASE(12)
        VPM_UP_CASE(13) VPM_UP_CASE(14) VPM_UP_CASE(15) VPM_UP_CASE(16) VPM_UP_CASE(17) VPM_UP_CASE(18)
#undef VPM_UP_CASE
        default: return full();
    }
    if (r != cudaSuccess) {   // cooperative launch refused: the level loop over all cells instead
        (void)cudaGetLastError();
        return full();
    }
    *launches += 2;
    return r;
}

// Upward pass: P2M of every active leaf, then M2M level by level from the
// deepest possible level up to level 1 (levels below the tree's depth exit
// at once; the launch count does not depend on the data, so the sequence can
// be captured in a CUDA graph).
cudaError_t fmm2d_upward(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches) {
    cudaError_t r = cudaMemsetAsync(e.a, 0, sizeof(double2) * (size_t)t.cap_cells * (P + 1), st);
    if (r != cudaSuccess) return r;
    const size_t smem = sizeof(double2) * kP2MWarps * (P + 1) * kAccPad;
    p2m2d<<<148 * 16, 32 * kP2MWarps, smem, st>>>(t, e.a, P, err);
    *launches += 1;
    if (t.gbar) {
        int grid = 0;
        r = launch_coop(m2m_levels_coop, 32 * kLevelWarps, 0, st, 1, &grid, t, e.a, (const double*)e.coef, P,
                        t.gbar + 2, err);
        if (r == cudaSuccess) {
            *launches += 1;
            return cudaGetLastError();
        }
        (void)cudaGetLastError();  // cooperative launch refused: one launch per level instead
    }
    for (int L = t.key_levels - 1; L >= 1; --L) {
        m2m_level2d<<<148 * 4, 128, 0, st>>>(t, e.a, e.coef, P, L, err);
        *launches += 1;
    }
    return cudaGetLastError();
}

// List-2 operators T_tau (see m2l2d_op) for the 49 offset slots, from the
// same M2L coefficients as the direct formula (so the reference's binomials
// carry over). Upload synchronises `st`.
cudaError_t set_m2l_operators2d(int P, bool exact, double2* dst, cudaStream_t st) {
    std::vector<double2> op((size_t)49 * (P + 1) * P);
    for (int slot = 0; slot < 49; ++slot) {
        const int dx = slot % 7 - 3, dy = slot / 7 - 3;
        std::complex<double> tau(dx, dy), inv = (dx == 0 && dy == 0) ? 0.0 : 1.0 / tau;
        std::vector<std::complex<double>> ip(2 * P + 2);
        ip[0] = 1.0;
        for (int m = 1; m <= 2 * P; ++m) ip[m] = ip[m - 1] * inv;
        for (int p = 1; p <= P; ++p) {
            for (int k = 0; k <= P; ++k) {
                std::complex<double> v;
                if (k == 0) v = -(1.0 / (double)p) * ip[p];
                else v = -((double)binom_host(p + k - 1, k - 1, exact) * ((k & 1) ? -1.0 : 1.0) / (double)k) * ip[p + k];
                op[((size_t)slot * (P + 1) + k) * P + (p - 1)] = make_double2(v.real(), v.imag());
            }
        }
    }
    cudaError_t e = cudaMemcpyAsync(dst, op.data(), sizeof(double2) * op.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t fmm2d_m2l_only(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err,
                           cudaStream_t st, int* launches) {
    const int G = 32 / P;
    if (e.op) {
        const size_t smem = sizeof(double2) * 4 * (size_t)(2 * G * (P + 1) + G * (2 * P + 1));
        m2l2d_op<<<148 * 16, 128, smem, st>>>(t, l, e.a, e.b, e.op, e.coef, P, err);
    } else {
        const size_t smem = sizeof(double2) * 4 * (size_t)(G * (2 * P + 1) + 2 * G * (P + 1));
        m2l2d<<<148 * 16, 128, smem, st>>>(t, l, e.a, e.b, e.coef, P, err);
    }
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_l2l(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches) {
    if (t.gbar) {
        int grid = 0;
        cudaError_t r = launch_coop(l2l_levels_coop, 32 * kLevelWarps, 0, st, 1, &grid, t, e.b,
                                    (const double*)e.coef, P, t.gbar + 4, err);
        if (r == cudaSuccess) {
            *launches += 1;
            return cudaGetLastError();
        }
        (void)cudaGetLastError();  // cooperative launch refused: one launch per level instead
    }
    for (int L = 3; L <= t.key_levels; ++L) {
        l2l_level2d<<<148 * 4, 128, 0, st>>>(t, e.b, e.coef, P, L, err);
        *launches += 1;
    }
    return cudaGetLastError();
}

// Full local expansion of every leaf straight from the M2L parts of its
// ancestors: b(leaf) = b_M2L(leaf) + sum over ancestors a at levels 2..L-1 of
// the L2L shift of b_M2L(a) by z_leaf - z_a. Shifts of a degree-P polynomial
// compose exactly (shift by t1 then t2 = shift by t1 + t2) when the binomials
// C(k, p) are exact, which the reference's 32-bit binComb gives for k <= 17;
// the result then equals the level-by-level pull of fmm2D.cpp:587-651 up to
// rounding, without a level loop or grid barrier. G = 32/(P+1) leaves per
// warp, lane k of group g holds coefficient k of leaf g. Ancestors come from
// the dense grid (written for every cell of levels <= dense_levels by the
// tree build, so an ancestor's entry is always current) and the parent chain
// below it; their centres and coefficients are staged in shared memory in
// chunks of kL2LChunk levels.
constexpr int kL2LChunk = 4;
constexpr int kL2LWarps = 4;
constexpr int kL2LGroups = 16;   // leaves per warp at most (P >= 1)

__global__ void __launch_bounds__(32 * kL2LWarps)
l2l_leaves2d(Tree2D t, double2* __restrict__ b, const double* __restrict__ coef, int P) {
    __shared__ int s_anc[kL2LWarps][kL2LGroups][kMaxLevels2D + 1];  // [warp][group][level]
    __shared__ int s_lev[kL2LWarps][kL2LGroups];                    // leaf level per group
    __shared__ double2 s_ctr[kL2LWarps][kL2LGroups][kL2LChunk];     // ancestor centres
    __shared__ double2 s_cf[kL2LWarps][kL2LChunk * 32];             // chunk coefficients, all groups
    const double* g_l2l = coef + kCoefL2L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int Q = P + 1, G = 32 / Q, g = lane / Q, k = lane - g * Q;
    const bool in_grp = g < G;
    const int nl = t.info->n_leaves, nc = t.info->n_cells;
    const int dlev = t.dense ? t.dense_levels : 1;
    const int warps = gridDim.x * kL2LWarps;
    for (int lb = (blockIdx.x * kL2LWarps + wib) * G; lb < nl; lb += warps * G) {
        const int li = lb + g;
        const bool has = in_grp && li < nl;
        const int c = has ? t.leaf_cells[li] : 0;
        const int L = has ? (int)t.c_level[c] : 0;
        const int na = L > 2 ? L - 2 : 0;   // ancestors at levels 2..L-1
        int ix = 0, iy = 0;
        double zx = 0.0, zy = 0.0;
        double2 acc = make_double2(0.0, 0.0);
        if (in_grp && k == 0) s_lev[wib][g] = L;
        if (na) {
            ix = t.c_ix[c];
            iy = t.c_iy[c];
            zx = t.c_cx[c];
            zy = t.c_cy[c];
            acc = b[(size_t)c * Q + k];
            // dense-grid ancestors, one level per lane of the group
            for (int m = 2 + k; m < L && m <= dlev; m += Q) {
                const int sh = L - m;
                const int a = t.dense[start_id2(m) + (ix >> sh) + ((int64_t)(iy >> sh) << m)];
                s_anc[wib][g][m] = (a >= 0 && a < nc) ? a : -1;
            }
            // deeper ancestors by the parent chain
            if (k == 0) {
                int a = t.c_parent[c];
                for (int m = L - 1; m > dlev && m >= 2; --m) {
                    s_anc[wib][g][m] = a;
                    a = t.c_parent[a];
                }
            }
        }
        __syncwarp();
        const int na_max = __reduce_max_sync(0xffffffffu, na);
        for (int m0 = 0; m0 < na_max; m0 += kL2LChunk) {
            const int mc = min(kL2LChunk, na_max - m0);
            // stage: centres (one ancestor per lane of the group), then coefficients of all groups
            if (k < mc && 2 + m0 + k < L) {
                const int a = s_anc[wib][g][2 + m0 + k];
                s_ctr[wib][g][k] = a >= 0 ? make_double2(t.c_cx[a], t.c_cy[a]) : make_double2(zx, zy);
            }
            for (int j = lane; j < G * mc * Q; j += 32) {
                const int gj = j / (mc * Q), r = j - gj * (mc * Q), mj = r / Q, kj = r - mj * Q;
                double2 v = make_double2(0.0, 0.0);
                if (2 + m0 + mj < s_lev[wib][gj]) {
                    const int a = s_anc[wib][gj][2 + m0 + mj];
                    if (a >= 0) v = b[(size_t)a * Q + kj];
                }
                s_cf[wib][(gj * kL2LChunk + mj) * Q + kj] = v;
            }
            __syncwarp();
            if (has) {
                const double* cf = g_l2l + k * W;
                for (int mj = 0; mj < mc && m0 + mj < na; ++mj) {
                    const double2 ctr = s_ctr[wib][g][mj];
                    const double2 tt = make_double2(zx - ctr.x, zy - ctr.y);
                    const double2* par = &s_cf[wib][(g * kL2LChunk + mj) * Q];
                    double2 S = cscale(par[P], cf[P]);
                    for (int kk = P - 1; kk >= k; --kk) S = cfma(S, tt, cscale(par[kk], cf[kk]));
                    acc = cadd(acc, S);
                }
            }
            __syncwarp();
        }
        if (na) b[(size_t)c * Q + k] = acc;
    }
}

bool l2l_direct_ok(int P, bool exact) { return P >= 1 && (exact || P <= 17); }

cudaError_t fmm2d_l2l_leaves(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches) {
    (void)err;
    l2l_leaves2d<<<148 * 8, 32 * kL2LWarps, 0, st>>>(t, e.b, e.coef, P);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_m2l(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches) {
    cudaError_t r = fmm2d_m2l_only(t, l, e, P, err, st, launches);
    if (r != cudaSuccess) return r;
    return fmm2d_l2l(t, e, P, err, st, launches);
}

cudaError_t fmm2d_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                       int* launches) {
    eval2d<kEvalFull><<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, P, nullptr, nullptr, nullptr,
                                                         nullptr, 0, 0.0, 0.0, kP2PListCsr, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_m2p(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches, int lists) {
    eval2d<kEvalM2P><<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, P, nullptr, nullptr, nullptr,
                                                        nullptr, 0, 0.0, 0.0, lists, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_eval_combine(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, const double* nx,
                               const double* ny, double* out0, double* out1, int velocity, double u_inf, double v_inf,
                               unsigned* err, cudaStream_t st, int* launches, bool m2p_done) {
    if (m2p_done)
        eval2d<kEvalL2P><<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, P, nx, ny, out0, out1, velocity,
                                                            u_inf, v_inf, kP2PListCsr, err);
    else
        eval2d<kEvalFull><<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, P, nx, ny, out0, out1,
                                                             velocity, u_inf, v_inf, kP2PListCsr, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p_out(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* out0, double* out1,
                          int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st, int* launches) {
    p2p2d<<<148 * 16, kP2PThreads, 0, st>>>(t, l, e.fx, e.fy, out0, out1, velocity, u_inf, v_inf, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p_f32(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* out0, double* out1,
                          int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st, int* launches,
                          bool near_only, int lists) {
    Expansions2D en = e;
    if (near_only) en.fx = en.fy = nullptr;
    // Many short blocks (a leaf or a few per warp) rather than one persistent
    // wave: blocks retire all through the launch, so the far-field kernels
    // running concurrently on the other streams get SM room as they queue.
    // the pass over the few leaves whose list 1 outgrew its slots: one wave
    const int grid = lists == kP2PListSpill ? 148 : 148 * 3 * 8;
    p2p2d_tile_f32<<<grid, 32 * kTileWarps, 0, st>>>(t, l, en.fx, en.fy, out0, out1, velocity, u_inf, v_inf, lists,
                                                    err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p_f64_tma(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double4* aos, double* out0,
                              double* out1, int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st,
                              int* launches, int max_par, bool near_only) {
    particles_aos<<<148 * 8, 256, 0, st>>>(t, aos, err);
    *launches += 2;
    Expansions2D en = e;
    if (near_only) en.fx = en.fy = nullptr;
    if (max_par < 0) return launch_p2p_tma<P2PF64>(t, l, aos, en, out0, out1, velocity, u_inf, v_inf, err, st, -max_par);
    p2p2d_warp<P2PF64><<<148 * 64 / P2PF64::kWarps, 32 * P2PF64::kWarps, 0, st>>>(
        t, l, aos, en.fx, en.fy, out0, out1, velocity, u_inf, v_inf, err);
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* ex, double* ey,
                      unsigned* err, cudaStream_t st, int* launches) {
    return fmm2d_p2p_out(t, l, e, ex, ey, 0, 0.0, 0.0, err, st, launches);
}

}  // namespace vpm
