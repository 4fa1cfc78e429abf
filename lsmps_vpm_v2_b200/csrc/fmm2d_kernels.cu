// FP64 (plain form) translation and evaluation kernels of the 2D Laurent FMM
// (reference src/FMM/fmm2D.cpp). Expansions are complex: multipole
//   a_k = sum_j q_j (z_j - z_c)^k                      (P2M, fmm2D.cpp:237-284)
// and local coefficients b_p, with the field at z taken as
//   E_x = Re F, E_y = -Im F,  F = sum of q/(z - z_j) terms.
//
// Stage map:
//   fmm2d_upward  P2M of every active leaf fused with M2M (fmm2D.cpp:309-379):
//                 the last child to finish computes its parent, so the whole
//                 upward pass is one launch.
//   fmm2d_m2l     lists 2 and 4 of every cell at level >= 2 (fmm2D.cpp:396-556).
//   fmm2d_eval    per leaf: the L2L chain from its level-2 ancestor
//                 (fmm2D.cpp:587-651), then M2P over list 3 (fmm2D.cpp:1040-1066)
//                 and L2P (fmm2D.cpp:1076-1093) for its particles.
//   fmm2d_p2p     per leaf: direct sum over list 1, j != i (fmm2D.cpp:135-179),
//                 added to the far field and written in the caller's order.
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

// Newton-Raphson reciprocal: hardware seed refined twice by y <- y + y(1 - a y).
__device__ __forceinline__ double rcp_nr(double a) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double e = fma(-a, y, 1.0);
    y = fma(y, e, y);
    e = fma(-a, y, 1.0);
    y = fma(y, e, y);
    return y;
}

__device__ __forceinline__ double2 ldcg2(const double2* p) { return __ldcg(p); }

__device__ __forceinline__ double2 warp_sum2(double2 v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
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

// M2M into the active non-leaf cells of level L (fmm2D.cpp:309-379), one warp
// per cell, lane p computing a_p by Horner's rule in t = z_child - z_parent:
//   a_p += a0 t^p + sum_{k=1..p} m2m[p][k] a_k t^(p-k).
__global__ void __launch_bounds__(128)
m2m_level2d(Tree2D t, double2* __restrict__ a, const double* __restrict__ coef, int P, int L, unsigned* err) {
    __shared__ double2 s_child[4][W];
    if (fatal(err)) return;
    const double* g_m2m = coef + kCoefM2M;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int c0 = t.info->level_start[L], c1 = t.info->level_start[L + 1];
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c0 + blockIdx.x * (blockDim.x >> 5) + wib; c < c1; c += warps) {
        const uint8_t f = t.c_flags[c];
        if ((f & CELL_LEAF) || !(f & CELL_ACTIVE)) continue;
        const double px = t.c_cx[c], py = t.c_cy[c];
        const unsigned m = t.c_chmask[c];
        const int ch0 = t.c_child0[c];
        if (ch0 < 0) continue;
        double2 acc = make_double2(0.0, 0.0);
        for (int r = 0; r < __popc(m); ++r) {
            const int ch = ch0 + r;
            if (lane <= P) s_child[wib][lane] = a[(size_t)ch * (P + 1) + lane];
            __syncwarp();
            const double2 tt = make_double2(t.c_cx[ch] - px, t.c_cy[ch] - py);
            if (lane == 0) {
                acc = cadd(acc, s_child[wib][0]);
            } else if (lane <= P) {
                const int p = lane;
                double2 S = s_child[wib][0];
                for (int j = p - 1; j >= 0; --j) {
                    const int k = p - j;
                    S = cfma(S, tt, cscale(s_child[wib][k], g_m2m[p * W + k]));
                }
                acc = cadd(acc, S);
            }
            __syncwarp();
        }
        if (lane <= P) a[(size_t)c * (P + 1) + lane] = acc;
    }
}

// L2L pull into every cell of level L >= 3 from its parent (fmm2D.cpp:587-651,
// where each non-leaf parent at levels 2..max-1 pushes into its children):
//   b_p(c) += sum_{k=p..P} l2l[p][k] b_k(parent) t^(k-p),  t = z_c - z_parent.
// The parent's expansion is final because level L-1 ran in the previous launch.
__global__ void __launch_bounds__(128)
l2l_level2d(Tree2D t, double2* __restrict__ b, const double* __restrict__ coef, int P, int L, unsigned* err) {
    __shared__ double2 s_par[4][W];
    if (fatal(err)) return;
    const double* g_l2l = coef + kCoefL2L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int c0 = t.info->level_start[L], c1 = t.info->level_start[L + 1];
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c0 + blockIdx.x * (blockDim.x >> 5) + wib; c < c1; c += warps) {
        const int par = t.c_parent[c];
        if (lane <= P) s_par[wib][lane] = b[(size_t)par * (P + 1) + lane];
        __syncwarp();
        if (lane <= P) {
            const double2 tt = make_double2(t.c_cx[c] - t.c_cx[par], t.c_cy[c] - t.c_cy[par]);
            const int pp = lane;
            const double* cf = g_l2l + pp * W;
            double2 S = cscale(s_par[wib][P], cf[P]);
            for (int kk = P - 1; kk >= pp; --kk) S = cfma(S, tt, cscale(s_par[wib][kk], cf[kk]));
            double2* bc = &b[(size_t)c * (P + 1) + pp];
            *bc = cadd(*bc, S);
        }
        __syncwarp();
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

constexpr int kEvalThreads = 64;

// Far field of every particle of a leaf: M2P over list 3 (fmm2D.cpp:1040-1066)
// and L2P of the leaf's complete local expansion (fmm2D.cpp:1076-1093). Cells
// above level 2 carry no local expansion (M2L starts at level 2).
__global__ void __launch_bounds__(kEvalThreads)
eval2d(Tree2D t, Lists2D l, const double2* __restrict__ a, const double2* __restrict__ b, double* __restrict__ fx,
       double* __restrict__ fy, int P, unsigned* err) {
    __shared__ double2 s_b[W];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int L = t.c_level[c];
        if (threadIdx.x <= P)
            s_b[threadIdx.x] = L >= 2 ? b[(size_t)c * (P + 1) + threadIdx.x] : make_double2(0.0, 0.0);
        __syncthreads();
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        const uint32_t o3 = l.l3_off[li], e3 = l.l3_off[li + 1];
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double x = t.px[i], y = t.py[i];
            double ex = 0.0, ey = 0.0;
            for (uint32_t k = o3; k < e3; ++k) {
                const int s = l.l3_src[k];
                const double2 w = cinv(make_double2(x - t.c_cx[s], y - t.c_cy[s]));
                const double2* A = a + (size_t)s * (P + 1);
                double2 S = A[P];
                for (int pp = P - 1; pp >= 0; --pp) S = cfma(S, w, A[pp]);
                S = cmul(S, w);
                ex += S.x;
                ey -= S.y;
            }
            const double2 w = make_double2(x - zx, y - zy);
            double2 S = cscale(s_b[P], (double)P);
            for (int pp = P - 1; pp >= 1; --pp) S = cfma(S, w, cscale(s_b[pp], (double)pp));
            ex += S.x;
            ey -= S.y;
            fx[i] = ex;
            fy[i] = ey;
        }
        __syncthreads();
    }
}

// ---- P2P over list 1 --------------------------------------------------------

constexpr int kP2PThreads = 128;

// One block per leaf (grid-stride). Thread (t, split) owns target t and the
// sources split, split + ns, ... of every list-1 cell; sources are read from
// global memory (L1-resident, nearly warp-uniform addresses), so the pair
// loop has no barrier. The partial sums of a target's splits are combined in
// a fixed order at the end.
__global__ void __launch_bounds__(kP2PThreads)
p2p2d(Tree2D t, Lists2D l, const double* __restrict__ fx, const double* __restrict__ fy, double* __restrict__ out0,
      double* __restrict__ out1, int velocity, double u_inf, double v_inf, unsigned* err) {
    __shared__ double s_px[kP2PThreads], s_py[kP2PThreads];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    const double* __restrict__ px = t.px;
    const double* __restrict__ py = t.py;
    const double* __restrict__ pq = t.pq;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        for (int tb = lo; tb < hi; tb += kP2PThreads) {
            const int T = min(kP2PThreads, hi - tb);
            const int ns = kP2PThreads / T;
            const int tt = threadIdx.x % T, split = threadIdx.x / T;
            const bool on = split < ns;
            const int ti = tb + tt;
            const double xt = px[ti], yt = py[ti];
            double ex0 = 0.0, ey0 = 0.0, ex1 = 0.0, ey1 = 0.0;
            if (on) {
                for (uint32_t k = o1; k < e1; ++k) {
                    const int sc = l.l1_src[k];
                    const int s_hi = t.c_hi[sc];
                    int j = t.c_lo[sc] + split;
                    for (; j + ns < s_hi; j += 2 * ns) {
                        const int j1 = j + ns;
                        const double dx0 = xt - __ldg(px + j), dy0 = yt - __ldg(py + j);
                        const double dx1 = xt - __ldg(px + j1), dy1 = yt - __ldg(py + j1);
                        const double r0 = fma(dx0, dx0, dy0 * dy0), r1 = fma(dx1, dx1, dy1 * dy1);
                        const double f0 = (j == ti) ? 0.0 : __ldg(pq + j) * rcp_nr(r0);
                        const double f1 = (j1 == ti) ? 0.0 : __ldg(pq + j1) * rcp_nr(r1);
                        ex0 = fma(f0, dx0, ex0);
                        ey0 = fma(f0, dy0, ey0);
                        ex1 = fma(f1, dx1, ex1);
                        ey1 = fma(f1, dy1, ey1);
                    }
                    if (j < s_hi) {
                        const double dx0 = xt - __ldg(px + j), dy0 = yt - __ldg(py + j);
                        const double r0 = fma(dx0, dx0, dy0 * dy0);
                        const double f0 = (j == ti) ? 0.0 : __ldg(pq + j) * rcp_nr(r0);
                        ex0 = fma(f0, dx0, ex0);
                        ey0 = fma(f0, dy0, ey0);
                    }
                }
            }
            double ex = ex0 + ex1, ey = ey0 + ey1;
            if (on && split > 0) { s_px[threadIdx.x] = ex; s_py[threadIdx.x] = ey; }
            __syncthreads();
            if (split == 0) {
                for (int s = 1; s < ns; ++s) { ex += s_px[s * T + tt]; ey += s_py[s * T + tt]; }
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
            __syncthreads();
        }
    }
}

// ---- mixed form: FP32 near field ---------------------------------------------

// Leaf-relative FP32 coordinates and FP32 strengths: x - c_leaf is formed in
// FP64 (exact enough: |x - c| <= cell size) and rounded once.
__global__ void leaf_relative_f32(Tree2D t, float4* __restrict__ rel, unsigned* err) {
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const double cx = t.c_cx[c], cy = t.c_cy[c];
        for (int i = t.c_lo[c] + threadIdx.x; i < t.c_hi[c]; i += blockDim.x)
            rel[i] = make_float4((float)(t.px[i] - cx), (float)(t.py[i] - cy), (float)t.pq[i], __int_as_float(i));
    }
}

// FP32 P2P over list 1. Targets and sources are expressed relative to the
// target leaf's centre: source = (c_src - c_tgt) [FP64 difference, rounded
// once per source cell] + (x - c_src) [FP32, precomputed], so every pair
// offset keeps ~1e-7 relative accuracy. Each thread sums one source cell's
// contributions in FP32 and adds that block sum into an FP64 accumulator
// (compensated per-target summation). Same thread mapping as p2p2d.
__global__ void __launch_bounds__(kP2PThreads)
p2p2d_f32(Tree2D t, Lists2D l, const float4* __restrict__ rel, const double* __restrict__ fx,
          const double* __restrict__ fy, double* __restrict__ out0, double* __restrict__ out1, int velocity,
          double u_inf, double v_inf, unsigned* err) {
    __shared__ double s_px[kP2PThreads], s_py[kP2PThreads];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const double ccx = t.c_cx[c], ccy = t.c_cy[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        for (int tb = lo; tb < hi; tb += kP2PThreads) {
            const int T = min(kP2PThreads, hi - tb);
            const int ns = kP2PThreads / T;
            const int tt = threadIdx.x % T, split = threadIdx.x / T;
            const bool on = split < ns;
            const int ti = tb + tt;
            const float4 tg = rel[ti];
            double ex = 0.0, ey = 0.0;
            if (on) {
                for (uint32_t k = o1; k < e1; ++k) {
                    const int sc = l.l1_src[k];
                    const int s_hi = t.c_hi[sc];
                    // target minus source offset, per source cell
                    const float ox = tg.x - (float)(t.c_cx[sc] - ccx), oy = tg.y - (float)(t.c_cy[sc] - ccy);
                    float bx0 = 0.f, by0 = 0.f, bx1 = 0.f, by1 = 0.f;
                    int j = t.c_lo[sc] + split;
                    for (; j + ns < s_hi; j += 2 * ns) {
                        const int j1 = j + ns;
                        const float4 s0 = __ldg(rel + j), s1 = __ldg(rel + j1);
                        const float dx0 = ox - s0.x, dy0 = oy - s0.y;
                        const float dx1 = ox - s1.x, dy1 = oy - s1.y;
                        const float r0 = fmaf(dx0, dx0, dy0 * dy0), r1 = fmaf(dx1, dx1, dy1 * dy1);
                        float i0, i1;
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(i0) : "f"(r0));
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(i1) : "f"(r1));
                        const float f0 = (j == ti) ? 0.f : s0.z * i0;
                        const float f1 = (j1 == ti) ? 0.f : s1.z * i1;
                        bx0 = fmaf(f0, dx0, bx0);
                        by0 = fmaf(f0, dy0, by0);
                        bx1 = fmaf(f1, dx1, bx1);
                        by1 = fmaf(f1, dy1, by1);
                    }
                    if (j < s_hi) {
                        const float4 s0 = __ldg(rel + j);
                        const float dx0 = ox - s0.x, dy0 = oy - s0.y;
                        const float r0 = fmaf(dx0, dx0, dy0 * dy0);
                        float i0;
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(i0) : "f"(r0));
                        const float f0 = (j == ti) ? 0.f : s0.z * i0;
                        bx0 = fmaf(f0, dx0, bx0);
                        by0 = fmaf(f0, dy0, by0);
                    }
                    ex += (double)bx0 + (double)bx1;
                    ey += (double)by0 + (double)by1;
                }
            }
            if (on && split > 0) { s_px[threadIdx.x] = ex; s_py[threadIdx.x] = ey; }
            __syncthreads();
            if (split == 0) {
                for (int s2 = 1; s2 < ns; ++s2) { ex += s_px[s2 * T + tt]; ey += s_py[s2 * T + tt]; }
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
            __syncthreads();
        }
    }
}

__global__ void zero_u32(unsigned* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
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

cudaError_t fmm2d_m2l(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches) {
    const int G = 32 / P;
    if (e.op) {
        const size_t smem = sizeof(double2) * 4 * (size_t)(2 * G * (P + 1) + G * (2 * P + 1));
        m2l2d_op<<<148 * 16, 128, smem, st>>>(t, l, e.a, e.b, e.op, e.coef, P, err);
    } else {
        const size_t smem = sizeof(double2) * 4 * (size_t)(G * (2 * P + 1) + 2 * G * (P + 1));
        m2l2d<<<148 * 16, 128, smem, st>>>(t, l, e.a, e.b, e.coef, P, err);
    }
    *launches += 1;
    for (int L = 3; L <= t.key_levels; ++L) {
        l2l_level2d<<<148 * 4, 128, 0, st>>>(t, e.b, e.coef, P, L, err);
        *launches += 1;
    }
    return cudaGetLastError();
}

cudaError_t fmm2d_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                       int* launches) {
    eval2d<<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, P, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p_out(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* out0, double* out1,
                          int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st, int* launches) {
    p2p2d<<<148 * 16, kP2PThreads, 0, st>>>(t, l, e.fx, e.fy, out0, out1, velocity, u_inf, v_inf, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p_f32(const Tree2D& t, const Lists2D& l, const Expansions2D& e, float4* rel, double* out0,
                          double* out1, int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st,
                          int* launches) {
    leaf_relative_f32<<<148 * 8, 128, 0, st>>>(t, rel, err);
    p2p2d_f32<<<148 * 16, kP2PThreads, 0, st>>>(t, l, rel, e.fx, e.fy, out0, out1, velocity, u_inf, v_inf, err);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t fmm2d_p2p(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* ex, double* ey,
                      unsigned* err, cudaStream_t st, int* launches) {
    return fmm2d_p2p_out(t, l, e, ex, ey, 0, 0.0, 0.0, err, st, launches);
}

}  // namespace vpm
