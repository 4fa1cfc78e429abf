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

// One warp per leaf. Lane k holds coefficient k (P <= 30 < 32).
__global__ void __launch_bounds__(128)
upward2d(Tree2D t, double2* __restrict__ a, unsigned* __restrict__ cnt, const double* __restrict__ coef, int P,
         unsigned* err) {
    const double* g_m2m = coef + kCoefM2M;
    __shared__ double2 s_child[4][W];
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nl = t.info->n_leaves;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int li = blockIdx.x * (blockDim.x >> 5) + wib; li < nl; li += warps) {
        const int c = t.leaf_cells[li];
        if (t.c_flags[c] & CELL_ACTIVE) {
            const double zx = t.c_cx[c], zy = t.c_cy[c];
            const int lo = t.c_lo[c], hi = t.c_hi[c];
            double2 acc = make_double2(0.0, 0.0);
            for (int j0 = lo; j0 < hi; j0 += 32) {
                const int j = j0 + lane;
                double q = 0.0;
                double2 w = make_double2(0.0, 0.0);
                if (j < hi && t.pact[j]) {
                    q = t.pq[j];
                    w = make_double2(t.px[j] - zx, t.py[j] - zy);
                }
                double2 wk = make_double2(q, 0.0);  // q w^k
                for (int k = 0; k <= P; ++k) {
                    double2 s = warp_sum2(wk);
                    if (lane == k) acc = cadd(acc, s);
                    wk = cmul(wk, w);
                }
            }
            if (lane <= P) a[(size_t)c * (P + 1) + lane] = acc;
        }
        // Walk up: the last child of a parent to finish computes the parent.
        int cur = c;
        for (;;) {
            const int par = t.c_parent[cur];
            if (par <= 0) break;  // the root's expansion is never used
            __threadfence();
            __syncwarp();
            unsigned old = 0;
            if (lane == 0) old = atomicAdd(&cnt[par], 1u);
            old = __shfl_sync(0xffffffffu, old, 0);
            const unsigned m = t.c_chmask[par];
            if (old != (unsigned)__popc(m) - 1u) break;
            __threadfence();
            if (t.c_flags[par] & CELL_ACTIVE) {
                const double px = t.c_cx[par], py = t.c_cy[par];
                double2 acc = make_double2(0.0, 0.0);
                const int c0 = t.c_child0[par];
                for (int r = 0; r < __popc(m); ++r) {
                    const int ch = c0 + r;
                    if (lane <= P) s_child[wib][lane] = ldcg2(&a[(size_t)ch * (P + 1) + lane]);
                    __syncwarp();
                    const double2 tt = make_double2(t.c_cx[ch] - px, t.c_cy[ch] - py);
                    if (lane == 0) {
                        acc = cadd(acc, s_child[wib][0]);
                    } else if (lane <= P) {
                        // sum_{j=0..p} coef_j t^j with coef_p = a0, coef_{p-k} = m2m[p][k] a_k
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
                if (lane <= P) a[(size_t)par * (P + 1) + lane] = acc;
            }
            cur = par;
        }
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

// ---- leaf evaluation: L2L chain, M2P (list 3), L2P --------------------------

constexpr int kEvalThreads = 64;

__global__ void __launch_bounds__(kEvalThreads)
eval2d(Tree2D t, Lists2D l, const double2* __restrict__ a, const double2* __restrict__ b, double* __restrict__ fx,
       double* __restrict__ fy, const double* __restrict__ coef, int P, unsigned* err) {
    const double* g_l2l = coef + kCoefL2L;
    __shared__ double2 s_b[W];
    __shared__ double2 s_nb[W];
    __shared__ int s_path[kMaxLevels2D + 1];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int L = t.c_level[c];
        // Local expansion of the leaf: b(level 2 ancestor) pushed down.
        if (threadIdx.x == 0) {
            int cur = c;
            for (int k = L; k >= 0; --k) {
                s_path[k] = cur < 0 ? 0 : cur;
                if (cur >= 0) cur = t.c_parent[cur];
            }
        }
        __syncthreads();
        if (L >= 2) {
            const int lane = threadIdx.x;
            if (lane <= P) s_b[lane] = b[(size_t)s_path[2] * (P + 1) + lane];
            __syncthreads();
            for (int k = 3; k <= L; ++k) {
                const int ch = s_path[k], par = s_path[k - 1];
                if (lane <= P) {
                    const double2 tt = make_double2(t.c_cx[ch] - t.c_cx[par], t.c_cy[ch] - t.c_cy[par]);
                    const int pp = lane;
                    const double* cf = g_l2l + pp * W;
                    double2 S = cscale(s_b[P], cf[P]);
                    for (int kk = P - 1; kk >= pp; --kk) S = cfma(S, tt, cscale(s_b[kk], cf[kk]));
                    s_nb[pp] = cadd(b[(size_t)ch * (P + 1) + pp], S);
                }
                __syncthreads();
                if (lane <= P) s_b[lane] = s_nb[lane];
                __syncthreads();
            }
        } else {
            if (threadIdx.x <= P) s_b[threadIdx.x] = make_double2(0.0, 0.0);
            __syncthreads();
        }
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
constexpr int kP2PStage = 256;

__global__ void __launch_bounds__(kP2PThreads)
p2p2d(Tree2D t, Lists2D l, const double* __restrict__ fx, const double* __restrict__ fy, double* __restrict__ out0,
      double* __restrict__ out1, int velocity, double u_inf, double v_inf, unsigned* err) {
    __shared__ double s_x[kP2PStage], s_y[kP2PStage], s_q[kP2PStage];
    __shared__ int s_i[kP2PStage];
    __shared__ double s_px[kP2PThreads], s_py[kP2PThreads];
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
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
            const double xt = t.px[ti], yt = t.py[ti];
            double ex = 0.0, ey = 0.0;
            // Stage list-1 sources in chunks.
            uint32_t k = o1;
            int s_lo = 0, s_hi = 0;  // remaining range of the current source cell
            if (k < e1) { const int sc = l.l1_src[k]; s_lo = t.c_lo[sc]; s_hi = t.c_hi[sc]; }
            while (k < e1) {
                int m = 0;
                __syncthreads();
                // fill the stage (uniform control flow: all threads walk the same ranges)
                while (k < e1 && m < kP2PStage) {
                    const int take = min(kP2PStage - m, s_hi - s_lo);
                    for (int j = threadIdx.x; j < take; j += blockDim.x) {
                        const int gj = s_lo + j;
                        s_x[m + j] = t.px[gj];
                        s_y[m + j] = t.py[gj];
                        s_q[m + j] = t.pq[gj];
                        s_i[m + j] = gj;
                    }
                    m += take;
                    s_lo += take;
                    if (s_lo >= s_hi) {
                        ++k;
                        if (k < e1) { const int sc = l.l1_src[k]; s_lo = t.c_lo[sc]; s_hi = t.c_hi[sc]; }
                    }
                }
                __syncthreads();
                if (on) {
                    for (int j = split; j < m; j += ns) {
                        if (s_i[j] == ti) continue;
                        const double dx = xt - s_x[j], dy = yt - s_y[j];
                        const double r2 = fma(dx, dx, dy * dy);
                        const double f = s_q[j] * rcp_nr(r2);
                        ex = fma(f, dx, ex);
                        ey = fma(f, dy, ey);
                    }
                }
            }
            // Reduce the splits of each target.
            __syncthreads();
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

constexpr int kP2PStageF = 512;

// FP32 P2P over list 1. Targets and sources are expressed relative to the
// target leaf's centre: source = (c_src - c_tgt) [FP64 difference, rounded
// once] + (x - c_src) [FP32], so every pair offset keeps ~1e-7 relative
// accuracy. Each thread sums a staged block of sources in FP32 and adds the
// block sum into an FP64 accumulator (compensated per-target summation).
__global__ void __launch_bounds__(kP2PThreads)
p2p2d_f32(Tree2D t, Lists2D l, const float4* __restrict__ rel, const double* __restrict__ fx,
          const double* __restrict__ fy, double* __restrict__ out0, double* __restrict__ out1, int velocity,
          double u_inf, double v_inf, unsigned* err) {
    __shared__ float4 s_src[kP2PStageF];
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
            const int tid = __float_as_int(tg.w);
            double ex = 0.0, ey = 0.0;
            uint32_t k = o1;
            int s_lo = 0, s_hi = 0;
            float ox = 0.f, oy = 0.f;
            if (k < e1) {
                const int sc = l.l1_src[k];
                s_lo = t.c_lo[sc]; s_hi = t.c_hi[sc];
                ox = (float)(t.c_cx[sc] - ccx); oy = (float)(t.c_cy[sc] - ccy);
            }
            while (k < e1) {
                int m = 0;
                __syncthreads();
                while (k < e1 && m < kP2PStageF) {
                    const int take = min(kP2PStageF - m, s_hi - s_lo);
                    for (int j = threadIdx.x; j < take; j += blockDim.x) {
                        float4 v = rel[s_lo + j];
                        v.x += ox;
                        v.y += oy;
                        s_src[m + j] = v;
                    }
                    m += take;
                    s_lo += take;
                    if (s_lo >= s_hi) {
                        ++k;
                        if (k < e1) {
                            const int sc = l.l1_src[k];
                            s_lo = t.c_lo[sc]; s_hi = t.c_hi[sc];
                            ox = (float)(t.c_cx[sc] - ccx); oy = (float)(t.c_cy[sc] - ccy);
                        }
                    }
                }
                __syncthreads();
                if (on) {
                    float bx = 0.f, by = 0.f;
                    for (int j = split; j < m; j += ns) {
                        const float4 sv = s_src[j];
                        const float dx = tg.x - sv.x, dy = tg.y - sv.y;
                        const float r2 = fmaf(dx, dx, dy * dy);
                        float inv;
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(r2));
                        const float f = (__float_as_int(sv.w) == tid) ? 0.f : sv.z * inv;
                        bx = fmaf(f, dx, bx);
                        by = fmaf(f, dy, by);
                    }
                    ex += bx;
                    ey += by;
                }
            }
            __syncthreads();
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

cudaError_t fmm2d_upward(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches) {
    cudaError_t r = cudaMemsetAsync(e.a, 0, sizeof(double2) * (size_t)t.cap_cells * (P + 1), st);
    if (r != cudaSuccess) return r;
    zero_u32<<<148, 256, 0, st>>>(e.up_count, t.cap_cells);
    upward2d<<<148 * 8, 128, 0, st>>>(t, e.a, e.up_count, e.coef, P, err);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t fmm2d_m2l(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches) {
    const int G = 32 / P;
    const size_t smem = sizeof(double2) * 4 * (size_t)(G * (2 * P + 1) + 2 * G * (P + 1));
    m2l2d<<<148 * 16, 128, smem, st>>>(t, l, e.a, e.b, e.coef, P, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                       int* launches) {
    eval2d<<<148 * 16, kEvalThreads, 0, st>>>(t, l, e.a, e.b, e.fx, e.fy, e.coef, P, err);
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
