// 2D FMM potential (fmm2D::calcPotential, src/FMM/fmm2D.cpp:681-896): the
// same tree, lists, P2M, M2M and list-2/4 M2L as the field, plus
//   b_0 += a_0 log(z_t - z_s) - sum_{k>=1} a_k / k (-1)^k (z_s - z_t)^-k   (fmm2D.cpp:465-470, 504-509)
//   L2L including p = 0                                                 (fmm2D.cpp:637-641)
//   M2P   phi += Re[ a_0 log(w) - sum_{p>=1} a_p / p w^-p ]             (fmm2D.cpp:826-834)
//   L2P   phi += Re[ sum_{p>=0} b_p w^p ]                               (fmm2D.cpp:858-866)
//   P2P   phi += q_j log(r^2) / 2, j != i, list 1                       (fmm2D.cpp:77-122)
// All in FP64.
#include "fmm2d.cuh"

namespace vpm {

namespace {

__device__ __forceinline__ double2 clog2(double2 z) { return make_double2(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

// b_0 of every cell at level >= 2 from its list-2 and list-4 sources; one warp
// per cell, lane per source, summed across the warp.
__global__ void __launch_bounds__(128)
m2l_b0_2d(Tree2D t, Lists2D l, const double2* __restrict__ a, double2* __restrict__ b, int P, unsigned* err) {
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31;
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c_begin + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < c_end; c += warps) {
        const int n2 = l.l2_n[c], ns = n2 + l.l4_n[c];
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        double2 acc = make_double2(0.0, 0.0);
        for (int si = lane; si < ns; si += 32) {
            const int s = si < n2 ? l.l2_src[(size_t)c * kList2Cap + si] : l.l4_src[(size_t)c * kList4Cap + (si - n2)];
            const double2* A = a + (size_t)s * (P + 1);
            const double2 d = make_double2(zx - t.c_cx[s], zy - t.c_cy[s]);   // z_t - z_s
            const double2 tinv = cinv(make_double2(-d.x, -d.y));             // (z_s - z_t)^-1
            // sum_{k=1..P} (-1)^k a_k / k tinv^k by Horner in tinv
            double2 S = cscale(A[P], ((P & 1) ? -1.0 : 1.0) / (double)P);
            for (int k = P - 1; k >= 1; --k) S = cfma(S, tinv, cscale(A[k], ((k & 1) ? -1.0 : 1.0) / (double)k));
            S = cmul(S, tinv);
            acc = cadd(acc, csub(cmul(A[0], clog2(d)), S));
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (lane == 0) b[(size_t)c * (P + 1)] = acc;
    }
}

// Far-field potential of every particle of a leaf: M2P over list 3 and L2P.
__global__ void __launch_bounds__(64)
eval_pot2d(Tree2D t, Lists2D l, const double2* __restrict__ a, const double2* __restrict__ b,
           double* __restrict__ far, int P, unsigned* err) {
    __shared__ double2 s_b[kMaxP + 1];
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
            double phi = 0.0;
            for (uint32_t k = o3; k < e3; ++k) {
                const int s = l.l3_src[k];
                const double2 w = make_double2(x - t.c_cx[s], y - t.c_cy[s]);
                const double2 winv = cinv(w);
                const double2* A = a + (size_t)s * (P + 1);
                double2 S = cscale(A[P], 1.0 / (double)P);
                for (int p = P - 1; p >= 1; --p) S = cfma(S, winv, cscale(A[p], 1.0 / (double)p));
                S = cmul(S, winv);
                phi += (cmul(A[0], clog2(w)).x - S.x);
            }
            const double2 w = make_double2(x - zx, y - zy);
            double2 S = s_b[P];
            for (int p = P - 1; p >= 0; --p) S = cfma(S, w, s_b[p]);
            far[i] = phi + S.x;
        }
        __syncthreads();
    }
}

// Near-field potential over list 1 plus the far field, written in the
// caller's order. One block per leaf, one thread per target.
__global__ void __launch_bounds__(128)
p2p_pot2d(Tree2D t, Lists2D l, const double* __restrict__ far, double* __restrict__ out, unsigned* err) {
    if (fatal(err)) return;
    const int nl = t.info->n_leaves;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = t.leaf_cells[li];
        const int lo = t.c_lo[c], hi = t.c_hi[c];
        const uint32_t o1 = l.l1_off[li], e1 = l.l1_off[li + 1];
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double x = t.px[i], y = t.py[i];
            double phi = 0.0;
            for (uint32_t k = o1; k < e1; ++k) {
                const int sc = l.l1_src[k];
                for (int j = t.c_lo[sc]; j < t.c_hi[sc]; ++j) {
                    if (j == i) continue;
                    const double dx = x - t.px[j], dy = y - t.py[j];
                    phi += t.pq[j] * log(dx * dx + dy * dy) / 2.0;
                }
            }
            const uint32_t orig = t.perm[i];
            if (orig >= (uint32_t)t.n) set_err(err, ERR_INDEX);
            else out[orig] = phi + far[i];
        }
    }
}

}  // namespace

// Potential stages after the field's M2L: b_0, then L2L (shared), then these.
cudaError_t fmm2d_m2l_b0(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                         int* launches) {
    m2l_b0_2d<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, P, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_potential_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, double* out,
                                 unsigned* err, cudaStream_t st, int* launches) {
    eval_pot2d<<<148 * 16, 64, 0, st>>>(t, l, e.a, e.b, e.fx, P, err);
    p2p_pot2d<<<148 * 16, 128, 0, st>>>(t, l, e.fx, out, err);
    *launches += 2;
    return cudaGetLastError();
}

}  // namespace vpm
