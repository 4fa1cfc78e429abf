// 3D treecode evaluation (fastFMM3Dutils::evaluateFMM, src/FMM/fast3DFMM.cpp:318-472):
// every particle is a target; from the root's children down, each active
// child k of a cell on the target's list is
//   far   if R^2 > (s size_k)^2   -> M2P with the derivative multipliers of
//                                    fmm3D::M2P_mul_calc (fmm3D.cpp:147-200)
//   else a non-leaf               -> onto the target's list for the next level
//   else a leaf                   -> P2P  u += (alpha_j x r) / |r|^3, j != i,
//                                    active j only (fast3DFMM.cpp:440-460)
// The reference's TreeCell path (fmm3D::calcVelocity, VELOCITY_CALCULATION_TYPE
// 2, fmm3D.cpp:1264-1360; calcVelocityNearBody, fmm3D.cpp:1406-1606) walks
// its TreeCell the same way, with every particle of a near leaf a source.
// (level-1 cells themselves are never evaluated, as in the reference).
// s is the reference's support factor 2 (fast3DFMM.cpp:4) unless the caller
// asks for a stricter far test (a larger s: more accurate, slower).
//
// One warp per 32 consecutive particles in leaf order (leaves hold about 8
// particles on average, so a warp spans a few neighbouring leaves), one lane
// per target. The warp walks the union of its targets' lists level by level,
// each entry carrying the mask of the lanes whose own list holds it; every
// lane therefore makes exactly its own reference decisions, in its own order,
// whichever other targets share its warp (results do not depend on the
// grouping). The far/near test uses separately rounded IEEE operations (no
// contraction) so it decides as the reference does.
#include "fmm3d.cuh"

#include <algorithm>
#include <cmath>

namespace vpm {

namespace {

struct Src3 {
    const double *px, *py, *pz, *ax, *ay, *az;
    const uint8_t* act;
};

// M2P of one far cell, FP64: multipliers g of r / |r|^3 and its first two
// derivatives paired with the ten moments of each source component, then
// u += M_y g_z - M_z g_y etc. (fast3DFMM.cpp:395-425).
__device__ __forceinline__ void m2p64(const double* __restrict__ M, double R2, double dx, double dy, double dz,
                                      double& vx, double& vy, double& vz) {
    const double R = sqrt(R2);
    const double i2 = 1.0 / R2;
    const double i3 = 1.0 / (R * R2);
    const double i5 = i3 * i2, i7 = i5 * i2;
    double gx[10], gy[10], gz[10];
    gx[0] = dx * i3;
    gx[1] = -(3 * dx * dx * i5) + i3;
    gx[2] = -(3 * dx * dy * i5);
    gx[3] = -(3 * dx * dz * i5);
    gx[4] = (15 * dx * dx * dx * i7) - (9 * dx * i5);
    gx[5] = (15 * dx * dy * dy * i7) - (3 * dx * i5);
    gx[6] = (15 * dx * dz * dz * i7) - (3 * dx * i5);
    gx[7] = (15 * dx * dx * dy * i7) - (3 * dy * i5);
    gx[8] = (15 * dx * dy * dz * i7);
    gx[9] = (15 * dx * dx * dz * i7) - (3 * dz * i5);
    gy[0] = dy * i3;
    gy[1] = -(3 * dy * dx * i5);
    gy[2] = -(3 * dy * dy * i5) + i3;
    gy[3] = -(3 * dy * dz * i5);
    gy[4] = (15 * dy * dx * dx * i7) - (3 * dy * i5);
    gy[5] = (15 * dy * dy * dy * i7) - (9 * dy * i5);
    gy[6] = (15 * dy * dz * dz * i7) - (3 * dy * i5);
    gy[7] = (15 * dy * dx * dy * i7) - (3 * dx * i5);
    gy[8] = (15 * dy * dy * dz * i7) - (3 * dz * i5);
    gy[9] = (15 * dy * dx * dz * i7);
    gz[0] = dz * i3;
    gz[1] = -(3 * dz * dx * i5);
    gz[2] = -(3 * dz * dy * i5);
    gz[3] = -(3 * dz * dz * i5) + i3;
    gz[4] = (15 * dz * dx * dx * i7) - (3 * dz * i5);
    gz[5] = (15 * dz * dy * dy * i7) - (3 * dz * i5);
    gz[6] = (15 * dz * dz * dz * i7) - (9 * dz * i5);
    gz[7] = (15 * dz * dx * dy * i7);
    gz[8] = (15 * dz * dy * dz * i7) - (3 * dy * i5);
    gz[9] = (15 * dz * dx * dz * i7) - (3 * dx * i5);
    const double* Mx = M;
    const double* My = M + 10;
    const double* Mz = M + 20;
    #pragma unroll
    for (int m = 0; m < 10; ++m) {
        const double mx = Mx[m], my = My[m], mz = Mz[m];
        vx += my * gz[m] - mz * gy[m];
        vy += mz * gx[m] - mx * gz[m];
        vz += mx * gy[m] - my * gx[m];
    }
}

// The same in FP32 (mixed form): offsets rounded to float after the FP64
// subtraction, moments from their FP32 copy, the cell's sum formed in FP32
// and added to the FP64 total.
__device__ __forceinline__ void m2p32(const float* __restrict__ M, double dxd, double dyd, double dzd,
                                      double& vx, double& vy, double& vz) {
    const float dx = (float)dxd, dy = (float)dyd, dz = (float)dzd;
    const float R2 = dx * dx + dy * dy + dz * dz;
    const float iR = rsqrtf(R2);
    const float i2 = iR * iR;
    const float i3 = i2 * iR;
    const float i5 = i3 * i2, i7 = i5 * i2;
    const float a5x = 3.f * i5 * dx, a5y = 3.f * i5 * dy, a5z = 3.f * i5 * dz;
    const float b7 = 15.f * i7;
    float gx[10], gy[10], gz[10];
    gx[0] = dx * i3;
    gx[1] = -(a5x * dx) + i3;
    gx[2] = -(a5x * dy);
    gx[3] = -(a5x * dz);
    gx[4] = (b7 * dx * dx * dx) - 3.f * a5x;
    gx[5] = (b7 * dx * dy * dy) - a5x;
    gx[6] = (b7 * dx * dz * dz) - a5x;
    gx[7] = (b7 * dx * dx * dy) - a5y;
    gx[8] = (b7 * dx * dy * dz);
    gx[9] = (b7 * dx * dx * dz) - a5z;
    gy[0] = dy * i3;
    gy[1] = -(a5y * dx);
    gy[2] = -(a5y * dy) + i3;
    gy[3] = -(a5y * dz);
    gy[4] = (b7 * dy * dx * dx) - a5y;
    gy[5] = (b7 * dy * dy * dy) - 3.f * a5y;
    gy[6] = (b7 * dy * dz * dz) - a5y;
    gy[7] = (b7 * dy * dx * dy) - a5x;
    gy[8] = (b7 * dy * dy * dz) - a5z;
    gy[9] = (b7 * dy * dx * dz);
    gz[0] = dz * i3;
    gz[1] = -(a5z * dx);
    gz[2] = -(a5z * dy);
    gz[3] = -(a5z * dz) + i3;
    gz[4] = (b7 * dz * dx * dx) - a5z;
    gz[5] = (b7 * dz * dy * dy) - a5z;
    gz[6] = (b7 * dz * dz * dz) - 3.f * a5z;
    gz[7] = (b7 * dz * dx * dy);
    gz[8] = (b7 * dz * dy * dz) - a5y;
    gz[9] = (b7 * dz * dx * dz) - a5x;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    #pragma unroll
    for (int m = 0; m < 10; ++m) {
        const float mx = M[m], my = M[10 + m], mz = M[20 + m];
        sx += my * gz[m] - mz * gy[m];
        sy += mz * gx[m] - mx * gz[m];
        sz += mx * gy[m] - my * gx[m];
    }
    vx += sx;
    vy += sy;
    vz += sz;
}

// P2P of one near leaf [lo, hi) onto target slot `self` at (xp, yp, zp);
// ALL: inactive particles are sources too (TreeCell path).
// F32: the target's offset from the leaf's centre (cx, cy, cz) is formed in
// FP64 once and rounded; the sources' offsets and alphas come from their FP32
// copies (prep3d_f32), so the pair loop is FP32 only.
template <bool F32, bool ALL>
__device__ __forceinline__ void p2p3(const Src3& s, const float4* __restrict__ ps32, const float4* __restrict__ as32,
                                     int lo, int hi, int self, double xp, double yp, double zp, double cx, double cy,
                                     double cz, double& vx, double& vy, double& vz) {
    if (F32) {
        const float tx = (float)(xp - cx), ty = (float)(yp - cy), tz = (float)(zp - cz);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        for (int j = lo; j < hi; ++j) {
            const float4 sp = ps32[j];
            if ((!ALL && sp.w == 0.f) || j == self) continue;
            const float ex = tx - sp.x, ey = ty - sp.y, ez = tz - sp.z;
            const float r2 = ex * ex + ey * ey + ez * ez;
            const float ir = rsqrtf(r2);
            const float ir3 = ir * ir * ir;
            const float4 al = as32[j];
            sx += (al.y * ez - al.z * ey) * ir3;
            sy += (al.z * ex - al.x * ez) * ir3;
            sz += (al.x * ey - al.y * ex) * ir3;
        }
        vx += sx;
        vy += sy;
        vz += sz;
    } else {
        for (int j = lo; j < hi; ++j) {
            if ((!ALL && !s.act[j]) || j == self) continue;
            const double ex = xp - s.px[j], ey = yp - s.py[j], ez = zp - s.pz[j];
            const double r2 = ex * ex + ey * ey + ez * ez;
            const double ir3 = 1.0 / (sqrt(r2) * r2);
            vx += (s.ay[j] * ez - s.az[j] * ey) * ir3;
            vy += (s.az[j] * ex - s.ax[j] * ez) * ir3;
            vz += (s.ax[j] * ey - s.ay[j] * ex) * ir3;
        }
    }
}

// One warp per cell: for a leaf (no children), the offsets from its centre
// and the alphas of its particles; then every cell's moments (grid-stride).
__global__ void __launch_bounds__(256) prep3d_f32_kernel(Tree3D t, unsigned* err) {
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31;
    const int nc = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nc; c += warps) {
        if (t.c_chmask[c] != 0) continue;
        const double cx = t.c_x[c], cy = t.c_y[c], cz = t.c_z[c];
        for (int j = t.c_lo[c] + lane; j < t.c_hi[c]; j += 32) {
            t.ps32[j] = make_float4((float)(t.px[j] - cx), (float)(t.py[j] - cy), (float)(t.pz[j] - cz),
                                    t.pact[j] ? 1.f : 0.f);
            t.as32[j] = make_float4((float)t.ax[j], (float)t.ay[j], (float)t.az[j], 0.f);
        }
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)nc * 30;
         i += (long long)gridDim.x * blockDim.x)
        t.mom32[i] = (float)t.mom[i];
}

template <bool F32, bool ALL>
__global__ void __launch_bounds__(32 * kEval3DWarps)
eval3d_kernel(Tree3D t, const uint8_t* __restrict__ target, double support, int cap, double* __restrict__ u,
              double* __restrict__ v, double* __restrict__ w, double uinf, double vinf, double winf, unsigned* ticket,
              unsigned* err) {
    // per warp two work lists of `cap` entries (cell, lane mask): dynamic
    // shared memory sized from the support factor by the launcher
    extern __shared__ int s_work[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int* s_cell0 = s_work + (size_t)wib * 4 * cap;
    unsigned* s_mask0 = reinterpret_cast<unsigned*>(s_cell0 + 2 * cap);
    int stop = 0;
    if (lane == 0) stop = fatal(err);
    if (__shfl_sync(0xffffffffu, stop, 0)) return;  // warp-uniform
    const int depth = t.info->depth;
    const int nchunks = (t.n + 31) >> 5;
    const Src3 src{t.px, t.py, t.pz, t.ax, t.ay, t.az, t.pact};
    const unsigned rm = t.c_chmask[0];
    const int r0 = t.c_child0[0];
    for (;;) {
        int c = 0;
        if (lane == 0) c = (int)atomicAdd(ticket, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= nchunks) break;
        const int lo = c * 32, hi = min(t.n, lo + 32);
        for (int tb = lo; tb < hi; tb += 32) {
            const int slot = tb + lane;
            const bool has = slot < hi;
            const bool tgt = has && (target == nullptr || target[t.perm[slot]] != 0);
            const double xp = has ? t.px[slot] : 0.0, yp = has ? t.py[slot] : 0.0, zp = has ? t.pz[slot] : 0.0;
            const unsigned full = __ballot_sync(0xffffffffu, tgt);
            double vx = 0.0, vy = 0.0, vz = 0.0;
            int which = 0;
            int ncur = __popc(rm);
            if (lane < ncur) {
                s_cell0[lane] = r0 + lane;
                s_mask0[lane] = full;
            }
            __syncwarp();
            for (int lv = 1; lv < depth && ncur > 0; ++lv) {
                const int* cur_c = s_cell0 + which * cap;
                const unsigned* cur_m = s_mask0 + which * cap;
                int* nxt_c = s_cell0 + (which ^ 1) * cap;
                unsigned* nxt_m = s_mask0 + (which ^ 1) * cap;
                int nn = 0;
                for (int e = 0; e < ncur; ++e) {
                    const int cc = cur_c[e];
                    const bool mine = (cur_m[e] >> lane) & 1u;
                    const unsigned cm = t.c_chmask[cc];
                    const int k0 = t.c_child0[cc];
                    int r = 0;
                    for (int o = 0; o < 8; ++o) {
                        if (!((cm >> o) & 1u)) continue;
                        const int k = k0 + r++;
                        if (!t.c_active[k]) continue;
                        bool far = false;
                        double dx = 0.0, dy = 0.0, dz = 0.0, R2 = 0.0;
                        if (mine) {
                            dx = xsub(xp, t.c_x[k]);
                            dy = xsub(yp, t.c_y[k]);
                            dz = xsub(zp, t.c_z[k]);
                            R2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                            const double Rc = xmul(t.c_size[k], support);
                            far = R2 > xmul(Rc, Rc);
                            if (far) {
                                if (F32) m2p32(&t.mom32[(size_t)k * 30], dx, dy, dz, vx, vy, vz);
                                else m2p64(&t.mom[(size_t)k * 30], R2, dx, dy, dz, vx, vy, vz);
                            }
                        }
                        const unsigned near = __ballot_sync(0xffffffffu, mine && !far);
                        if (!near) continue;
                        if (t.c_chmask[k] != 0) {
                            if (nn < cap) {
                                if (lane == 0) {
                                    nxt_c[nn] = k;
                                    nxt_m[nn] = near;
                                }
                            } else if (lane == 0) {
                                set_err(err, ERR_QUEUE);
                            }
                            ++nn;
                        } else if ((near >> lane) & 1u) {
                            p2p3<F32, ALL>(src, t.ps32, t.as32, t.c_lo[k], t.c_hi[k], slot, xp, yp, zp, t.c_x[k],
                                           t.c_y[k], t.c_z[k], vx, vy, vz);
                        }
                    }
                }
                __syncwarp();
                which ^= 1;
                ncur = min(nn, cap);
            }
            if (has) {
                const uint32_t i = t.perm[slot];
                u[i] = tgt ? vx + uinf : 0.0;
                v[i] = tgt ? vy + vinf : 0.0;
                w[i] = tgt ? vz + winf : 0.0;
            }
            __syncwarp();
        }
    }
}

}  // namespace

cudaError_t prep3d_f32(const Tree3D& t, unsigned* err, cudaStream_t st, int* launches) {
    prep3d_f32_kernel<<<148 * 8, 256, 0, st>>>(t, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t eval3d(const Tree3D& t, bool mixed, bool all_src, const uint8_t* target, double support, double* u,
                   double* v, double* w, double uinf, double vinf, double winf, unsigned* err, cudaStream_t st,
                   int* launches) {
    unsigned* ticket = t.gbar + 4;
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    // work-list entries per level: kWork3DCap at the reference's factor 2
    // (which needs a few dozen), times (factor / 2)^1.5 beyond it (the near
    // shell of a level widens with the factor; on the 2M-particle ring 3.5
    // and 4 fit with room to spare, and an overflow sets ERR_QUEUE)
    const double f = support > 2.0 ? support / 2.0 : 1.0;
    const int cap = std::min(8 * kWork3DCap, (int)std::ceil(kWork3DCap * std::pow(f, 1.5) / 32.0) * 32);
    const size_t smem = sizeof(int) * 4 * (size_t)cap * kEval3DWarps;
    const dim3 g(148 * 8), b(32 * kEval3DWarps);
#define VPM_EVAL3D(F, A)                                                                                     \
    do {                                                                                                     \
        e = cudaFuncSetAttribute(eval3d_kernel<F, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                                      \
        eval3d_kernel<F, A><<<g, b, smem, st>>>(t, target, support, cap, u, v, w, uinf, vinf, winf, ticket, err); \
    } while (0)
    if (mixed && all_src) VPM_EVAL3D(true, true);
    else if (mixed) VPM_EVAL3D(true, false);
    else if (all_src) VPM_EVAL3D(false, true);
    else VPM_EVAL3D(false, false);
#undef VPM_EVAL3D
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace vpm
