// Learned (leaf caps, p) selector of the mixed 2D form, and the FP64 direct
// sum that labels and checks it. No counterpart in the reference, which
// always evaluates with its fixed caps 50/75 and p = 10 (global.cpp:311-313);
// that pair stays the fallback.
//
//   features   228 floats: log10 N, log10 root length, log10 max|q|,
//              log10 target error, then for levels 3..9 a 32-bin histogram
//              (fractions) of floor(log2 count) over the occupied cells of
//              the uniform grid of that level on the root box.
//   network    228 -> 64 -> 64 -> 64 -> 2 x kCand, GELU (erf form) after the
//              hidden layers, FP32 weights; outputs are the standardised
//              log10 error and log10 time of every candidate (caps, p).
//   training   minibatch Adam on the GPU: forward, MSE gradient, backward
//              and update are the kernels below.
//   inference  BF16 weights, FP32 accumulation, one block.
//   selection  the candidate with the least predicted time among those whose
//              predicted error is below the target (minus a margin); none ->
//              the reference pair.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "context.h"

namespace vpm {

namespace {

constexpr int kFeat = 228;
constexpr int kHid = 64;
constexpr int kCand = 35;
constexpr int kOut = 2 * kCand;
constexpr int kLayers = 4;
// Width of layer l (0 = input, kLayers = output).
__host__ __device__ constexpr int kdim(int l) { return l == 0 ? kFeat : (l == kLayers ? kOut : kHid); }
constexpr int kFeatLevelLo = 3, kFeatLevelHi = 9, kFeatBins = 32;

// Candidate (caps, p): max_src = cap, max_par = 3 cap / 2.
constexpr int kCapsList[5] = {25, 50, 100, 200, 400};
constexpr int kPList[7] = {4, 6, 8, 10, 12, 16, 20};

__host__ __device__ inline int param_count() {
    int n = 0;
    for (int l = 0; l < kLayers; ++l) n += kdim(l + 1) * kdim(l) + kdim(l + 1);
    return n;
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// ---- features ----------------------------------------------------------------

__global__ void feat_reduce(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ q,
                            int n, double* partial) {
    __shared__ double s[5][256];
    double v[5] = {INFINITY, -INFINITY, INFINITY, -INFINITY, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        v[0] = fmin(v[0], x[i]);
        v[1] = fmax(v[1], x[i]);
        v[2] = fmin(v[2], y[i]);
        v[3] = fmax(v[3], y[i]);
        v[4] = fmax(v[4], fabs(q[i]));
    }
    for (int k = 0; k < 5; ++k) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[0][threadIdx.x] = fmin(s[0][threadIdx.x], s[0][threadIdx.x + o]);
            s[1][threadIdx.x] = fmax(s[1][threadIdx.x], s[1][threadIdx.x + o]);
            s[2][threadIdx.x] = fmin(s[2][threadIdx.x], s[2][threadIdx.x + o]);
            s[3][threadIdx.x] = fmax(s[3][threadIdx.x], s[3][threadIdx.x + o]);
            s[4][threadIdx.x] = fmax(s[4][threadIdx.x], s[4][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 5) partial[blockIdx.x * 5 + threadIdx.x] = s[threadIdx.x][0];
}

// Particle counts of the level-9 grid cells on the square root box
// [x0, x0 + len) x [y0, y0 + len).
__global__ void feat_count9(const double* __restrict__ x, const double* __restrict__ y, int n, double x0, double y0,
                            double len, unsigned* counts) {
    const int G = 1 << kFeatLevelHi;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ix = (int)((x[i] - x0) / len * G), iy = (int)((y[i] - y0) / len * G);
        ix = min(max(ix, 0), G - 1);
        iy = min(max(iy, 0), G - 1);
        atomicAdd(&counts[iy * G + ix], 1u);
    }
}

// Level L from level L+1 (2x2 sums).
__global__ void feat_coarsen(const unsigned* __restrict__ fine, unsigned* __restrict__ coarse, int L) {
    const int G = 1 << L;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < G * G; c += gridDim.x * blockDim.x) {
        const int ix = c % G, iy = c / G, F = 2 * G;
        coarse[c] = fine[(2 * iy) * F + 2 * ix] + fine[(2 * iy) * F + 2 * ix + 1] + fine[(2 * iy + 1) * F + 2 * ix] +
                    fine[(2 * iy + 1) * F + 2 * ix + 1];
    }
}

__global__ void feat_hist(const unsigned* __restrict__ counts, int cells, unsigned* hist /*33: bins, occupied*/) {
    __shared__ unsigned h[kFeatBins + 1];
    if (threadIdx.x <= kFeatBins) h[threadIdx.x] = 0;
    __syncthreads();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
        const unsigned k = counts[c];
        if (!k) continue;
        const int b = min(kFeatBins - 1, 31 - __clz(k));  // floor(log2 k)
        atomicAdd(&h[b], 1u);
        atomicAdd(&h[kFeatBins], 1u);
    }
    __syncthreads();
    if (threadIdx.x <= kFeatBins && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// ---- network -----------------------------------------------------------------

// Z = X W^T + b (row-major X [B x in], W [out x in]); A = gelu(Z) or Z.
__global__ void lin_fwd(const float* __restrict__ X, int B, int in, const float* __restrict__ W,
                        const float* __restrict__ bias, int out, float* __restrict__ Z, float* __restrict__ A,
                        int act) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B * out; k += gridDim.x * blockDim.x) {
        const int r = k / out, o = k - r * out;
        const float* xr = X + (size_t)r * in;
        const float* wr = W + (size_t)o * in;
        float z = bias[o];
        for (int i = 0; i < in; ++i) z = fmaf(wr[i], xr[i], z);
        Z[k] = z;
        A[k] = act ? gelu(z) : z;
    }
}

// Masked MSE: dY = 2 (Yhat - Y) m / count, loss += (Yhat - Y)^2 m / count.
__global__ void mse_grad(const float* __restrict__ Yh, const float* __restrict__ Y, const float* __restrict__ M,
                         int n, float inv_count, float* __restrict__ dY, float* loss) {
    float acc = 0.f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float m = M ? M[k] : 1.f;
        const float d = (Yh[k] - Y[k]) * m;
        dY[k] = 2.f * d * inv_count;
        acc += d * d * inv_count;
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(loss, acc);
}

__global__ void act_bwd(const float* __restrict__ dA, const float* __restrict__ Z, int n, float* __restrict__ dZ,
                        int act) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        dZ[k] = act ? dA[k] * gelu_grad(Z[k]) : dA[k];
}

// dW[o][i] = sum_r dZ[r][o] X[r][i]; db[o] = sum_r dZ[r][o]  (fixed order: deterministic)
__global__ void lin_bwd_w(const float* __restrict__ dZ, const float* __restrict__ X, int B, int in, int out,
                          float* __restrict__ dW, float* __restrict__ db) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < out * (in + 1); k += gridDim.x * blockDim.x) {
        const int o = k / (in + 1), i = k - o * (in + 1);
        float s = 0.f;
        if (i < in) {
            for (int r = 0; r < B; ++r) s = fmaf(dZ[(size_t)r * out + o], X[(size_t)r * in + i], s);
            dW[(size_t)o * in + i] = s;
        } else {
            for (int r = 0; r < B; ++r) s += dZ[(size_t)r * out + o];
            db[o] = s;
        }
    }
}

// dX[r][i] = sum_o dZ[r][o] W[o][i]
__global__ void lin_bwd_x(const float* __restrict__ dZ, const float* __restrict__ W, int B, int in, int out,
                          float* __restrict__ dX) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B * in; k += gridDim.x * blockDim.x) {
        const int r = k / in, i = k - r * in;
        float s = 0.f;
        for (int o = 0; o < out; ++o) s = fmaf(dZ[(size_t)r * out + o], W[(size_t)o * in + i], s);
        dX[k] = s;
    }
}

__global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    }
}

__global__ void gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int rows, int width,
                            float* __restrict__ dst) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < rows * width; k += gridDim.x * blockDim.x) {
        const int r = k / width, c = k - r * width;
        dst[k] = src[(size_t)idx[r] * width + c];
    }
}

__global__ void to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) wb[k] = __float2bfloat16(w[k]);
}

// BF16-weight inference of B rows (one block per row, FP32 accumulation).
__global__ void __launch_bounds__(128)
infer_bf16(const float* __restrict__ X, int B, const __nv_bfloat16* __restrict__ wb, float* __restrict__ Y) {
    __shared__ float s_a[kFeat], s_b[kFeat];
    for (int r = blockIdx.x; r < B; r += gridDim.x) {
        for (int i = threadIdx.x; i < kFeat; i += blockDim.x) s_a[i] = X[(size_t)r * kFeat + i];
        __syncthreads();
        const __nv_bfloat16* p = wb;
        float* cur = s_a;
        float* nxt = s_b;
        for (int l = 0; l < kLayers; ++l) {
            const int in = kdim(l), out = kdim(l + 1);
            const __nv_bfloat16* W = p;
            const __nv_bfloat16* bias = p + (size_t)out * in;
            for (int o = threadIdx.x; o < out; o += blockDim.x) {
                float z = __bfloat162float(bias[o]);
                for (int i = 0; i < in; ++i) z = fmaf(__bfloat162float(W[(size_t)o * in + i]), cur[i], z);
                nxt[o] = l + 1 < kLayers ? gelu(z) : z;
            }
            __syncthreads();
            p += (size_t)out * in + out;
            float* t = cur;
            cur = nxt;
            nxt = t;
        }
        for (int o = threadIdx.x; o < kOut; o += blockDim.x) Y[(size_t)r * kOut + o] = cur[o];
        __syncthreads();
    }
}

// ---- FP64 direct sum at sampled targets ----------------------------------------

constexpr int kDirTargets = 32;   // targets per block
constexpr int kDirSplits = 16;    // source ranges per target block

// partial[split][k] = sum over active j != t_k in the split's source range of
// q_j (x_t - x_j) / |x_t - x_j|^2 (x and y parts).
__global__ void __launch_bounds__(256)
direct2d_partial(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ q,
                 const uint8_t* __restrict__ act, int n, const int64_t* __restrict__ tgt, int m,
                 double* __restrict__ part) {
    __shared__ double s_x[kDirTargets], s_y[kDirTargets];
    __shared__ int64_t s_t[kDirTargets];
    __shared__ double s_red[2][8][kDirTargets];
    const int t0 = blockIdx.x * kDirTargets;
    if (threadIdx.x < kDirTargets) {
        const int k = t0 + threadIdx.x;
        const int64_t ti = k < m ? tgt[k] : -1;
        s_t[threadIdx.x] = ti;
        s_x[threadIdx.x] = ti >= 0 ? x[ti] : 0.0;
        s_y[threadIdx.x] = ti >= 0 ? y[ti] : 0.0;
    }
    __syncthreads();
    const int split = blockIdx.y;
    const long long per = (n + kDirSplits - 1) / kDirSplits;
    const long long j0 = split * per, j1 = min((long long)n, j0 + per);
    double ex[kDirTargets], ey[kDirTargets];
    #pragma unroll
    for (int k = 0; k < kDirTargets; ++k) ex[k] = ey[k] = 0.0;
    for (long long j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        if (!act[j]) continue;
        const double xj = x[j], yj = y[j], qj = q[j];
        #pragma unroll
        for (int k = 0; k < kDirTargets; ++k) {
            const double dx = s_x[k] - xj, dy = s_y[k] - yj;
            const double r2 = dx * dx + dy * dy;
            const double f = (j == s_t[k]) ? 0.0 : qj / r2;
            ex[k] = fma(f, dx, ex[k]);
            ey[k] = fma(f, dy, ey[k]);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int k = 0; k < kDirTargets; ++k) {
        double a = ex[k], b = ey[k];
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            s_red[0][warp][k] = a;
            s_red[1][warp][k] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x < kDirTargets) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            a += s_red[0][w][threadIdx.x];
            b += s_red[1][w][threadIdx.x];
        }
        const int k = t0 + threadIdx.x;
        if (k < m) {
            part[((size_t)split * m + k) * 2] = a;
            part[((size_t)split * m + k) * 2 + 1] = b;
        }
    }
}

__global__ void direct2d_sum(const double* __restrict__ part, int m, double* __restrict__ ex, double* __restrict__ ey) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        double a = 0.0, b = 0.0;
        for (int s = 0; s < kDirSplits; ++s) {
            a += part[((size_t)s * m + k) * 2];
            b += part[((size_t)s * m + k) * 2 + 1];
        }
        ex[k] = a;
        ey[k] = b;
    }
}

// The 3D Biot-Savart sum at sampled targets in the same arrangement:
// partial[split][k] = sum over active j != t_k of alpha_j x r / |r|^3,
// r = x_t - x_j (fast3DFMM.cpp:437-459 over all sources).
__global__ void __launch_bounds__(256)
direct3d_partial(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                 const double* __restrict__ ax, const double* __restrict__ ay, const double* __restrict__ az,
                 const uint8_t* __restrict__ act, int n, const int64_t* __restrict__ tgt, int m,
                 double* __restrict__ part) {
    constexpr int T = kDirTargets / 2;   // targets per block (three sums each)
    __shared__ double s_p[3][T];
    __shared__ int64_t s_t[T];
    __shared__ double s_red[3][8][T];
    const int t0 = blockIdx.x * T;
    if (threadIdx.x < T) {
        const int k = t0 + threadIdx.x;
        const int64_t ti = k < m ? tgt[k] : -1;
        s_t[threadIdx.x] = ti;
        s_p[0][threadIdx.x] = ti >= 0 ? x[ti] : 0.0;
        s_p[1][threadIdx.x] = ti >= 0 ? y[ti] : 0.0;
        s_p[2][threadIdx.x] = ti >= 0 ? z[ti] : 0.0;
    }
    __syncthreads();
    const int split = blockIdx.y;
    const long long per = (n + kDirSplits - 1) / kDirSplits;
    const long long j0 = split * per, j1 = min((long long)n, j0 + per);
    double u[T], v[T], w[T];
    #pragma unroll
    for (int k = 0; k < T; ++k) u[k] = v[k] = w[k] = 0.0;
    for (long long j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        if (!act[j]) continue;
        const double xj = x[j], yj = y[j], zj = z[j], a1 = ax[j], a2 = ay[j], a3 = az[j];
        #pragma unroll
        for (int k = 0; k < T; ++k) {
            const double ex = s_p[0][k] - xj, ey = s_p[1][k] - yj, ez = s_p[2][k] - zj;
            const double r2 = ex * ex + ey * ey + ez * ez;
            const double r3 = sqrt(r2) * r2;
            const double f = (j == s_t[k]) ? 0.0 : 1.0 / r3;
            u[k] = fma(f, a2 * ez - a3 * ey, u[k]);
            v[k] = fma(f, a3 * ex - a1 * ez, v[k]);
            w[k] = fma(f, a1 * ey - a2 * ex, w[k]);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int k = 0; k < T; ++k) {
        double a = u[k], b = v[k], c = w[k];
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (lane == 0) {
            s_red[0][warp][k] = a;
            s_red[1][warp][k] = b;
            s_red[2][warp][k] = c;
        }
    }
    __syncthreads();
    if (threadIdx.x < T) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int wv = 0; wv < 8; ++wv) {
            a += s_red[0][wv][threadIdx.x];
            b += s_red[1][wv][threadIdx.x];
            c += s_red[2][wv][threadIdx.x];
        }
        const int k = t0 + threadIdx.x;
        if (k < m) {
            double* o = part + ((size_t)split * m + k) * 3;
            o[0] = a;
            o[1] = b;
            o[2] = c;
        }
    }
}

__global__ void direct3d_sum(const double* __restrict__ part, int m, double* __restrict__ u, double* __restrict__ v,
                             double* __restrict__ w) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int sp = 0; sp < kDirSplits; ++sp) {
            const double* o = part + ((size_t)sp * m + k) * 3;
            a += o[0];
            b += o[1];
            c += o[2];
        }
        u[k] = a;
        v[k] = b;
        w[k] = c;
    }
}

}  // namespace

// ---- host side -------------------------------------------------------------------

struct Selector {
    int device = 0;
    float* params = nullptr;   // [param_count]
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    __nv_bfloat16* wb = nullptr;
    bool wb_fresh = false;
    int adam_t = 0;
    int bmax = 0;
    float* act[kLayers + 1] = {};   // A_l  [bmax x dim_l]
    float* pre[kLayers + 1] = {};   // Z_l
    float* dA = nullptr;            // [bmax x kFeat]
    float* dZ = nullptr;
    float* ybatch = nullptr;
    float* mbatch = nullptr;
    float* loss = nullptr;          // device scalars
    int* idx = nullptr;
    // training set
    float *X = nullptr, *Y = nullptr, *M = nullptr;
    long long rows = 0, rows_cap = 0;
    // normalisation
    std::vector<float> in_mean, in_std, out_mean, out_std;
    // feature scratch
    unsigned* counts = nullptr;     // level 9 .. 3 grids
    unsigned* hist = nullptr;       // [7][33]
    double* partial = nullptr;      // [296 * 5]
    double* dir_part = nullptr;
    size_t dir_part_cap = 0;
    void* staging = nullptr;
    size_t staging_cap = 0;

    ~Selector() {
        cudaSetDevice(device);
        for (void* p : {(void*)params, (void*)grads, (void*)adam_m, (void*)adam_v, (void*)wb, (void*)dA, (void*)dZ,
                        (void*)ybatch, (void*)mbatch, (void*)loss, (void*)idx, (void*)X, (void*)Y, (void*)M,
                        (void*)counts, (void*)hist, (void*)partial, (void*)dir_part, staging})
            if (p) cudaFree(p);
        for (int l = 0; l <= kLayers; ++l) {
            if (act[l]) cudaFree(act[l]);
            if (pre[l]) cudaFree(pre[l]);
        }
    }
};

namespace {

int grid_for(long long n, int block = 256) { return (int)std::max<long long>(1, std::min<long long>(1184, (n + block - 1) / block)); }

cudaError_t sel_alloc(Selector& s) {
    if (s.params) return cudaSuccess;
    const int P = param_count();
    cudaError_t e;
    if ((e = cudaMalloc(&s.params, sizeof(float) * P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.grads, sizeof(float) * P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.adam_m, sizeof(float) * P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.adam_v, sizeof(float) * P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.wb, sizeof(__nv_bfloat16) * P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.loss, sizeof(float) * 4)) != cudaSuccess) return e;
    const int G = 1 << kFeatLevelHi;
    if ((e = cudaMalloc(&s.counts, sizeof(unsigned) * 2 * G * G)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.hist, sizeof(unsigned) * 7 * (kFeatBins + 1))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.partial, sizeof(double) * 296 * 5)) != cudaSuccess) return e;
    s.in_mean.assign(kFeat, 0.f);
    s.in_std.assign(kFeat, 1.f);
    s.out_mean.assign(kOut, 0.f);
    s.out_std.assign(kOut, 1.f);
    return cudaSuccess;
}

cudaError_t sel_batch(Selector& s, int B) {
    if (B <= s.bmax) return cudaSuccess;
    for (int l = 0; l <= kLayers; ++l) {
        if (s.act[l]) cudaFree(s.act[l]);
        if (s.pre[l]) cudaFree(s.pre[l]);
        s.act[l] = s.pre[l] = nullptr;
    }
    for (float** p : {&s.dA, &s.dZ, &s.ybatch, &s.mbatch})
        if (*p) { cudaFree(*p); *p = nullptr; }
    if (s.idx) { cudaFree(s.idx); s.idx = nullptr; }
    s.bmax = 0;
    cudaError_t e;
    for (int l = 0; l <= kLayers; ++l) {
        if ((e = cudaMalloc(&s.act[l], sizeof(float) * (size_t)B * kdim(l))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s.pre[l], sizeof(float) * (size_t)B * kdim(l))) != cudaSuccess) return e;
    }
    if ((e = cudaMalloc(&s.dA, sizeof(float) * (size_t)B * kFeat)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.dZ, sizeof(float) * (size_t)B * kFeat)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.ybatch, sizeof(float) * (size_t)B * kOut)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.mbatch, sizeof(float) * (size_t)B * kOut)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s.idx, sizeof(int) * (size_t)B)) != cudaSuccess) return e;
    s.bmax = B;
    return cudaSuccess;
}

// Forward of the B rows in s.act[0]; outputs in s.act[kLayers].
void sel_forward(Selector& s, int B, cudaStream_t st) {
    const float* p = s.params;
    for (int l = 0; l < kLayers; ++l) {
        const int in = kdim(l), out = kdim(l + 1);
        lin_fwd<<<grid_for((long long)B * out), 256, 0, st>>>(s.act[l], B, in, p, p + (size_t)out * in, out, s.pre[l + 1],
                                                             s.act[l + 1], l + 1 < kLayers);
        p += (size_t)out * in + out;
    }
}

// Gradient of the masked MSE of s.act[kLayers] against s.ybatch into s.grads;
// the loss is added to s.loss[slot].
void sel_backward(Selector& s, int B, const float* mask, int slot, cudaStream_t st) {
    const int n = B * kOut;
    mse_grad<<<grid_for(n), 256, 0, st>>>(s.act[kLayers], s.ybatch, mask, n, 1.f / (float)n, s.dA, s.loss + slot);
    // parameter offsets per layer
    size_t off[kLayers];
    size_t o = 0;
    for (int l = 0; l < kLayers; ++l) {
        off[l] = o;
        o += (size_t)kdim(l + 1) * kdim(l) + kdim(l + 1);
    }
    for (int l = kLayers - 1; l >= 0; --l) {
        const int in = kdim(l), out = kdim(l + 1);
        act_bwd<<<grid_for((long long)B * out), 256, 0, st>>>(s.dA, s.pre[l + 1], B * out, s.dZ, l + 1 < kLayers);
        lin_bwd_w<<<grid_for((long long)out * (in + 1)), 256, 0, st>>>(s.dZ, s.act[l], B, in, out, s.grads + off[l],
                                                                      s.grads + off[l] + (size_t)out * in);
        if (l > 0)
            lin_bwd_x<<<grid_for((long long)B * in), 256, 0, st>>>(s.dZ, s.params + off[l], B, in, out, s.dA);
    }
}

}  // namespace

}  // namespace vpm

using vpm::Ctx;
using vpm::Selector;

namespace {

Selector* selector_of(Ctx* c) {
    if (!c->selector) {
        c->selector = new (std::nothrow) Selector();
        if (c->selector) c->selector->device = c->device;
    }
    return c->selector;
}

#define SEL_TRY(expr)                                           \
    do {                                                        \
        cudaError_t _e = (expr);                                \
        if (_e != cudaSuccess) return c->fail_cuda(_e, #expr);  \
    } while (0)

}  // namespace

extern "C" {

int64_t vpm_mlp_param_count(void) { return vpm::param_count(); }

int vpm_selector_candidates(int32_t* caps, int32_t* ps, int32_t count) {
    if (count < vpm::kCand || !caps || !ps) return VPM_EINVAL;
    int k = 0;
    for (int ci = 0; ci < 5; ++ci)
        for (int pi = 0; pi < 7; ++pi, ++k) {
            caps[k] = vpm::kCapsList[ci];
            ps[k] = vpm::kPList[pi];
        }
    return VPM_OK;
}

int vpm_mlp_init(vpm_ctx* ctx, uint64_t seed) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    std::mt19937_64 rng(seed);
    std::vector<float> h(vpm::param_count());
    size_t o = 0;
    for (int l = 0; l < vpm::kLayers; ++l) {
        const int in = vpm::kdim(l), out = vpm::kdim(l + 1);
        const double a = std::sqrt(6.0 / (in + out));
        std::uniform_real_distribution<double> U(-a, a);
        for (int k = 0; k < out * in; ++k) h[o++] = (float)U(rng);
        for (int k = 0; k < out; ++k) h[o++] = 0.f;
    }
    SEL_TRY(cudaMemcpy(s->params, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
    SEL_TRY(cudaMemset(s->adam_m, 0, sizeof(float) * h.size()));
    SEL_TRY(cudaMemset(s->adam_v, 0, sizeof(float) * h.size()));
    s->adam_t = 0;
    s->wb_fresh = false;
    return VPM_OK;
}

int vpm_mlp_set_params(vpm_ctx* ctx, const float* params, int64_t count) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!params || count != vpm::param_count()) return c->fail(VPM_EINVAL, "parameter count");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    SEL_TRY(cudaMemcpy(s->params, params, sizeof(float) * count, cudaMemcpyHostToDevice));
    SEL_TRY(cudaMemset(s->adam_m, 0, sizeof(float) * count));
    SEL_TRY(cudaMemset(s->adam_v, 0, sizeof(float) * count));
    s->adam_t = 0;
    s->wb_fresh = false;
    return VPM_OK;
}

int vpm_mlp_get_params(vpm_ctx* ctx, float* params, int64_t count) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    Selector* s = c->selector;
    if (!s || !s->params) return c->fail(VPM_EINVAL, "no network on this context");
    if (!params || count != vpm::param_count()) return c->fail(VPM_EINVAL, "parameter count");
    SEL_TRY(cudaSetDevice(c->device));
    SEL_TRY(cudaMemcpy(params, s->params, sizeof(float) * count, cudaMemcpyDeviceToHost));
    return VPM_OK;
}

int vpm_mlp_set_norm(vpm_ctx* ctx, const float* in_mean, const float* in_std, const float* out_mean,
                     const float* out_std) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!in_mean || !in_std || !out_mean || !out_std) return c->fail(VPM_EINVAL, "null buffer");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    s->in_mean.assign(in_mean, in_mean + vpm::kFeat);
    s->in_std.assign(in_std, in_std + vpm::kFeat);
    s->out_mean.assign(out_mean, out_mean + vpm::kOut);
    s->out_std.assign(out_std, out_std + vpm::kOut);
    return VPM_OK;
}

// Forward of B rows (already normalised inputs, host arrays). bf16 != 0 uses
// the BF16 inference kernel, else the FP32 training forward.
int vpm_mlp_forward(vpm_ctx* ctx, const float* X, int32_t B, float* Y, int32_t bf16) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    Selector* s = c->selector;
    if (!s || !s->params) return c->fail(VPM_EINVAL, "no network on this context");
    if (B <= 0 || !X || !Y) return c->fail(VPM_EINVAL, "bad batch");
    SEL_TRY(cudaSetDevice(c->device));
    SEL_TRY(vpm::sel_batch(*s, B));
    cudaStream_t st = c->stream;
    SEL_TRY(cudaMemcpyAsync(s->act[0], X, sizeof(float) * (size_t)B * vpm::kFeat, cudaMemcpyHostToDevice, st));
    const float* out = s->act[vpm::kLayers];
    if (bf16) {
        if (!s->wb_fresh) {
            vpm::to_bf16<<<vpm::grid_for(vpm::param_count()), 256, 0, st>>>(s->params, s->wb, vpm::param_count());
            s->wb_fresh = true;
        }
        vpm::infer_bf16<<<std::min(B, 1184), 128, 0, st>>>(s->act[0], B, s->wb, s->dA);
        out = s->dA;
    } else {
        vpm::sel_forward(*s, B, st);
    }
    SEL_TRY(cudaGetLastError());
    SEL_TRY(cudaMemcpyAsync(Y, out, sizeof(float) * (size_t)B * vpm::kOut, cudaMemcpyDeviceToHost, st));
    SEL_TRY(cudaStreamSynchronize(st));
    return VPM_OK;
}

// Gradient of the masked MSE loss over B rows (host arrays; mask may be NULL).
int vpm_mlp_grads(vpm_ctx* ctx, const float* X, const float* Y, const float* mask, int32_t B, float* grads,
                  float* loss) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    Selector* s = c->selector;
    if (!s || !s->params) return c->fail(VPM_EINVAL, "no network on this context");
    if (B <= 0 || !X || !Y || !grads) return c->fail(VPM_EINVAL, "bad batch");
    SEL_TRY(cudaSetDevice(c->device));
    SEL_TRY(vpm::sel_batch(*s, B));
    cudaStream_t st = c->stream;
    SEL_TRY(cudaMemcpyAsync(s->act[0], X, sizeof(float) * (size_t)B * vpm::kFeat, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemcpyAsync(s->ybatch, Y, sizeof(float) * (size_t)B * vpm::kOut, cudaMemcpyHostToDevice, st));
    if (mask)
        SEL_TRY(cudaMemcpyAsync(s->mbatch, mask, sizeof(float) * (size_t)B * vpm::kOut, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemsetAsync(s->loss, 0, sizeof(float), st));
    vpm::sel_forward(*s, B, st);
    vpm::sel_backward(*s, B, mask ? s->mbatch : nullptr, 0, st);
    SEL_TRY(cudaGetLastError());
    SEL_TRY(cudaMemcpyAsync(grads, s->grads, sizeof(float) * vpm::param_count(), cudaMemcpyDeviceToHost, st));
    float l = 0.f;
    SEL_TRY(cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    SEL_TRY(cudaStreamSynchronize(st));
    if (loss) *loss = l;
    return VPM_OK;
}

// Minibatch Adam on the GPU over the rows (normalised X, Y; mask may be
// NULL): `steps` steps of `batch` rows drawn without replacement per epoch
// (seeded). loss_hist (may be NULL) receives the loss of every step.
int vpm_mlp_train(vpm_ctx* ctx, const float* X, const float* Y, const float* mask, int64_t rows, int32_t batch,
                  int32_t steps, float lr, uint64_t seed, float* loss_hist) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    Selector* s = c->selector;
    if (!s || !s->params) return c->fail(VPM_EINVAL, "no network on this context");
    if (rows <= 0 || batch <= 0 || batch > rows || steps < 0 || !X || !Y) return c->fail(VPM_EINVAL, "bad training set");
    SEL_TRY(cudaSetDevice(c->device));
    SEL_TRY(vpm::sel_batch(*s, batch));
    cudaStream_t st = c->stream;
    if (rows > s->rows_cap) {
        for (float** p : {&s->X, &s->Y, &s->M})
            if (*p) { cudaFree(*p); *p = nullptr; }
        s->rows_cap = 0;
        SEL_TRY(cudaMalloc(&s->X, sizeof(float) * rows * vpm::kFeat));
        SEL_TRY(cudaMalloc(&s->Y, sizeof(float) * rows * vpm::kOut));
        SEL_TRY(cudaMalloc(&s->M, sizeof(float) * rows * vpm::kOut));
        s->rows_cap = rows;
    }
    SEL_TRY(cudaMemcpyAsync(s->X, X, sizeof(float) * rows * vpm::kFeat, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemcpyAsync(s->Y, Y, sizeof(float) * rows * vpm::kOut, cudaMemcpyHostToDevice, st));
    if (mask) SEL_TRY(cudaMemcpyAsync(s->M, mask, sizeof(float) * rows * vpm::kOut, cudaMemcpyHostToDevice, st));
    float* d_hist = nullptr;
    SEL_TRY(cudaMalloc(&d_hist, sizeof(float) * std::max(1, steps)));
    cudaError_t e = cudaMemsetAsync(d_hist, 0, sizeof(float) * std::max(1, steps), st);
    std::mt19937_64 rng(seed);
    std::vector<int> perm(rows), idx(batch);
    for (long long i = 0; i < rows; ++i) perm[i] = (int)i;
    long long pos = rows;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<int*> idx_bufs;
    for (int step = 0; step < steps && e == cudaSuccess; ++step) {
        for (int k = 0; k < batch; ++k) {
            if (pos >= rows) {
                std::shuffle(perm.begin(), perm.end(), rng);
                pos = 0;
            }
            idx[k] = perm[pos++];
        }
        // the index upload must not be overwritten before the gather ran: one sync per step
        e = cudaMemcpyAsync(s->idx, idx.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) break;
        vpm::gather_rows<<<vpm::grid_for((long long)batch * vpm::kFeat), 256, 0, st>>>(s->X, s->idx, batch, vpm::kFeat,
                                                                                    s->act[0]);
        vpm::gather_rows<<<vpm::grid_for((long long)batch * vpm::kOut), 256, 0, st>>>(s->Y, s->idx, batch, vpm::kOut,
                                                                                   s->ybatch);
        if (mask)
            vpm::gather_rows<<<vpm::grid_for((long long)batch * vpm::kOut), 256, 0, st>>>(s->M, s->idx, batch,
                                                                                       vpm::kOut, s->mbatch);
        vpm::sel_forward(*s, batch, st);
        SEL_TRY(cudaMemsetAsync(s->loss + 1, 0, sizeof(float), st));
        vpm::sel_backward(*s, batch, mask ? s->mbatch : nullptr, 1, st);
        ++s->adam_t;
        const float c1 = 1.f - std::pow(b1, (float)s->adam_t), c2 = 1.f - std::pow(b2, (float)s->adam_t);
        vpm::adam_step<<<vpm::grid_for(vpm::param_count()), 256, 0, st>>>(s->params, s->grads, s->adam_m, s->adam_v,
                                                                       vpm::param_count(), lr, b1, b2, eps, c1, c2);
        e = cudaMemcpyAsync(d_hist + step, s->loss + 1, sizeof(float), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && loss_hist && steps > 0)
        e = cudaMemcpy(loss_hist, d_hist, sizeof(float) * steps, cudaMemcpyDeviceToHost);
    cudaFree(d_hist);
    s->wb_fresh = false;
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_mlp_train");
    return VPM_OK;
}

namespace {

// The 228 features of a 2D particle set in device memory (see the top of the
// file); synchronises the context's stream.
int features_device(Ctx* c, Selector* s, const double* x, const double* y, const double* q, const uint8_t* act,
                     int n, double target_err, float* feat) {
    (void)act;
    cudaStream_t st = c->stream;
    const int nb = std::max(1, std::min(296, (n + 255) / 256));
    vpm::feat_reduce<<<nb, 256, 0, st>>>(x, y, q, n, s->partial);
    std::vector<double> part((size_t)nb * 5);
    SEL_TRY(cudaMemcpyAsync(part.data(), s->partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
    SEL_TRY(cudaStreamSynchronize(st));
    double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY, mq = 0.0;
    for (int b = 0; b < nb; ++b) {
        mnx = std::min(mnx, part[b * 5 + 0]);
        mxx = std::max(mxx, part[b * 5 + 1]);
        mny = std::min(mny, part[b * 5 + 2]);
        mxy = std::max(mxy, part[b * 5 + 3]);
        mq = std::max(mq, part[b * 5 + 4]);
    }
    double len = std::max(mxx - mnx, mxy - mny) * 1.01;
    if (!(len > 0.0)) len = 1.0;
    const double x0 = 0.5 * (mnx + mxx) - 0.5 * len, y0 = 0.5 * (mny + mxy) - 0.5 * len;
    const int G9 = 1 << vpm::kFeatLevelHi;
    unsigned* bufA = s->counts;
    unsigned* bufB = s->counts + G9 * G9;
    SEL_TRY(cudaMemsetAsync(bufA, 0, sizeof(unsigned) * G9 * G9, st));
    SEL_TRY(cudaMemsetAsync(s->hist, 0, sizeof(unsigned) * 7 * (vpm::kFeatBins + 1), st));
    vpm::feat_count9<<<vpm::grid_for(n), 256, 0, st>>>(x, y, n, x0, y0, len, bufA);
    unsigned* cur = bufA;
    for (int L = vpm::kFeatLevelHi; L >= vpm::kFeatLevelLo; --L) {
        const int cells = 1 << (2 * L);
        vpm::feat_hist<<<vpm::grid_for(cells), 256, 0, st>>>(cur, cells,
                                                            s->hist + (L - vpm::kFeatLevelLo) * (vpm::kFeatBins + 1));
        if (L > vpm::kFeatLevelLo) {
            unsigned* nxt = cur == bufA ? bufB : bufA;
            vpm::feat_coarsen<<<vpm::grid_for(cells / 4), 256, 0, st>>>(cur, nxt, L - 1);
            cur = nxt;
        }
    }
    SEL_TRY(cudaGetLastError());
    std::vector<unsigned> h(7 * (vpm::kFeatBins + 1));
    SEL_TRY(cudaMemcpyAsync(h.data(), s->hist, sizeof(unsigned) * h.size(), cudaMemcpyDeviceToHost, st));
    SEL_TRY(cudaStreamSynchronize(st));
    feat[0] = (float)std::log10((double)n);
    feat[1] = (float)std::log10(len);
    feat[2] = (float)std::log10(std::max(mq, 1e-300));
    feat[3] = (float)std::log10(target_err);
    for (int L = 0; L < 7; ++L) {
        const unsigned* hl = &h[L * (vpm::kFeatBins + 1)];
        const double occ = std::max(1u, hl[vpm::kFeatBins]);
        for (int b = 0; b < vpm::kFeatBins; ++b) feat[4 + L * vpm::kFeatBins + b] = (float)(hl[b] / occ);
    }
    return VPM_OK;
}

}  // namespace

int vpm_selector_features2d_device(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                                   const uint8_t* active, int64_t n, double target_err, float* feat) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!x || !y || !q || !active || !feat || n < 1 || n >= (1ll << 31) || !(target_err > 0.0))
        return c->fail(VPM_EINVAL, "bad feature request");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    return features_device(c, s, x, y, q, active, (int)n, target_err, feat);
}

int vpm_selector_features2d(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                            const uint8_t* active, int64_t n, double target_err, float* feat) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!x || !y || !q || !active || !feat || n < 1 || n >= (1ll << 31) || !(target_err > 0.0))
        return c->fail(VPM_EINVAL, "bad feature request");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    const size_t need = (size_t)n * (3 * sizeof(double) + 1) + 64;
    if (s->staging_cap < need) {
        if (s->staging) cudaFree(s->staging);
        s->staging = nullptr;
        s->staging_cap = 0;
        SEL_TRY(cudaMalloc(&s->staging, need));
        s->staging_cap = need;
    }
    double* dx = (double*)s->staging;
    double* dy = dx + n;
    double* dq = dy + n;
    uint8_t* da = (uint8_t*)(dq + n);
    cudaStream_t st = c->stream;
    SEL_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemcpyAsync(dy, y, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemcpyAsync(dq, q, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SEL_TRY(cudaMemcpyAsync(da, active, n, cudaMemcpyHostToDevice, st));
    return features_device(c, s, dx, dy, dq, da, (int)n, target_err, feat);
}

// Selection from raw features: normalise, BF16 inference, then the cheapest
// candidate whose predicted log10 error is at most log10(target) - margin.
// Falls back to the reference pair (50/75, p = 10) when none qualifies.
// pred (may be NULL) receives the 2 x 35 de-normalised predictions.
int vpm_select2d(vpm_ctx* ctx, const float* feat, double target_err, double margin_decades, int32_t* max_src,
                 int32_t* max_par, int32_t* p, float* pred) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    Selector* s = c->selector;
    if (!feat || !max_src || !max_par || !p || !(target_err > 0.0)) return c->fail(VPM_EINVAL, "bad selection request");
    *max_src = 50;
    *max_par = 75;
    *p = 10;
    if (!s || !s->params) return VPM_OK;  // no network: the reference pair
    std::vector<float> xn(vpm::kFeat), y(vpm::kOut);
    for (int i = 0; i < vpm::kFeat; ++i) {
        const float v = i == 3 ? (float)std::log10(target_err) : feat[i];
        xn[i] = (v - s->in_mean[i]) / s->in_std[i];
    }
    int r = vpm_mlp_forward(ctx, xn.data(), 1, y.data(), 1);
    if (r) return r;
    const double lim = std::log10(target_err) - margin_decades;
    int best = -1;
    double best_t = INFINITY;
    for (int k = 0; k < vpm::kCand; ++k) {
        const double le = y[k] * s->out_std[k] + s->out_mean[k];
        const double lt = y[vpm::kCand + k] * s->out_std[vpm::kCand + k] + s->out_mean[vpm::kCand + k];
        if (pred) {
            pred[k] = (float)le;
            pred[vpm::kCand + k] = (float)lt;
        }
        if (le <= lim && lt < best_t) {
            best_t = lt;
            best = k;
        }
    }
    if (best >= 0) {
        const int cap = vpm::kCapsList[best / 7];
        *max_src = cap;
        *max_par = cap * 3 / 2;
        *p = vpm::kPList[best % 7];
    }
    return VPM_OK;
}

// FP64 direct field at m sampled targets (device pointers; targets int64 on
// the device), E = sum over active j != t of q_j (x_t - x_j) / |x_t - x_j|^2.
int vpm_direct2d_field_device(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                              const uint8_t* active, int64_t n, const int64_t* targets, int64_t m, double* ex,
                              double* ey) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (n < 1 || n >= (1ll << 31) || m < 0 || m >= (1ll << 31)) return c->fail(VPM_EINVAL, "n or m out of range");
    if (m == 0) return VPM_OK;
    if (!x || !y || !q || !active || !targets || !ex || !ey) return c->fail(VPM_EINVAL, "null buffer");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    const size_t need = sizeof(double) * 2 * vpm::kDirSplits * (size_t)m;
    if (s->dir_part_cap < need) {
        if (s->dir_part) cudaFree(s->dir_part);
        s->dir_part = nullptr;
        s->dir_part_cap = 0;
        SEL_TRY(cudaMalloc(&s->dir_part, need));
        s->dir_part_cap = need;
    }
    dim3 grid((unsigned)((m + vpm::kDirTargets - 1) / vpm::kDirTargets), vpm::kDirSplits);
    vpm::direct2d_partial<<<grid, 256, 0, c->stream>>>(x, y, q, active, (int)n, targets, (int)m, s->dir_part);
    vpm::direct2d_sum<<<vpm::grid_for(m), 256, 0, c->stream>>>(s->dir_part, (int)m, ex, ey);
    SEL_TRY(cudaGetLastError());
    return VPM_OK;
}

// FP64 direct 3D velocity at m sampled targets (device pointers).
int vpm_direct3d_velocity_device(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                                 const double* ay, const double* az, const uint8_t* active, int64_t n,
                                 const int64_t* targets, int64_t m, double* u, double* v, double* w) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (n < 1 || n >= (1ll << 31) || m < 0 || m >= (1ll << 31)) return c->fail(VPM_EINVAL, "n or m out of range");
    if (m == 0) return VPM_OK;
    if (!x || !y || !z || !ax || !ay || !az || !active || !targets || !u || !v || !w)
        return c->fail(VPM_EINVAL, "null buffer");
    SEL_TRY(cudaSetDevice(c->device));
    Selector* s = selector_of(c);
    if (!s) return c->fail(VPM_ENOMEM, "selector");
    SEL_TRY(vpm::sel_alloc(*s));
    const size_t need = sizeof(double) * 3 * vpm::kDirSplits * (size_t)m;
    if (s->dir_part_cap < need) {
        if (s->dir_part) cudaFree(s->dir_part);
        s->dir_part = nullptr;
        s->dir_part_cap = 0;
        SEL_TRY(cudaMalloc(&s->dir_part, need));
        s->dir_part_cap = need;
    }
    const int T = vpm::kDirTargets / 2;
    dim3 grid((unsigned)((m + T - 1) / T), vpm::kDirSplits);
    vpm::direct3d_partial<<<grid, 256, 0, c->stream>>>(x, y, z, ax, ay, az, active, (int)n, targets, (int)m,
                                                       s->dir_part);
    vpm::direct3d_sum<<<vpm::grid_for(m), 256, 0, c->stream>>>(s->dir_part, (int)m, u, v, w);
    SEL_TRY(cudaGetLastError());
    return VPM_OK;
}

}  // extern "C"

namespace vpm {
void drop_selector(Selector* s) { delete s; }
}  // namespace vpm
