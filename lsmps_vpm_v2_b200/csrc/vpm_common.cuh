// Shared device/host helpers for the B200 FMM velocity step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vpm_fmm.h"

namespace vpm {

// ---------------------------------------------------------------------------
// Device error word: kernels never trap; they OR a bit into the context's
// error word and skip the offending access. The host maps bits to a status.
// ---------------------------------------------------------------------------
enum ErrBits : unsigned {
    ERR_DEPTH = 1u << 0,        // tree deeper than the key resolution
    ERR_CELL_CAP = 1u << 1,     // cell arrays too small
    ERR_QUEUE = 1u << 2,        // list BFS queue overflow
    ERR_LIST4 = 1u << 3,        // list 4 longer than its fixed slots
    ERR_INDEX = 1u << 4,        // an index fell outside its array
    ERR_TIMEOUT = 1u << 5,      // a bounded spin-wait gave up
    ERR_NONFINITE = 1u << 6,    // NaN / Inf in positions
    ERR_LIST2 = 1u << 7,        // list 2 longer than 27 (cannot happen)
    ERR_LIST_CAP = 1u << 8,     // CSR list storage too small
    ERR_RANGE = 1u << 9,        // a particle index fell outside its level box
};

// Every spin-wait in this library is bounded by this many polls; on expiry the
// kernel sets ERR_TIMEOUT and continues with what it has.
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ void set_err(unsigned* err, unsigned bit) { atomicOr(err, bit); }

// Errors after which the tree or list arrays are incomplete: every later
// kernel returns at once instead of indexing into them.
constexpr unsigned kFatalBits = ERR_DEPTH | ERR_CELL_CAP | ERR_LIST_CAP | ERR_NONFINITE | ERR_RANGE | ERR_TIMEOUT |
                                ERR_INDEX;
__device__ __forceinline__ bool fatal(const unsigned* err) {
    return (*(volatile const unsigned*)err & kFatalBits) != 0;
}

// ---------------------------------------------------------------------------
// Exact IEEE double operations (round-to-nearest, never contracted): used for
// every value that decides an integer (cell index, adjacency, separation).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// ---------------------------------------------------------------------------
// Complex double as double2 (x = real, y = imag).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// acc + a*b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
__device__ __forceinline__ double2 cinv(double2 a) {
    double d = a.x * a.x + a.y * a.y;
    double r = 1.0 / d;
    return make_double2(a.x * r, -a.y * r);
}

// ---------------------------------------------------------------------------
// Morton interleave helpers (x in the even bits, matching the reference's
// child order (0,0),(1,0),(0,1),(1,1) = x + 2y, treeCell.cpp:407-409).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t spread2(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
__host__ __device__ __forceinline__ uint64_t morton2(uint32_t ix, uint32_t iy) {
    return spread2(ix) | (spread2(iy) << 1);
}

__host__ __device__ __forceinline__ int64_t start_id2(int L) { return (((int64_t)1 << (2 * L)) - 1) / 3; }

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace vpm

#define VPM_CUDA_TRY(expr)                                             \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) return fail_cuda(_e, #expr);            \
    } while (0)
