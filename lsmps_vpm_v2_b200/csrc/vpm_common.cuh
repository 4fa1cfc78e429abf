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
    ERR_LEAF1 = 1u << 10,       // 3D TreeCell: a level-1 leaf in a deeper tree
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
// Grid-wide barrier for cooperative (co-resident) launches: bar[0] counts
// arrivals, bar[1] is the generation. The last block to arrive resets the
// count and bumps the generation; the others poll the generation, at most
// kSpinLimit times (then ERR_TIMEOUT and continue). bar[0] must be zero at
// launch. Every block must call it the same number of times.
// ---------------------------------------------------------------------------
// Device-scope relaxed accesses for look-back status words, which carry their
// flag and value in one word.
__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Decoupled look-back by one warp: the sum of the values published by tiles
// tile-1, tile-2, ... down to and including the nearest inclusive prefix.
// Status words are FLAG_A | aggregate or FLAG_P | inclusive prefix in the
// bits above VMASK (0: not yet published). Each round reads 32 predecessors
// at once, so a chain of published aggregates costs one load round per 32
// tiles. Call with the whole warp; the result is in every lane. A wait that
// exceeds kSpinLimit rounds sets ERR_TIMEOUT and returns the partial sum.
template <uint64_t FLAG_P, uint64_t VMASK>
__device__ __forceinline__ uint64_t warp_lookback(const uint64_t* status, int tile, unsigned* err) {
    const int lane = threadIdx.x & 31;
    uint64_t prefix = 0;
    int k = tile - 1;
    long long spins = 0;
    while (k >= 0) {
        const int idx = k - lane;
        const uint64_t w = idx >= 0 ? ld_relaxed64(&status[idx]) : FLAG_P;  // before tile 0: empty prefix
        const uint64_t f = w & ~VMASK;
        const unsigned notready = __ballot_sync(0xffffffffu, f == 0);
        const unsigned incl = __ballot_sync(0xffffffffu, f == FLAG_P);
        // lanes 0 .. first inclusive prefix (all 32 when there is none)
        const unsigned upto = ((incl & (0u - incl)) << 1) - 1u;
        if (notready & upto) {
            if (++spins > kSpinLimit) {
                if (lane == 0) set_err(err, ERR_TIMEOUT);
                break;
            }
            continue;
        }
        uint64_t v = ((upto >> lane) & 1u) ? (w & VMASK) : 0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        prefix += v;
        if (incl) break;
        k -= 32;
    }
    return prefix;
}

// The error word's fatal bits, read once per block so that every thread of
// the block takes the same branch (safe around __syncthreads).
__device__ __forceinline__ bool block_fatal(const unsigned* err) {
    __shared__ int s_fatal;
    __syncthreads();
    if (threadIdx.x == 0) s_fatal = fatal(err);
    __syncthreads();
    return s_fatal != 0;
}

// Grid barrier on a counter that only grows: the G blocks of barrier i take
// it from i G to (i + 1) G, and a block waits until it reaches the next
// multiple of G above the value its own arrival saw. One atomic per block and
// no reset step, so the wait ends one memory round trip after the last
// arrival. The arrival is a release at GPU scope and the polls are acquires,
// with the block barriers on either side carrying the ordering to the other
// threads of the block (no full fences: 2.4 us per phase against 2.7 with
// them, measured on the B200). The counter must be zero at launch and used by
// one kernel only (a word of its own, zeroed before every evaluation).
__device__ __forceinline__ void grid_sync_counter(unsigned* bar, unsigned* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned old;
        asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
        const unsigned target = (old / gridDim.x + 1u) * gridDim.x;
        long long spins = 0;
        for (;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if ((int)(v - target) >= 0) break;
            if (++spins > kSpinLimit) {
                set_err(err, ERR_TIMEOUT);
                break;
            }
            __nanosleep(16);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void grid_sync(unsigned* bar, unsigned* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > kSpinLimit) {
                    set_err(err, ERR_TIMEOUT);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
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

// Cooperative launch with every block co-resident: grid = SMs x the
// occupancy of `kernel` at `block` threads (at most max_blocks_per_sm), and at
// most max_grid blocks. The grid size is returned in *grid. Fails (no launch)
// when the device cannot make the blocks co-resident.
template <typename... KArgs, typename... Args>
cudaError_t launch_coop_max(void (*kernel)(KArgs...), int block, size_t smem, cudaStream_t st, int max_blocks_per_sm,
                            int max_grid, int* grid, Args... args) {
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorCooperativeLaunchTooLarge;
    if (occ > max_blocks_per_sm) occ = max_blocks_per_sm;
    const int g = sms * occ < max_grid ? sms * occ : (max_grid > 0 ? max_grid : 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (grid) *grid = g;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename... KArgs, typename... Args>
cudaError_t launch_coop(void (*kernel)(KArgs...), int block, size_t smem, cudaStream_t st, int max_blocks_per_sm,
                        int* grid, Args... args) {
    return launch_coop_max(kernel, block, smem, st, max_blocks_per_sm, 1 << 30, grid, args...);
}

}  // namespace vpm

#define VPM_CUDA_TRY(expr)                                             \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) return fail_cuda(_e, #expr);            \
    } while (0)
