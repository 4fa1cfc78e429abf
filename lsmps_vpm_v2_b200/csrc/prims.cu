// Exclusive scan and onesweep-style LSD radix sort (see prims.cuh).
#include "prims.cuh"

#include <algorithm>

namespace vpm {

namespace {

constexpr uint64_t kFlagA = 1ull << 62;   // tile aggregate published
constexpr uint64_t kFlagP = 2ull << 62;   // inclusive prefix published
constexpr uint64_t kValMask = (1ull << 62) - 1;

// Status words carry flag and value together, so relaxed device-scope
// accesses are sufficient.
__device__ __forceinline__ uint64_t load_volatile(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void store_volatile(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t load_volatile32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void store_volatile32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Exclusive block scan of one value per thread (256 threads).
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t* warp_sums, uint64_t* agg) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = w;  // inclusive
    }
    __syncthreads();
    uint64_t base = warp ? warp_sums[warp - 1] : 0;
    *agg = warp_sums[(blockDim.x >> 5) - 1];
    return base + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n, uint32_t* total,
            uint64_t* status, unsigned* ticket, unsigned* err) {
    __shared__ uint64_t warp_sums[kScanThreads / 32];
    __shared__ unsigned s_tile;
    __shared__ uint64_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const int tile = (int)s_tile;
    const long long base = (long long)tile * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint64_t sum = 0;
    #pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0u;
        sum += v[k];
    }
    uint64_t agg;
    uint64_t excl = block_excl_scan(sum, warp_sums, &agg);
    if (threadIdx.x == 0) {
        uint64_t prefix = 0;
        if (tile == 0) {
            store_volatile(&status[0], kFlagP | agg);
        } else {
            store_volatile(&status[tile], kFlagA | agg);
            int k = tile - 1;
            long long spins = 0;
            while (k >= 0) {
                uint64_t w = load_volatile(&status[k]);
                if ((w & ~kValMask) == 0) {
                    if (++spins > kSpinLimit) { set_err(err, ERR_TIMEOUT); break; }
                    continue;
                }
                prefix += w & kValMask;
                if ((w & ~kValMask) == kFlagP) break;
                --k;
            }
            store_volatile(&status[tile], kFlagP | (prefix + agg));
        }
        s_prefix = prefix;
        int ntiles = scan_tiles(n);
        if (total && tile == ntiles - 1) *total = (uint32_t)(prefix + agg);
    }
    __syncthreads();
    uint64_t run = s_prefix + excl;
    #pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        if (i < n) out[i] = (uint32_t)run;
        run += v[k];
    }
}

// ---- radix sort ------------------------------------------------------------

constexpr uint32_t kRsA = 1u << 30;
constexpr uint32_t kRsP = 2u << 30;
constexpr uint32_t kRsMask = (1u << 30) - 1;

__global__ void __launch_bounds__(256)
rs_histogram(const uint64_t* __restrict__ keys, int n, int passes, uint32_t* hist) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 255], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        uint32_t c = (&h[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// hist[p][d] -> exclusive offsets within pass p (one block of 256 threads).
__global__ void rs_hist_scan(uint32_t* hist, int passes) {
    __shared__ uint64_t warp_sums[8];
    for (int p = 0; p < passes; ++p) {
        uint64_t agg;
        uint64_t v = hist[p * 256 + threadIdx.x];
        uint64_t e = block_excl_scan(v, warp_sums, &agg);
        __syncthreads();
        hist[p * 256 + threadIdx.x] = (uint32_t)e;
        __syncthreads();
    }
}

// One 8-bit digit pass. Items are arranged warp-striped: item j of lane l in
// warp w is tile_base + w*256 + j*32 + l, so processing j in order ranks keys
// in index order (stability).
__global__ void __launch_bounds__(kSortThreads)
rs_pass(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
        uint32_t* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ digit_offset,
        uint32_t* status, unsigned* ticket, unsigned* err) {
    __shared__ uint32_t s_wh[kSortThreads / 32][256];  // per-warp digit counts, then warp prefixes
    __shared__ uint32_t s_base[256];
    __shared__ unsigned s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    for (int i = threadIdx.x; i < (kSortThreads / 32) * 256; i += blockDim.x) (&s_wh[0][0])[i] = 0;
    __syncthreads();
    const int tile = (int)s_tile;
    const long long tbase = (long long)tile * kSortTile + warp * (32 * kSortItems);
    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
    int dig[kSortItems];
    const unsigned lt = (1u << lane) - 1u;
    #pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        long long i = tbase + j * 32 + lane;
        bool ok = i < n;
        key[j] = ok ? kin[i] : 0ull;
        val[j] = ok ? vin[i] : 0u;
        dig[j] = ok ? (int)((key[j] >> shift) & 255) : 256;
        unsigned m = __match_any_sync(0xffffffffu, dig[j]);
        uint32_t prior = 0;
        if (ok) prior = s_wh[warp][dig[j]];
        __syncwarp();
        if (ok && (m & lt) == 0) s_wh[warp][dig[j]] = prior + __popc(m);
        __syncwarp();
        rank[j] = prior + __popc(m & lt);
    }
    __syncthreads();
    // thread d: warp-exclusive prefixes for digit d and the tile total.
    const int d = threadIdx.x;
    uint32_t run = 0;
    #pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        uint32_t c = s_wh[w][d];
        s_wh[w][d] = run;
        run += c;
    }
    uint32_t* st = status + (size_t)tile * 256;
    if (tile == 0) {
        store_volatile32(&st[d], kRsP | run);
        s_base[d] = digit_offset[d];
    } else {
        store_volatile32(&st[d], kRsA | run);
        uint32_t prefix = 0;
        int k = tile - 1;
        long long spins = 0;
        while (k >= 0) {
            uint32_t w = load_volatile32(&status[(size_t)k * 256 + d]);
            if ((w & ~kRsMask) == 0) {
                if (++spins > kSpinLimit) { set_err(err, ERR_TIMEOUT); break; }
                continue;
            }
            prefix += w & kRsMask;
            if ((w & ~kRsMask) == kRsP) break;
            --k;
        }
        store_volatile32(&st[d], kRsP | (prefix + run));
        s_base[d] = digit_offset[d] + prefix;
    }
    __syncthreads();
    #pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (dig[j] < 256) {
            uint32_t pos = s_base[dig[j]] + s_wh[warp][dig[j]] + rank[j];
            if (pos < (uint32_t)n) {
                kout[pos] = key[j];
                vout[pos] = val[j];
            } else {
                set_err(err, ERR_INDEX);
            }
        }
    }
}

}  // namespace

cudaError_t scan_exclusive(const uint32_t* in, uint32_t* out, int n, uint32_t* total,
                           const ScanScratch& s, unsigned* err, cudaStream_t st) {
    int tiles = scan_tiles(n);
    if (tiles > s.max_tiles) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(s.status, 0, sizeof(uint64_t) * tiles, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.ticket, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    scan_kernel<<<tiles, kScanThreads, 0, st>>>(in, out, n, total, s.status, s.ticket, err);
    return cudaGetLastError();
}

cudaError_t radix_sort_pairs(uint64_t** keys, uint32_t** vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             int n, int bits, const SortScratch& s, unsigned* err, cudaStream_t st,
                             int* launches) {
    int passes = (bits + 7) / 8;
    if (passes < 1 || passes > 8) return cudaErrorInvalidValue;
    int tiles = sort_tiles(n);
    if (tiles > s.max_tiles) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(s.status, 0, sizeof(uint32_t) * (size_t)passes * tiles * 256, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.tickets, 0, sizeof(unsigned) * 8, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 8 * 256, st);
    if (e != cudaSuccess) return e;
    int hblocks = std::min(1184, ceil_div(n, 256 * 8));
    if (hblocks < 1) hblocks = 1;
    rs_histogram<<<hblocks, 256, 0, st>>>(*keys, n, passes, s.hist);
    rs_hist_scan<<<1, 256, 0, st>>>(s.hist, passes);
    if (launches) *launches += 2;
    uint64_t* ka = *keys;
    uint32_t* va = *vals;
    uint64_t* kb = keys_alt;
    uint32_t* vb = vals_alt;
    for (int p = 0; p < passes; ++p) {
        rs_pass<<<tiles, kSortThreads, 0, st>>>(ka, va, kb, vb, n, 8 * p, s.hist + 256 * p,
                                                s.status + (size_t)p * tiles * 256, s.tickets + p, err);
        if (launches) *launches += 1;
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    *keys = ka;
    *vals = va;
    return cudaGetLastError();
}

}  // namespace vpm
