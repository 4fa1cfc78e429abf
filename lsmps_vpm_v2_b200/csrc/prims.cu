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
    if (threadIdx.x < 32) {
        uint64_t prefix = 0;
        if (tile == 0) {
            if (threadIdx.x == 0) store_volatile(&status[0], kFlagP | agg);
        } else {
            if (threadIdx.x == 0) store_volatile(&status[tile], kFlagA | agg);
            prefix = warp_lookback<kFlagP, kValMask>(status, tile, err);
            if (threadIdx.x == 0) store_volatile(&status[tile], kFlagP | (prefix + agg));
        }
        if (threadIdx.x == 0) {
            s_prefix = prefix;
            int ntiles = scan_tiles(n);
            if (total && tile == ntiles - 1) *total = (uint32_t)(prefix + agg);
        }
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

template <typename K>
__global__ void __launch_bounds__(256)
rs_histogram(const K* __restrict__ keys, int n, int passes, uint32_t* hist) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const K k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 255], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        uint32_t c = (&h[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// One 8-bit digit pass. Items are arranged warp-striped: item j of lane l in
// warp w is tile_base + w*256 + j*32 + l, so processing j in order ranks keys
// in index order (stability). The tile is first reordered by digit in shared
// memory, then written out so that consecutive threads store consecutive
// addresses within each digit's run.
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
rs_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
        uint32_t* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ digit_hist,
        uint32_t* status, unsigned* ticket, unsigned* err) {
    constexpr int kSortItems = SortItems<K>::value;
    constexpr int kSortTile = kSortThreads * kSortItems;
    __shared__ uint32_t s_wh[kSortThreads / 32][256];  // per-warp digit counts, then warp prefixes
    __shared__ uint32_t s_local[256];                   // tile-local start of each digit
    __shared__ uint32_t s_base[256];                    // global start minus tile-local start
    __shared__ K s_key[kSortTile];
    __shared__ uint32_t s_val[kSortTile];
    __shared__ uint64_t s_warp_sums[kSortThreads / 32];
    __shared__ unsigned s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    for (int i = threadIdx.x; i < (kSortThreads / 32) * 256; i += blockDim.x) (&s_wh[0][0])[i] = 0;
    __syncthreads();
    const int tile = (int)s_tile;
    const long long tile0 = (long long)tile * kSortTile;
    const long long tbase = tile0 + warp * (32 * kSortItems);
    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
    int dig[kSortItems];
    const unsigned lt = (1u << lane) - 1u;
    #pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        long long i = tbase + j * 32 + lane;
        bool ok = i < n;
        key[j] = ok ? kin[i] : (K)0;
        val[j] = ok ? vin[i] : 0u;
        dig[j] = ok ? (int)((key[j] >> shift) & 255) : 256;
    }
    #pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const bool ok = dig[j] < 256;
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
    uint64_t agg;
    const uint32_t local = (uint32_t)block_excl_scan(run, s_warp_sums, &agg);
    s_local[d] = local;
    uint32_t* st = status + (size_t)tile * 256;
    uint32_t prefix = 0;
    if (tile == 0) {
        store_volatile32(&st[d], kRsP | run);
    } else {
        store_volatile32(&st[d], kRsA | run);
        // Look-back for digit d, reading 16 predecessors per round (independent
        // loads) and consuming them in order up to the first one not yet
        // published or the first inclusive prefix.
        int k = tile - 1;
        long long spins = 0;
        bool done = false;
        while (!done && k >= 0) {
            uint32_t w[16];
            #pragma unroll
            for (int j = 0; j < 16; ++j) w[j] = k - j >= 0 ? load_volatile32(&status[(size_t)(k - j) * 256 + d]) : kRsP;
            bool stalled = false;
            #pragma unroll
            for (int j = 0; j < 16; ++j) {
                if (done || stalled) continue;
                const uint32_t f = w[j] & ~kRsMask;
                if (f == 0) { stalled = true; continue; }
                prefix += w[j] & kRsMask;
                --k;
                if (f == kRsP) done = true;
            }
            if (stalled && ++spins > kSpinLimit) { set_err(err, ERR_TIMEOUT); break; }
        }
        store_volatile32(&st[d], kRsP | (prefix + run));
    }
    // exclusive scan of the pass's global digit histogram (every block: 256 values)
    __syncthreads();   // s_warp_sums is reused
    uint64_t agg2;
    const uint32_t dig_off = (uint32_t)block_excl_scan(digit_hist[d], s_warp_sums, &agg2);
    s_base[d] = dig_off + prefix - local;  // modulo 2^32; adding a tile-local index gives the output index
    __syncthreads();
    #pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (dig[j] < 256) {
            const uint32_t lp = s_local[dig[j]] + s_wh[warp][dig[j]] + rank[j];
            s_key[lp] = key[j];
            s_val[lp] = val[j];
        }
    }
    __syncthreads();
    const int cnt = (int)min((long long)kSortTile, (long long)n - tile0);
    for (int i = threadIdx.x; i < cnt; i += kSortThreads) {
        const K k = s_key[i];
        const uint32_t pos = s_base[(int)((k >> shift) & 255)] + (uint32_t)i;
        if (pos < (uint32_t)n) {
            kout[pos] = k;
            vout[pos] = s_val[i];
        } else {
            set_err(err, ERR_INDEX);
        }
    }
}

template <typename K>
cudaError_t sort_pairs(K** keys, uint32_t** vals, K* keys_alt, uint32_t* vals_alt, int n, int bits,
                       const SortScratch& s, unsigned* err, cudaStream_t st, int* launches) {
    int passes = (bits + 7) / 8;
    if (passes < 1 || passes > (int)sizeof(K)) return cudaErrorInvalidValue;
    const int tiles = ceil_div(n > 0 ? n : 1, kSortThreads * SortItems<K>::value);
    if (tiles > s.max_tiles) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(s.status, 0, sizeof(uint32_t) * (size_t)passes * tiles * 256, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.tickets, 0, sizeof(unsigned) * 8, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 8 * 256, st);
    if (e != cudaSuccess) return e;
    int hblocks = std::min(1184, ceil_div(n, 256 * 8));
    if (hblocks < 1) hblocks = 1;
    rs_histogram<K><<<hblocks, 256, 0, st>>>(*keys, n, passes, s.hist);
    if (launches) *launches += 1;
    K* ka = *keys;
    uint32_t* va = *vals;
    K* kb = keys_alt;
    uint32_t* vb = vals_alt;
    for (int p = 0; p < passes; ++p) {
        rs_pass<K><<<tiles, kSortThreads, 0, st>>>(ka, va, kb, vb, n, 8 * p, s.hist + 256 * p,
                                                   s.status + (size_t)p * tiles * 256, s.tickets + p, err);
        if (launches) *launches += 1;
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    *keys = ka;
    *vals = va;
    return cudaGetLastError();
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
    return sort_pairs<uint64_t>(keys, vals, keys_alt, vals_alt, n, bits, s, err, st, launches);
}

cudaError_t radix_sort_pairs(uint32_t** keys, uint32_t** vals, uint32_t* keys_alt, uint32_t* vals_alt,
                             int n, int bits, const SortScratch& s, unsigned* err, cudaStream_t st,
                             int* launches) {
    return sort_pairs<uint32_t>(keys, vals, keys_alt, vals_alt, n, bits, s, err, st, launches);
}

}  // namespace vpm
