// Device-wide primitives: exclusive scan and LSD radix sort of (key, value)
// pairs. Both are single-pass-per-digit designs with decoupled look-back: a
// tile publishes its aggregate, then accumulates predecessors' published
// values until it meets an inclusive prefix. Tiles take their index from an
// atomic ticket, so a tile only ever waits on tiles that are already running;
// every wait is bounded by kSpinLimit polls (ERR_TIMEOUT on expiry).
#pragma once

#include "vpm_common.cuh"

namespace vpm {

struct ScanScratch {
    uint64_t* status = nullptr;   // one word per tile
    unsigned* ticket = nullptr;   // one counter
    int max_tiles = 0;
};

struct SortScratch {
    uint32_t* status = nullptr;   // passes * tiles * 256 words
    unsigned* tickets = nullptr;  // one counter per pass
    uint32_t* hist = nullptr;     // 8 * 256 counts, then offsets
    int max_tiles = 0;
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kSortThreads = 256;
// Items per thread of a radix pass: 16 for 32-bit keys, 8 for 64-bit keys
// (shared-memory staging of one tile stays under 48 KB).
template <typename K>
struct SortItems { static constexpr int value = sizeof(K) == 4 ? 16 : 8; };
constexpr int kSortTileMin = kSortThreads * 8;  // smallest tile: sizes the look-back scratch

__host__ __device__ inline int scan_tiles(long long n) { return ceil_div(n > 0 ? n : 1, kScanTile); }
// Upper bound on the tiles of any radix pass over n keys.
__host__ __device__ inline int sort_tiles(long long n) { return ceil_div(n > 0 ? n : 1, kSortTileMin); }

// out[i] = sum_{j<i} in[i]; *total (if non-null) = sum of all. Values are
// 32-bit; sums must stay below 2^62. The scratch must be zeroed by the caller
// before each call (status words and ticket); scan_exclusive does that.
cudaError_t scan_exclusive(const uint32_t* in, uint32_t* out, int n, uint32_t* total,
                           const ScanScratch& s, unsigned* err, cudaStream_t st);

// Stable LSD sort of (key, value) pairs on the low `bits` bits of the keys
// (8-bit digits; 64- or 32-bit keys). Inputs are overwritten; on return the sorted data is in
// (*keys, *vals), which may point at either buffer pair.
cudaError_t radix_sort_pairs(uint64_t** keys, uint32_t** vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             int n, int bits, const SortScratch& s, unsigned* err, cudaStream_t st,
                             int* launches);
cudaError_t radix_sort_pairs(uint32_t** keys, uint32_t** vals, uint32_t* keys_alt, uint32_t* vals_alt,
                             int n, int bits, const SortScratch& s, unsigned* err, cudaStream_t st,
                             int* launches);

}  // namespace vpm
