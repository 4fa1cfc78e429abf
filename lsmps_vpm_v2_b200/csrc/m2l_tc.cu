// List-2 M2L of the mixed form on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulator in TMEM).
//
// With scaled expansions a~_k = a_k / r^k and b~_p = r^p b_p (r the cell
// length of the level) a list-2 pair at the integer offset tau in {-3..3}^2
// translates as b~ = T_tau a~ with 49 level-independent operators (the
// algebra of fmm2D.cpp:471-481, the same operators as the FP64 kernel). As
// real matrices, [Re b~; Im b~] = [[Tr, -Ti], [Ti, Tr]] [Re a~; Im a~]:
// N = 2P output rows, K = 2(P+1) inputs.
//
// A block owns a tile of 128 target cells (one per TMEM lane / thread) and
// loops over the 49 offsets: for offset tau, row m of the A tile is a~ of
// the list-2 source of cell m at that offset (zero if none), B is T_tau, and
// D[128 x N] += A B^T accumulates in TMEM across all offsets. Each product is
// split as 3xTF32 (a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulation), so
// the result carries about 21 significant bits. Operands are staged into
// shared memory in the canonical K-major no-swizzle layout by cp.async with
// zero fill, two stages deep: the copies for offset tau overlap the MMAs of
// the previous offset, whose completion (tcgen05.commit -> mbarrier) frees
// the stage. List-4 sources (coarser leaves at arbitrary offsets) are added
// afterwards in FP64 by m2l_list4_add.
#include "fmm2d.cuh"

#include <complex>
#include <cstring>
#include <vector>

namespace vpm {

namespace {

// The reference's binComb (32-bit, wrapping, truncating divisions) or the
// exact binomial coefficient, for the M2L coefficients on the host.
long long binom_m2l_host(int n, int k, bool exact) {
    if (k > n) return 0;
    if (exact) {
        long long c = 1;
        for (int i = 1; i <= k; ++i) c = c * (n - k + i) / i;
        return c;
    }
    const int inv = n - k, mx = inv > k ? inv : k, mn = inv > k ? k : inv;
    int32_t c = 1;
    for (int i = n; i > mx; --i) c = (int32_t)((uint32_t)c * (uint32_t)i);
    for (int i = mn; i > 1; --i) c /= i;
    return c;
}

constexpr int kTcRows = 128;
constexpr int kTcStages = 2;
constexpr int kTcMaxK = 48;   // K_pad = round_up(2 (P+1), 8)
constexpr int kTcMaxN = 48;   // N_pad = round_up(2 P, 16)

__host__ __device__ inline int tc_kpad(int P) { return ((2 * (P + 1) + 7) / 8) * 8; }
__host__ __device__ inline int tc_npad(int P) { return ((2 * P + 15) / 16) * 16; }

// Float offset of element (row, k) in a canonical K-major no-swizzle tile:
// 8-row x 16-byte core matrices, K-adjacent ones 128 B apart (LBO), row
// groups KC * 128 B apart (SBO), KC = K_pad / 4.
__host__ __device__ inline int canon_off(int row, int k, int KC) {
    return (((row >> 3) * KC + (k >> 2)) * 32) + (row & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool full) {
    const int n = full ? 16 : 0;  // 0: zero-fill the 16 bytes
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;  // descriptor version
    return d;         // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = n.
__host__ __device__ inline uint32_t make_idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    #pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Scaled multipole rows of every cell: hi and lo TF32 parts of
// [Re a~_0..Re a~_P, Im a~_0..Im a~_P, 0...] (K_pad floats each).
__global__ void m2l_rows_tf32(Tree2D t, const double2* __restrict__ a, float* __restrict__ rows, int P, int KP,
                              unsigned* err) {
    if (fatal(err)) return;
    const int nc = t.info->n_cells;
    const double root = t.geom->root;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)nc * KP;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i / KP), k = (int)(i - (long long)c * KP);
        float v = 0.f;
        if (k < 2 * (P + 1)) {
            const int kk = k <= P ? k : k - (P + 1);
            const double rinv = ldexp(1.0, (int)t.c_level[c]) / root;
            double s = 1.0;
            for (int e = 0; e < kk; ++e) s *= rinv;
            const double2 ak = a[(size_t)c * (P + 1) + kk];
            v = (float)((k <= P ? ak.x : ak.y) * s);
        }
        const float hi = tf32_round(v);
        rows[(size_t)c * 2 * KP + k] = hi;
        rows[(size_t)c * 2 * KP + KP + k] = v - hi;
    }
}

__global__ void __launch_bounds__(kTcRows)
m2l2d_tc(Tree2D t, Lists2D l, const float* __restrict__ rows, const float* __restrict__ ops,
         double2* __restrict__ b, int P, int KP, int NP, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ uint64_t s_bar[kTcStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_any[49];
    __shared__ int s_stop;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int KC = KP / 4;
    const int a_floats = kTcRows * KP, b_floats = NP * KP;
    const int stage_floats = 2 * a_floats + 2 * b_floats;
    float* stage0 = reinterpret_cast<float*>(tc_smem);
    int* s_src = reinterpret_cast<int*>(stage0 + kTcStages * stage_floats);  // [49][128]
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int ntiles = c_end > c_begin ? (c_end - c_begin + kTcRows - 1) / kTcRows : 0;
    if (tid == 0) s_stop = fatal(err);
    if (tid < kTcStages) mbar_init(&s_bar[tid], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    if (s_stop || (int)blockIdx.x >= ntiles) return;  // uniform, before any TMEM is held
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(64u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = make_idesc_tf32(NP);
    uint32_t phase[kTcStages] = {0u, 0u};
    bool pending[kTcStages] = {false, false};
    bool ok = true;
    const double root = t.geom->root;

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int c = c_begin + tile * kTcRows + tid;
        const bool valid = c < c_end;
        // offset table of the tile
        for (int i = tid; i < 49; i += kTcRows) s_any[i] = 0;
        for (int s = 0; s < 49; ++s) s_src[s * kTcRows + tid] = -1;
        __syncthreads();
        if (valid) {
            const int n2 = l.l2_n[c];
            for (int k = 0; k < n2; ++k) {
                const int slot = l.l2_slot[(size_t)c * kList2Cap + k];
                s_src[slot * kTcRows + tid] = l.l2_src[(size_t)c * kList2Cap + k];
                s_any[slot] = 1;
            }
        }
        __syncthreads();
        int issued = 0;   // MMA groups issued for this tile
        int it = 0;       // staged offsets
        int prev_stage = -1;
        for (int slot = 0; slot <= 49; ++slot) {
            const bool have = slot < 49 && s_any[slot];
            if (have) {
                const int st = it % kTcStages;
                // the stage's previous MMAs must be done before it is overwritten
                if (pending[st]) {
                    if (!mbar_wait(&s_bar[st], phase[st])) ok = false;
                    phase[st] ^= 1u;
                    pending[st] = false;
                }
                float* A_hi = stage0 + st * stage_floats;
                float* A_lo = A_hi + a_floats;
                float* B_hi = A_lo + a_floats;
                float* B_lo = B_hi + b_floats;
                const int src = s_src[slot * kTcRows + tid];
                const float* row = rows + (size_t)(src >= 0 ? src : 0) * 2 * KP;
                for (int kc = 0; kc < KC; ++kc) {
                    const int off = canon_off(tid, 4 * kc, KC);
                    cp_async16(smem_u32(A_hi + off), row + 4 * kc, src >= 0);
                    cp_async16(smem_u32(A_lo + off), row + KP + 4 * kc, src >= 0);
                }
                const float* op = ops + (size_t)slot * 2 * b_floats;  // hi then lo, canonical
                for (int q = tid; q < 2 * b_floats / 4; q += kTcRows)
                    cp_async16(smem_u32(B_hi + 4 * q), op + 4 * q, true);
                cp_async_commit();
            }
            // issue the MMAs of the previously staged offset
            if (prev_stage >= 0) {
                if (have) cp_async_wait<1>();
                else cp_async_wait<0>();
                fence_proxy_async();
                __syncthreads();
                if (tid == 0 && ok) {
                    tc_fence_after();
                    const float* A_hi = stage0 + prev_stage * stage_floats;
                    const float* A_lo = A_hi + a_floats;
                    const float* B_hi = A_lo + a_floats;
                    const float* B_lo = B_hi + b_floats;
                    const uint32_t sbo = (uint32_t)KC * 128u;
                    for (int ks = 0; ks < KP / 8; ++ks) {
                        const uint32_t ko = (uint32_t)ks * 256u;
                        const uint64_t ah = make_desc(smem_u32(A_hi) + ko, 128u, sbo);
                        const uint64_t al = make_desc(smem_u32(A_lo) + ko, 128u, sbo);
                        const uint64_t bh = make_desc(smem_u32(B_hi) + ko, 128u, sbo);
                        const uint64_t bl = make_desc(smem_u32(B_lo) + ko, 128u, sbo);
                        mma_tf32(tmem, ah, bh, idesc, issued > 0 || ks > 0 ? 1u : 0u);
                        mma_tf32(tmem, ah, bl, idesc, 1u);
                        mma_tf32(tmem, al, bh, idesc, 1u);
                    }
                    mma_commit(&s_bar[prev_stage]);
                }
                pending[prev_stage] = true;
                ++issued;
                __syncthreads();
                prev_stage = -1;
            }
            if (have) {
                prev_stage = it % kTcStages;
                ++it;
            }
        }
        // all MMAs of the tile complete
        for (int st = 0; st < kTcStages; ++st) {
            if (pending[st]) {
                if (!mbar_wait(&s_bar[st], phase[st])) ok = false;
                phase[st] ^= 1u;
                pending[st] = false;
            }
        }
        ok = __syncthreads_and(ok) != 0;  // block-uniform from here on
        tc_fence_after();
        // epilogue: this thread's TMEM lane holds row tid of D
        float d[kTcMaxN];
        for (int j = 0; j < NP; ++j) d[j] = 0.f;
        if (issued > 0 && ok) {
            const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
            for (int j = 0; j < NP; j += 16) tmem_ld16(lane_addr + (uint32_t)j, d + j);
        }
        if (valid && ok) {
            const double rinv = ldexp(1.0, (int)t.c_level[c]) / root;
            double rk = 1.0;
            b[(size_t)c * (P + 1)] = make_double2(0.0, 0.0);
            for (int p = 1; p <= P; ++p) {
                rk *= rinv;
                b[(size_t)c * (P + 1) + p] = make_double2((double)d[p - 1] * rk, (double)d[P + p - 1] * rk);
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0) set_err(err, ERR_TIMEOUT);
    // every MMA was waited for above (or gave up after a bounded wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u) : "memory");
}

// ---- list-2 M2L per parent: one dense product over all parents ------------
//
// The list-2 sources of the (up to) four children of a parent P are children
// of P's eight neighbours: 32 positions of the 6 x 6 block of child-level
// cells around P's own 2 x 2 children. Position j = 4 k + d (child d of
// neighbour k) sits at (sx, sy) = (2 (k % 3 - 1) + (d & 1), 2 (k / 3 - 1) +
// (d >> 1)) relative to P's first child, and for child q = (qx, qy) it is
// the offset tau = (sx - qx, sy - qy); it is in q's list 2 exactly when it
// is not adjacent to q (some |tau| >= 2). So, with the scaled rows a~ of the
// 32 positions laid side by side (K = 32 x K_pad), all four children's
// b~ come out of one fixed operator:
//   D[parent][q 2P + r] = sum_j sum_k a~_j[k] Op_j[q 2P + r][k],
//   Op_j = T_tau(q, j) for separated (q, j), 0 otherwise,
// a dense GEMM with M = parents, N = 4 x 2P outputs, K = 32 x K_pad. A block
// takes 128 parents (one TMEM lane each) and walks the 32 positions; at
// position j the A tile holds the row of each parent's source there (zero
// when missing), the B tile is Op_j (precomputed, hi and lo TF32 parts), and
// three tcgen05.mma kind::tf32 per 8 K columns (a_hi b_hi + a_hi b_lo +
// a_lo b_hi) accumulate into TMEM. A source row is read once per parent
// that has it in its block (at most 9 parents) instead of once per list-2
// pair. Stages (as many as 220 KB of shared memory hold, up to 6) are filled
// by cp.async (zero fill for missing sources), 8 rows x 4 chunks per warp
// instruction; the MMAs of the last two positions stay in flight while the
// other stages load, and tcgen05.commit on a stage's mbarrier releases it.
// The epilogue unscales in FP64 and writes b of every child.
constexpr int kParRows = 128;
constexpr int kParMaxP = 16;
constexpr int kParMaxStages = 6;
constexpr int kParPos = 32;

__host__ __device__ inline int par_npad(int P) { return ((8 * P + 15) / 16) * 16; }
__host__ __device__ inline int par_tmem_cols(int P) {
    const int n = par_npad(P);
    int c = 32;
    while (c < n) c <<= 1;
    return c;
}
__host__ __device__ inline size_t par_stage_floats(int P) {
    const int KP = tc_kpad(P);
    return (size_t)2 * kParRows * KP + (size_t)2 * par_npad(P) * KP;
}
inline int par_stages(int P) {
    const size_t budget = 220 * 1024 - sizeof(int) * kParPos * kParRows;
    const int s = (int)(budget / (sizeof(float) * par_stage_floats(P)));
    return s < 2 ? 0 : (s > kParMaxStages ? kParMaxStages : s);
}

template <int N>
__device__ __forceinline__ void cp_async_wait_n(int pending) {
    if (pending >= N) cp_async_wait<N>();
    else if constexpr (N > 0) cp_async_wait_n<N - 1>(pending);
}

__global__ void __launch_bounds__(kParRows)
m2l_parent_tc(Tree2D t, const int32_t* __restrict__ blk, const float* __restrict__ rows,
              const float* __restrict__ ops, double2* __restrict__ b, int P, int KP, int NP, int S, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char par_smem[];
    __shared__ uint64_t s_bar[kParMaxStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_any[kParPos];
    __shared__ int s_stop;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int KC = KP / 4;
    const int a_floats = kParRows * KP, b_floats = NP * KP;
    const int stage_floats = 2 * a_floats + 2 * b_floats;
    float* stage0 = reinterpret_cast<float*>(par_smem);
    int* s_src = reinterpret_cast<int*>(stage0 + (size_t)S * stage_floats);   // [32][128]
    const int np = t.info->n_cells - t.info->n_leaves;   // non-leaf cells; the root is the first
    const int nparents = np > 1 ? np - 1 : 0;
    const int ntiles = (nparents + kParRows - 1) / kParRows;
    // list 2 not given by the offset rule: every b is zeroed here and
    // m2l_list4_add adds lists 2 and 4 pair by pair
    const bool irregular = t.info->l2_irregular != 0;
    const uint32_t tcols = (uint32_t)par_tmem_cols(P);
    if (tid == 0) s_stop = fatal(err);
    if (tid < S) mbar_init(&s_bar[tid], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    if (s_stop || (int)blockIdx.x >= ntiles) return;  // uniform, before any TMEM is held
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = make_idesc_tf32(NP);
    uint32_t phase_bits = 0u;     // bit st: parity of stage st's next completion
    uint32_t pending_bits = 0u;   // bit st: MMAs of stage st issued and not yet waited for
    bool ok = true;
    const double root = t.geom->root;
    const uint32_t sbo = (uint32_t)KC * 128u;

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int pi = 1 + tile * kParRows + tid;
        const int par = pi < np ? t.nonleaf[pi] : -1;
        if (tid < kParPos) s_any[tid] = 0;
        __syncthreads();
        if (par >= 0 && !irregular) {
            const int4* bp = reinterpret_cast<const int4*>(blk + (size_t)par * kParPos);
            #pragma unroll
            for (int q = 0; q < kParPos / 4; ++q) {
                const int4 v = __ldg(bp + q);
                const int vv[4] = {v.x, v.y, v.z, v.w};
                #pragma unroll
                for (int u = 0; u < 4; ++u) {
                    s_src[(4 * q + u) * kParRows + tid] = vv[u];
                    if (vv[u] >= 0) s_any[4 * q + u] = 1;
                }
            }
        } else {
            for (int j = 0; j < kParPos; ++j) s_src[j * kParRows + tid] = -1;
        }
        __syncthreads();
        // positions that hold a source for some parent of the tile, in order
        uint32_t pos_mask = 0u;
        for (int j = 0; j < kParPos; ++j)
            if (s_any[j]) pos_mask |= 1u << j;
        const int npos = __popc(pos_mask);
        auto pos_at = [&](int i) {   // the i-th set bit of pos_mask
            uint32_t m = pos_mask;
            for (int r = 0; r < i; ++r) m &= m - 1u;
            return __ffs(m) - 1;
        };
        // stage i of the walk: position pos_at(i) into stage i % S
        auto load = [&](int i) {
            const int st = i % S;
            if (pending_bits & (1u << st)) {   // the stage's previous MMAs must be done
                if (!mbar_wait(&s_bar[st], (phase_bits >> st) & 1u)) ok = false;
                phase_bits ^= 1u << st;
                pending_bits &= ~(1u << st);
            }
            const int j = pos_at(i);
            float* A_hi = stage0 + (size_t)st * stage_floats;
            float* A_lo = A_hi + a_floats;
            float* B_hi = A_lo + a_floats;
            // A rows: warp w copies rows 32 w .. 32 w + 31 in groups of 8, lane
            // (r = lane & 7, c = lane >> 3) chunks c, c + 4, ... of row r (hi
            // chunks, then lo): one instruction touches 8 rows (not 32 scattered
            // ones) and writes 8 distinct 16-byte bank groups.
            const int lane = tid & 31;
            for (int g = 0; g < 4; ++g) {
                const int row = 32 * warp + 8 * g + (lane & 7);
                const int src = s_src[j * kParRows + row];
                const float* rp = rows + (size_t)(src >= 0 ? src : 0) * 2 * KP;
                for (int c = lane >> 3; c < 2 * KC; c += 4) {
                    const int part = c >= KC ? 1 : 0, kc = c - part * KC;
                    cp_async16(smem_u32((part ? A_lo : A_hi) + canon_off(row, 4 * kc, KC)), rp + part * KP + 4 * kc,
                               src >= 0);
                }
            }
            const float* op = ops + (size_t)j * 2 * b_floats;   // hi then lo, canonical
            for (int q = tid; q < 2 * b_floats / 4; q += kParRows) cp_async16(smem_u32(B_hi + 4 * q), op + 4 * q, true);
        };
        // positions staged ahead of the MMAs: S - lag, where the MMAs of the
        // last `lag` positions may still run while their stages wait for reuse
        const int ahead = S - (S >= 4 ? 2 : 1);
        int loaded = 0;
        for (; loaded < npos && loaded < ahead; ++loaded) {
            load(loaded);
            cp_async_commit();
        }
        for (int i = 0; i < npos; ++i) {
            // loads issued: 0 .. loaded-1; the ones after i may stay in flight
            cp_async_wait_n<kParMaxStages - 1>(loaded - 1 - i);
            fence_proxy_async();
            __syncthreads();
            const int st = i % S;
            if (tid == 0 && ok) {
                tc_fence_after();
                const float* A_hi = stage0 + (size_t)st * stage_floats;
                const float* A_lo = A_hi + a_floats;
                const float* B_hi = A_lo + a_floats;
                const float* B_lo = B_hi + b_floats;
                for (int ks = 0; ks < KP / 8; ++ks) {
                    const uint32_t ko = (uint32_t)ks * 256u;
                    const uint64_t ah = make_desc(smem_u32(A_hi) + ko, 128u, sbo);
                    const uint64_t al = make_desc(smem_u32(A_lo) + ko, 128u, sbo);
                    const uint64_t bh = make_desc(smem_u32(B_hi) + ko, 128u, sbo);
                    const uint64_t bl = make_desc(smem_u32(B_lo) + ko, 128u, sbo);
                    mma_tf32(tmem, ah, bh, idesc, i > 0 || ks > 0 ? 1u : 0u);
                    mma_tf32(tmem, ah, bl, idesc, 1u);
                    mma_tf32(tmem, al, bh, idesc, 1u);
                }
                mma_commit(&s_bar[st]);
            }
            pending_bits |= 1u << st;
            if (loaded < npos) {
                load(loaded);
                ++loaded;
            }
            cp_async_commit();   // one group per iteration (possibly empty)
        }
        // all MMAs of the tile complete
        for (int st = 0; st < S; ++st) {
            if (pending_bits & (1u << st)) {
                if (!mbar_wait(&s_bar[st], (phase_bits >> st) & 1u)) ok = false;
                phase_bits ^= 1u << st;
                pending_bits &= ~(1u << st);
            }
        }
        ok = __syncthreads_and(ok) != 0;   // block-uniform from here on
        tc_fence_after();
        // epilogue: this thread's TMEM lane holds the row of parent `par`
        if (ok) {
            int chi[4] = {-1, -1, -1, -1};
            double rinv = 0.0;
            if (par >= 0) {
                const unsigned m = t.c_chmask[par];
                const int c0 = t.c_child0[par];
                #pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (m & (1u << q)) chi[q] = c0 + __popc(m & ((1u << q) - 1u));
                rinv = ldexp(1.0, (int)t.c_level[par] + 1) / root;   // 1 / child cell length
                #pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (chi[q] >= 0) b[(size_t)chi[q] * (P + 1)] = make_double2(0.0, 0.0);
            }
            const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
            for (int j0 = 0; j0 < NP; j0 += 16) {
                float d[16];
                if (npos > 0) tmem_ld16(lane_addr + (uint32_t)j0, d);
                else
                    for (int u = 0; u < 16; ++u) d[u] = 0.f;
                if (par < 0) continue;
                #pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int n = j0 + u;
                    const int q = n / (2 * P), r = n - q * 2 * P;
                    if (q >= 4 || chi[q] < 0) continue;
                    const int pp = r < P ? r + 1 : r - P + 1;
                    double rk = 1.0;
                    for (int e = 0; e < pp; ++e) rk *= rinv;
                    double* bc = reinterpret_cast<double*>(b + (size_t)chi[q] * (P + 1));
                    bc[2 * pp + (r < P ? 0 : 1)] = (double)d[u] * rk;
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0) set_err(err, ERR_TIMEOUT);
    // every MMA was waited for above (or gave up after a bounded wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
}

// ---- list-2 M2L per parent on the FP32 pipes ----------------------------------
//
// The same per-parent contraction as m2l_parent_tc, evaluated through the
// structure of the operator: with C[p][0] = -1/p and C[p][k] = -m2l[p][k]
// (k >= 1, the reference's M2L coefficients, fmm2D.cpp:471-481),
//   T_tau[p][k] = tau^-p C[p][k] tau^-k,
// so a source's contribution to one child is a diagonal scaling of its
// scaled moments by tau^-k, one real P x (P+1) matrix applied to the real
// and imaginary parts, and a diagonal scaling by tau^-p: about 212 FP32
// operations per (child, source) instead of 288 for the dense 2P x 2(P+1)
// operator. C and the powers tau^-k of the 49 offsets are kernel parameters
// (constant bank, read as broadcast operands). A block takes 32 parents, one
// per lane; warps q and q + 4 compute child q of every parent over positions
// 0..15 and 16..31. The block first gathers the scaled moments of all 32 x 32
// (position, parent) sources into shared memory (one round of independent
// loads, FP64 moments rounded once after scaling by the child level's
// 1 / length^k); then each warp walks its positions not adjacent to its
// child, and the first half's sums are added to the second's. Sums run in
// position order, so the result does not depend on the schedule.
constexpr int kPF32MaxP = 16;

template <int P>
struct ParF32Args {
    float C[P][P + 1];      // C[p - 1][k]
    float2 tp[49][P + 1];   // tau^-k, k = 0 .. P, slot = (tau_y + 3) 7 + tau_x + 3
};

template <int P>
__global__ void __launch_bounds__(256)
m2l_parent_f32(Tree2D t, const int32_t* __restrict__ blk, const double2* __restrict__ a, double2* __restrict__ b,
               const __grid_constant__ ParF32Args<P> args, int part, const unsigned* __restrict__ top_level,
               unsigned* err) {
    constexpr int Q = P + 1;
    extern __shared__ float2 pf_A[];             // [32 positions][Q][32 parents]
    __shared__ int s_src[kParPos][32];           // [position][parent]
    __shared__ double s_rp[32][Q];               // [parent][k]: (1 / child length)^k
    __shared__ float s_half[4][2 * P][32];       // the first position half's sums [child][output][parent]
    if (fatal(err)) return;
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int q = wq & 3, half = wq >> 2;
    const int qx = q & 1, qy = q >> 1;
    const int np = t.info->n_cells - t.info->n_leaves;   // non-leaf cells; the root is the first
    // parents [pb, pe) of the non-leaf list (level-major): all, or those at
    // levels >= *top_level (part 1: their children's sources are final once
    // the small cells' moments are), or the others (part 2)
    int pb = 1, pe = np;
    if (part != 0) {
        const int top = (int)*top_level;
        const int split = max(1, t.info->level_start[top] - t.info->leaf_start[top]);
        if (part == 1) pb = max(pb, split);
        else pe = min(pe, split);
    }
    const bool irregular = t.info->l2_irregular != 0;
    const double root = t.geom->root;
    for (int tile = blockIdx.x; pb + tile * 32 < pe; tile += gridDim.x) {
        const int pi = pb + tile * 32 + lane;
        const int par = pi < pe ? t.nonleaf[pi] : -1;
        if (wq == 0) {
            const double rinv = par >= 0 ? ldexp(1.0, (int)t.c_level[par] + 1) / root : 0.0;
            double r = 1.0;
            #pragma unroll
            for (int k = 0; k < Q; ++k) {
                s_rp[lane][k] = r;
                r *= rinv;
            }
        }
        if (wq == 1) {
            if (par >= 0 && !irregular) {
                const int4* bp = reinterpret_cast<const int4*>(blk + (size_t)par * kParPos);
                #pragma unroll
                for (int u = 0; u < kParPos / 4; ++u) {
                    const int4 v = __ldg(bp + u);
                    s_src[4 * u][lane] = v.x;
                    s_src[4 * u + 1][lane] = v.y;
                    s_src[4 * u + 2][lane] = v.z;
                    s_src[4 * u + 3][lane] = v.w;
                }
            } else {
                for (int j = 0; j < kParPos; ++j) s_src[j][lane] = -1;
            }
        }
        __syncthreads();
        // gather: item (j, m, k), k fastest (a source's moments are contiguous)
        for (int idx = threadIdx.x; idx < kParPos * 32 * Q; idx += blockDim.x) {
            const int jm = idx / Q, k = idx - jm * Q;
            const int j = jm >> 5, m = jm & 31;
            const int src = s_src[j][m];
            float2 v = make_float2(0.f, 0.f);
            if (src >= 0) {
                const double2 av = __ldg(a + (size_t)src * Q + k);
                const double sc = s_rp[m][k];
                v = make_float2((float)(av.x * sc), (float)(av.y * sc));
            }
            pf_A[(j * Q + k) * 32 + m] = v;
        }
        __syncthreads();
        float accr[P], acci[P];
        #pragma unroll
        for (int p = 0; p < P; ++p) accr[p] = acci[p] = 0.f;
        for (int j = half * (kParPos / 2); j < (half + 1) * (kParPos / 2); ++j) {
            const int k8 = j >> 2, d = j & 3, nb = k8 < 4 ? k8 : k8 + 1;
            const int tx = 2 * (nb % 3 - 1) + (d & 1) - qx, ty = 2 * (nb / 3 - 1) + (d >> 1) - qy;
            if (tx >= -1 && tx <= 1 && ty >= -1 && ty <= 1) continue;   // adjacent: not in this child's list 2
            const int slot = (ty + 3) * 7 + tx + 3;
            float ar[Q], ai[Q];
            #pragma unroll
            for (int k = 0; k < Q; ++k) {
                const float2 v = pf_A[(j * Q + k) * 32 + lane];
                const float2 w = args.tp[slot][k];
                ar[k] = v.x * w.x - v.y * w.y;
                ai[k] = v.x * w.y + v.y * w.x;
            }
            #pragma unroll
            for (int p = 0; p < P; ++p) {
                float br = 0.f, bi = 0.f;
                #pragma unroll
                for (int k = 0; k < Q; ++k) {
                    br = fmaf(args.C[p][k], ar[k], br);
                    bi = fmaf(args.C[p][k], ai[k], bi);
                }
                const float2 w = args.tp[slot][p + 1];
                accr[p] = fmaf(w.x, br, fmaf(-w.y, bi, accr[p]));
                acci[p] = fmaf(w.x, bi, fmaf(w.y, br, acci[p]));
            }
        }
        if (half == 0) {
            #pragma unroll
            for (int p = 0; p < P; ++p) {
                s_half[q][p][lane] = accr[p];
                s_half[q][P + p][lane] = acci[p];
            }
        }
        __syncthreads();
        if (half == 1 && par >= 0) {
            #pragma unroll
            for (int p = 0; p < P; ++p) {
                accr[p] = s_half[q][p][lane] + accr[p];
                acci[p] = s_half[q][P + p][lane] + acci[p];
            }
            const unsigned m = t.c_chmask[par];
            if (m & (1u << q)) {
                const int ch = t.c_child0[par] + __popc(m & ((1u << q) - 1u));
                double2* bc = b + (size_t)ch * Q;
                bc[0] = make_double2(0.0, 0.0);
                #pragma unroll
                for (int p = 0; p < P; ++p) {
                    const double rk = s_rp[lane][p + 1];
                    bc[p + 1] = make_double2((double)accr[p] * rk, (double)acci[p] * rk);
                }
            }
        }
        __syncthreads();
    }
}

template <int P>
cudaError_t launch_m2l_parent_f32(const Tree2D& t, const Lists2D& l, Expansions2D& e, bool exact, unsigned* err,
                                  cudaStream_t st, int part) {
    ParF32Args<P> args;
    for (int p = 1; p <= P; ++p) {
        args.C[p - 1][0] = (float)(-1.0 / (double)p);
        for (int k = 1; k <= P; ++k)
            args.C[p - 1][k] =
                (float)(-(double)binom_m2l_host(p + k - 1, k - 1, exact) * ((k & 1) ? -1.0 : 1.0) / (double)k);
    }
    for (int slot = 0; slot < 49; ++slot) {
        const int dx = slot % 7 - 3, dy = slot / 7 - 3;
        const std::complex<double> inv = (dx == 0 && dy == 0) ? 0.0 : 1.0 / std::complex<double>(dx, dy);
        std::complex<double> w = 1.0;
        for (int k = 0; k <= P; ++k) {
            args.tp[slot][k] = make_float2((float)w.real(), (float)w.imag());
            w *= inv;
        }
    }
    const size_t smem = sizeof(float2) * (size_t)kParPos * (P + 1) * 32;
    cudaError_t r = cudaFuncSetAttribute(m2l_parent_f32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    int occ = 0;
    r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, m2l_parent_f32<P>, 256, smem);
    if (r != cudaSuccess) return r;
    m2l_parent_f32<P><<<148 * (occ > 0 ? occ : 1), 256, smem, st>>>(t, l.l2_blk, e.a, e.b, args, part,
                                                                     t.gbar ? t.gbar + 3 : nullptr, err);
    return cudaGetLastError();
}

// List 4 of every cell (FP64, direct formula of fmm2D.cpp:504-520), added
// to b; with with_list2 on a tree flagged l2_irregular, list 2 as well (the
// per-parent M2L then left b at zero). One warp per cell with sources; the
// warp's lanes form
// G = 32 / P groups, group g takes sources g, g + G, ... and its lane p - 1
// computes that part of b_p; the groups' parts are summed in group order.
__global__ void __launch_bounds__(128)
m2l_list4_add(Tree2D t, Lists2D l, const double2* __restrict__ a, double2* __restrict__ b,
              const double* __restrict__ coef, int P, bool with_list2, unsigned* err) {
    if (fatal(err)) return;
    const double* g_m2l = coef + kCoefM2L;
    const int lane = threadIdx.x & 31;
    const int G = P <= 32 ? 32 / P : 1;
    const int grp = lane / P, p = lane - grp * P + 1;
    const bool on = grp < G;
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const bool with_l2 = with_list2 && t.info->l2_irregular != 0;
    for (int c = c_begin + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < c_end; c += warps) {
        const int n2 = with_l2 ? l.l2_n[c] : 0;
        const int ns = n2 + l.l4_n[c];
        if (ns == 0) continue;
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        double2 acc = make_double2(0.0, 0.0);
        if (on) {
            for (int si = grp; si < ns; si += G) {
                const int src = si < n2 ? l.l2_src[(size_t)c * kList2Cap + si]
                                        : l.l4_src[(size_t)c * kList4Cap + (si - n2)];
                const double2 w = cinv(make_double2(t.c_cx[src] - zx, t.c_cy[src] - zy));
                const double2* A = a + (size_t)src * (P + 1);
                double2 wp = make_double2(1.0, 0.0);
                for (int e = 0; e < p; ++e) wp = cmul(wp, w);   // w^p
                double2 sv = cscale(cmul(A[0], wp), 1.0 / (double)p);
                const double* cf = g_m2l + p * (kMaxP + 1);
                double2 wk = wp;
                for (int k = 1; k <= P; ++k) {
                    wk = cmul(wk, w);  // w^(p+k)
                    sv = cfma(cscale(A[k], cf[k]), wk, sv);
                }
                acc = csub(acc, sv);
            }
        }
        // lane p - 1 of group 0 adds the other groups' parts in group order
        for (int g = 1; g < G; ++g) {
            const int from = g * P + (lane < P ? lane : 0);
            const double vx = __shfl_sync(0xffffffffu, acc.x, from), vy = __shfl_sync(0xffffffffu, acc.y, from);
            if (lane < P) acc = make_double2(acc.x + vx, acc.y + vy);
        }
        if (lane < P) {
            double2* bp = &b[(size_t)c * (P + 1) + lane + 1];
            *bp = cadd(*bp, acc);
        }
    }
}

}  // namespace

bool m2l_tc_supported(int P) { return P >= 1 && P <= 20; }
bool m2l_parent_supported(int P) { return P >= 1 && P <= kParMaxP && par_stages(P) >= 2; }

size_t m2l_tc_rows_bytes(int cap_cells) { return sizeof(float) * (size_t)cap_cells * 2 * kTcMaxK; }
size_t m2l_tc_ops_bytes() {
    const size_t per_offset = sizeof(float) * (size_t)49 * 2 * kTcMaxN * kTcMaxK;
    const size_t per_parent = sizeof(float) * (size_t)kParPos * 2 * par_npad(kParMaxP) * tc_kpad(kParMaxP);
    return per_offset > per_parent ? per_offset : per_parent;
}

// Op_j of m2l_parent_tc for the 32 block positions j: rows q 2P + r (child q,
// output r: Re b~_1..P, Im b~_1..P), columns k (Re a~_0..P, Im a~_0..P), the
// real form of T_tau with tau = position - child, zero where the position is
// adjacent to the child; TF32 hi and lo parts, each in the canonical layout
// (from the same double operators as set_m2l_operators2d: op[slot][k][p-1],
// slot = (tau_y + 3) 7 + tau_x + 3). Synchronises.
cudaError_t set_m2l_parent_operators(int P, const double2* op_dev, float* dst, cudaStream_t st) {
    if (!m2l_parent_supported(P)) return cudaErrorInvalidValue;
    const int KP = tc_kpad(P), NP = par_npad(P), KC = KP / 4;
    std::vector<double2> op((size_t)49 * (P + 1) * P);
    cudaError_t e = cudaMemcpyAsync(op.data(), op_dev, sizeof(double2) * op.size(), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    const int bf = NP * KP;
    std::vector<float> h((size_t)kParPos * 2 * bf, 0.f);
    auto tf32 = [](float x) {
        uint32_t u;
        std::memcpy(&u, &x, 4);
        if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
        float r;
        std::memcpy(&r, &u, 4);
        return r;
    };
    for (int j = 0; j < kParPos; ++j) {
        const int k8 = j >> 2, d = j & 3, nb = k8 < 4 ? k8 : k8 + 1;
        const int sx = 2 * (nb % 3 - 1) + (d & 1), sy = 2 * (nb / 3 - 1) + (d >> 1);
        float* hi = h.data() + (size_t)j * 2 * bf;
        float* lo = hi + bf;
        for (int q = 0; q < 4; ++q) {
            const int tx = sx - (q & 1), ty = sy - (q >> 1);
            if (tx >= -1 && tx <= 1 && ty >= -1 && ty <= 1) continue;   // adjacent: not in q's list 2
            const int slot = (ty + 3) * 7 + (tx + 3);
            for (int p = 1; p <= P; ++p) {
                for (int k = 0; k <= P; ++k) {
                    const double2 T = op[((size_t)slot * (P + 1) + k) * P + (p - 1)];
                    // Re b_p: Tr Re a_k - Ti Im a_k ; Im b_p: Ti Re a_k + Tr Im a_k
                    const double v[4] = {T.x, -T.y, T.y, T.x};
                    const int rows_[4] = {q * 2 * P + p - 1, q * 2 * P + p - 1, q * 2 * P + P + p - 1,
                                          q * 2 * P + P + p - 1};
                    const int cols_[4] = {k, P + 1 + k, k, P + 1 + k};
                    for (int u = 0; u < 4; ++u) {
                        const float f = (float)v[u];
                        const float fh = tf32(f);
                        const int o = canon_off(rows_[u], cols_[u], KC);
                        hi[o] = fh;
                        lo[o] = f - fh;
                    }
                }
            }
        }
    }
    e = cudaMemcpyAsync(dst, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

bool m2l_parent_f32_supported(int P) { return P >= 1 && P <= kPF32MaxP; }

cudaError_t fmm2d_m2l_parent_f32(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, bool exact,
                                 unsigned* err, cudaStream_t st, int* launches, int part) {
    if (!m2l_parent_f32_supported(P) || !l.l2_blk || !t.nonleaf || (part != 0 && !t.gbar))
        return cudaErrorInvalidValue;
    cudaError_t r;
    switch (P) {
#define VPM_PF32_CASE(PP) \
    case PP: r = launch_m2l_parent_f32<PP>(t, l, e, exact, err, st, part); break;
        VPM_PF32_CASE(1) VPM_PF32_CASE(2) VPM_PF32_CASE(3) VPM_PF32_CASE(4) VPM_PF32_CASE(5) VPM_PF32_CASE(6)
        VPM_PF32_CASE(7) VPM_PF32_CASE(8) VPM_PF32_CASE(9) VPM_PF32_CASE(10) VPM_PF32_CASE(11) VPM_PF32_CASE(12)
        VPM_PF32_CASE(13) VPM_PF32_CASE(14) VPM_PF32_CASE(15) VPM_PF32_CASE(16)
#undef VPM_PF32_CASE
        default: return cudaErrorInvalidValue;
    }
    if (r != cudaSuccess) return r;
    *launches += 1;
    if (part != 0) return cudaGetLastError();
    return fmm2d_m2l_list4(t, l, e, P, err, st, launches);
}

cudaError_t fmm2d_m2l_list4(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                            int* launches) {
    m2l_list4_add<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, e.coef, P, true, err);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t fmm2d_m2l_parent(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, float* rows,
                             const float* ops, unsigned* err, cudaStream_t st, int* launches) {
    if (!m2l_parent_supported(P) || !l.l2_blk || !t.nonleaf) return cudaErrorInvalidValue;
    const int KP = tc_kpad(P), NP = par_npad(P), S = par_stages(P);
    m2l_rows_tf32<<<148 * 8, 256, 0, st>>>(t, e.a, rows, P, KP, err);
    const size_t smem = sizeof(float) * (size_t)S * par_stage_floats(P) + sizeof(int) * kParPos * kParRows;
    cudaError_t r = cudaFuncSetAttribute(m2l_parent_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    m2l_parent_tc<<<148, kParRows, smem, st>>>(t, l.l2_blk, rows, ops, e.b, P, KP, NP, S, err);
    m2l_list4_add<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, e.coef, P, true, err);
    *launches += 3;
    return cudaGetLastError();
}

// The 49 list-2 operators as real N_pad x K_pad matrices, split into TF32 hi
// and lo parts, each in the canonical shared-memory layout (from the same
// double operators as set_m2l_operators2d: op[slot][k][p-1]). Synchronises.
cudaError_t set_m2l_tc_operators(int P, const double2* op_dev, float* dst, cudaStream_t st) {
    const int KP = tc_kpad(P), NP = tc_npad(P), KC = KP / 4;
    std::vector<double2> op((size_t)49 * (P + 1) * P);
    cudaError_t e = cudaMemcpyAsync(op.data(), op_dev, sizeof(double2) * op.size(), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    const int bf = NP * KP;
    std::vector<float> h((size_t)49 * 2 * bf, 0.f);
    auto tf32 = [](float x) {
        // round to nearest (ties away) at 10 mantissa bits, as cvt.rna.tf32.f32
        uint32_t u;
        std::memcpy(&u, &x, 4);
        if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
        float r;
        std::memcpy(&r, &u, 4);
        return r;
    };
    for (int slot = 0; slot < 49; ++slot) {
        float* hi = h.data() + (size_t)slot * 2 * bf;
        float* lo = hi + bf;
        for (int p = 1; p <= P; ++p) {
            for (int k = 0; k <= P; ++k) {
                const double2 T = op[((size_t)slot * (P + 1) + k) * P + (p - 1)];
                // Re b_p: Tr Re a_k - Ti Im a_k ; Im b_p: Ti Re a_k + Tr Im a_k
                const double v[4] = {T.x, -T.y, T.y, T.x};
                const int rows_[4] = {p - 1, p - 1, P + p - 1, P + p - 1};
                const int cols_[4] = {k, P + 1 + k, k, P + 1 + k};
                for (int q = 0; q < 4; ++q) {
                    const float f = (float)v[q];
                    const float fh = tf32(f);
                    const int o = canon_off(rows_[q], cols_[q], KC);
                    hi[o] = fh;
                    lo[o] = f - fh;
                }
            }
        }
    }
    e = cudaMemcpyAsync(dst, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t fmm2d_m2l_tc(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, float* rows, const float* ops,
                         unsigned* err, cudaStream_t st, int* launches) {
    const int KP = tc_kpad(P), NP = tc_npad(P);
    m2l_rows_tf32<<<148 * 8, 256, 0, st>>>(t, e.a, rows, P, KP, err);
    const size_t smem = sizeof(float) * (size_t)kTcStages * (2 * kTcRows * KP + 2 * NP * KP) +
                        sizeof(int) * 49 * kTcRows;
    cudaError_t r = cudaFuncSetAttribute(m2l2d_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    m2l2d_tc<<<148 * 2, kTcRows, smem, st>>>(t, l, rows, ops, e.b, P, KP, NP, err);
    m2l_list4_add<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, e.coef, P, false, err);
    *launches += 3;
    return cudaGetLastError();
}

}  // namespace vpm
