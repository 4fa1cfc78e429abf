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

#include <cstring>
#include <vector>

namespace vpm {

namespace {

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

// ---- the same scaled list-2 M2L on the FP32 pipes (orders 1..kF32MaxP) ----
//
// b~ = sum over offsets tau of T_tau a~ in FP32. A warp takes 32 / NG
// consecutive target cells, NG = (2P rounded up to 4) / 4 lanes per target,
// each lane four of the target's 2P real outputs. The warp walks the offsets
// present in its targets' lists in increasing order; at offset tau every
// lane applies its four rows of the same operator (shared memory, one
// 16-byte read per input) to the scaled row of its target's source (zero
// when it has none), accumulating in registers. The next offset's rows are
// loaded while the current one is applied. FP32 products and sums carry
// about 24 bits, as the 3xTF32 tensor-core form; the order of the sums is
// fixed.
constexpr int kF32MaxP = 12;
constexpr int kF32Warps = 8;

__host__ __device__ constexpr int f32_rp(int P) { return ((2 * (P + 1) + 3) / 4) * 4; }   // row stride (floats)
__host__ __device__ constexpr int f32_nrp(int P) { return ((2 * P + 3) / 4) * 4; }       // outputs, padded

// Scaled multipole rows [Re a~_0..Re a~_P, Im a~_0..Im a~_P, 0..] in FP32, and
// after the last cell (row n_cells) a row of zeros: the source of an empty slot.
__global__ void m2l_rows_f32(Tree2D t, const double2* __restrict__ a, float* __restrict__ rows, int P, int RP,
                             unsigned* err) {
    if (fatal(err)) return;
    const int nc = t.info->n_cells;
    const double root = t.geom->root;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)(nc + 1) * RP;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i / RP), k = (int)(i - (long long)c * RP);
        float v = 0.f;
        if (c < nc && k < 2 * (P + 1)) {
            const int kk = k <= P ? k : k - (P + 1);
            const double rinv = ldexp(1.0, (int)t.c_level[c]) / root;
            double sc = 1.0;
            for (int e = 0; e < kk; ++e) sc *= rinv;
            const double2 ak = a[(size_t)c * (P + 1) + kk];
            v = (float)((k <= P ? ak.x : ak.y) * sc);
        }
        rows[i] = v;
    }
}

// One instantiation per order P (all loops have constant bounds).
template <int P>
__global__ void __launch_bounds__(32 * kF32Warps)
m2l2d_f32(Tree2D t, Lists2D l, const float* __restrict__ rows, const float* __restrict__ ops,
          double2* __restrict__ b, unsigned* err) {
    extern __shared__ __align__(16) float f32_smem[];
    constexpr int NRP = f32_nrp(P), NG = NRP / 4, TPW = 32 / NG;
    constexpr int RP = f32_rp(P), RQ = RP / 4, K2 = 2 * (P + 1);
    float* s_op = f32_smem;                                                         // [49][K2][NRP]
    int* s_src = reinterpret_cast<int*>(s_op + (size_t)49 * K2 * NRP);              // [warps][49][TPW]
    if (fatal(err)) return;
    for (int i = threadIdx.x; i < 49 * K2 * NRP / 4; i += blockDim.x)
        reinterpret_cast<float4*>(s_op)[i] = reinterpret_cast<const float4*>(ops)[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int tl = lane / NG, g = lane - tl * NG;   // target of the lane, output group
    int* my_src = s_src + (size_t)wib * 49 * TPW;
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int ntasks = (c_end - c_begin + TPW - 1) / TPW;
    const double root = t.geom->root;
    for (int task = blockIdx.x * kF32Warps + wib; task < ntasks; task += gridDim.x * kF32Warps) {
        const int c = c_begin + task * TPW + tl;
        const bool valid = tl < TPW && c < c_end;
        for (int i = lane; i < 49 * TPW; i += 32) my_src[i] = c_end;   // the zero row
        __syncwarp();
        uint32_t m_lo = 0, m_hi = 0;   // offsets present in this target's list
        if (valid && g == 0) {
            const int n2 = l.l2_n[c];
            for (int k = 0; k < n2; ++k) {
                const int slot = l.l2_slot[(size_t)c * kList2Cap + k];
                my_src[slot * TPW + tl] = l.l2_src[(size_t)c * kList2Cap + k];
                if (slot < 32) m_lo |= 1u << slot;
                else m_hi |= 1u << (slot - 32);
            }
        }
        __syncwarp();
        uint64_t mask = ((uint64_t)__reduce_or_sync(0xffffffffu, m_hi) << 32) | __reduce_or_sync(0xffffffffu, m_lo);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        // row of this lane's target's source at offset tau (the zero row when it has none)
        auto load_row = [&](int tau, float4* dst) {
            const int src = valid ? my_src[tau * TPW + tl] : c_end;
            const float4* row = reinterpret_cast<const float4*>(rows + (size_t)src * RP);
            #pragma unroll
            for (int q = 0; q < RQ; ++q) dst[q] = __ldg(row + q);
        };
        auto apply = [&](int tau, const float4* row) {
            const float4* T = reinterpret_cast<const float4*>(s_op + (size_t)tau * K2 * NRP) + g;
            #pragma unroll
            for (int q = 0; q < RQ; ++q) {
                const float av[4] = {row[q].x, row[q].y, row[q].z, row[q].w};
                #pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = 4 * q + u;
                    if (k >= K2) break;
                    const float4 w = T[k * NG];
                    acc[0] = fmaf(w.x, av[u], acc[0]);
                    acc[1] = fmaf(w.y, av[u], acc[1]);
                    acc[2] = fmaf(w.z, av[u], acc[2]);
                    acc[3] = fmaf(w.w, av[u], acc[3]);
                }
            }
        };
        auto next_tau = [&]() {
            const int tt = mask ? __ffsll((long long)mask) - 1 : 49;
            mask &= mask - 1;
            return tt;
        };
        // offsets in increasing order, two row buffers in turn (the next row
        // loads while the current one is applied)
        float4 ra[RQ], rb[RQ];
        int ta = next_tau();
        if (ta < 49) load_row(ta, ra);
        while (ta < 49) {
            const int tb = next_tau();
            if (tb < 49) load_row(tb, rb);
            apply(ta, ra);
            if (tb >= 49) break;
            ta = next_tau();
            if (ta < 49) load_row(ta, ra);
            apply(tb, rb);
        }
        if (valid) {
            // output r = 4 g + i is Re b~_{r+1} (r < P) or Im b~_{r-P+1} (P <= r < 2P)
            const double rinv = ldexp(1.0, (int)t.c_level[c]) / root;
            double* bc = reinterpret_cast<double*>(b + (size_t)c * (P + 1));
            if (g == 0) {
                bc[0] = 0.0;
                bc[1] = 0.0;
            }
            #pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = 4 * g + i;
                if (r < 2 * P) {
                    const int pp = r < P ? r + 1 : r - P + 1;
                    double rk = 1.0;
                    for (int e = 0; e < pp; ++e) rk *= rinv;
                    bc[2 * pp + (r < P ? 0 : 1)] = (double)acc[i] * rk;
                }
            }
        }
        __syncwarp();
    }
}

// List 4 of every cell (FP64, direct formula of fmm2D.cpp:504-520), added
// to b. One warp per cell with list-4 sources; the warp's lanes form
// G = 32 / P groups, group g takes sources g, g + G, ... and its lane p - 1
// computes that part of b_p; the groups' parts are summed in group order.
__global__ void __launch_bounds__(128)
m2l_list4_add(Tree2D t, Lists2D l, const double2* __restrict__ a, double2* __restrict__ b,
              const double* __restrict__ coef, int P, unsigned* err) {
    if (fatal(err)) return;
    const double* g_m2l = coef + kCoefM2L;
    const int lane = threadIdx.x & 31;
    const int G = P <= 32 ? 32 / P : 1;
    const int grp = lane / P, p = lane - grp * P + 1;
    const bool on = grp < G;
    const int c_begin = t.info->level_start[2], c_end = t.info->n_cells;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = c_begin + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < c_end; c += warps) {
        const int n4 = l.l4_n[c];
        if (n4 == 0) continue;
        const double zx = t.c_cx[c], zy = t.c_cy[c];
        double2 acc = make_double2(0.0, 0.0);
        if (on) {
            for (int si = grp; si < n4; si += G) {
                const int src = l.l4_src[(size_t)c * kList4Cap + si];
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
bool m2l_f32_supported(int P) { return P >= 1 && P <= kF32MaxP; }

size_t m2l_tc_rows_bytes(int cap_cells) { return sizeof(float) * (size_t)cap_cells * 2 * kTcMaxK; }
size_t m2l_tc_ops_bytes() { return sizeof(float) * (size_t)49 * 2 * kTcMaxN * kTcMaxK; }

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
    m2l_list4_add<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, e.coef, P, err);
    *launches += 3;
    return cudaGetLastError();
}


// The 49 list-2 operators for m2l2d_f32 as FP32 [slot][k][r]: k the input
// (Re a~_0..P, Im a~_0..P), r the output (Re b~_1..P, Im b~_1..P, padding).
// Synchronises.
cudaError_t set_m2l_f32_operators(int P, const double2* op_dev, float* dst, cudaStream_t st) {
    const int K2 = 2 * (P + 1), NRP = f32_nrp(P);
    std::vector<double2> op((size_t)49 * (P + 1) * P);
    cudaError_t e = cudaMemcpyAsync(op.data(), op_dev, sizeof(double2) * op.size(), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    std::vector<float> h((size_t)49 * K2 * NRP, 0.f);
    for (int slot = 0; slot < 49; ++slot) {
        float* T = h.data() + (size_t)slot * K2 * NRP;
        for (int p = 1; p <= P; ++p) {
            for (int k = 0; k <= P; ++k) {
                const double2 Tc = op[((size_t)slot * (P + 1) + k) * P + (p - 1)];
                // Re b_p = Tr Re a_k - Ti Im a_k ; Im b_p = Ti Re a_k + Tr Im a_k
                T[(size_t)k * NRP + (p - 1)] = (float)Tc.x;
                T[(size_t)(P + 1 + k) * NRP + (p - 1)] = (float)(-Tc.y);
                T[(size_t)k * NRP + (P + p - 1)] = (float)Tc.y;
                T[(size_t)(P + 1 + k) * NRP + (P + p - 1)] = (float)Tc.x;
            }
        }
    }
    e = cudaMemcpyAsync(dst, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

template <int P>
cudaError_t launch_m2l_f32(const Tree2D& t, const Lists2D& l, Expansions2D& e, const float* rows, const float* ops,
                           unsigned* err, cudaStream_t st) {
    const size_t smem = sizeof(float) * (size_t)49 * 2 * (P + 1) * f32_nrp(P) + sizeof(int) * kF32Warps * 49 * (32 / (f32_nrp(P) / 4));
    cudaError_t r = cudaFuncSetAttribute(m2l2d_f32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    int occ = 0;
    r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, m2l2d_f32<P>, 32 * kF32Warps, smem);
    if (r != cudaSuccess) return r;
    m2l2d_f32<P><<<148 * (occ > 0 ? occ : 1), 32 * kF32Warps, smem, st>>>(t, l, rows, ops, e.b, err);
    return cudaGetLastError();
}

cudaError_t fmm2d_m2l_f32(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, float* rows, const float* ops,
                          unsigned* err, cudaStream_t st, int* launches) {
    if (!m2l_f32_supported(P)) return cudaErrorInvalidValue;
    const int RP = f32_rp(P);
    m2l_rows_f32<<<148 * 8, 256, 0, st>>>(t, e.a, rows, P, RP, err);
    cudaError_t r;
    switch (P) {
#define VPM_M2L_F32_CASE(PP) \
    case PP: r = launch_m2l_f32<PP>(t, l, e, rows, ops, err, st); break;
        VPM_M2L_F32_CASE(1) VPM_M2L_F32_CASE(2) VPM_M2L_F32_CASE(3) VPM_M2L_F32_CASE(4) VPM_M2L_F32_CASE(5)
        VPM_M2L_F32_CASE(6) VPM_M2L_F32_CASE(7) VPM_M2L_F32_CASE(8) VPM_M2L_F32_CASE(9) VPM_M2L_F32_CASE(10)
        VPM_M2L_F32_CASE(11) VPM_M2L_F32_CASE(12)
#undef VPM_M2L_F32_CASE
        default: return cudaErrorInvalidValue;
    }
    if (r != cudaSuccess) return r;
    m2l_list4_add<<<148 * 8, 128, 0, st>>>(t, l, e.a, e.b, e.coef, P, err);
    *launches += 3;
    return cudaGetLastError();
}

}  // namespace vpm
