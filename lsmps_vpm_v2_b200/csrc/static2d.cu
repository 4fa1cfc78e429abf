// vpm_fmm2d_field_device_static: the 2D evaluation of vpm_fmm2d_field_device
// for callers that cannot allocate device memory. Two kinds of caller need
// it: programs whose device memory belongs to another allocator (a solver
// that hands its whole budget to a framework's caching allocator, so a
// cudaMalloc here would fail or fragment that pool), and time-step loops that
// must not stall, since cudaMalloc and cudaFree can synchronise the device.
//
// All scratch (sorted particles, cells, lists, expansions, sort and scan
// status words, the error word) lives in one file-scope static device array
// of kStaticBytes, which every GPU that loads this library holds until the
// process exits. The caller passes only its input and output device buffers.
// No cudaMalloc, cudaFree or allocating library routine is called, on the
// device or the host.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (set-up, once per device, with that device current);
// make that first call before any stream capture begins. Each call ends by
// reading the device error word back and waiting for its stream.
//
// Limits: n <= kStaticMaxN particles, at most kStaticMaxCells tree cells,
// p <= kStaticMaxP; larger requests are rejected with VPM_EINVAL, and a tree
// that outgrows the cell or list space returns VPM_EOVERFLOW.
//
// Every call shares the one array and overwrites it (the state of the last
// call stays there); everything that must start at zero is cleared by the
// stages themselves at the start of each call. Two calls whose work overlaps
// on the GPU (different streams, or different host threads) race on the
// array and corrupt each other: serialise them.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "context.h"

namespace vpm {
namespace {

constexpr int kStaticMaxN = 8192;
constexpr int kStaticMaxCells = 8192;
constexpr int kStaticMaxP = 12;
constexpr size_t kStaticBytes = 8u << 20;  // 8 MiB
constexpr int kStaticMaxDevices = 64;

__device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// Device address of g_static_scratch per device. In host code the symbol's
// name is a host-side stand-in, not a device address: a kernel given it would
// fault or silently use the wrong memory, so the address is looked up with
// cudaGetSymbolAddress once per device, with that device current.
void* g_static_addr[kStaticMaxDevices] = {};
std::mutex g_static_mutex;

struct Carve {
    size_t total = 0;
    template <class T>
    T* take(char* base, size_t count) {
        size_t off = (total + 255) & ~(size_t)255;
        total = off + sizeof(T) * (count > 0 ? count : 1);
        return base ? (T*)(base + off) : nullptr;
    }
};

// The reference's binComb (32-bit, wrapping) or the exact value.
long long binom_static(int n, int k, bool exact) {
    if (k > n) return 0;
    if (exact) {
        long long c = 1;
        for (int i = 1; i <= k; ++i) c = c * (n - k + i) / i;
        return c;
    }
    int inv = n - k;
    int mx = inv > k ? inv : k, mn = inv > k ? k : inv;
    int32_t c = 1;
    for (int i = n; i > mx; --i) c = (int32_t)((uint32_t)c * (uint32_t)i);
    for (int i = mn; i > 1; --i) c /= i;
    return c;
}

void set_msg(char* buf, size_t len, const char* msg) {
    if (buf && len) std::snprintf(buf, len, "%s", msg);
}

}  // namespace
}  // namespace vpm

extern "C" int vpm_fmm2d_field_device_static(const double* x, const double* y, const double* q,
                                             const uint8_t* active, int64_t n64, const vpm_fmm_params* prm,
                                             double* ex, double* ey, void* cuda_stream, char* errbuf,
                                             size_t errlen) {
    using namespace vpm;
    vpm_fmm_params p;
    if (prm) p = *prm;
    else vpm_fmm_params_default(&p);
    if (!x || !y || !q || !active || !ex || !ey) {
        set_msg(errbuf, errlen, "null buffer");
        return VPM_EINVAL;
    }
    if (n64 < 2 || n64 > kStaticMaxN) {
        set_msg(errbuf, errlen, "n must be in 2..8192 for the static-scratch entry point");
        return VPM_EINVAL;
    }
    if (p.p < 1 || p.p > kStaticMaxP) {
        set_msg(errbuf, errlen, "p must be in 1..12 for the static-scratch entry point");
        return VPM_EINVAL;
    }
    if (p.max_src < 0 || p.max_par < 1) {
        set_msg(errbuf, errlen, "leaf caps must be max_src >= 0, max_par >= 1");
        return VPM_EINVAL;
    }
    if (p.precision != VPM_PREC_FP64 && p.precision != VPM_PREC_MIXED && p.precision != VPM_PREC_MIXED_FP64_M2L) {
        set_msg(errbuf, errlen, "precision must be VPM_PREC_FP64, VPM_PREC_MIXED or VPM_PREC_MIXED_FP64_M2L");
        return VPM_EINVAL;
    }
    const int K = (p.max_depth == 31) ? 31 : 16;
    const int n = (int)n64;
    const int P = p.p;
    cudaStream_t st = (cudaStream_t)cuda_stream;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kStaticMaxDevices) {
        set_msg(errbuf, errlen, "no usable current CUDA device");
        return VPM_EDEVICE;
    }
    void* base_ptr = nullptr;
    {
        // Set-up, once per device, with that device current (the first call
        // on a device; it should come before any stream capture begins).
        std::lock_guard<std::mutex> lock(g_static_mutex);
        if (!g_static_addr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_static_scratch);
            if (e != cudaSuccess || !ptr) {
                set_msg(errbuf, errlen, "cudaGetSymbolAddress of the static scratch array failed");
                return VPM_EDEVICE;
            }
            g_static_addr[dev] = ptr;
        }
        base_ptr = g_static_addr[dev];
    }

    // Carve the static array (same buffers as the context arena).
    char* base = (char*)base_ptr;
    const size_t C = kStaticMaxCells;
    const int s_tiles = sort_tiles(kStaticMaxN);
    const int sc_tiles = scan_tiles(kStaticMaxCells + 1);
    Carve cv;
    Tree2D t{};
    TreeScratch2D ts{};
    Lists2D l{};
    Expansions2D xe{};
    unsigned* err = cv.take<unsigned>(base, 64);
    t.key = cv.take<uint64_t>(base, kStaticMaxN);
    t.perm = cv.take<uint32_t>(base, kStaticMaxN);
    t.px = cv.take<double>(base, kStaticMaxN);
    t.py = cv.take<double>(base, kStaticMaxN);
    t.pq = cv.take<double>(base, kStaticMaxN);
    t.pact = cv.take<uint8_t>(base, kStaticMaxN);
    t.actscan = cv.take<uint32_t>(base, kStaticMaxN + 1);
    ts.key_alt = cv.take<uint64_t>(base, kStaticMaxN);
    ts.val_alt = cv.take<uint32_t>(base, kStaticMaxN);
    ts.act_u32 = cv.take<uint32_t>(base, kStaticMaxN);
    ts.bbox_partial = cv.take<double>(base, kBBoxBlocks * 4);
    ts.lvl_ticket = cv.take<unsigned>(base, kTicketWords);
    ts.flat_tiles = ceil_div(kStaticMaxN, kFlatTile);
    ts.pinfo = cv.take<uint32_t>(base, kStaticMaxN);
    ts.tile_cnt = cv.take<uint32_t>(base, (size_t)2 * (kMaxLevels2D + 1) * ts.flat_tiles);
    ts.level_tot = cv.take<uint32_t>(base, 2 * (kMaxLevels2D + 1));
    ts.sort.status = cv.take<uint32_t>(base, (size_t)8 * s_tiles * 256);
    ts.sort.tickets = cv.take<unsigned>(base, 8);
    ts.sort.hist = cv.take<uint32_t>(base, 8 * 256);
    ts.sort.max_tiles = s_tiles;
    ts.scan.status = cv.take<uint64_t>(base, sc_tiles);
    ts.scan.ticket = cv.take<unsigned>(base, 1);
    ts.scan.max_tiles = sc_tiles;
    t.c_lo = cv.take<int32_t>(base, C); t.c_hi = cv.take<int32_t>(base, C); t.c_src = cv.take<int32_t>(base, C);
    t.c_parent = cv.take<int32_t>(base, C); t.c_child0 = cv.take<int32_t>(base, C);
    t.c_ix = cv.take<int32_t>(base, C); t.c_iy = cv.take<int32_t>(base, C); t.c_leafidx = cv.take<int32_t>(base, C);
    t.c_flags = cv.take<uint8_t>(base, C); t.c_chmask = cv.take<uint8_t>(base, C);
    t.c_level = cv.take<uint8_t>(base, C);
    t.c_cx = cv.take<double>(base, C); t.c_cy = cv.take<double>(base, C); t.c_code = cv.take<uint64_t>(base, C);
    t.leaf_cells = cv.take<int32_t>(base, C);
    t.geom = cv.take<Geom2D>(base, 1);
    t.info = cv.take<TreeInfo2D>(base, 1);
    t.cap_cells = kStaticMaxCells;
    t.dense = nullptr;  // lookups fall back to binary search
    t.dense_levels = 0;
    t.gbar = ts.lvl_ticket + kBarrierWordsAt;
    l.l2_src = cv.take<int32_t>(base, C * kList2Cap); l.l2_slot = cv.take<uint8_t>(base, C * kList2Cap);
    l.l2_n = cv.take<uint8_t>(base, C);
    l.l4_src = cv.take<int32_t>(base, C * kList4Cap); l.l4_n = cv.take<uint8_t>(base, C);
    l.cap_leaves = kStaticMaxCells;
    l.cap_l1 = 16ll * kStaticMaxCells;
    l.cap_l3 = 8ll * kStaticMaxCells;
    l.l1_cnt = cv.take<uint32_t>(base, C); l.l1_off = cv.take<uint32_t>(base, C + 1);
    l.l1_src = cv.take<int32_t>(base, l.cap_l1);
    l.l3_cnt = cv.take<uint32_t>(base, C); l.l3_off = cv.take<uint32_t>(base, C + 1);
    l.l3_src = cv.take<int32_t>(base, l.cap_l3);
    xe.a = cv.take<double2>(base, C * (kStaticMaxP + 1));
    xe.b = cv.take<double2>(base, C * (kStaticMaxP + 1));
    xe.up_count = cv.take<unsigned>(base, C);
    xe.fx = cv.take<double>(base, kStaticMaxN);
    xe.fy = cv.take<double>(base, kStaticMaxN);
    xe.coef = cv.take<double>(base, 3 * kCoefTable);
    xe.op = nullptr;  // direct M2L formula
    if (cv.total > kStaticBytes) {
        set_msg(errbuf, errlen, "static scratch layout exceeds its array");
        return VPM_EDEVICE;
    }
    t.n = n;
    t.key_levels = K;

    // Translation coefficients, built on the stack and copied (no allocation).
    double tab[3 * kCoefTable];
    std::memset(tab, 0, sizeof(tab));
    const bool exact = p.binom == VPM_BINOM_EXACT;
    const int W = kMaxP + 1;
    for (int pp = 0; pp <= P; ++pp) {
        for (int k = 1; k <= pp; ++k)
            tab[kCoefM2M + pp * W + k] = (double)binom_static(pp - 1, k - 1, exact) * ((double)pp / (double)k);
        for (int k = 1; k <= P; ++k)
            tab[kCoefM2L + pp * W + k] =
                (double)binom_static(pp + k - 1, k - 1, exact) * ((k & 1) ? -1.0 : 1.0) / (double)k;
        for (int k = pp; k <= P; ++k) tab[kCoefL2L + pp * W + k] = (double)binom_static(k, pp, exact);
    }
    int launches = 0;
    cudaError_t r = cudaMemsetAsync(err, 0, 64 * sizeof(unsigned), st);
    if (r == cudaSuccess) r = cudaMemcpyAsync(xe.coef, tab, sizeof(tab), cudaMemcpyHostToDevice, st);
    if (r == cudaSuccess)
        r = build_tree2d(x, y, q, active, t, ts, p.max_src, p.max_par, p.exp_tree_pct, err, st, &launches);
    if (r == cudaSuccess) r = build_lists2d(t, l, ts.scan, p.eps, err, st, &launches);
    if (r == cudaSuccess) r = fmm2d_upward(t, xe, P, err, st, &launches);
    if (r == cudaSuccess) r = fmm2d_m2l(t, l, xe, P, err, st, &launches);
    if (r == cudaSuccess) r = fmm2d_eval(t, l, xe, P, err, st, &launches);
    if (r == cudaSuccess) {
        if (p.precision == VPM_PREC_MIXED || p.precision == VPM_PREC_MIXED_FP64_M2L)
            r = fmm2d_p2p_f32(t, l, xe, ex, ey, 0, 0.0, 0.0, err, st, &launches);
        else
            r = fmm2d_p2p(t, l, xe, ex, ey, err, st, &launches);
    }
    unsigned bits = 0;
    if (r == cudaSuccess) r = cudaMemcpyAsync(&bits, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (r == cudaSuccess) r = cudaStreamSynchronize(st);
    if (r != cudaSuccess) {
        set_msg(errbuf, errlen, cudaGetErrorString(r));
        return r == cudaErrorMemoryAllocation ? VPM_ENOMEM : VPM_EDEVICE;
    }
    if (bits & (ERR_CELL_CAP | ERR_LIST_CAP | ERR_DEPTH | ERR_QUEUE | ERR_LIST4 | ERR_LIST2)) {
        set_msg(errbuf, errlen, "the tree outgrew the static scratch (cells, lists or key depth)");
        return VPM_EOVERFLOW;
    }
    if (bits & (ERR_NONFINITE | ERR_RANGE)) {
        set_msg(errbuf, errlen, "non-finite positions or a degenerate domain");
        return VPM_EINVAL;
    }
    if (bits & ERR_TIMEOUT) {
        set_msg(errbuf, errlen, "a bounded device-side wait gave up");
        return VPM_ETIMEDOUT;
    }
    if (bits) {
        set_msg(errbuf, errlen, "device index check failed");
        return VPM_EDEVICE;
    }
    set_msg(errbuf, errlen, "ok");
    return VPM_OK;
}
