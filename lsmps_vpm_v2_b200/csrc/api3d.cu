// C ABI of the 3D velocity step (include/vpm_fmm.h): arena, driver and the
// octree dump.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"

namespace vpm {

namespace {

// alpha = omega s^3 / (4 pi)   (velocity_calc.cpp:2432-2434), in place over omega
__global__ void alpha_from_vorticity(double* __restrict__ w0, double* __restrict__ w1, double* __restrict__ w2,
                                     const double* __restrict__ s, int n) {
    const double four_pi = 4 * 3.14159265358979323846;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double s3 = pow(s[i], 3.0);
        w0[i] = w0[i] * s3 / four_pi;
        w1[i] = w1[i] * s3 / four_pi;
        w2[i] = w2[i] * s3 / four_pi;
    }
}

struct Layout3D {
    size_t total = 0;
    template <class T>
    size_t take(size_t count) {
        size_t off = (total + 255) & ~(size_t)255;
        total = off + sizeof(T) * std::max<size_t>(count, 1);
        return off;
    }
};

int bits_for(long long v) {
    int b = 1;
    while ((1ll << b) < v) ++b;
    return b;
}

}  // namespace

int Ctx::reserve3d(int n, int cap_cells) {
    if (arena3d && n <= cap3.n && cap_cells <= cap3.cells) return VPM_OK;
    n = std::max(n, cap3.n);
    cap_cells = std::max(cap_cells, cap3.cells);
    const int s_tiles = sort_tiles(n);
    Layout3D L;
    size_t o_in[7], o_out[3];
    for (auto& o : o_in) o = L.take<double>(n);
    size_t o_act = L.take<uint8_t>(n);
    for (auto& o : o_out) o = L.take<double>(n);
    size_t o_perm = L.take<uint32_t>(n), o_p[6];
    for (auto& o : o_p) o = L.take<double>(n);
    size_t o_pact = L.take<uint8_t>(n), o_pcell = L.take<int32_t>(n), o_set = L.take<uint8_t>(n),
           o_oct = L.take<uint8_t>(n);
    const size_t C = cap_cells;
    size_t o_cx = L.take<double>(C), o_cy = L.take<double>(C), o_cz = L.take<double>(C), o_cs = L.take<double>(C);
    size_t o_np = L.take<int32_t>(C), o_par = L.take<int32_t>(C), o_ch0 = L.take<int32_t>(C),
           o_lo = L.take<int32_t>(C), o_hi = L.take<int32_t>(C);
    size_t o_mask = L.take<uint32_t>(C), o_act2 = L.take<uint8_t>(C), o_lev = L.take<uint8_t>(C);
    size_t o_mom = L.take<double>(C * 30), o_leaves = L.take<int32_t>(C);
    size_t o_ps32 = L.take<float4>(n), o_as32 = L.take<float4>(n), o_mom32 = L.take<float>(C * 30);
    size_t o_gbar = L.take<unsigned>(8), o_blk = L.take<uint32_t>(kCoopMaxBlocks3D);
    size_t o_geom = L.take<Geom3D>(1), o_info = L.take<TreeInfo3D>(1), o_bbox = L.take<double>(296 * 6);
    size_t o_ka = L.take<uint32_t>(n), o_kb = L.take<uint32_t>(n), o_va = L.take<uint32_t>(n),
           o_vb = L.take<uint32_t>(n);
    size_t o_sstat = L.take<uint32_t>((size_t)4 * s_tiles * 256), o_stick = L.take<unsigned>(8),
           o_hist = L.take<uint32_t>(8 * 256);
    const int tc_tiles = ceil_div(n, kTcTile);
    size_t o_tgt = L.take<uint8_t>(n), o_tcact = L.take<uint32_t>(n), o_tcscan = L.take<uint32_t>((size_t)n + 1),
           o_tcpinfo = L.take<uint32_t>(n), o_tctile = L.take<uint32_t>((size_t)2 * (kTcLevels + 1) * tc_tiles),
           o_tctot = L.take<uint32_t>(32), o_tccode = L.take<uint32_t>(C),
           o_scst = L.take<uint64_t>(scan_tiles(n)), o_sctk = L.take<unsigned>(8);

    if (arena3d) cudaFree(arena3d);
    arena3d = nullptr;
    cap3 = Caps3D{};
    have_tree3 = false;
    cudaError_t e = cudaMalloc(&arena3d, L.total);
    if (e != cudaSuccess) {
        arena3d = nullptr;
        return fail_cuda(e, "cudaMalloc of the 3D arena");
    }
    char* base = (char*)arena3d;
    auto P_ = [&](size_t off) { return (void*)(base + off); };
    for (int k = 0; k < 7; ++k) in3[k] = (double*)P_(o_in[k]);
    in3_act = (uint8_t*)P_(o_act);
    for (int k = 0; k < 3; ++k) out3[k] = (double*)P_(o_out[k]);
    Tree3D& t = tree3;
    t.perm = (uint32_t*)P_(o_perm);
    t.px = (double*)P_(o_p[0]); t.py = (double*)P_(o_p[1]); t.pz = (double*)P_(o_p[2]);
    t.ax = (double*)P_(o_p[3]); t.ay = (double*)P_(o_p[4]); t.az = (double*)P_(o_p[5]);
    t.pact = (uint8_t*)P_(o_pact); t.pcell = (int32_t*)P_(o_pcell); t.settled = (uint8_t*)P_(o_set);
    t.poct = (uint8_t*)P_(o_oct);
    t.c_x = (double*)P_(o_cx); t.c_y = (double*)P_(o_cy); t.c_z = (double*)P_(o_cz); t.c_size = (double*)P_(o_cs);
    t.c_npar = (int32_t*)P_(o_np); t.c_parent = (int32_t*)P_(o_par); t.c_child0 = (int32_t*)P_(o_ch0);
    t.c_lo = (int32_t*)P_(o_lo); t.c_hi = (int32_t*)P_(o_hi);
    t.c_chmask = (uint32_t*)P_(o_mask); t.c_active = (uint8_t*)P_(o_act2); t.c_level = (uint8_t*)P_(o_lev);
    t.mom = (double*)P_(o_mom); t.leaf_cells = (int32_t*)P_(o_leaves);
    t.ps32 = (float4*)P_(o_ps32); t.as32 = (float4*)P_(o_as32); t.mom32 = (float*)P_(o_mom32);
    t.gbar = (unsigned*)P_(o_gbar); t.blk = (uint32_t*)P_(o_blk);
    t.geom = (Geom3D*)P_(o_geom); t.info = (TreeInfo3D*)P_(o_info);
    t.cap_cells = cap_cells;
    bbox3 = (double*)P_(o_bbox);
    s3.key_a = (uint32_t*)P_(o_ka); s3.key_b = (uint32_t*)P_(o_kb);
    s3.val_a = (uint32_t*)P_(o_va); s3.val_b = (uint32_t*)P_(o_vb);
    s3.sort.status = (uint32_t*)P_(o_sstat); s3.sort.tickets = (unsigned*)P_(o_stick);
    s3.sort.hist = (uint32_t*)P_(o_hist); s3.sort.max_tiles = s_tiles;
    in3_tgt = (uint8_t*)P_(o_tgt);
    s3.tc_act = (uint32_t*)P_(o_tcact); s3.tc_scan = (uint32_t*)P_(o_tcscan); s3.tc_pinfo = (uint32_t*)P_(o_tcpinfo);
    s3.tc_tile = (uint32_t*)P_(o_tctile); s3.tc_tot = (uint32_t*)P_(o_tctot); s3.tc_code = (uint32_t*)P_(o_tccode);
    s3.scan.status = (uint64_t*)P_(o_scst); s3.scan.ticket = (unsigned*)P_(o_sctk); s3.scan.max_tiles = scan_tiles(n);
    s3.tc_tiles = tc_tiles;
    cap3.n = n;
    cap3.cells = cap_cells;
    return VPM_OK;
}

int Ctx::enqueue3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                   const double* az, const uint8_t* act, int n, const vpm_fmm_params& p, double* u, double* v,
                   double* w, double uinf, double vinf, double winf, bool tree_only, bool treecell,
                   const uint8_t* target) {
    cudaStream_t st = stream;
    int launches = 0;
    tree3.n = n;
    tree3.leaf_cap = p.leaf_cap_3d;
    VPM_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(unsigned), st));
    VPM_CUDA_TRY(cudaEventRecord(ev[0], st));
    if (treecell)
        VPM_CUDA_TRY(build_treecell3d(x, y, z, ax, ay, az, act, p.max_src, p.max_par, p.exp_tree_pct, tree3, s3,
                                      bbox3, d_err, st, &launches));
    else
        VPM_CUDA_TRY(build_tree3d(x, y, z, ax, ay, az, act, p.center_3d, p.exp_tree_pct, tree3, s3, bbox3, d_err,
                                  st, &launches));
    if (!tree_only) {
        const bool mixed = p.precision == VPM_PREC_MIXED;
        if (mixed) VPM_CUDA_TRY(prep3d_f32(tree3, d_err, st, &launches));
        VPM_CUDA_TRY(eval3d(tree3, mixed, treecell, target, p.support_3d, u, v, w, uinf, vinf, winf, d_err, st,
                            &launches));
    }
    VPM_CUDA_TRY(cudaEventRecord(ev[1], st));
    last_launches3 = launches;
    have_tree3 = true;
    last_treecell3 = treecell;
    last_n3 = n;
    return VPM_OK;
}

int Ctx::run3d_host(const double* x, const double* y, const double* z, const double* a0, const double* a1,
                    const double* a2, const double* s, const uint8_t* act, int64_t n64, const vpm_fmm_params* prm,
                    double* u, double* v, double* w, double uinf, double vinf, double winf, vpm_fmm_stats* stats,
                    bool tree_only, bool treecell, const uint8_t* target) {
    vpm_fmm_params p;
    int r = check_params(prm, p);
    if (r) return r;
    if (p.leaf_cap_3d < 1) return fail(VPM_EINVAL, "leaf_cap_3d must be >= 1");
    if (n64 < 0 || n64 >= (1ll << 30)) return fail(VPM_EINVAL, "n out of range");
    if (!x || !y || !z || !act || (!tree_only && (!a0 || !a1 || !a2 || !u || !v || !w)))
        return fail(VPM_EINVAL, "null buffer");
    const int n = (int)n64;
    if (n == 0) return VPM_OK;
    long long cells = std::max<long long>(4096, 2ll * n);
    for (int attempt = 0; attempt < 5; ++attempt) {
        if (cells > (1ll << 30)) return fail(VPM_EINVAL, "too many cells");
        r = reserve3d(n, (int)cells);
        if (r) return r;
        const double* src[7] = {x, y, z, a0, a1, a2, s};
        for (int k = 0; k < 7; ++k) {
            if (k >= 3 && tree_only) {
                VPM_CUDA_TRY(cudaMemsetAsync(in3[k], 0, sizeof(double) * n, stream));
                continue;
            }
            if (k == 6 && !s) continue;
            VPM_CUDA_TRY(cudaMemcpyAsync(in3[k], src[k], sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        }
        VPM_CUDA_TRY(cudaMemcpyAsync(in3_act, act, n, cudaMemcpyHostToDevice, stream));
        if (target) VPM_CUDA_TRY(cudaMemcpyAsync(in3_tgt, target, n, cudaMemcpyHostToDevice, stream));
        if (s && !tree_only) {
            alpha_from_vorticity<<<std::min(1184, ceil_div(n, 256)), 256, 0, stream>>>(in3[3], in3[4], in3[5],
                                                                                       in3[6], n);
            VPM_CUDA_TRY(cudaGetLastError());
        }
        r = enqueue3d(in3[0], in3[1], in3[2], in3[3], in3[4], in3[5], in3_act, n, p, out3[0], out3[1], out3[2], uinf,
                      vinf, winf, tree_only, treecell, target ? in3_tgt : nullptr);
        if (r) return r;
        unsigned bits = 0;
        VPM_CUDA_TRY(cudaMemcpyAsync(&bits, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        VPM_CUDA_TRY(cudaStreamSynchronize(stream));
        if (bits & ERR_CELL_CAP) {
            cells *= 2;
            continue;
        }
        if ((bits & ERR_DEPTH) && treecell)
            return fail(VPM_EINVAL, "TreeCell deeper than level 10: the reference's 32-bit cell IDs overflow there");
        if (bits & ERR_DEPTH) return fail(VPM_EINVAL, "octree deeper than 60 levels (coincident particles)");
        if ((bits & ERR_LEAF1) && !tree_only)
            return fail(VPM_EINVAL, "a level-1 cell is a leaf: the reference's TreeCell traversal cannot take its "
                                    "children (fmm3D.cpp:1286 throws)");
        bits &= ~(unsigned)ERR_LEAF1;
        if (bits) return map_err(bits);
        VPM_CUDA_TRY(cudaEventElapsedTime(&last_ms3, ev[0], ev[1]));
        if (!tree_only) {
            VPM_CUDA_TRY(cudaMemcpyAsync(u, out3[0], sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
            VPM_CUDA_TRY(cudaMemcpyAsync(v, out3[1], sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
            VPM_CUDA_TRY(cudaMemcpyAsync(w, out3[2], sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
            VPM_CUDA_TRY(cudaStreamSynchronize(stream));
        }
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            TreeInfo3D info;
            VPM_CUDA_TRY(cudaMemcpy(&info, tree3.info, sizeof(info), cudaMemcpyDeviceToHost));
            stats->n = n;
            stats->n_cells = info.n_cells;
            stats->n_leaves = info.n_leaves;
            stats->max_level = info.depth;
            stats->ms_total = last_ms3;
            stats->kernels = last_launches3;
        }
        return VPM_OK;
    }
    return fail(VPM_EOVERFLOW, "capacity retries exhausted");
}

}  // namespace vpm

using vpm::Ctx;

extern "C" {

int vpm_fmm3d_velocity(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                       const double* ay, const double* az, const uint8_t* active, const uint8_t* target, int64_t n,
                       const vpm_fmm_params* prm, double* u, double* v, double* w, vpm_fmm_stats* stats) {
    (void)target;  // every particle is a target (fast3DFMM.cpp:341-343 ignores the flags)
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run3d_host(x, y, z, ax, ay, az, nullptr, active, n, prm, u, v, w, 0.0, 0.0, 0.0, stats, false, false,
                         nullptr);
}

int vpm_velocity3d(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* omega_x,
                   const double* omega_y, const double* omega_z, const double* s, const uint8_t* active, int64_t n,
                   const vpm_fmm_params* prm, double u_inf, double v_inf, double w_inf, double* u, double* v,
                   double* w, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!s) return c->fail(VPM_EINVAL, "null buffer");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run3d_host(x, y, z, omega_x, omega_y, omega_z, s, active, n, prm, u, v, w, u_inf, v_inf, w_inf, stats,
                         false, false, nullptr);
}

int vpm_fmm3d_velocity_device(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                              const double* ay, const double* az, const uint8_t* active, int64_t n64,
                              const vpm_fmm_params* prm, double* u, double* v, double* w) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    vpm_fmm_params p;
    int r = c->check_params(prm, p);
    if (r) return r;
    if (p.leaf_cap_3d < 1) return c->fail(VPM_EINVAL, "leaf_cap_3d must be >= 1");
    if (n64 < 0 || n64 >= (1ll << 30)) return c->fail(VPM_EINVAL, "n out of range");
    if (!x || !y || !z || !ax || !ay || !az || !active || !u || !v || !w) return c->fail(VPM_EINVAL, "null buffer");
    const int n = (int)n64;
    if (n == 0) return VPM_OK;
    r = c->reserve3d(n, std::max(4096, 2 * n));
    if (r) return r;
    return c->enqueue3d(x, y, z, ax, ay, az, active, n, p, u, v, w, 0.0, 0.0, 0.0, false, false, nullptr);
}

int vpm_tree3d_build(vpm_ctx* ctx, const double* x, const double* y, const double* z, const uint8_t* active,
                     int64_t n, const vpm_fmm_params* prm, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run3d_host(x, y, z, nullptr, nullptr, nullptr, nullptr, active, n, prm, nullptr, nullptr, nullptr, 0.0,
                         0.0, 0.0, stats, true, false, nullptr);
}

int vpm_tree3d_counts(vpm_ctx* ctx, int64_t* n_cells, int64_t* n_leaves, int32_t* depth) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!c->have_tree3) return c->fail(VPM_EINVAL, "no 3D tree on this context yet");
    vpm::TreeInfo3D info;
    cudaError_t e = cudaMemcpyAsync(&info, c->tree3.info, sizeof(info), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_tree3d_counts");
    if (n_cells) *n_cells = info.n_cells;
    if (n_leaves) *n_leaves = info.n_leaves;
    if (depth) *depth = info.depth;
    return VPM_OK;
}

int vpm_tree3d_cells(vpm_ctx* ctx, int32_t* ints6, double* geom4, int64_t* leaf_offs, int32_t* pids) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!c->have_tree3) return c->fail(VPM_EINVAL, "no 3D tree on this context yet");
    const vpm::Tree3D& t = c->tree3;
    vpm::TreeInfo3D info;
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(&info, t.info, sizeof(info), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_tree3d_cells");
    const int nc = info.n_cells, n = c->last_n3;
    std::vector<int32_t> npar(nc), par(nc), lo(nc), hi(nc);
    std::vector<uint32_t> mask(nc), perm(n);
    std::vector<uint8_t> act(nc), lev(nc);
    std::vector<double> g[4];
    for (auto& x : g) x.resize(nc);
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    };
    cp(npar.data(), t.c_npar, 4ull * nc);
    cp(par.data(), t.c_parent, 4ull * nc);
    cp(lo.data(), t.c_lo, 4ull * nc);
    cp(hi.data(), t.c_hi, 4ull * nc);
    cp(mask.data(), t.c_chmask, 4ull * nc);
    cp(act.data(), t.c_active, nc);
    cp(lev.data(), t.c_level, nc);
    cp(g[0].data(), t.c_x, 8ull * nc);
    cp(g[1].data(), t.c_y, 8ull * nc);
    cp(g[2].data(), t.c_z, 8ull * nc);
    cp(g[3].data(), t.c_size, 8ull * nc);
    cp(perm.data(), t.perm, 4ull * n);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_tree3d_cells");
    int64_t off = 0;
    for (int k = 0; k < nc; ++k) {
        if (ints6) {
            int32_t* r = ints6 + 6 * (size_t)k;
            r[0] = npar[k]; r[1] = (int32_t)mask[k]; r[2] = par[k]; r[3] = act[k]; r[4] = lev[k];
            r[5] = k == 0 ? info.depth : 0;
        }
        if (geom4)
            for (int d = 0; d < 4; ++d) geom4[4 * (size_t)k + d] = g[d][k];
        if (leaf_offs) {
            leaf_offs[k] = off;
            if (mask[k] == 0 && k > 0) {
                for (int j = lo[k]; j < hi[k]; ++j) {
                    if (pids) pids[off] = (int32_t)perm[j];
                    ++off;
                }
            }
        }
    }
    if (leaf_offs) leaf_offs[nc] = off;
    return VPM_OK;
}

int vpm_fmm3d_velocity_treecell(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                                const double* ay, const double* az, const uint8_t* active, const uint8_t* target,
                                int64_t n, const vpm_fmm_params* prm, double* u, double* v, double* w,
                                vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run3d_host(x, y, z, ax, ay, az, nullptr, active, n, prm, u, v, w, 0.0, 0.0, 0.0, stats, false, true,
                         target);
}

int vpm_fmm3d_velocity_treecell_device(vpm_ctx* ctx, const double* x, const double* y, const double* z,
                                       const double* ax, const double* ay, const double* az, const uint8_t* active,
                                       const uint8_t* target, int64_t n64, const vpm_fmm_params* prm, double* u,
                                       double* v, double* w) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    vpm_fmm_params p;
    int r = c->check_params(prm, p);
    if (r) return r;
    if (n64 < 0 || n64 >= (1ll << 30)) return c->fail(VPM_EINVAL, "n out of range");
    if (!x || !y || !z || !ax || !ay || !az || !active || !u || !v || !w) return c->fail(VPM_EINVAL, "null buffer");
    const int n = (int)n64;
    if (n == 0) return VPM_OK;
    r = c->reserve3d(n, std::max(4096, 2 * n));
    if (r) return r;
    return c->enqueue3d(x, y, z, ax, ay, az, active, n, p, u, v, w, 0.0, 0.0, 0.0, false, true, target);
}

int vpm_treecell3d_build(vpm_ctx* ctx, const double* x, const double* y, const double* z, const uint8_t* active,
                         int64_t n, const vpm_fmm_params* prm, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run3d_host(x, y, z, nullptr, nullptr, nullptr, nullptr, active, n, prm, nullptr, nullptr, nullptr, 0.0,
                         0.0, 0.0, stats, true, true, nullptr);
}

int vpm_tree3d_cell_ids(vpm_ctx* ctx, int64_t* ids) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    if (!c->have_tree3) return c->fail(VPM_EINVAL, "no 3D tree on this context yet");
    if (!c->last_treecell3) return c->fail(VPM_EINVAL, "the octree of the default 3D path has no TreeCell IDs");
    if (!ids) return c->fail(VPM_EINVAL, "null buffer");
    const vpm::Tree3D& t = c->tree3;
    vpm::TreeInfo3D info;
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(&info, t.info, sizeof(info), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_tree3d_cell_ids");
    const int nc = info.n_cells;
    std::vector<uint32_t> code(nc);
    std::vector<uint8_t> lev(nc);
    e = cudaMemcpyAsync(code.data(), c->s3.tc_code, 4ull * nc, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lev.data(), t.c_level, nc, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_tree3d_cell_ids");
    ids[0] = 0;
    for (int k = 1; k < nc; ++k) {
        const int L = lev[k];
        const uint32_t pre = code[k] & 0x7fffffffu;
        int64_t ix = 0, iy = 0, iz = 0;
        for (int b = 0; b < L; ++b) {
            ix |= (int64_t)((pre >> (3 * b)) & 1u) << b;
            iy |= (int64_t)((pre >> (3 * b + 1)) & 1u) << b;
            iz |= (int64_t)((pre >> (3 * b + 2)) & 1u) << b;
        }
        ids[k] = ((int64_t)1 << (3 * L)) / 7 + ix + (iy << L) + (iz << (2 * L));   // treeCell.cpp:114-148, 223-250
    }
    return VPM_OK;
}

}  // extern "C"

