// C ABI of the 2D velocity step (include/vpm_fmm.h): context, device memory
// arena, the evaluation driver and the parity dumps.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"

namespace vpm {

namespace {

// q = -omega s^2 / (2 pi)   (velocity_calc.cpp:477)
__global__ void source_from_vorticity(const double* __restrict__ omega, const double* __restrict__ s, int n,
                                      double* __restrict__ q) {
    const double two_pi = 2 * 3.14159265358979323846;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s2 = __dmul_rn(s[i], s[i]);
        q[i] = __ddiv_rn(__dmul_rn(-omega[i], s2), two_pi);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Arena layout of the 2D buffers for (n particles, cap cells, order P).
// ---------------------------------------------------------------------------
struct Layout2D {
    size_t total = 0;
    template <class T>
    size_t take(size_t count) {
        size_t off = (total + 255) & ~(size_t)255;
        total = off + sizeof(T) * std::max<size_t>(count, 1);
        return off;
    }
};

static const char* status_text(int s) {
    switch (s) {
        case VPM_OK: return "ok";
        case VPM_EDEVICE: return "device error";
        case VPM_ENOMEM: return "out of device memory";
        case VPM_EINVAL: return "invalid argument";
        case VPM_EOVERFLOW: return "capacity exceeded";
        case VPM_ETIMEDOUT: return "device wait timed out";
    }
    return "unknown";
}

int Ctx::fail(int status, const std::string& msg) {
    last_error = std::string(status_text(status)) + ": " + msg;
    return status;
}

int Ctx::fail_cuda(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? VPM_ENOMEM : VPM_EDEVICE,
                std::string(what) + ": " + cudaGetErrorString(e));
}

int Ctx::reserve2d(int n, int cap_cells, int P, long long cap_l1, long long cap_l3) {
    if (n <= cap.n && cap_cells <= cap.cells && P <= cap.P && cap_l1 <= cap.l1 && cap_l3 <= cap.l3 && arena2d)
        return VPM_OK;
    n = std::max(n, cap.n);
    cap_cells = std::max(cap_cells, cap.cells);
    P = std::max(P, cap.P);
    cap_l1 = std::max(cap_l1, cap.l1);
    cap_l3 = std::max(cap_l3, cap.l3);
    const int K = kMaxLevels2D;
    const int s_tiles = sort_tiles(n);
    const int sc_tiles = scan_tiles(std::max(n, cap_cells) + 1);
    Layout2D L;
    size_t o_x = L.take<double>(n), o_y = L.take<double>(n), o_q = L.take<double>(n), o_act = L.take<uint8_t>(n);
    size_t o_o0 = L.take<double>(n), o_o1 = L.take<double>(n);
    size_t o_key = L.take<uint64_t>(n), o_perm = L.take<uint32_t>(n);
    size_t o_px = L.take<double>(n), o_py = L.take<double>(n), o_pq = L.take<double>(n), o_pact = L.take<uint8_t>(n);
    size_t o_actscan = L.take<uint32_t>((size_t)n + 1);
    size_t o_keyalt = L.take<uint64_t>(n), o_valalt = L.take<uint32_t>(n), o_actu = L.take<uint32_t>(n);
    size_t o_bbox = L.take<double>(kBBoxBlocks * 4), o_coop = L.take<uint32_t>(kCoopSortWords);
    size_t o_ltick = L.take<unsigned>(kTicketWords);
    const int flat_tiles = ceil_div(n, kFlatTile);
    size_t o_pinfo = L.take<uint32_t>(n), o_tcnt = L.take<uint32_t>((size_t)2 * (K + 1) * flat_tiles),
           o_ltot = L.take<uint32_t>(2 * (K + 1));
    size_t o_sstat = L.take<uint32_t>((size_t)8 * s_tiles * 256), o_stick = L.take<unsigned>(8),
           o_hist = L.take<uint32_t>(8 * 256);
    size_t o_scstat = L.take<uint64_t>(sc_tiles), o_sctick = L.take<unsigned>(1);
    const size_t C = cap_cells;
    size_t o_clo = L.take<int32_t>(C), o_chi = L.take<int32_t>(C), o_csrc = L.take<int32_t>(C),
           o_cpar = L.take<int32_t>(C), o_cch = L.take<int32_t>(C), o_cix = L.take<int32_t>(C),
           o_ciy = L.take<int32_t>(C), o_cleaf = L.take<int32_t>(C);
    size_t o_cfl = L.take<uint8_t>(C), o_cmask = L.take<uint8_t>(C), o_clev = L.take<uint8_t>(C);
    size_t o_ccx = L.take<double>(C), o_ccy = L.take<double>(C), o_ccode = L.take<uint64_t>(C);
    size_t o_leaves = L.take<int32_t>(C), o_nonleaf = L.take<int32_t>(C);
    size_t o_l2blk = L.take<int32_t>(C * 32);
    size_t o_l2 = L.take<int32_t>(C * kList2Cap), o_l2s = L.take<uint8_t>(C * kList2Cap), o_l2n = L.take<uint8_t>(C);
    size_t o_l4 = L.take<int32_t>(C * kList4Cap), o_l4n = L.take<uint8_t>(C);
    size_t o_l1c = L.take<uint32_t>(C), o_l1o = L.take<uint32_t>(C + 1), o_l1s = L.take<int32_t>(cap_l1);
    size_t o_l3c = L.take<uint32_t>(C), o_l3o = L.take<uint32_t>(C + 1), o_l3s = L.take<int32_t>(cap_l3);
    size_t o_l1slot = L.take<int32_t>(C * kListSlot1), o_l3slot = L.take<int32_t>(C * kListSlot3);
    size_t o_a = L.take<double2>(C * (P + 1)), o_b = L.take<double2>(C * (P + 1)), o_cnt = L.take<unsigned>(C);
    size_t o_fx = L.take<double>(n), o_fy = L.take<double>(n);
    size_t o_nx = L.take<double>(n), o_ny = L.take<double>(n);
    size_t o_geom = L.take<Geom2D>(1), o_info = L.take<TreeInfo2D>(1);
    size_t o_coef = L.take<double>(3 * kCoefTable);
    size_t o_op = L.take<double2>((size_t)49 * (P + 1) * P);
    const int dlev = dense_levels_for(n);
    size_t o_dense = L.take<int32_t>((size_t)dense_entries(dlev));
    size_t o_mixed = L.take<char>(mixed_bytes(n, cap_cells, P));

    drop_graph();
    if (arena2d) cudaFree(arena2d);
    arena2d = nullptr;
    cap = Caps2D{};
    cudaError_t e = cudaMalloc(&arena2d, L.total);
    if (e != cudaSuccess) {
        arena2d = nullptr;
        return fail_cuda(e, "cudaMalloc of the 2D arena");
    }
    arena2d_bytes = L.total;
    char* base = (char*)arena2d;
    auto P_ = [&](size_t off) { return (void*)(base + off); };
    in_x = (double*)P_(o_x); in_y = (double*)P_(o_y); in_q = (double*)P_(o_q); in_act = (uint8_t*)P_(o_act);
    out0 = (double*)P_(o_o0); out1 = (double*)P_(o_o1);
    tree.key = (uint64_t*)P_(o_key); tree.perm = (uint32_t*)P_(o_perm);
    tree.px = (double*)P_(o_px); tree.py = (double*)P_(o_py); tree.pq = (double*)P_(o_pq);
    tree.pact = (uint8_t*)P_(o_pact); tree.actscan = (uint32_t*)P_(o_actscan);
    ts.key_alt = (uint64_t*)P_(o_keyalt); ts.val_alt = (uint32_t*)P_(o_valalt); ts.act_u32 = (uint32_t*)P_(o_actu);
    ts.bbox_partial = (double*)P_(o_bbox); ts.coop_words = (uint32_t*)P_(o_coop);
    ts.lvl_ticket = (unsigned*)P_(o_ltick);
    ts.pinfo = (uint32_t*)P_(o_pinfo); ts.tile_cnt = (uint32_t*)P_(o_tcnt); ts.level_tot = (uint32_t*)P_(o_ltot);
    ts.flat_tiles = flat_tiles;
    ts.sort.status = (uint32_t*)P_(o_sstat); ts.sort.tickets = (unsigned*)P_(o_stick);
    ts.sort.hist = (uint32_t*)P_(o_hist); ts.sort.max_tiles = s_tiles;
    ts.scan.status = (uint64_t*)P_(o_scstat); ts.scan.ticket = (unsigned*)P_(o_sctick); ts.scan.max_tiles = sc_tiles;
    tree.c_lo = (int32_t*)P_(o_clo); tree.c_hi = (int32_t*)P_(o_chi); tree.c_src = (int32_t*)P_(o_csrc);
    tree.c_parent = (int32_t*)P_(o_cpar); tree.c_child0 = (int32_t*)P_(o_cch); tree.c_ix = (int32_t*)P_(o_cix);
    tree.c_iy = (int32_t*)P_(o_ciy); tree.c_leafidx = (int32_t*)P_(o_cleaf);
    tree.c_flags = (uint8_t*)P_(o_cfl); tree.c_chmask = (uint8_t*)P_(o_cmask); tree.c_level = (uint8_t*)P_(o_clev);
    tree.c_cx = (double*)P_(o_ccx); tree.c_cy = (double*)P_(o_ccy); tree.c_code = (uint64_t*)P_(o_ccode);
    tree.leaf_cells = (int32_t*)P_(o_leaves);
    tree.nonleaf = (int32_t*)P_(o_nonleaf);
    lists.l2_blk = (int32_t*)P_(o_l2blk);
    tree.geom = (Geom2D*)P_(o_geom); tree.info = (TreeInfo2D*)P_(o_info);
    tree.dense = (int32_t*)P_(o_dense);
    tree.gbar = ts.lvl_ticket + kBarrierWordsAt;
    tree.dense_levels = dlev;
    tree.cap_cells = cap_cells;
    lists.l2_src = (int32_t*)P_(o_l2); lists.l2_slot = (uint8_t*)P_(o_l2s); lists.l2_n = (uint8_t*)P_(o_l2n);
    lists.l4_src = (int32_t*)P_(o_l4); lists.l4_n = (uint8_t*)P_(o_l4n);
    lists.l1_cnt = (uint32_t*)P_(o_l1c); lists.l1_off = (uint32_t*)P_(o_l1o); lists.l1_src = (int32_t*)P_(o_l1s);
    lists.l3_cnt = (uint32_t*)P_(o_l3c); lists.l3_off = (uint32_t*)P_(o_l3o); lists.l3_src = (int32_t*)P_(o_l3s);
    lists.l1_slot = (int32_t*)P_(o_l1slot); lists.l3_slot = (int32_t*)P_(o_l3slot);
    lists.cap_leaves = cap_cells;
    lists.cap_l1 = cap_l1;
    lists.cap_l3 = cap_l3;
    ex2.a = (double2*)P_(o_a); ex2.b = (double2*)P_(o_b); ex2.up_count = (unsigned*)P_(o_cnt);
    ex2.fx = (double*)P_(o_fx); ex2.fy = (double*)P_(o_fy);
    near_x = (double*)P_(o_nx); near_y = (double*)P_(o_ny);
    ex2.coef = (double*)P_(o_coef);
    ex2.op = (double2*)P_(o_op);
    coef_P = -1;  // the new arena holds no coefficients yet
    mixed_base = P_(o_mixed);
    {
        const size_t r0 = ((sizeof(double4) * (size_t)n + 1023) & ~(size_t)1023);
        tc_rows = (float*)((char*)mixed_base + r0);
        tc_ops = (float*)((char*)tc_rows + ((m2l_tc_rows_bytes(cap_cells) + 1023) & ~(size_t)1023));
    }
    cap.n = n; cap.cells = cap_cells; cap.P = P; cap.l1 = cap_l1; cap.l3 = cap_l3;
    return VPM_OK;
}

int Ctx::map_err(unsigned bits) {
    if (!bits) return VPM_OK;
    if (bits & (ERR_NONFINITE | ERR_RANGE))
        return fail(VPM_EINVAL, "non-finite positions or a degenerate domain (all particles coincide)");
    if (bits & ERR_TIMEOUT) return fail(VPM_ETIMEDOUT, "a bounded device-side wait gave up");
    if (bits & ERR_DEPTH) return fail(VPM_EOVERFLOW, "tree deeper than the key resolution (coincident particles?)");
    if (bits & (ERR_CELL_CAP | ERR_LIST_CAP)) return fail(VPM_EOVERFLOW, "cell or list capacity exceeded");
    if (bits & (ERR_QUEUE | ERR_LIST4 | ERR_LIST2)) return fail(VPM_EOVERFLOW, "interaction-list queue overflow");
    if (bits & ERR_LEAF1)
        return fail(VPM_EINVAL, "3D TreeCell: a level-1 cell is a leaf of a deeper tree (the reference's traversal "
                                "throws there)");
    return fail(VPM_EDEVICE, "device index check failed");
}

int Ctx::check_params(const vpm_fmm_params* prm, vpm_fmm_params& out) {
    if (prm) out = *prm;
    else vpm_fmm_params_default(&out);
    if (out.p < 1 || out.p > kMaxP) return fail(VPM_EINVAL, "p must be in 1..30");
    if (out.max_src < 0 || out.max_par < 1) return fail(VPM_EINVAL, "leaf caps must be max_src >= 0, max_par >= 1");
    if (out.max_depth != 16 && out.max_depth != 31) out.max_depth = 16;
    if (!(out.exp_tree_pct >= 0.0) || !std::isfinite(out.exp_tree_pct)) return fail(VPM_EINVAL, "exp_tree_pct");
    if (out.support_3d == 0.0) out.support_3d = 2.0;
    if (!(out.support_3d >= 1.0) || !std::isfinite(out.support_3d))
        return fail(VPM_EINVAL, "support_3d must be a finite factor >= 1");
    if (out.precision != VPM_PREC_FP64 && out.precision != VPM_PREC_MIXED && out.precision != VPM_PREC_MIXED_FP64_M2L &&
        out.precision != VPM_PREC_MIXED_TC)
        return fail(VPM_EINVAL, "precision");
    return VPM_OK;
}

int Ctx::plan_caps(int n, const vpm_fmm_params& p, int& cells, long long& l1, long long& l3) {
    int m = std::max(1, std::min(p.max_src, p.max_par));
    long long c = 8ll * n / m + 4096;
    c = std::max<long long>(c, (long long)cap.cells);
    if (c > (1ll << 30)) return fail(VPM_EINVAL, "too many cells");
    cells = (int)c;
    l1 = std::max<long long>(16ll * cells, cap.l1);
    l3 = std::max<long long>(8ll * cells, cap.l3);
    return VPM_OK;
}

// Enqueue one 2D evaluation on device buffers. mode: 0 field, 1 velocity.
int Ctx::enqueue2d(const double* x, const double* y, const double* q, const uint8_t* act, int n,
                   const vpm_fmm_params& p, int K, double* o0, double* o1, int velocity, double uinf,
                   double vinf, bool tree_only) {
    cudaStream_t st = stream;
    int launches = 0;
    tree.n = n;
    tree.key_levels = K;
    VPM_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(unsigned), st));
    if (int r = ensure_coefs(p)) return r;
    if (int r = record(0)) return r;
    // Strengths still in flight on `upload` (q_ready): sort without them and
    // gather them in tree order just before their first reader.
    const bool deferred = q_ready != nullptr && !tree_only;
    const unsigned wait_flags = capturing ? cudaEventWaitExternal : 0u;
    VPM_CUDA_TRY(keys_sort2d(x, y, deferred ? nullptr : q, act, tree, ts, p.exp_tree_pct, d_err, st, &launches,
                             std::min(p.max_src, p.max_par), sort_items));
    if (int r = record(1)) return r;
    VPM_CUDA_TRY(levels2d(tree, ts, p.max_src, p.max_par, d_err, st, &launches));
    if (int r = record(2)) return r;
    if (capturing && !split_capture && !tree_only && velocity != kModePotential) {
        // One captured graph: the near field (lists 1/3, P2P) runs on the side
        // stream concurrently with lists 2/4 and the far field (P2M, M2M, M2L,
        // L2L); M2P follows lists 2/4 on the third stream once the upward pass
        // and list 3 are done (the mixed form: list 3 from the slots, the few
        // leaves that outgrew them after the CSR on the fourth stream; its M2L
        // of the levels below the large cells also runs on the third stream,
        // beside the large cells' M2M loop); L2P then adds the M2P and
        // near-field sums and writes the output.
        VPM_CUDA_TRY(cudaEventRecord(fork2, st));
        VPM_CUDA_TRY(cudaStreamWaitEvent(side, fork2, 0));
        if (deferred) {
            VPM_CUDA_TRY(cudaStreamWaitEvent(st, q_ready, wait_flags));
            VPM_CUDA_TRY(gather_strengths2d(tree, q, d_err, st, &launches));
            VPM_CUDA_TRY(cudaEventRecord(ev_qg, st));
        }
        const bool slots = p.precision != VPM_PREC_FP64 && int_lists_slotted(lists);
        if (slots) {
            // the mixed near field and M2P start from the list slots; the CSR
            // (for the few leaves whose lists outgrew their slots) is built on
            // a third side stream meanwhile
            VPM_CUDA_TRY(build_int_slots2d(tree, lists, p.eps, d_err, side, &launches));
            VPM_CUDA_TRY(cudaEventRecord(ev_slots, side));
            if (deferred) VPM_CUDA_TRY(cudaStreamWaitEvent(side, ev_qg, 0));
            VPM_CUDA_TRY(fmm2d_p2p_f32(tree, lists, ex2, near_x, near_y, 0, 0.0, 0.0, d_err, side, &launches, true,
                                       kP2PListSlots));
            VPM_CUDA_TRY(cudaStreamWaitEvent(side3, ev_slots, 0));
            VPM_CUDA_TRY(build_int_csr2d(tree, lists, ts.scan, p.eps, d_err, side3, &launches));
            VPM_CUDA_TRY(cudaEventRecord(ev_l13, side3));
            if (deferred) VPM_CUDA_TRY(cudaStreamWaitEvent(side3, ev_qg, 0));
            VPM_CUDA_TRY(fmm2d_p2p_f32(tree, lists, ex2, near_x, near_y, 0, 0.0, 0.0, d_err, side3, &launches, true,
                                       kP2PListSpill));
        } else {
            VPM_CUDA_TRY(build_int_lists2d(tree, lists, ts.scan, p.eps, d_err, side, &launches));
            VPM_CUDA_TRY(cudaEventRecord(ev_l13, side));
            if (deferred) VPM_CUDA_TRY(cudaStreamWaitEvent(side, ev_qg, 0));
            if (p.precision != VPM_PREC_FP64)
                VPM_CUDA_TRY(fmm2d_p2p_f32(tree, lists, ex2, near_x, near_y, 0, 0.0, 0.0, d_err, side, &launches, true));
            else
                VPM_CUDA_TRY(fmm2d_p2p_f64_tma(tree, lists, ex2, (double4*)mixed_base, near_x, near_y, 0, 0.0, 0.0,
                                               d_err, side, &launches, p.max_par, true));
        }
        VPM_CUDA_TRY(cudaEventRecord(join2, side));
        VPM_CUDA_TRY(cudaStreamWaitEvent(side2, fork2, 0));
        VPM_CUDA_TRY(build_ext_lists2d(tree, lists, p.eps, d_err, side2, &launches));
        VPM_CUDA_TRY(cudaEventRecord(join3, side2));
        // mixed form: the per-parent M2L of the levels below the cells left
        // to the M2M loop runs on the lists-2/4 stream as soon as the other
        // moments are final, beside that loop; the rest follows it
        const bool split = split_m2l && p.precision == VPM_PREC_MIXED && m2l_parent_f32_supported(p.p) &&
                           lists.l2_blk && tree.nonleaf && tree.gbar;
        VPM_CUDA_TRY(fmm2d_upward_direct(tree, ex2, p.p, p.binom == VPM_BINOM_EXACT, d_err, st, &launches,
                                         split ? ev_small : nullptr));
        VPM_CUDA_TRY(cudaEventRecord(ev_up, st));
        if (split) {
            VPM_CUDA_TRY(cudaStreamWaitEvent(side2, ev_small, 0));
            VPM_CUDA_TRY(fmm2d_m2l_parent_f32(tree, lists, ex2, p.p, p.binom == VPM_BINOM_EXACT, d_err, side2,
                                              &launches, 1));
            VPM_CUDA_TRY(cudaEventRecord(ev_m2ld, side2));
        }
        if (slots) {
            // M2P of the leaves whose list 3 outgrew its slots, after their
            // CSR (the others: from the slots on the third stream below)
            VPM_CUDA_TRY(cudaStreamWaitEvent(side3, ev_up, 0));
            VPM_CUDA_TRY(fmm2d_m2p(tree, lists, ex2, p.p, d_err, side3, &launches, kP2PListSpill));
            VPM_CUDA_TRY(cudaEventRecord(join5, side3));
        }
        VPM_CUDA_TRY(cudaStreamWaitEvent(side2, ev_up, 0));
        VPM_CUDA_TRY(cudaStreamWaitEvent(side2, slots ? ev_slots : ev_l13, 0));
        VPM_CUDA_TRY(fmm2d_m2p(tree, lists, ex2, p.p, d_err, side2, &launches, slots ? kP2PListSlots : kP2PListCsr));
        VPM_CUDA_TRY(cudaEventRecord(join4, side2));
        VPM_CUDA_TRY(cudaStreamWaitEvent(st, join3, 0));
        if (split) {
            VPM_CUDA_TRY(fmm2d_m2l_parent_f32(tree, lists, ex2, p.p, p.binom == VPM_BINOM_EXACT, d_err, st,
                                              &launches, 2));
            VPM_CUDA_TRY(cudaStreamWaitEvent(st, ev_m2ld, 0));
            VPM_CUDA_TRY(fmm2d_m2l_list4(tree, lists, ex2, p.p, d_err, st, &launches));
        } else if (int r = enqueue_m2l(p, st, &launches)) {
            return r;
        }
        if (l2l_direct_ok(p.p, p.binom == VPM_BINOM_EXACT))
            VPM_CUDA_TRY(fmm2d_l2l_leaves(tree, ex2, p.p, d_err, st, &launches));
        else
            VPM_CUDA_TRY(fmm2d_l2l(tree, ex2, p.p, d_err, st, &launches));
        VPM_CUDA_TRY(cudaStreamWaitEvent(st, join2, 0));
        VPM_CUDA_TRY(cudaStreamWaitEvent(st, join4, 0));
        if (slots) VPM_CUDA_TRY(cudaStreamWaitEvent(st, join5, 0));
        VPM_CUDA_TRY(fmm2d_eval_combine(tree, lists, ex2, p.p, near_x, near_y, o0, o1, velocity, uinf, vinf, d_err, st,
                                        &launches, true));
        last_launches = launches;
        last_params = p;
        last_n = n;
        have_tree = true;
        return VPM_OK;
    }
    VPM_CUDA_TRY(build_lists2d(tree, lists, ts.scan, p.eps, d_err, st, &launches));
    if (int r = record(3)) return r;
    if (tree_only) {
        for (int i = 4; i < kStageEvents; ++i)
            if (int r = record(i)) return r;
    } else {
        if (deferred) {
            VPM_CUDA_TRY(cudaStreamWaitEvent(st, q_ready, wait_flags));
            VPM_CUDA_TRY(gather_strengths2d(tree, q, d_err, st, &launches));
        }
        VPM_CUDA_TRY(fmm2d_upward_direct(tree, ex2, p.p, p.binom == VPM_BINOM_EXACT, d_err, st, &launches));
        if (int r = record(4)) return r;
        if (velocity == kModePotential) VPM_CUDA_TRY(fmm2d_m2l_only(tree, lists, ex2, p.p, d_err, st, &launches));
        else if (int r = enqueue_m2l(p, st, &launches)) return r;
        if (velocity == kModePotential) VPM_CUDA_TRY(fmm2d_m2l_b0(tree, lists, ex2, p.p, d_err, st, &launches));
        if (int r = record(5)) return r;
        if (l2l_direct_ok(p.p, p.binom == VPM_BINOM_EXACT))
            VPM_CUDA_TRY(fmm2d_l2l_leaves(tree, ex2, p.p, d_err, st, &launches));
        else
            VPM_CUDA_TRY(fmm2d_l2l(tree, ex2, p.p, d_err, st, &launches));
        if (int r = record(6)) return r;
        if (velocity == kModePotential) {
            // far field and near field in one stage pair: the events keep their slots
            VPM_CUDA_TRY(fmm2d_potential_eval(tree, lists, ex2, p.p, o0, d_err, st, &launches));
            if (int r = record(7)) return r;
        } else {
            VPM_CUDA_TRY(fmm2d_eval(tree, lists, ex2, p.p, d_err, st, &launches));
            if (int r = record(7)) return r;
        }
        if (velocity == kModePotential) {
        } else if (p.precision != VPM_PREC_FP64) {
            VPM_CUDA_TRY(fmm2d_p2p_f32(tree, lists, ex2, o0, o1, velocity, uinf, vinf, d_err, st, &launches));
        } else {
            VPM_CUDA_TRY(fmm2d_p2p_f64_tma(tree, lists, ex2, (double4*)mixed_base, o0, o1, velocity, uinf, vinf, d_err,
                                           st, &launches, p.max_par));
        }
        if (int r = record(8)) return r;
    }
    last_launches = launches;
    last_params = p;
    last_n = n;
    have_tree = true;
    return VPM_OK;
}

// M2L of lists 2 and 4 for the precision setting: the mixed form per parent
// on the FP32 pipes (orders 1..16), the tensor-core variants for
// VPM_PREC_MIXED_TC (per parent, orders 1..16) and for the mixed orders 17..20
// (per offset), FP64 otherwise.
int Ctx::enqueue_m2l(const vpm_fmm_params& p, cudaStream_t st, int* launches) {
    const bool exact = p.binom == VPM_BINOM_EXACT;
    if (p.precision == VPM_PREC_MIXED && m2l_parent_f32_supported(p.p))
        VPM_CUDA_TRY(fmm2d_m2l_parent_f32(tree, lists, ex2, p.p, exact, d_err, st, launches));
    else if (p.precision == VPM_PREC_MIXED_TC && m2l_parent_supported(p.p))
        VPM_CUDA_TRY(fmm2d_m2l_parent(tree, lists, ex2, p.p, tc_rows, tc_ops, d_err, st, launches));
    else if ((p.precision == VPM_PREC_MIXED || p.precision == VPM_PREC_MIXED_TC) && m2l_tc_supported(p.p))
        VPM_CUDA_TRY(fmm2d_m2l_tc(tree, lists, ex2, p.p, tc_rows, tc_ops, d_err, st, launches));
    else
        VPM_CUDA_TRY(fmm2d_m2l_only(tree, lists, ex2, p.p, d_err, st, launches));
    return VPM_OK;
}

// Translation coefficients, list-2 operators (FP64 and tensor-core forms) of
// order p.p on this context's arena; uploaded when the order, the binomials
// or the arena changed. The uploads synchronise the stream, so callers that
// capture graphs call this before the capture begins.
int Ctx::ensure_coefs(const vpm_fmm_params& p) {
    if (coef_P == p.p && coef_binom == p.binom) return VPM_OK;
    if (capturing) return fail(VPM_EINVAL, "coefficient upload inside a graph capture");
    VPM_CUDA_TRY(set_coefficients2d(p.p, p.binom == VPM_BINOM_EXACT, ex2.coef, stream));
    VPM_CUDA_TRY(set_m2l_operators2d(p.p, p.binom == VPM_BINOM_EXACT, ex2.op, stream));
    if (m2l_parent_supported(p.p)) VPM_CUDA_TRY(set_m2l_parent_operators(p.p, ex2.op, tc_ops, stream));
    else if (m2l_tc_supported(p.p)) VPM_CUDA_TRY(set_m2l_tc_operators(p.p, ex2.op, tc_ops, stream));
    coef_P = p.p;
    coef_binom = p.binom;
    return VPM_OK;
}

// Stage mark i. Eager launches record event i. While one graph is being
// captured (use_graph = 1) marks are skipped: event nodes inside the graph
// would cost more than the stages they time. While per-stage graphs are
// being captured (use_graph = 2) a mark closes the graph of the previous
// stage and opens the next; replay records the events between stage graphs.
int Ctx::record(int i) {
    if (!capturing) {
        VPM_CUDA_TRY(cudaEventRecord(ev[i], stream));
        if (ring_cur >= 0) VPM_CUDA_TRY(cudaEventRecord(ring[ring_cur][i], stream));
        return VPM_OK;
    }
    if (!split_capture || i == 0) return VPM_OK;
    cudaGraph_t g = nullptr;
    VPM_CUDA_TRY(cudaStreamEndCapture(stream, &g));
    cudaGraphExec_t x = nullptr;
    cudaError_t e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGraphInstantiate (stage)");
    stage_exec[i - 1] = x;
    if (i < kStageEvents - 1) VPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    return VPM_OK;
}

// The ring slot for the evaluation about to be enqueued (if the ring is on).
void Ctx::begin_ring() {
    ring_cur = -1;
    if (!ring_on) return;
    if (!ring[0][0]) {
        for (auto& row : ring)
            for (auto& e : row) cudaEventCreate(&e);
    }
    ring_cur = (ring_head + ring_count) % kRing;
    if (ring_count == kRing) ring_head = (ring_head + 1) % kRing;
    else ++ring_count;
}

void Ctx::end_ring() { ring_cur = -1; }

void Ctx::drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    for (auto& x : stage_exec) {
        if (x) cudaGraphExecDestroy(x);
        x = nullptr;
    }
}

// Enqueue (or replay) one evaluation on device buffers. With p.use_graph the
// whole evaluation is captured once per (buffers, n, parameters, stream,
// arena) and replayed as a CUDA graph: every launch in it reads its sizes from
// device memory, so the same graph is valid for any particle set of this size.
int Ctx::launch2d(const double* x, const double* y, const double* q, const uint8_t* act, int n,
                  const vpm_fmm_params& p, int K, double* o0, double* o1, int velocity, double uinf,
                  double vinf) {
    if (!p.use_graph) {
        last_timed = true;
        begin_ring();
        int r = enqueue2d(x, y, q, act, n, p, K, o0, o1, velocity, uinf, vinf, false);
        end_ring();
        return r;
    }
    GraphKey k;
    std::memset(&k, 0, sizeof(k));  // padding included: the key is compared bytewise
    k.ptr[0] = x; k.ptr[1] = y; k.ptr[2] = q; k.ptr[3] = act; k.ptr[4] = o0; k.ptr[5] = o1;
    k.n = n; k.K = K; k.velocity = velocity; k.uinf = uinf; k.vinf = vinf; k.p = p; k.stream = stream;
    k.arena = arena2d;
    k.deferred = q_ready != nullptr;
    const bool split = p.use_graph == 2;
    const bool have = split ? stage_exec[0] != nullptr : gexec != nullptr;
    if (have && std::memcmp(&k, &gkey, sizeof(k)) == 0) {
        if (split) {
            begin_ring();
            if (int r = record(0)) return r;
            for (int i = 0; i < kStageEvents - 1; ++i) {
                VPM_CUDA_TRY(cudaGraphLaunch(stage_exec[i], stream));
                if (int r = record(i + 1)) return r;
            }
            end_ring();
        } else {
            VPM_CUDA_TRY(cudaGraphLaunch(gexec, stream));
        }
        last_launches = graph_launches;
        last_n = n;
        last_timed = split;
        return VPM_OK;
    }
    drop_graph();
    if (int r = ensure_coefs(p)) return r;  // uploads synchronise: never inside a capture
    VPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    split_capture = split;
    int r = enqueue2d(x, y, q, act, n, p, K, o0, o1, velocity, uinf, vinf, false);
    capturing = false;
    split_capture = false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(stream, &cs);
    if (r != VPM_OK) {
        if (cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
        }
        drop_graph();
        return r;
    }
    if (!split) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            gexec = nullptr;
            return fail_cuda(e, "cudaGraphInstantiate");
        }
    }
    std::memcpy(&gkey, &k, sizeof(k));
    graph_launches = last_launches;
    return launch2d(x, y, q, act, n, p, K, o0, o1, velocity, uinf, vinf);
}

int Ctx::collect_stats(vpm_fmm_stats* s) {
    std::memset(s, 0, sizeof(*s));
    if (!have_tree) return VPM_OK;
    TreeInfo2D info;
    VPM_CUDA_TRY(cudaMemcpyAsync(&info, tree.info, sizeof(info), cudaMemcpyDeviceToHost, stream));
    VPM_CUDA_TRY(cudaStreamSynchronize(stream));
    s->n = last_n;
    s->n_cells = info.n_cells;
    s->n_leaves = info.n_leaves;
    s->min_level = info.min_leaf_level;
    s->max_level = info.max_leaf_level;
    s->list1_len = (int64_t)info.list1_len;
    s->list3_len = (int64_t)info.list3_len;
    float ms[kStageEvents] = {0};
    if (last_timed)
        for (int i = 1; i < kStageEvents; ++i) cudaEventElapsedTime(&ms[i], ev[i - 1], ev[i]);
    s->ms_keys_sort = ms[1];
    s->ms_levels = ms[2];
    s->ms_tree = ms[1] + ms[2];
    s->ms_lists = ms[3];
    s->ms_upward = ms[4];
    s->ms_m2l = ms[5];
    s->ms_l2l = ms[6];
    s->ms_eval = ms[7];
    s->ms_p2p = ms[8];
    if (last_timed) cudaEventElapsedTime(&s->ms_total, ev[0], ev[kStageEvents - 1]);
    s->kernels = last_launches;
    s->depth_retry = depth_retry;
    // Interaction counts (exact, from the lists).
    return count_interactions(s);
}

// Host-synchronous driver: copies, enqueue, sync, error handling with
// capacity / depth retries.
int Ctx::run2d_host(const double* x, const double* y, const double* q_or_omega, const double* s,
                    const uint8_t* act, int64_t n64, const vpm_fmm_params* prm, double* o0, double* o1,
                    int velocity, double uinf, double vinf, vpm_fmm_stats* stats, bool tree_only) {
    vpm_fmm_params p;
    int r = check_params(prm, p);
    if (r) return r;
    if (n64 < 0 || n64 >= (1ll << 30)) return fail(VPM_EINVAL, "n out of range");
    if (!x || !y || !act || (!tree_only && (!q_or_omega || !o0 || (!o1 && velocity != kModePotential))) ||
        (velocity == 1 && !s))
        return fail(VPM_EINVAL, "null buffer");
    const int n = (int)n64;
    if (n == 0) return VPM_OK;
    if (n == 1) return fail(VPM_EINVAL, "a single particle gives a zero-size root cell (the reference fails there too)");
    depth_retry = 0;
    int K = p.max_depth;
    for (int attempt = 0; attempt < 6; ++attempt) {
        int cells;
        long long l1, l3;
        r = plan_caps(n, p, cells, l1, l3);
        if (r) return r;
        if (attempt > 0 && grow) {
            cells = (int)std::min<long long>(2ll * cap.cells, 1ll << 30);
            l1 = 2 * cap.l1;
            l3 = 2 * cap.l3;
            grow = false;
        }
        r = reserve2d(n, cells, p.p, l1, l3);
        if (r) return r;
        // Positions and flags first on the main stream: the sort and the tree
        // and list builds need nothing else. The strengths (or vorticity and
        // core size) follow on `upload`, ordered after them on the copy
        // engine, and are waited for only where P2M and P2P first read them.
        VPM_CUDA_TRY(cudaMemcpyAsync(in_x, x, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        VPM_CUDA_TRY(cudaMemcpyAsync(in_y, y, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        VPM_CUDA_TRY(cudaMemcpyAsync(in_act, act, n, cudaMemcpyHostToDevice, stream));
        if (tree_only) {
            VPM_CUDA_TRY(cudaMemsetAsync(in_q, 0, sizeof(double) * n, stream));
        } else {
            VPM_CUDA_TRY(cudaEventRecord(ev_upload, stream));
            VPM_CUDA_TRY(cudaStreamWaitEvent(upload, ev_upload, 0));
            VPM_CUDA_TRY(cudaMemcpyAsync(in_q, q_or_omega, sizeof(double) * n, cudaMemcpyHostToDevice, upload));
            if (velocity == 1) {
                // the core sizes pass through out0, which the evaluation
                // writes only after it has waited for ev_q
                VPM_CUDA_TRY(cudaMemcpyAsync(out0, s, sizeof(double) * n, cudaMemcpyHostToDevice, upload));
                source_from_vorticity<<<std::min(1184, ceil_div(n, 256)), 256, 0, upload>>>(in_q, out0, n, in_q);
                VPM_CUDA_TRY(cudaGetLastError());
            }
            VPM_CUDA_TRY(cudaEventRecord(ev_q, upload));
            q_ready = ev_q;
        }
        last_was_graph = p.use_graph != 0 && !tree_only;
        if (tree_only) last_timed = true;
        r = tree_only ? enqueue2d(in_x, in_y, in_q, in_act, n, p, K, out0, out1, velocity, uinf, vinf, true)
                      : launch2d(in_x, in_y, in_q, in_act, n, p, K, out0, out1, velocity, uinf, vinf);
        q_ready = nullptr;
        if (r) {
            cudaStreamSynchronize(upload);
            return r;
        }
        // The error word and the outputs in one round trip: on an error the
        // outputs are discarded (retried, or the call fails).
        unsigned bits = 0;
        VPM_CUDA_TRY(cudaMemcpyAsync(&bits, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        if (!tree_only) {
            VPM_CUDA_TRY(cudaMemcpyAsync(o0, out0, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
            if (o1) VPM_CUDA_TRY(cudaMemcpyAsync(o1, out1, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        }
        VPM_CUDA_TRY(cudaStreamSynchronize(stream));
        if (bits & ERR_DEPTH) {
            if (K < kMaxLevels2D) { K = kMaxLevels2D; depth_retry = 1; continue; }
            return map_err(bits);
        }
        if (bits & (ERR_CELL_CAP | ERR_LIST_CAP)) { grow = true; continue; }
        if (bits) return map_err(bits);
        if (tree_only) return stats ? collect_stats(stats) : VPM_OK;
        if (stats) return collect_stats(stats);
        return VPM_OK;
    }
    return fail(VPM_EOVERFLOW, "capacity retries exhausted");
}

// ---------------------------------------------------------------------------
// Dumps (host-side reconstruction of the reference's vocabulary).
// ---------------------------------------------------------------------------
int Ctx::fetch_tree(HostTree2D& h) {
    if (!have_tree) return fail(VPM_EINVAL, "no 2D tree on this context yet");
    TreeInfo2D info;
    VPM_CUDA_TRY(cudaMemcpyAsync(&info, tree.info, sizeof(info), cudaMemcpyDeviceToHost, stream));
    VPM_CUDA_TRY(cudaStreamSynchronize(stream));
    const int nc = info.n_cells, nl = info.n_leaves, n = last_n;
    h.nc = nc; h.nl = nl; h.n = n;
    h.lo.resize(nc); h.hi.resize(nc); h.src.resize(nc); h.ix.resize(nc); h.iy.resize(nc); h.leafidx.resize(nc);
    h.flags.resize(nc); h.level.resize(nc); h.cx.resize(nc); h.cy.resize(nc); h.perm.resize(n);
    h.leaf_cells.resize(nl); h.l2n.resize(nc); h.l4n.resize(nc);
    h.l2.resize((size_t)nc * kList2Cap); h.l4.resize((size_t)nc * kList4Cap);
    h.l1off.resize(nl + 1); h.l3off.resize(nl + 1);
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
    };
    VPM_CUDA_TRY(cp(h.lo.data(), tree.c_lo, 4ull * nc));
    VPM_CUDA_TRY(cp(h.hi.data(), tree.c_hi, 4ull * nc));
    VPM_CUDA_TRY(cp(h.src.data(), tree.c_src, 4ull * nc));
    VPM_CUDA_TRY(cp(h.ix.data(), tree.c_ix, 4ull * nc));
    VPM_CUDA_TRY(cp(h.iy.data(), tree.c_iy, 4ull * nc));
    VPM_CUDA_TRY(cp(h.leafidx.data(), tree.c_leafidx, 4ull * nc));
    VPM_CUDA_TRY(cp(h.flags.data(), tree.c_flags, nc));
    VPM_CUDA_TRY(cp(h.level.data(), tree.c_level, nc));
    VPM_CUDA_TRY(cp(h.cx.data(), tree.c_cx, 8ull * nc));
    VPM_CUDA_TRY(cp(h.cy.data(), tree.c_cy, 8ull * nc));
    VPM_CUDA_TRY(cp(h.perm.data(), tree.perm, 4ull * n));
    VPM_CUDA_TRY(cp(h.leaf_cells.data(), tree.leaf_cells, 4ull * nl));
    VPM_CUDA_TRY(cp(h.l2n.data(), lists.l2_n, nc));
    VPM_CUDA_TRY(cp(h.l4n.data(), lists.l4_n, nc));
    VPM_CUDA_TRY(cp(h.l2.data(), lists.l2_src, 4ull * nc * kList2Cap));
    VPM_CUDA_TRY(cp(h.l4.data(), lists.l4_src, 4ull * nc * kList4Cap));
    VPM_CUDA_TRY(cp(h.l1off.data(), lists.l1_off, 4ull * (nl + 1)));
    VPM_CUDA_TRY(cp(h.l3off.data(), lists.l3_off, 4ull * (nl + 1)));
    VPM_CUDA_TRY(cudaStreamSynchronize(stream));
    h.l1.resize(h.l1off[nl]);
    h.l3.resize(h.l3off[nl]);
    if (!h.l1.empty()) VPM_CUDA_TRY(cp(h.l1.data(), lists.l1_src, 4ull * h.l1.size()));
    if (!h.l3.empty()) VPM_CUDA_TRY(cp(h.l3.data(), lists.l3_src, 4ull * h.l3.size()));
    VPM_CUDA_TRY(cudaStreamSynchronize(stream));
    h.id.resize(nc);
    for (int c = 0; c < nc; ++c) h.id[c] = start_id2(h.level[c]) + h.ix[c] + ((int64_t)h.iy[c] << h.level[c]);
    h.by_id.resize(nc);
    for (int c = 0; c < nc; ++c) h.by_id[c] = c;
    std::sort(h.by_id.begin(), h.by_id.end(), [&](int a, int b) { return h.id[a] < h.id[b]; });
    return VPM_OK;
}

}  // namespace vpm

using vpm::Ctx;

extern "C" {

void vpm_fmm_params_default(vpm_fmm_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->p = 10;
    p->max_src = 50;
    p->max_par = 75;
    p->leaf_cap_3d = 30;
    p->exp_tree_pct = 1.0;
    p->eps = 10e-10;
    p->precision = VPM_PREC_FP64;
    p->binom = VPM_BINOM_REFERENCE;
    p->max_depth = 16;
    p->support_3d = 2.0;
}

int vpm_ctx_create(int device, vpm_ctx** out) {
    if (!out) return VPM_EINVAL;
    *out = nullptr;
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) return VPM_ENOMEM;
    int r = c->init(device);
    if (r != VPM_OK) {
        delete c;
        return r;
    }
    *out = (vpm_ctx*)c;
    return VPM_OK;
}

int vpm_ctx_destroy(vpm_ctx* ctx) {
    if (!ctx) return VPM_EINVAL;
    delete (Ctx*)ctx;
    return VPM_OK;
}

int vpm_ctx_set_stream(vpm_ctx* ctx, void* s) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return VPM_OK;
}

int vpm_ctx_sync(vpm_ctx* ctx) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    unsigned bits = 0;
    e = cudaMemcpyAsync(&bits, c->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail_cuda(e, "vpm_ctx_sync");
    if (c->batch_subs > 0) {  // errors of the sub-contexts of the last batch
        unsigned b = 0;
        int r = c->batch_errors(&b);
        if (r) return r;
        bits |= b;
        c->batch_subs = 0;
    }
    return c->map_err(bits);
}

const char* vpm_last_error(vpm_ctx* ctx) {
    if (!ctx) return "null context";
    return ((Ctx*)ctx)->last_error.c_str();
}

int vpm_fmm2d_field(vpm_ctx* ctx, const double* x, const double* y, const double* q, const uint8_t* active,
                    int64_t n, const vpm_fmm_params* prm, double* ex, double* ey, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run2d_host(x, y, q, nullptr, active, n, prm, ex, ey, 0, 0.0, 0.0, stats, false);
}

int vpm_tree2d_build(vpm_ctx* ctx, const double* x, const double* y, const uint8_t* active, int64_t n,
                     const vpm_fmm_params* prm, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run2d_host(x, y, nullptr, nullptr, active, n, prm, nullptr, nullptr, 0, 0.0, 0.0, stats, true);
}

int vpm_velocity2d(vpm_ctx* ctx, const double* x, const double* y, const double* omega, const double* s,
                   const uint8_t* active, int64_t n, const vpm_fmm_params* prm, double u_inf, double v_inf,
                   double* u, double* v, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run2d_host(x, y, omega, s, active, n, prm, u, v, 1, u_inf, v_inf, stats, false);
}

int vpm_fmm2d_potential(vpm_ctx* ctx, const double* x, const double* y, const double* q, const uint8_t* active,
                        int64_t n, const vpm_fmm_params* prm, double* phi, vpm_fmm_stats* stats) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->run2d_host(x, y, q, nullptr, active, n, prm, phi, nullptr, vpm::kModePotential, 0.0, 0.0, stats, false);
}

int vpm_fmm2d_field_device(vpm_ctx* ctx, const double* x, const double* y, const double* q, const uint8_t* active,
                           int64_t n64, const vpm_fmm_params* prm, double* ex, double* ey) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    vpm_fmm_params p;
    int r = c->check_params(prm, p);
    if (r) return r;
    if (n64 < 2 || n64 >= (1ll << 30)) return c->fail(VPM_EINVAL, "n must be in 2..2^30-1 for the device entry point");
    if (!x || !y || !q || !active || !ex || !ey) return c->fail(VPM_EINVAL, "null buffer");
    const int n = (int)n64;
    int cells;
    long long l1, l3;
    r = c->plan_caps(n, p, cells, l1, l3);
    if (r) return r;
    r = c->reserve2d(n, cells, p.p, l1, l3);
    if (r) return r;
    c->last_was_graph = p.use_graph != 0;
    return c->launch2d(x, y, q, active, n, p, p.max_depth, ex, ey, 0, 0.0, 0.0);
}

int vpm_stage_history(vpm_ctx* ctx, int32_t enable, int32_t max_entries, float* ms, int32_t* count) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    int got = 0;
    if (ms && max_entries > 0 && c->ring_count > 0) {
        e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return c->fail_cuda(e, "vpm_stage_history");
        for (int k = 0; k < c->ring_count && got < max_entries; ++k) {
            const int slot = (c->ring_head + k) % Ctx::kRing;
            for (int i = 0; i + 1 < vpm::kStageEvents; ++i) {
                float v = 0.f;
                cudaEventElapsedTime(&v, c->ring[slot][i], c->ring[slot][i + 1]);
                ms[(size_t)got * (vpm::kStageEvents - 1) + i] = v;
            }
            ++got;
        }
    }
    if (count) *count = got;
    c->ring_head = 0;
    c->ring_count = 0;
    c->ring_on = enable ? 1 : 0;
    return VPM_OK;
}

int vpm_last_stats(vpm_ctx* ctx, vpm_fmm_stats* stats) {
    if (!ctx || !stats) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return c->collect_stats(stats);
}

int vpm_tree2d_counts(vpm_ctx* ctx, int64_t* n_cells, int64_t* n_leaves, int64_t list_len[4]) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    vpm::HostTree2D& h = c->host_tree;
    int r = c->fetch_tree(h);
    if (r) return r;
    if (n_cells) *n_cells = h.nc;
    if (n_leaves) *n_leaves = h.nl;
    if (list_len) {
        int64_t s2 = 0, s4 = 0;
        for (int i = 0; i < h.nc; ++i) { s2 += h.l2n[i]; s4 += h.l4n[i]; }
        list_len[0] = (int64_t)h.l1.size();
        list_len[1] = s2;
        list_len[2] = (int64_t)h.l3.size();
        list_len[3] = s4;
    }
    return VPM_OK;
}

int vpm_tree2d_cells(vpm_ctx* ctx, int64_t* ids, int32_t* ints6, double* centers2) {
    if (!ctx || !ids || !ints6 || !centers2) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    vpm::HostTree2D& h = c->host_tree;
    if (h.nc == 0) return c->fail(VPM_EINVAL, "call vpm_tree2d_counts first");
    for (int k = 0; k < h.nc; ++k) {
        const int i = h.by_id[k];
        ids[k] = h.id[i];
        int32_t* r = ints6 + 6 * k;
        r[0] = h.level[i]; r[1] = h.ix[i]; r[2] = h.iy[i]; r[3] = h.hi[i] - h.lo[i]; r[4] = h.src[i];
        r[5] = (h.flags[i] & vpm::CELL_LEAF ? 1 : 0) | (h.flags[i] & vpm::CELL_ACTIVE ? 2 : 0);
        centers2[2 * k] = h.cx[i];
        centers2[2 * k + 1] = h.cy[i];
    }
    return VPM_OK;
}

int vpm_tree2d_leaves(vpm_ctx* ctx, int64_t* leaf_ids, int64_t* offs, int32_t* pids) {
    if (!ctx || !leaf_ids || !offs || !pids) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    vpm::HostTree2D& h = c->host_tree;
    if (h.nc == 0) return c->fail(VPM_EINVAL, "call vpm_tree2d_counts first");
    // The reference creates the cells of a level in the order of their first
    // (lowest-index) unsettled particle (treeCell.cpp:1152-1171), which is the
    // order of leafList within a level.
    struct LeafKey { int level; uint32_t first; int cell; };
    std::vector<LeafKey> keys(h.nl);
    for (int li = 0; li < h.nl; ++li) {
        const int cc = h.leaf_cells[li];
        uint32_t mn = 0xFFFFFFFFu;
        for (int j = h.lo[cc]; j < h.hi[cc]; ++j) mn = std::min(mn, h.perm[j]);
        keys[li] = {h.level[cc], mn, cc};
    }
    std::sort(keys.begin(), keys.end(), [](const LeafKey& a, const LeafKey& b) {
        return a.level != b.level ? a.level < b.level : a.first < b.first;
    });
    int64_t o = 0;
    std::vector<uint32_t> tmp;
    for (int k = 0; k < h.nl; ++k) {
        const int cc = keys[k].cell;
        leaf_ids[k] = h.id[cc];
        offs[k] = o;
        tmp.assign(h.perm.begin() + h.lo[cc], h.perm.begin() + h.hi[cc]);
        std::sort(tmp.begin(), tmp.end());
        for (uint32_t v : tmp) pids[o++] = (int32_t)v;
    }
    offs[h.nl] = o;
    return VPM_OK;
}

int vpm_tree2d_list(vpm_ctx* ctx, int which, int64_t* cell_ids, int64_t* offs, int64_t* ids) {
    if (!ctx || !cell_ids || !offs || !ids || which < 1 || which > 4) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    vpm::HostTree2D& h = c->host_tree;
    if (h.nc == 0) return c->fail(VPM_EINVAL, "call vpm_tree2d_counts first");
    int64_t m = 0, o = 0;
    for (int k = 0; k < h.nc; ++k) {
        const int i = h.by_id[k];
        const bool leaf = h.flags[i] & vpm::CELL_LEAF;
        if ((which == 1 || which == 3) && !leaf) continue;
        if ((which == 2 || which == 4) && h.level[i] < 2) continue;
        cell_ids[m] = h.id[i];
        offs[m] = o;
        if (which == 1 || which == 3) {
            const int li = h.leafidx[i];
            const std::vector<uint32_t>& off = which == 1 ? h.l1off : h.l3off;
            const std::vector<int32_t>& src = which == 1 ? h.l1 : h.l3;
            for (uint32_t e = off[li]; e < off[li + 1]; ++e) ids[o++] = h.id[src[e]];
        } else if (which == 2) {
            for (int e = 0; e < h.l2n[i]; ++e) ids[o++] = h.id[h.l2[(size_t)i * vpm::kList2Cap + e]];
        } else {
            for (int e = 0; e < h.l4n[i]; ++e) ids[o++] = h.id[h.l4[(size_t)i * vpm::kList4Cap + e]];
        }
        ++m;
    }
    offs[m] = o;
    return VPM_OK;
}

}  // extern "C"
