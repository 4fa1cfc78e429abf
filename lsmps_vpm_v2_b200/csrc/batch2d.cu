// Batched independent 2D solves: many uneven particle sets (one velocity
// evaluation each) in one call. Solves are dealt round-robin to up to
// kBatchStreams sub-contexts, each with its own stream and arena, forked
// from and joined back into the caller's stream by events, so solves of
// different sizes overlap on the GPU. With use_graph the whole batch - every
// solve's launches on every stream - is captured once as one CUDA graph and
// replayed by a single graph launch while the batch layout is unchanged.
#include <algorithm>
#include <cstring>

#include "context.h"

namespace vpm {

namespace {

constexpr int kBatchStreams = 8;

// Word 1 of a context's error buffer collects the error bits of every solve
// the context ran in the current batch (word 0 is reset by each solve).
__global__ void collect_err(unsigned* err) { err[1] |= err[0]; }

}  // namespace

int Ctx::batch2d(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                 const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey) {
    if (ns <= 0) return VPM_OK;
    if (!offs || offs[0] != 0) return fail(VPM_EINVAL, "offsets must start at 0");
    for (int i = 0; i < ns; ++i) {
        const int64_t n = offs[i + 1] - offs[i];
        if (n < 0 || n == 1 || n >= (1ll << 30)) return fail(VPM_EINVAL, "each solve needs 0 or 2..2^30-1 particles");
    }
    const int S = std::min(kBatchStreams, ns);
    while ((int)subs.size() < S) {
        Ctx* c = new (std::nothrow) Ctx();
        if (!c) return fail(VPM_ENOMEM, "sub-context");
        if (int r = c->init(device)) {
            std::string m = c->last_error;
            delete c;
            return fail(r, "sub-context: " + m);
        }
        subs.push_back(c);
        cudaEvent_t e = nullptr;
        VPM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        join_ev.push_back(e);
    }
    if (!fork_ev) VPM_CUDA_TRY(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    // arenas and coefficients of every sub-context before anything is enqueued
    for (int s = 0; s < S; ++s) {
        Ctx* c = subs[s];
        int maxn = 0;
        for (int i = s; i < ns; i += S) maxn = std::max<int>(maxn, (int)(offs[i + 1] - offs[i]));
        if (maxn < 2) continue;
        int cells;
        long long l1, l3;
        if (int r = c->plan_caps(maxn, p, cells, l1, l3)) return fail(r, c->last_error);
        if (int r = c->reserve2d(maxn, cells, p.p, l1, l3)) return fail(r, c->last_error);
        if (int r = c->ensure_coefs(p)) return fail(r, c->last_error);
    }
    batch_subs = S;

    // replay
    std::vector<int64_t> key;
    if (p.use_graph) {
        key.assign(offs, offs + ns + 1);
        const int64_t extra[] = {(int64_t)(intptr_t)x, (int64_t)(intptr_t)y,  (int64_t)(intptr_t)q,
                                 (int64_t)(intptr_t)act, (int64_t)(intptr_t)ex, (int64_t)(intptr_t)ey,
                                 (int64_t)(intptr_t)stream};
        key.insert(key.end(), extra, extra + 7);
        std::vector<int64_t> pk((sizeof(p) + 7) / 8, 0);
        std::memcpy(pk.data(), &p, sizeof(p));
        key.insert(key.end(), pk.begin(), pk.end());
        for (int s = 0; s < S; ++s) key.push_back((int64_t)(intptr_t)subs[s]->arena2d);
        if (batch_exec && key == batch_key) {
            VPM_CUDA_TRY(cudaGraphLaunch(batch_exec, stream));
            return VPM_OK;
        }
        if (batch_exec) cudaGraphExecDestroy(batch_exec);
        batch_exec = nullptr;
        batch_key.clear();
        VPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < S; ++s) subs[s]->capturing = true;
    }
    int r = VPM_OK;
    cudaError_t e = cudaEventRecord(fork_ev, stream);
    for (int s = 0; s < S && e == cudaSuccess; ++s) {
        e = cudaStreamWaitEvent(subs[s]->stream, fork_ev, 0);
        if (e == cudaSuccess) e = cudaMemsetAsync(subs[s]->d_err + 1, 0, sizeof(unsigned), subs[s]->stream);
    }
    for (int i = 0; i < ns && e == cudaSuccess && r == VPM_OK; ++i) {
        const int64_t o = offs[i], n = offs[i + 1] - offs[i];
        if (n == 0) continue;
        Ctx* c = subs[i % S];
        c->last_was_graph = false;
        r = c->enqueue2d(x + o, y + o, q + o, act + o, (int)n, p, p.max_depth, ex + o, ey + o, 0, 0.0, 0.0, false);
        if (r != VPM_OK) {
            last_error = c->last_error;
            break;
        }
        collect_err<<<1, 1, 0, c->stream>>>(c->d_err);
        e = cudaGetLastError();
    }
    for (int s = 0; s < S && e == cudaSuccess; ++s) {
        e = cudaEventRecord(join_ev[s], subs[s]->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join_ev[s], 0);
    }
    if (p.use_graph) {
        for (int s = 0; s < S; ++s) subs[s]->capturing = false;
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && r == VPM_OK) {
            e = cudaGraphInstantiate(&batch_exec, g, 0);
            if (e != cudaSuccess) batch_exec = nullptr;
        }
        if (g) cudaGraphDestroy(g);
        if (e == cudaSuccess && r == VPM_OK) {
            batch_key = key;
            e = cudaGraphLaunch(batch_exec, stream);
        }
    }
    if (r != VPM_OK) return r;
    if (e != cudaSuccess) return fail_cuda(e, "batched solves");
    return VPM_OK;
}

// Error bits of the last batch (all sub-contexts); synchronises their streams.
int Ctx::batch_errors(unsigned* bits) {
    *bits = 0;
    for (int s = 0; s < batch_subs && s < (int)subs.size(); ++s) {
        unsigned b = 0;
        VPM_CUDA_TRY(cudaMemcpyAsync(&b, subs[s]->d_err + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, subs[s]->stream));
        VPM_CUDA_TRY(cudaStreamSynchronize(subs[s]->stream));
        *bits |= b;
    }
    return VPM_OK;
}

void Ctx::drop_batch() {
    if (batch_exec) cudaGraphExecDestroy(batch_exec);
    batch_exec = nullptr;
    for (auto* c : subs) delete c;
    subs.clear();
    for (auto e : join_ev)
        if (e) cudaEventDestroy(e);
    join_ev.clear();
    if (fork_ev) cudaEventDestroy(fork_ev);
    fork_ev = nullptr;
    if (batch_in) cudaFree(batch_in);
    batch_in = nullptr;
    batch_in_bytes = 0;
}

}  // namespace vpm

using vpm::Ctx;

extern "C" {

int vpm_fmm2d_field_batched_device(vpm_ctx* ctx, int32_t n_solves, const int64_t* offsets, const double* x,
                                   const double* y, const double* q, const uint8_t* active,
                                   const vpm_fmm_params* prm, double* ex, double* ey) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    vpm_fmm_params p;
    int r = c->check_params(prm, p);
    if (r) return r;
    if (n_solves < 0) return c->fail(VPM_EINVAL, "n_solves < 0");
    if (n_solves > 0 && (!x || !y || !q || !active || !ex || !ey)) return c->fail(VPM_EINVAL, "null buffer");
    return c->batch2d(n_solves, offsets, x, y, q, active, p, ex, ey);
}

int vpm_fmm2d_field_batched(vpm_ctx* ctx, int32_t n_solves, const int64_t* offsets, const double* x,
                            const double* y, const double* q, const uint8_t* active, const vpm_fmm_params* prm,
                            double* ex, double* ey) {
    if (!ctx) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    vpm_fmm_params p;
    int r = c->check_params(prm, p);
    if (r) return r;
    if (n_solves <= 0) return n_solves == 0 ? VPM_OK : c->fail(VPM_EINVAL, "n_solves < 0");
    if (!offsets || !x || !y || !q || !active || !ex || !ey) return c->fail(VPM_EINVAL, "null buffer");
    const int64_t N = offsets[n_solves];
    if (N < 0 || N >= (1ll << 31)) return c->fail(VPM_EINVAL, "total particle count out of range");
    const size_t need = (size_t)N * (5 * sizeof(double) + 1) + 1024;
    if (c->batch_in_bytes < need) {
        if (c->batch_in) cudaFree(c->batch_in);
        c->batch_in = nullptr;
        c->batch_in_bytes = 0;
        e = cudaMalloc(&c->batch_in, need);
        if (e != cudaSuccess) return c->fail_cuda(e, "cudaMalloc of the batch buffers");
        c->batch_in_bytes = need;
    }
    double* dx = (double*)c->batch_in;
    double* dy = dx + N;
    double* dq = dy + N;
    double* dex = dq + N;
    double* dey = dex + N;
    uint8_t* da = (uint8_t*)(dey + N);
    cudaStream_t st = c->stream;
    const size_t b8 = sizeof(double) * (size_t)N;
    if ((e = cudaMemcpyAsync(dx, x, b8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dy, y, b8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dq, q, b8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(da, active, (size_t)N, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return c->fail_cuda(e, "batch inputs");
    for (int attempt = 0; attempt < 2; ++attempt) {
        r = c->batch2d(n_solves, offsets, dx, dy, dq, da, p, dex, dey);
        if (r) return r;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return c->fail_cuda(e, "batched solves");
        unsigned bits = 0;
        if ((r = c->batch_errors(&bits))) return r;
        if ((bits & vpm::ERR_DEPTH) && p.max_depth < vpm::kMaxLevels2D) {
            p.max_depth = vpm::kMaxLevels2D;  // coincident clusters: resolve 31 levels
            continue;
        }
        if (bits) return c->map_err(bits);
        break;
    }
    if ((e = cudaMemcpyAsync(ex, dex, b8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(ey, dey, b8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return c->fail_cuda(e, "batch outputs");
    return VPM_OK;
}

}  // extern "C"
