// Batched independent 2D solves: many uneven particle sets (one velocity
// evaluation each) in one call. Each solve runs on one of S sub-contexts, each
// with its own stream and arena, forked from and joined back into the
// caller's stream by events, so solves of different sizes overlap on the
// GPU. Solves are dealt longest first to the least-loaded stream (the load of
// a solve modelled as its particle count plus kSolveFixed, the fixed latency
// of one evaluation's launch chain), and each stream runs its solves largest
// first. With use_graph the whole batch - every solve's launches on every
// stream - is captured once as one CUDA graph and replayed by a single graph
// launch while the batch layout is unchanged; the first call for a layout
// tunes S: it captures the batch for each S in kBatchStreamChoices, times two
// replays of each and keeps the fastest graph (the choice is remembered per
// layout for the life of the context).
#include <algorithm>
#include <cstring>
#include <numeric>

#include "context.h"

namespace vpm {

namespace {

constexpr int kBatchStreamChoices[] = {4, 8, 12, 16};
constexpr int kBatchStreamsMax = 16;
constexpr int kBatchStreamsEager = 8;
constexpr int64_t kSolveFixed = 150000;

// Word 1 of a context's error buffer collects the error bits of every solve
// the context ran in the current batch (word 0 is reset by each solve).
__global__ void collect_err(unsigned* err) { err[1] |= err[0]; }

// Stream of each solve (longest first to the least-loaded of S streams) and
// the order solves are enqueued in (largest first).
void plan_batch(int ns, const int64_t* offs, int S, std::vector<int>& stream_of, std::vector<int>& order) {
    order.resize(ns);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return offs[a + 1] - offs[a] > offs[b + 1] - offs[b];
    });
    stream_of.assign(ns, 0);
    std::vector<int64_t> load(S, 0);
    for (int i : order) {
        const int64_t n = offs[i + 1] - offs[i];
        if (n == 0) continue;
        const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        stream_of[i] = s;
        load[s] += n + kSolveFixed;
    }
}

}  // namespace

// Sub-contexts 0..S-1 with arenas and coefficients for the solves `plan`
// gives them.
int Ctx::prepare_batch(int ns, const int64_t* offs, const vpm_fmm_params& p, int S, const std::vector<int>& stream_of) {
    while ((int)subs.size() < S) {
        Ctx* c = new (std::nothrow) Ctx();
        if (!c) return fail(VPM_ENOMEM, "sub-context");
        if (int r = c->init(device)) {
            std::string m = c->last_error;
            delete c;
            return fail(r, "sub-context: " + m);
        }
        // 8192 particles per sort block: a batch's sorts run side by side
        // (64 uneven solves: 5.11 -> 4.54 ms against 2048)
        c->sort_items = 8192;
        c->split_m2l = false;
        subs.push_back(c);
        cudaEvent_t e = nullptr;
        VPM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        join_ev.push_back(e);
    }
    if (!fork_ev) VPM_CUDA_TRY(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    for (int s = 0; s < S; ++s) {
        Ctx* c = subs[s];
        int maxn = 0;
        for (int i = 0; i < ns; ++i)
            if (stream_of[i] == s) maxn = std::max<int>(maxn, (int)(offs[i + 1] - offs[i]));
        if (maxn < 2) continue;
        int cells;
        long long l1, l3;
        if (int r = c->plan_caps(maxn, p, cells, l1, l3)) return fail(r, c->last_error);
        if (int r = c->reserve2d(maxn, cells, p.p, l1, l3)) return fail(r, c->last_error);
        if (int r = c->ensure_coefs(p)) return fail(r, c->last_error);
    }
    return VPM_OK;
}

// Enqueue every solve on its sub-context's stream (fork, solves, join).
int Ctx::enqueue_batch(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                       const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey, int S,
                       const std::vector<int>& stream_of, const std::vector<int>& order) {
    cudaError_t e = cudaEventRecord(fork_ev, stream);
    for (int s = 0; s < S && e == cudaSuccess; ++s) {
        e = cudaStreamWaitEvent(subs[s]->stream, fork_ev, 0);
        if (e == cudaSuccess) e = cudaMemsetAsync(subs[s]->d_err + 1, 0, sizeof(unsigned), subs[s]->stream);
    }
    int r = VPM_OK;
    for (int k = 0; k < ns && e == cudaSuccess && r == VPM_OK; ++k) {
        const int i = order[k];
        const int64_t o = offs[i], n = offs[i + 1] - offs[i];
        if (n == 0) continue;
        Ctx* c = subs[stream_of[i]];
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
    if (r != VPM_OK) return r;
    if (e != cudaSuccess) return fail_cuda(e, "batched solves");
    return VPM_OK;
}

// One CUDA graph of the whole batch with S streams.
int Ctx::capture_batch(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                       const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey, int S,
                       cudaGraphExec_t* out) {
    *out = nullptr;
    std::vector<int> stream_of, order;
    plan_batch(ns, offs, S, stream_of, order);
    if (int r = prepare_batch(ns, offs, p, S, stream_of)) return r;
    VPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < S; ++s) subs[s]->capturing = true;
    int r = enqueue_batch(ns, offs, x, y, q, act, p, ex, ey, S, stream_of, order);
    for (int s = 0; s < S; ++s) subs[s]->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (r == VPM_OK && e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (g) cudaGraphDestroy(g);
    if (r != VPM_OK) return r;
    if (e != cudaSuccess) {
        *out = nullptr;
        return fail_cuda(e, "batch graph");
    }
    return VPM_OK;
}

int Ctx::batch2d(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                 const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey) {
    if (ns <= 0) return VPM_OK;
    if (!offs || offs[0] != 0) return fail(VPM_EINVAL, "offsets must start at 0");
    for (int i = 0; i < ns; ++i) {
        const int64_t n = offs[i + 1] - offs[i];
        if (n < 0 || n == 1 || n >= (1ll << 30)) return fail(VPM_EINVAL, "each solve needs 0 or 2..2^30-1 particles");
    }
    if (!p.use_graph) {
        const int S = std::min(kBatchStreamsEager, ns);
        std::vector<int> stream_of, order;
        plan_batch(ns, offs, S, stream_of, order);
        if (int r = prepare_batch(ns, offs, p, S, stream_of)) return r;
        batch_subs = S;
        batch_streams = S;
        return enqueue_batch(ns, offs, x, y, q, act, p, ex, ey, S, stream_of, order);
    }
    // the layout key of the graph: offsets, buffers, stream, parameters
    std::vector<int64_t> key(offs, offs + ns + 1);
    const int64_t extra[] = {(int64_t)(intptr_t)x, (int64_t)(intptr_t)y,  (int64_t)(intptr_t)q,
                             (int64_t)(intptr_t)act, (int64_t)(intptr_t)ex, (int64_t)(intptr_t)ey,
                             (int64_t)(intptr_t)stream};
    key.insert(key.end(), extra, extra + 7);
    std::vector<int64_t> pk((sizeof(p) + 7) / 8, 0);
    std::memcpy(pk.data(), &p, sizeof(p));
    key.insert(key.end(), pk.begin(), pk.end());
    if (batch_exec && key == batch_key) {
        batch_subs = batch_streams;
        VPM_CUDA_TRY(cudaGraphLaunch(batch_exec, stream));
        return VPM_OK;
    }
    if (batch_exec) cudaGraphExecDestroy(batch_exec);
    batch_exec = nullptr;
    batch_key.clear();
    // tune the stream count: the fastest of two timed replays per choice
    if (!tune_ev[0]) {
        VPM_CUDA_TRY(cudaEventCreate(&tune_ev[0]));
        VPM_CUDA_TRY(cudaEventCreate(&tune_ev[1]));
    }
    float best_ms = 0.f;
    int best_s = 0;
    for (int S : kBatchStreamChoices) {
        if (S > std::max(1, ns) && S != kBatchStreamChoices[0]) break;
        const int SS = std::min(S, std::max(1, ns));
        cudaGraphExec_t g = nullptr;
        if (int r = capture_batch(ns, offs, x, y, q, act, p, ex, ey, SS, &g)) return r;
        float ms = 0.f;
        cudaError_t e = cudaGraphLaunch(g, stream);
        if (e == cudaSuccess) e = cudaEventRecord(tune_ev[0], stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(g, stream);
        if (e == cudaSuccess) e = cudaEventRecord(tune_ev[1], stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(tune_ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, tune_ev[0], tune_ev[1]);
        if (e != cudaSuccess) {
            cudaGraphExecDestroy(g);
            return fail_cuda(e, "batch tuning");
        }
        if (!batch_exec || ms < best_ms) {
            if (batch_exec) cudaGraphExecDestroy(batch_exec);
            batch_exec = g;
            best_ms = ms;
            best_s = SS;
        } else {
            cudaGraphExecDestroy(g);
        }
    }
    batch_subs = best_s;
    batch_streams = best_s;
    batch_key = key;
    VPM_CUDA_TRY(cudaGraphLaunch(batch_exec, stream));
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
    for (auto& e : tune_ev)
        if (e) cudaEventDestroy(e);
    tune_ev[0] = tune_ev[1] = nullptr;
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

int vpm_batch_streams(vpm_ctx* ctx, int32_t* streams) {
    if (!ctx || !streams) return VPM_EINVAL;
    Ctx* c = (Ctx*)ctx;
    *streams = c->batch_streams ? c->batch_streams : c->batch_subs;
    return VPM_OK;
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
