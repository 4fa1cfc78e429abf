// Context lifetime and interaction counting.
#include "context.h"

namespace vpm {

namespace {

// Exact interaction counts of the last 2D evaluation (for the statistics and
// the roofline figures): list-1 pairs j != i, M2L pairs, list-3 pairs.
__global__ void count2d(Tree2D t, Lists2D l, unsigned long long* out, const unsigned* err) {
    if (fatal(err)) return;
    const int nl = t.info->n_leaves, nc = t.info->n_cells;
    unsigned long long p2p = 0, m2p = 0, m2l = 0;
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < nl; li += gridDim.x * blockDim.x) {
        const int c = t.leaf_cells[li];
        const long long T = t.c_hi[c] - t.c_lo[c];
        long long S = 0;
        bool self = false;
        for (uint32_t k = l.l1_off[li]; k < l.l1_off[li + 1]; ++k) {
            const int s = l.l1_src[k];
            S += t.c_hi[s] - t.c_lo[s];
            self |= (s == c);
        }
        p2p += (unsigned long long)(T * S - (self ? T : 0));
        m2p += (unsigned long long)(T * (long long)(l.l3_off[li + 1] - l.l3_off[li]));
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        m2l += l.l2_n[c] + l.l4_n[c];
    atomicAdd(&out[0], p2p);
    atomicAdd(&out[1], m2l);
    atomicAdd(&out[2], m2p);
}

}  // namespace

Ctx::~Ctx() {
    if (device >= 0) cudaSetDevice(device);
    drop_batch();
    drop_selector(selector);
    selector = nullptr;
    drop_graph();
    if (arena2d) cudaFree(arena2d);
    if (arena3d) cudaFree(arena3d);
    if (d_err) cudaFree(d_err);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (side) cudaStreamDestroy(side);
    if (side2) cudaStreamDestroy(side2);
    if (side3) cudaStreamDestroy(side3);
    if (upload) cudaStreamDestroy(upload);
    if (join3) cudaEventDestroy(join3);
    if (fork2) cudaEventDestroy(fork2);
    if (join2) cudaEventDestroy(join2);
    for (cudaEvent_t x : {ev_up, ev_l13, join4, ev_slots, join5, ev_upload, ev_q, ev_qg, ev_small, ev_m2ld})
        if (x) cudaEventDestroy(x);
}

int Ctx::init(int dev) {
    device = dev;
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
    // A blocking stream: work the caller puts on the legacy default stream
    // (e.g. PyTorch's default) is ordered with the context's work.
    e = cudaStreamCreate(&own_stream);
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamCreate");
    stream = own_stream;
    e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&side2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&side3, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&upload, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamCreate");
    e = cudaEventCreateWithFlags(&fork2, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join2, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join3, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_up, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_l13, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join4, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_slots, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join5, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_upload, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_q, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_qg, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_small, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_m2ld, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventCreate");
    e = cudaMalloc(&d_err, 64);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc");
    e = cudaMemset(d_err, 0, 64);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemset");
    for (auto& x : ev) {
        e = cudaEventCreate(&x);
        if (e != cudaSuccess) return fail_cuda(e, "cudaEventCreate");
    }
    return VPM_OK;
}

int Ctx::count_interactions(vpm_fmm_stats* s) {
    unsigned long long* d = (unsigned long long*)(d_err + 2);  // 3 counters after the error word
    cudaError_t e = cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync");
    count2d<<<148, 256, 0, stream>>>(tree, lists, d, d_err);
    unsigned long long h[3];
    e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail_cuda(e, "count interactions");
    s->p2p_pairs = (int64_t)h[0];
    s->m2l_pairs = (int64_t)h[1];
    s->m2p_pairs = (int64_t)h[2];
    return VPM_OK;
}

// Mixed/near-field work area: leaf-relative FP32 particles (float4 per
// particle, mixed form) or the AoS FP64 copy (double4 per particle, plain
// form), then the tensor-core M2L rows and operators.
size_t mixed_bytes(int n, int cap_cells, int P) {
    return sizeof(double4) * (size_t)n + 1024 + m2l_tc_rows_bytes(cap_cells) + 1024 + m2l_tc_ops_bytes() + 1024;
}



}  // namespace vpm
