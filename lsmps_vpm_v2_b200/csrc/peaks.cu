// FMA-throughput microbenchmark: the FP64 and FP32 pipe peaks that the
// near-field (P2P) roofline fractions are quoted against. Each thread runs 8
// independent FMA chains; flops = 2 * chains * iterations * threads.
#include "context.h"

namespace vpm {
namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-12345.0) out[0] = s;  // keeps the chains alive
}

template <class T>
int run(Ctx* c, int iters, double* tflops) {
    const int blocks = 148 * 8, threads = 256;
    T* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 64);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaMalloc");
    fma_chains<T><<<blocks, threads, 0, c->stream>>>(d, 4, (T)0.999, (T)0.001);  // warm-up
    cudaEventRecord(c->ev[0], c->stream);
    fma_chains<T><<<blocks, threads, 0, c->stream>>>(d, iters, (T)0.999, (T)0.001);
    cudaEventRecord(c->ev[1], c->stream);
    e = cudaEventSynchronize(c->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    cudaFree(d);
    if (e != cudaSuccess) return c->fail_cuda(e, "fma_chains");
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return VPM_OK;
}

// Reciprocal-throughput microbenchmark (rcp.approx.ftz.f32, the special
// function unit the FP32 near field issues one reciprocal per pair to): 8
// independent chains x <- 1/x + 1 per thread (the add keeps consecutive
// reciprocals from cancelling and runs on the FMA pipe, which is 8x wider).
__global__ void __launch_bounds__(256) rcp_chains(float* out, int iters) {
    float x[8];
    #pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = 1.0f + 0.125f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int u = 0; u < 16; ++u) {
            #pragma unroll
            for (int k = 0; k < 8; ++k)
                asm volatile("rcp.approx.ftz.f32 %0, %0;\n\tadd.f32 %0, %0, 0f3F800000;" : "+f"(x[k]));
        }
    }
    float s = 0.f;
    #pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == -12345.0f) out[0] = s;
}

int run_rcp(Ctx* c, int iters, double* grcp) {
    const int blocks = 148 * 8, threads = 256;
    float* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 64);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaMalloc");
    rcp_chains<<<blocks, threads, 0, c->stream>>>(d, 4);  // warm-up
    cudaEventRecord(c->ev[0], c->stream);
    rcp_chains<<<blocks, threads, 0, c->stream>>>(d, iters);
    cudaEventRecord(c->ev[1], c->stream);
    e = cudaEventSynchronize(c->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    cudaFree(d);
    if (e != cudaSuccess) return c->fail_cuda(e, "rcp_chains");
    const double n = 8.0 * 16 * (double)iters * blocks * threads;
    *grcp = n / (ms * 1e-3) / 1e9;
    return VPM_OK;
}

}  // namespace
}  // namespace vpm

extern "C" int vpm_measure_rcp_peak(vpm_ctx* ctx, double* grcp_per_s) {
    if (!ctx || !grcp_per_s) return VPM_EINVAL;
    vpm::Ctx* c = (vpm::Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    return vpm::run_rcp(c, 1024, grcp_per_s);
}

extern "C" int vpm_measure_fma_peaks(vpm_ctx* ctx, double* fp64_tflops, double* fp32_tflops) {
    if (!ctx || !fp64_tflops || !fp32_tflops) return VPM_EINVAL;
    vpm::Ctx* c = (vpm::Ctx*)ctx;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->fail_cuda(e, "cudaSetDevice");
    int r = vpm::run<double>(c, 2048, fp64_tflops);
    if (r) return r;
    return vpm::run<float>(c, 4096, fp32_tflops);
}
