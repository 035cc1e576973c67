// probe.cu -- instruction-throughput probes for the roofline of the pair passes.
//
// The fused log-sum-exp passes are bound neither by HBM (their operands are a
// few MB and stay in L2) nor by the tensor cores; they are bound by the FP64
// pipe (the exponent is formed in FP64) and by the MUFU/XU pipe (ex2 and the
// FP64 -> FP32 conversion). These kernels measure those pipes' sustained rates
// on the running GPU so the bench can report achieved pairs/s against a
// measured, not nominal, ceiling.
#include <cuda_runtime.h>

#include "internal.h"

namespace {

constexpr int PROBE_ITERS = 4096;
constexpr int CHAINS = 8;

__global__ void probe_dfma(double *sink, double a, double b) {
    double v[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) v[k] = threadIdx.x * 1e-9 + k;
    for (int i = 0; i < PROBE_ITERS; ++i) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) v[k] = fma(v[k], a, b);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += v[k];
    if (s == 123.456) sink[0] = s;
}

__global__ void probe_ex2(float *sink, float a) {
    float v[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) v[k] = -1e-3f * (threadIdx.x + k);
    for (int i = 0; i < PROBE_ITERS; ++i) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) {
            float y;
            asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v[k]));
            v[k] = y * a;
        }
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += v[k];
    if (s == 123.456f) sink[0] = s;
}

// cvt.rn.f32.f64 of loop-invariant values (volatile asm keeps every instance),
// one FADD each into independent accumulators.
__global__ void probe_cvt(float *sink, double a) {
    double v[CHAINS];
    float acc[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) { v[k] = threadIdx.x * a + k; acc[k] = 0.f; }
    for (int i = 0; i < PROBE_ITERS; ++i) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) {
            float f;
            asm volatile("cvt.rn.f32.f64 %0, %1;" : "=f"(f) : "d"(v[k]));
            acc[k] += f;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += acc[k];
    if (s == 123.456f) sink[0] = s;
}

template <class F>
double time_ms(F launch, cudaStream_t st) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();   // warm
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3; ++r) launch();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / 3.0;
}

}  // namespace

extern "C" int culamp_probe_pipes(culamp_handle h, double *out, void *stream) {
    if (!h || !out) return CULAMP_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (h->tmpB.reserve(64) != cudaSuccess) return CULAMP_ERR_ALLOC;
    const int blocks = h->sm_count * 8, threads = 256;
    const double ops = (double)blocks * threads * PROBE_ITERS * CHAINS;
    double *ds = h->tmpB.as<double>();
    float *fs = h->tmpB.as<float>();
    const double t_dfma = time_ms([&] { probe_dfma<<<blocks, threads, 0, st>>>(ds, 0.999999, 1e-7); }, st);
    const double t_ex2 = time_ms([&] { probe_ex2<<<blocks, threads, 0, st>>>(fs, -1.0f); }, st);
    const double t_cvt = time_ms([&] { probe_cvt<<<blocks, threads, 0, st>>>(fs, 1e-3); }, st);
    if (cudaGetLastError() != cudaSuccess) return culamp_set_error(h, CULAMP_ERR_CUDA, "probe failed");
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, h->device);
    out[0] = ops / (t_dfma * 1e-3);   // DFMA / s
    out[1] = ops / (t_ex2 * 1e-3);    // MUFU ex2 / s
    out[2] = ops / (t_cvt * 1e-3);    // cvt.rn.f32.f64 / s (one FADD each)
    out[3] = (double)h->sm_count;
    return CULAMP_OK;
}
