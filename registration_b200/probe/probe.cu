// Measurement utility, not part of the LDDMM library: kernels that measure this
// GPU's FP32 FMA, MUFU ex2 and packed f32x2 FMA issue rates.  bench.py times
// them to get the measured peaks that the kernel-sum roofline fractions are
// quoted against.  Built into its own liblddmm_probe.so.
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 8 independent FMA chains per thread, unrolled: 8*iters FFMA per thread.
static __global__ void probe_ffma_kernel(float* out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = (threadIdx.x + j) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = fmaf(x[j], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += x[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// 8 independent ex2 chains per thread: 8*iters MUFU.EX2 per thread.
static __global__ void probe_ex2_kernel(float* out, int iters) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = (threadIdx.x + j) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = ex2(-x[j]);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += x[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// 8 independent packed-pair FMA chains (fma.rn.f32x2, sm_100a): 8*iters
// instructions, 16*iters FMAs per thread.
static __global__ void probe_ffma2_kernel(float* out, int iters) {
    unsigned long long x[8], a, b;
    asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(0.999f), "f"(0.998f));
    asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(1e-4f), "f"(2e-4f));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float u = (threadIdx.x + j) * 1e-3f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[j]) : "f"(u), "f"(u + 0.5f));
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[j]) : "l"(a), "l"(b));
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float p, q;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(p), "=f"(q) : "l"(x[j]));
        s += p + q;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Launches `blocks` x `threads` threads that each issue 8*iters FP32 FMAs
// (what = 0), 8*iters MUFU ex2 (what = 1) or 8*iters packed two-lane FMAs
// (what = 2) and write one float each to out[blocks*threads] (a device buffer).
// Returns 0, -1 for a bad launch shape or a non-device `out`, -3 for a CUDA error.
extern "C" __attribute__((visibility("default"))) int lddmm_probe_launch(int what, int blocks, int threads,
                                                                         int iters, float* out, void* stream) {
    if (blocks < 1 || threads < 32 || threads > 1024 || iters < 1 || what < 0 || what > 2) return -1;
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, out) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return -1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (what == 0)
        probe_ffma_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.999f, 1e-4f);
    else if (what == 1)
        probe_ex2_kernel<<<blocks, threads, 0, st>>>(out, iters);
    else
        probe_ffma2_kernel<<<blocks, threads, 0, st>>>(out, iters);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
