// Affine and euclidean parts of the kernel sums (KernelSpec affine = 'affine'
// or 'euclidean'): py-lddmm/kernelFunctions.py:334-367 (applyK) and :431-448
// (applyDiffKT) add, after the kernel sum, terms built from the moments
//   M = sum_l (x_l - c) a_l^T  (d x dimb)  and  s = sum_l a_l  (dimb)
// of the sources x with weights a about the kernel's centre c, applied to each
// target row u_k as  f_k += (u_k - c) W + b.  Two entry points:
//   lddmm_moments_f64     M and s (FP64, fixed block tree: deterministic);
//   lddmm_rows_affine_f64 f += (u - c) W + b for every row.
// The caller forms W and b from the moments (for 'affine' W = w1 M, b = w2 s;
// for 'euclidean' the projections onto the skew basis of the reference).
#include "host.h"
#include "pack.cuh"

namespace lddmm {

constexpr int kMomThreads = 256;
constexpr int kMomMaxQ = 16;   // d * dimb + dimb <= 3 * 4 + 4

static __global__ void moments_partial_kernel(const double* __restrict__ x, long long m, int d,
                                              const double* __restrict__ a, int dimb, const double* __restrict__ c,
                                              double* __restrict__ part) {
    const int Q = d * dimb + dimb;
    double acc[kMomMaxQ];
    for (int q = 0; q < kMomMaxQ; ++q) acc[q] = 0.0;
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < m;
         l += (long long)gridDim.x * blockDim.x) {
        double xx[3] = {0, 0, 0};
        for (int i = 0; i < d; ++i) xx[i] = x[l * d + i] - (c ? c[i] : 0.0);
        for (int j = 0; j < dimb; ++j) {
            const double aj = a[l * dimb + j];
            for (int i = 0; i < d; ++i) acc[i * dimb + j] += xx[i] * aj;
            acc[d * dimb + j] += aj;
        }
    }
    __shared__ double red[kMomThreads];
    for (int q = 0; q < Q; ++q) {
        red[threadIdx.x] = acc[q];
        __syncthreads();
        for (int s = kMomThreads / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * Q + q] = red[0];
        __syncthreads();
    }
}

static __global__ void moments_final_kernel(const double* __restrict__ part, int nb, int Q, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= Q) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(long long)b * Q + q];
    out[q] = s;
}

static __global__ void rows_affine_kernel(const double* __restrict__ u, long long n, int Q,
                                          const double* __restrict__ c, const double* __restrict__ W,
                                          const double* __restrict__ b, int J, double* __restrict__ f) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        for (int j = 0; j < J; ++j) {
            double v = b ? b[j] : 0.0;
            for (int q = 0; q < Q; ++q) v += (u[k * Q + q] - (c ? c[q] : 0.0)) * W[q * J + j];
            f[k * J + j] += v;
        }
    }
}

static int moments_blocks(long long m) {
    return (int)std::max<long long>(1, std::min<long long>(256, (m + kMomThreads - 1) / kMomThreads));
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_moments_f64_workspace(int64_t m, int d, int dimb) {
    if (m < 0 || d < 1 || d > 3 || dimb < 1 || dimb > 4) return 0;
    return sizeof(double) * (size_t)moments_blocks(m) * (size_t)(d * dimb + dimb) + 256;
}

int lddmm_moments_f64(const double* x, int64_t m, int d, const double* a, int dimb, const double* center, double* out,
                      void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    if (m < 0 || m > (1LL << 30) || d < 1 || d > 3 || dimb < 1 || dimb > 4) {
        set_error("moments: invalid arguments (m=%lld d=%d dimb=%d)", (long long)m, d, dimb);
        return LDDMM_ERR_ARG;
    }
    const int Q = d * dimb + dimb;
    LDDMM_TRY(check_device_ptr(out, "out"));
    cudaStream_t st = (cudaStream_t)stream;
    if (m == 0) return cuda_check(cudaMemsetAsync(out, 0, sizeof(double) * Q, st), "moments memset");
    LDDMM_TRY(check_device_ptr(x, "x"));
    LDDMM_TRY(check_device_ptr(a, "a"));
    if (center) LDDMM_TRY(check_device_ptr(center, "center"));
    const int nb = moments_blocks(m);
    if (workspace == nullptr || workspace_bytes < sizeof(double) * (size_t)nb * Q) {
        set_error("moments: workspace too small (need %zu bytes)", sizeof(double) * (size_t)nb * Q);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(workspace, "workspace"));
    double* part = static_cast<double*>(workspace);
    moments_partial_kernel<<<nb, kMomThreads, 0, st>>>(x, m, d, a, dimb, center, part);
    moments_final_kernel<<<1, 32, 0, st>>>(part, nb, Q, out);
    return cuda_check(cudaGetLastError(), "moments");
}

int lddmm_rows_affine_f64(const double* u, int64_t n, int Q, const double* center, const double* W, const double* b,
                          int J, double* f, lddmm_stream_t stream) {
    if (n < 0 || n > (1LL << 30) || Q < 1 || Q > 16 || J < 1 || J > 4) {
        set_error("rows_affine: invalid arguments (n=%lld Q=%d J=%d)", (long long)n, Q, J);
        return LDDMM_ERR_ARG;
    }
    if (n == 0) return LDDMM_OK;
    LDDMM_TRY(check_device_ptr(u, "u"));
    LDDMM_TRY(check_device_ptr(W, "W"));
    LDDMM_TRY(check_device_ptr(f, "f"));
    if (center) LDDMM_TRY(check_device_ptr(center, "center"));
    if (b) LDDMM_TRY(check_device_ptr(b, "b"));
    rows_affine_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(u, n, Q, center, W, b, J, f);
    return cuda_check(cudaGetLastError(), "rows_affine");
}

}  // extern "C"
