// C ABI for the dense-weight kernel sums kff.applykmat / kff.applykdiffmat
// (py-lddmm/kernelFunctions.f90:499-552, 554-610):
//
//   applykmat:     f[k,:] = sum_l K(x_k, y_l) beta[k,l,:]            beta (n, m, dimb)
//   applykdiffmat: f[k,:] = sum_l K'(x_k, y_l) 2 (x_k - y_l) beta[k,l] beta (n, m)
//
// The weights are a dense n x m (x dimb) FP64 array read once, so these sums
// are HBM-bound (8 dimb bytes per pair) rather than FMA-bound: one block per
// target row streams its weight row with coalesced loads while the source
// coordinates stay in L2.  `_f32c` evaluates K in FP32 on prescaled
// coordinates (ex2 on the MUFU, as the sweeps do) and accumulates K * beta in
// FP64; `_f64` evaluates K with the Fortran branches in FP64.  Each row is
// reduced by a fixed tree: deterministic, no atomics, no workspace.
#include "host.h"
#include "internal.h"
#include "kfun.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

constexpr int kMatThreads = 256;
constexpr int kMatMaxB = 8;

// squared prescaled distance of x_k and y_l: FP32 (from FP64 differences) or FP64
template <bool F32>
LDDMM_D auto mat_r2(const double* xk, const double* yl, int d, double scale) {
    if constexpr (F32) {
        float r2 = 0.f;
        for (int j = 0; j < d; ++j) {
            const float t = (float)((xk[j] - yl[j]) * scale);
            r2 = fmaf(t, t, r2);
        }
        return r2;
    } else {
        double r2 = 0.0;
        for (int j = 0; j < d; ++j) {
            const double t = (xk[j] - yl[j]) * scale;
            r2 += t * t;
        }
        return r2;
    }
}

// fixed-tree block sum of nv values per thread; every thread returns the totals
template <int NV>
LDDMM_D void mat_block_sum(double (&v)[NV], int nv) {
    __shared__ double red[kMatThreads];
    for (int c = 0; c < nv; ++c) {
        red[threadIdx.x] = v[c];
        __syncthreads();
        for (int s = kMatThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        v[c] = red[0];
        __syncthreads();
    }
}

struct MatParams {
    double scale, dscale;
    float pk32[5], pq32[4];
    double pk64[5], pq64[4];
};

template <bool F32, int KIND, int DEG>
static __global__ void __launch_bounds__(kMatThreads) kmat_kernel(const double* __restrict__ x, long long n,
                                                                  const double* __restrict__ y, long long m,
                                                                  const double* __restrict__ beta, int d, int dimb,
                                                                  MatParams P, double* __restrict__ f) {
    for (long long k = blockIdx.x; k < n; k += gridDim.x) {
        double xk[3] = {0, 0, 0};
        for (int j = 0; j < d; ++j) xk[j] = x[k * d + j];
        double acc[kMatMaxB];
        for (int c = 0; c < kMatMaxB; ++c) acc[c] = 0.0;
        const double* brow = beta + k * m * dimb;
        for (long long l = threadIdx.x; l < m; l += blockDim.x) {
            double K;
            if constexpr (F32) K = (double)kval32<KIND, DEG>(P.pk32, mat_r2<true>(xk, y + l * d, d, P.scale));
            else K = kval64<KIND, DEG>(P.pk64, mat_r2<false>(xk, y + l * d, d, P.scale));
            for (int c = 0; c < dimb; ++c) acc[c] += K * brow[l * dimb + c];
        }
        mat_block_sum(acc, dimb);
        if (threadIdx.x == 0)
            for (int c = 0; c < dimb; ++c) f[k * dimb + c] = acc[c];
    }
}

template <bool F32, int KIND, int QDEG>
static __global__ void __launch_bounds__(kMatThreads) kdiffmat_kernel(const double* __restrict__ x, long long n,
                                                                      const double* __restrict__ y, long long m,
                                                                      const double* __restrict__ beta, int d,
                                                                      MatParams P, double* __restrict__ f) {
    for (long long k = blockIdx.x; k < n; k += gridDim.x) {
        double xk[3] = {0, 0, 0};
        for (int j = 0; j < d; ++j) xk[j] = x[k * d + j];
        double acc[3] = {0, 0, 0};
        const double* brow = beta + k * m;
        for (long long l = threadIdx.x; l < m; l += blockDim.x) {
            const double* yl = y + l * d;
            double F;
            if constexpr (F32) F = (double)kdiff32<KIND, QDEG>(P.pq32, mat_r2<true>(xk, yl, d, P.scale));
            else F = kdiff64<KIND, QDEG>(P.pq64, mat_r2<false>(xk, yl, d, P.scale));
            F *= brow[l];
            for (int j = 0; j < d; ++j) acc[j] += F * ((xk[j] - yl[j]) * P.scale);
        }
        mat_block_sum(acc, d);
        if (threadIdx.x == 0)
            for (int j = 0; j < d; ++j) f[k * d + j] = P.dscale * acc[j];
    }
}

template <bool F32>
static MatParams mat_params(int kind, int order, double sigma) {
    const KScale ks = F32 ? kernel_scale<float>(kind, order, sigma) : kernel_scale<double>(kind, order, sigma);
    MatParams P{};
    P.scale = ks.scale;
    P.dscale = ks.dscale;
    for (int j = 0; j < 5; ++j) {
        P.pk32[j] = (float)ks.pk[j];
        P.pk64[j] = ks.pk[j];
    }
    for (int j = 0; j < 4; ++j) {
        P.pq32[j] = (float)ks.pq[j];
        P.pq64[j] = ks.pq[j];
    }
    return P;
}

static int mat_grid(long long n) { return (int)std::max<long long>(1, std::min<long long>(n, 148LL * 16)); }

static int mat_check(const char* who, const double* x, long long n, const double* y, long long m,
                     const double* beta, int d, double sigma, int order, double* f) {
    if (n < 0 || m < 0 || d < 1 || d > 3 || !(sigma > 0) || order < 0) {
        set_error("%s: invalid arguments (n=%lld m=%lld d=%d sigma=%g order=%d)", who, n, m, d, sigma, order);
        return LDDMM_ERR_ARG;
    }
    if (n == 0) return LDDMM_OK;
    LDDMM_TRY(check_device_ptr(x, "x"));
    LDDMM_TRY(check_device_ptr(f, "f"));
    if (m > 0) {
        LDDMM_TRY(check_device_ptr(y, "y"));
        LDDMM_TRY(check_device_ptr(beta, "beta"));
    }
    return LDDMM_OK;
}

template <bool F32>
static int kmat_run(const double* x, long long n, const double* y, long long m, const double* beta, int d, int dimb,
                    double sigma, int order, double* f, cudaStream_t st) {
    if (dimb < 1 || dimb > kMatMaxB) {
        set_error("applykmat: dimb must be in [1, %d] (got %d)", kMatMaxB, dimb);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(mat_check("applykmat", x, n, y, m, beta, d, sigma, order, f));
    if (n == 0) return LDDMM_OK;
    if (m == 0) return cuda_check(cudaMemsetAsync(f, 0, sizeof(double) * n * dimb, st), "applykmat");
    const MatParams P = mat_params<F32>(order > 4 ? KGAUSS : KLAP, order, sigma);
    dispatch_kind_p(order, [&](auto K, auto DG) {
        kmat_kernel<F32, decltype(K)::value, decltype(DG)::value><<<mat_grid(n), kMatThreads, 0, st>>>(
            x, n, y, m, beta, d, dimb, P, f);
        return LDDMM_OK;
    });
    return cuda_check(cudaGetLastError(), "applykmat");
}

template <bool F32>
static int kdiffmat_run(const double* x, long long n, const double* y, long long m, const double* beta, int d,
                        double sigma, int order, double* f, cudaStream_t st) {
    LDDMM_TRY(mat_check("applykdiffmat", x, n, y, m, beta, d, sigma, order, f));
    if (order == 0) {
        set_error("applykdiffmat: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    if (n == 0) return LDDMM_OK;
    if (m == 0) return cuda_check(cudaMemsetAsync(f, 0, sizeof(double) * n * d, st), "applykdiffmat");
    const MatParams P = mat_params<F32>(order > 4 ? KGAUSS : KLAP, order, sigma);
    dispatch_kind_q(order, [&](auto K, auto DG) {
        kdiffmat_kernel<F32, decltype(K)::value, decltype(DG)::value><<<mat_grid(n), kMatThreads, 0, st>>>(
            x, n, y, m, beta, d, P, f);
        return LDDMM_OK;
    });
    return cuda_check(cudaGetLastError(), "applykdiffmat");
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

int lddmm_applykmat_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                         double sigma, int order, double* f, lddmm_stream_t stream) {
    return kmat_run<true>(x, n, y, m, beta, d, dimb, sigma, order, f, (cudaStream_t)stream);
}

int lddmm_applykmat_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                        double sigma, int order, double* f, lddmm_stream_t stream) {
    return kmat_run<false>(x, n, y, m, beta, d, dimb, sigma, order, f, (cudaStream_t)stream);
}

int lddmm_applykdiffmat_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                             double sigma, int order, double* f, lddmm_stream_t stream) {
    return kdiffmat_run<true>(x, n, y, m, beta, d, sigma, order, f, (cudaStream_t)stream);
}

int lddmm_applykdiffmat_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                            double sigma, int order, double* f, lddmm_stream_t stream) {
    return kdiffmat_run<false>(x, n, y, m, beta, d, sigma, order, f, (cudaStream_t)stream);
}

}  // extern "C"
