// Metric inner products of momentum directions along a trajectory.
//
//   lddmm_metric_dots_* : SurfaceMatching.dotProduct / CurveMatching.dotProduct
//                         (py-lddmm/surfaceMatching.py:353-377,
//                         curveMatching.py:286-304, no affine part)
//     out[l] = sum_t sum_k <g2_l[t][k], u_t[k]>,  u_t[k] = sum_j K(x_t[k], x_t[j]) g1[t][j]
//
// The line search asks for two of these per iteration, on the device-resident
// trajectory; as T applyK calls plus dot products they are a dozen launches of
// a few microseconds each for a small point set.  Here the T time steps are
// one launch: block (b, t) owns the targets [32 b, 32 b + 32) of step t, its
// 512 threads are 32 target slots times 16 source groups, the sources of the
// step pass through shared memory in tiles of 256 records (position in a
// per-step frame, g1 weights).  Group sums are FP32 partials over 32 sources
// folded into TwoSum pairs (or FP64), added in group order in FP64; u_t[k] is
// dotted with every g2_l[t][k] in FP64, each block reduces its targets with a
// fixed tree, and a second one-block launch adds the (t, b) partials in order.
// The result depends on the shape and the data only.
#include "fused_small.cuh"
#include "host.h"
#include "sweep_dispatch.cuh"

namespace lddmm {

constexpr int kDotThreads = 512;
constexpr int kDotTargets = 32;   // target slots per block
constexpr int kDotGroups = kDotThreads / kDotTargets;
constexpr int kDotTile = 256;
constexpr int kDotMaxDirs = 8;
static_assert(kDotThreads == kFusedThreads, "fused_block_sum reduces kFusedThreads values");

struct DotDirs {
    const double* g2[kDotMaxDirs];
};

template <class Real, int KIND, int DEG, int D>
__global__ void __launch_bounds__(kDotThreads)
    metric_dots_kernel(const double* __restrict__ xt, long long n, const double* __restrict__ g1, DotDirs dirs, int m,
                       double scale, FusedCoef cf, double* __restrict__ partial) {
    __shared__ FusedRec<Real> rec[kDotTile];
    __shared__ double red[kDotThreads * D];
    __shared__ double scratch[kDotThreads];
    const int tid = threadIdx.x;
    const int local = tid % kDotTargets, g = tid / kDotTargets;
    const long long t = blockIdx.y, N = n * D;
    const long long k = (long long)blockIdx.x * kDotTargets + local;
    const bool owner = k < n;
    const double* x = xt + t * N;
    const double* w = g1 + t * N;
    // frame of step t: its first point (only differences of positions enter K)
    double c[3] = {0, 0, 0};
    for (int j = 0; j < D; ++j) c[j] = x[j];
    Real pk[5];
    for (int j = 0; j < 5; ++j) pk[j] = (Real)cf.pk[j];
    Real xk[3] = {0, 0, 0};
    if (owner)
        for (int j = 0; j < D; ++j) xk[j] = (Real)((x[k * D + j] - c[j]) * scale);
    FusedAcc<Real, D> acc;
    acc.zero();
    constexpr int FOLD = sizeof(Real) == 4 ? 32 : 1 << 30;
    for (long long t0 = 0; t0 < n; t0 += kDotTile) {
        const int len = (int)(n - t0 < kDotTile ? n - t0 : kDotTile);
        for (int i = tid; i < len; i += kDotThreads) fused_store<Real>(rec[i], x + (t0 + i) * D, D, scale, c,
                                                                        w + (t0 + i) * D, D);
        __syncthreads();
        if (owner) {
            const int jb0 = g * len / kDotGroups, je0 = (g + 1) * len / kDotGroups;
            for (int jb = jb0; jb < je0; jb += FOLD) {
                acc.begin_fold();
                const int je = jb + FOLD < je0 ? jb + FOLD : je0;
                for (int j = jb; j < je; ++j) {
                    Real y[3], v[6];
                    fused_pos<Real>(rec[j], y);
                    fused_vals<Real>(rec[j], v);
                    Real r2 = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        const Real dq = xk[q] - y[q];
                        r2 = q == 0 ? dq * dq : r2 + dq * dq;
                    }
                    const Real kv = fused_k<Real, KIND, DEG>(pk, r2);
#pragma unroll
                    for (int q = 0; q < D; ++q) acc.fma(q, kv, v[q]);
                }
                acc.end_fold();
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < D; ++q) red[tid * D + q] = owner ? acc.value(q) : 0.0;
    __syncthreads();
    double u[3] = {0, 0, 0};
    if (owner && g == 0)
        for (int q = 0; q < D; ++q)
            for (int gg = 0; gg < kDotGroups; ++gg) u[q] += red[(gg * kDotTargets + local) * D + q];
    for (int l = 0; l < m; ++l) {
        double e = 0.0;
        if (owner && g == 0)
            for (int q = 0; q < D; ++q) e += dirs.g2[l][t * N + k * D + q] * u[q];
        e = fused_block_sum(e, scratch);
        if (tid == 0) partial[(t * gridDim.x + blockIdx.x) * m + l] = e;
    }
}

// out[l] = the partials of direction l in (t, block) order
static __global__ void metric_dots_finalize_kernel(const double* __restrict__ partial, long long count, int m,
                                                   double* __restrict__ out) {
    const int l = threadIdx.x;
    if (l >= m) return;
    double s = 0.0;
    for (long long i = 0; i < count; ++i) s += partial[i * m + l];
    out[l] = s;
}

struct DotArgs {
    const double* xt;
    long long n;
    int d;
    int T;
    const double* g1;
    DotDirs dirs;
    int m;
    double sigma;
    int order;
    double* out;
};

template <class Real, int KIND, int DEG, int D>
int dots_impl(const DotArgs& a, Workspace& ws, cudaStream_t st) {
    const int nb = (int)((a.n + kDotTargets - 1) / kDotTargets);
    double* partial = ws.take<double>((size_t)nb * a.T * a.m);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    FusedCoef cf{};
    for (int j = 0; j < 5; ++j) cf.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) cf.pq[j] = ks.pq[j];
    metric_dots_kernel<Real, KIND, DEG, D><<<dim3(nb, a.T), kDotThreads, 0, st>>>(a.xt, a.n, a.g1, a.dirs, a.m,
                                                                                  ks.scale, cf, partial);
    metric_dots_finalize_kernel<<<1, 32, 0, st>>>(partial, (long long)nb * a.T, a.m, a.out);
    return cuda_check(cudaGetLastError(), "metric dots");
}

template <class Real>
int dots_run(const DotArgs& a, Workspace& ws, cudaStream_t st) {
    return dispatch_kind_p(a.order, [&](auto kind, auto deg) {
        return dispatch_d(a.d, [&](auto D) {
            constexpr int K_ = decltype(kind)::value, P_ = decltype(deg)::value, D_ = decltype(D)::value;
            return dots_impl<Real, K_, P_, D_>(a, ws, st);
        });
    });
}

static bool dots_shape_ok(long long n, int d, int T, double sigma, int order) {
    return n >= 1 && n <= (1LL << 30) && d >= 1 && d <= 3 && T >= 1 && T <= 65535 && sigma > 0 && order >= 0;
}

static int dots_validate(const DotArgs& a) {
    if (!dots_shape_ok(a.n, a.d, a.T, a.sigma, a.order)) {
        set_error("metric dots: invalid arguments (n=%lld d=%d T=%d sigma=%g order=%d); d must be 1..3", a.n, a.d,
                  a.T, a.sigma, a.order);
        return LDDMM_ERR_ARG;
    }
    if (a.m < 1 || a.m > kDotMaxDirs) {
        set_error("metric dots: 1 <= m <= %d directions (m=%d)", kDotMaxDirs, a.m);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(a.xt, "xt"));
    LDDMM_TRY(check_device_ptr(a.g1, "g1"));
    LDDMM_TRY(check_device_ptr(a.out, "out"));
    for (int l = 0; l < a.m; ++l) LDDMM_TRY(check_device_ptr(a.dirs.g2[l], "g2"));
    return LDDMM_OK;
}

template <class Real>
size_t dots_ws(int64_t n, int d, int T, int m) {
    DotArgs a{};
    a.n = n;
    a.d = d;
    a.T = T;
    a.m = m;
    a.sigma = 1.0;
    a.order = 10;
    if (!dots_shape_ok(n, d, T, 1.0, 10) || m < 1 || m > kDotMaxDirs) return 0;
    Workspace ws;
    dots_run<Real>(a, ws, 0);
    return ws.off + 256;
}

template <class Real>
int dots_entry(const double* xt, int64_t n, int d, int T, const double* g1, const double* const* g2, int m,
               double sigma, int order, double* out, void* wsp, size_t wsb, cudaStream_t st) {
    DotArgs a{};
    a.xt = xt;
    a.n = n;
    a.d = d;
    a.T = T;
    a.g1 = g1;
    a.m = m;
    a.sigma = sigma;
    a.order = order;
    a.out = out;
    if (g2 == nullptr || m < 1 || m > kDotMaxDirs) {
        set_error("metric dots: g2 must hold 1 to %d device pointers (m=%d)", kDotMaxDirs, m);
        return LDDMM_ERR_ARG;
    }
    for (int l = 0; l < m; ++l) a.dirs.g2[l] = g2[l];
    LDDMM_TRY(dots_validate(a));
    Workspace meas;
    LDDMM_TRY(dots_run<Real>(a, meas, st));
    if (wsp == nullptr || meas.off > wsb) {
        set_error("metric dots: workspace too small: need %zu bytes, got %zu", meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return dots_run<Real>(a, ws, st);
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_metric_dots_f32c_workspace(int64_t n, int d, int T, int m) { return dots_ws<float>(n, d, T, m); }
size_t lddmm_metric_dots_f64_workspace(int64_t n, int d, int T, int m) { return dots_ws<double>(n, d, T, m); }

int lddmm_metric_dots_f32c(const double* xt, int64_t n, int d, int T, const double* g1, const double* const* g2, int m,
                           double sigma, int order, double* out, void* workspace, size_t workspace_bytes,
                           lddmm_stream_t stream) {
    return dots_entry<float>(xt, n, d, T, g1, g2, m, sigma, order, out, workspace, workspace_bytes,
                             (cudaStream_t)stream);
}

int lddmm_metric_dots_f64(const double* xt, int64_t n, int d, int T, const double* g1, const double* const* g2, int m,
                          double sigma, int order, double* out, void* workspace, size_t workspace_bytes,
                          lddmm_stream_t stream) {
    return dots_entry<double>(xt, n, d, T, g1, g2, m, sigma, order, out, workspace, workspace_bytes,
                              (cudaStream_t)stream);
}

}  // extern "C"
