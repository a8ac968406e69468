// C ABI for the kernel sums kff.applyk / kff.applykdifft
// (py-lddmm/kernelFunctions.f90:1-54, 56-114).
#include <type_traits>

#include "host.h"
#include "internal.h"
#include "ops2.cuh"
#include "pack.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

// ---------------------------------------------------------------------------
// applyk
// ---------------------------------------------------------------------------
struct ApplyKArgs {
    const double* x;
    long long n;
    const double* y;
    long long m;
    const double* beta;
    int d, dimb;
    double sigma;
    int order;
    double* f;
    int split_cap;  // 0: no cap on the number of source chunks
};

template <class Real, int KIND, int DEG, int D, int DIMB>
int applyk_group(const ApplyKArgs& a, int col0, Workspace& ws, cudaStream_t st) {
    // FP32: packed-pair operator (two targets per slot, duplicated source records);
    // FP64: the plain operator on double records.
    using Op = std::conditional_t<sizeof(Real) == 4, OpApplyK2<KIND, DEG, D, DIMB>, OpApplyK<Real, KIND, DEG, D, DIMB>>;
    const SinglePlan pl = plan_single<Op>(a.n, a.m, a.split_cap);
    float4* tgt = ws.take<float4>((size_t)Op::PP * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n * DIMB);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    if (ws.overflow()) {
        set_error("workspace too small: need %zu bytes, got %zu", ws.off, ws.cap);
        return LDDMM_ERR_WORKSPACE;
    }
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    Gather g{};
    g.src = a.beta;
    g.row_stride = a.dimb;
    g.nvals = std::min(DIMB, a.dimb - col0);
    for (int c = 0; c < g.nvals; ++c) g.off[c] = col0 + c;
    g.mult = 1.0;
    launch_bbox_center(a.x, a.n, a.y, a.m, a.d, center, st);
    pack_points_kernel<Real><<<grid_for(pl.n_tpad), 256, 0, st>>>(a.x, a.n, a.d, ks.scale, center, tgt, pl.n_tpad,
                                                                  pl.n_tpad);
    if constexpr (sizeof(Real) == 4) {
        for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks.pk[j]);
        for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks.pq[j]);
        pack_dup_kernel<<<grid_for(pl.m_pad), 256, 0, st>>>(a.y, a.m, a.d, ks.scale, center, g, D, DIMB, src,
                                                            pl.m_pad, pl.m_pad);
    } else {
        for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
        for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
        pack_points_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(a.y, a.m, a.d, ks.scale, center, src, pl.m_pad,
                                                                     pl.m_pad);
        pack_values_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(g, a.m, src, pl.m_pad, pl.m_pad, Op::PP);
    }
    LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
    // combine writes only the group's own columns
    const int ncols = g.nvals;
    if (ncols == DIMB) {
        combine_kernel<<<grid_for(a.n * DIMB), 256, 0, st>>>(part, a.n, DIMB, pl.split, 1.0, a.f, a.dimb, col0);
    } else {
        combine_cols_kernel<<<grid_for(a.n * ncols), 256, 0, st>>>(part, a.n, DIMB, ncols, pl.split, 1.0, a.f,
                                                                  a.dimb, col0);
    }
    return cuda_check(cudaGetLastError(), "applyk");
}

template <class Real>
int applyk_run(const ApplyKArgs& a, Workspace& ws, cudaStream_t st) {
    // column groups of at most 4 weights; workspace is reused group after group
    const size_t off0 = ws.off;
    size_t peak = off0;
    for (int col0 = 0; col0 < a.dimb; col0 += 4) {
        ws.off = off0;
        const int g = std::min(4, a.dimb - col0);
        int rc = dispatch_kind_p(a.order, [&](auto kind, auto deg) {
            return dispatch_d(a.d, [&](auto D) {
                return dispatch_dimb(g, [&](auto B) {
                    return applyk_group<Real, decltype(kind)::value, decltype(deg)::value, decltype(D)::value,
                                        decltype(B)::value>(a, col0, ws, st);
                });
            });
        });
        if (rc != LDDMM_OK) return rc;
        peak = std::max(peak, ws.off);
    }
    ws.off = peak;
    return LDDMM_OK;
}

static int applyk_validate(const ApplyKArgs& a) {
    if (a.n < 0 || a.m < 0 || a.d < 1 || a.d > 3 || a.dimb < 1 || !(a.sigma > 0) || a.order < 0) {
        set_error("applyk: invalid arguments (n=%lld m=%lld d=%d dimb=%d sigma=%g order=%d); d must be 1..3",
                  a.n, a.m, a.d, a.dimb, a.sigma, a.order);
        return LDDMM_ERR_ARG;
    }
    if (a.n > (1LL << 30) || a.m > (1LL << 30)) {
        set_error("applyk: more than 2^30 points");
        return LDDMM_ERR_ARG;
    }
    if (a.n == 0) return LDDMM_OK;
    LDDMM_TRY(check_device_ptr(a.x, "x"));
    LDDMM_TRY(check_device_ptr(a.f, "f"));
    if (a.m > 0) {
        LDDMM_TRY(check_device_ptr(a.y, "y"));
        LDDMM_TRY(check_device_ptr(a.beta, "beta"));
    }
    return LDDMM_OK;
}

template <class Real>
size_t applyk_ws(int64_t n, int64_t m, int d, int dimb) {
    ApplyKArgs a{nullptr, n, nullptr, m, nullptr, d, dimb, 1.0, 10, nullptr, 0};
    if (n <= 0 || m <= 0 || d < 1 || d > 3 || dimb < 1) return 0;
    Workspace ws;
    applyk_run<Real>(a, ws, 0);
    return ws.off + 256;
}

template <class Real>
int applyk_entry(const ApplyKArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(applyk_validate(a));
    if (a.n == 0) return LDDMM_OK;
    if (a.m == 0)
        return cuda_check(cudaMemsetAsync(a.f, 0, sizeof(double) * a.n * a.dimb, st), "applyk memset");
    if (wsp == nullptr) {
        set_error("applyk: workspace is NULL (query the *_workspace function)");
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    // a first measuring pass so no launch happens with a short workspace
    Workspace meas;
    applyk_run<Real>(a, meas, st);
    if (meas.off > wsb) {
        set_error("applyk: workspace too small: need %zu bytes, got %zu", meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    return applyk_run<Real>(a, ws, st);
}

// ---------------------------------------------------------------------------
// applykdifft
// ---------------------------------------------------------------------------
struct DiffKTArgs {
    const double* x;
    long long n;
    const double* y;
    long long m;
    const double* a1;
    const double* a2;
    int na, d, dimb;
    double sigma;
    int order;
    double* f;
};

template <class Real, int KIND, int DEG, int D, int W>
int difft_impl(const DiffKTArgs& a, Workspace& ws, cudaStream_t st) {
    using Op = std::conditional_t<sizeof(Real) == 4, OpDiffKT2<KIND, DEG, D, W>, OpDiffKT<Real, KIND, DEG, D, W>>;
    constexpr int NT = (sizeof(Real) == 4) ? 1 + (W + 3) / 4 : Op::NS;  // target planes
    const SinglePlan pl = plan_single<Op>(a.n, a.m);
    float4* tgt = ws.take<float4>((size_t)NT * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n * D);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    // u_k / v_l: value w = c*na + i  <->  a[i, row, c]  (the Fortran sum order)
    Gather gu{}, gv{};
    gu.src = a.a1;
    gv.src = a.a2;
    gu.row_stride = gv.row_stride = a.dimb;
    gu.nvals = gv.nvals = a.na * a.dimb;
    gu.mult = gv.mult = 1.0;
    for (int w = 0; w < a.na * a.dimb; ++w) {
        const int i = w % a.na, c = w / a.na;
        gu.off[w] = (long long)i * a.n * a.dimb + c;
        gv.off[w] = (long long)i * a.m * a.dimb + c;
    }
    launch_bbox_center(a.x, a.n, a.y, a.m, a.d, center, st);
    pack_points_kernel<Real><<<grid_for(pl.n_tpad), 256, 0, st>>>(a.x, a.n, a.d, ks.scale, center, tgt, pl.n_tpad,
                                                                  pl.n_tpad);
    pack_values_kernel<Real><<<grid_for(pl.n_tpad), 256, 0, st>>>(gu, a.n, tgt, pl.n_tpad, pl.n_tpad,
                                                                  PointPlanes<Real>::N);
    if constexpr (sizeof(Real) == 4) {
        for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks.pk[j]);
        for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks.pq[j]);
        pack_dup_kernel<<<grid_for(pl.m_pad), 256, 0, st>>>(a.y, a.m, a.d, ks.scale, center, gv, D, W, src,
                                                            pl.m_pad, pl.m_pad);
    } else {
        for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
        for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
        pack_points_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(a.y, a.m, a.d, ks.scale, center, src, pl.m_pad,
                                                                     pl.m_pad);
        pack_values_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(gv, a.m, src, pl.m_pad, pl.m_pad, Op::PP);
    }
    LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
    const int dout = a.d;  // D may exceed d (d == 1 runs as D == 2)
    if (dout == D) {
        combine_kernel<<<grid_for(a.n * D), 256, 0, st>>>(part, a.n, D, pl.split, ks.dscale, a.f, a.d, 0);
    } else {
        combine_cols_kernel<<<grid_for(a.n * dout), 256, 0, st>>>(part, a.n, D, dout, pl.split, ks.dscale, a.f,
                                                                 a.d, 0);
    }
    return cuda_check(cudaGetLastError(), "applykdifft");
}

template <class Real>
int difft_run(const DiffKTArgs& a, Workspace& ws, cudaStream_t st) {
    return dispatch_kind_q(a.order, [&](auto kind, auto deg) {
        return dispatch_d(a.d, [&](auto D) {
            return dispatch_w(a.na * a.dimb, [&](auto W) {
                return difft_impl<Real, decltype(kind)::value, decltype(deg)::value, decltype(D)::value,
                                  decltype(W)::value>(a, ws, st);
            });
        });
    });
}

static int difft_validate(const DiffKTArgs& a) {
    if (a.n < 0 || a.m < 0 || a.d < 1 || a.d > 3 || a.dimb < 1 || a.na < 1 || !(a.sigma > 0) || a.order < 0) {
        set_error("applykdifft: invalid arguments (n=%lld m=%lld na=%d d=%d dimb=%d sigma=%g order=%d)", a.n, a.m,
                  a.na, a.d, a.dimb, a.sigma, a.order);
        return LDDMM_ERR_ARG;
    }
    if (a.order == 0) {
        set_error("applykdifft: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    if (a.na * a.dimb > 12) {
        set_error("applykdifft: na*dimb = %d exceeds 12", a.na * a.dimb);
        return LDDMM_ERR_UNSUPPORTED;
    }
    if (a.n > (1LL << 30) || a.m > (1LL << 30)) {
        set_error("applykdifft: more than 2^30 points");
        return LDDMM_ERR_ARG;
    }
    if (a.n == 0) return LDDMM_OK;
    LDDMM_TRY(check_device_ptr(a.x, "x"));
    LDDMM_TRY(check_device_ptr(a.a1, "a1"));
    LDDMM_TRY(check_device_ptr(a.f, "f"));
    if (a.m > 0) {
        LDDMM_TRY(check_device_ptr(a.y, "y"));
        LDDMM_TRY(check_device_ptr(a.a2, "a2"));
    }
    return LDDMM_OK;
}

template <class Real>
size_t difft_ws(int64_t n, int64_t m, int na, int d, int dimb) {
    if (n <= 0 || m <= 0 || d < 1 || d > 3 || dimb < 1 || na < 1 || na * dimb > 12) return 0;
    DiffKTArgs a{nullptr, n, nullptr, m, nullptr, nullptr, na, d, dimb, 1.0, 10, nullptr};
    Workspace ws;
    difft_run<Real>(a, ws, 0);
    return ws.off + 256;
}

template <class Real>
int difft_entry(const DiffKTArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(difft_validate(a));
    if (a.n == 0) return LDDMM_OK;
    if (a.m == 0)
        return cuda_check(cudaMemsetAsync(a.f, 0, sizeof(double) * a.n * a.d, st), "applykdifft memset");
    Workspace meas;
    difft_run<Real>(a, meas, st);
    if (wsp == nullptr || meas.off > wsb) {
        set_error("applykdifft: workspace too small: need %zu bytes, got %zu", meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return difft_run<Real>(a, ws, st);
}

// ---------------------------------------------------------------------------
// applyDivergence
// ---------------------------------------------------------------------------
template <class Real, int KIND, int DEG, int D>
int div_impl(const ApplyKArgs& a, Workspace& ws, cudaStream_t st) {
    using Op = OpDivergence<Real, KIND, DEG, D>;
    const SinglePlan pl = plan_single<Op>(a.n, a.m);
    float4* tgt = ws.take<float4>((size_t)Op::PP * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma, /*exact_tables=*/true);
    // (the reference's applyDivergence runs on its dense numpy matrices, which
    //  use the exact rational polynomials, kernelFunctions.py:75-88)
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
    launch_bbox_center(a.x, a.n, a.y, a.m, a.d, center, st);
    pack_points_kernel<Real><<<grid_for(pl.n_tpad), 256, 0, st>>>(a.x, a.n, a.d, ks.scale, center, tgt, pl.n_tpad,
                                                                  pl.n_tpad);
    pack_points_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(a.y, a.m, a.d, ks.scale, center, src, pl.m_pad,
                                                                 pl.m_pad);
    Gather g{};
    g.src = a.beta;
    g.row_stride = a.d;
    g.nvals = a.d;
    for (int c = 0; c < a.d; ++c) g.off[c] = c;
    g.mult = 1.0;  // K' 2 <x-y, a> = dscale * F * <x'-y', a>
    pack_values_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(g, a.m, src, pl.m_pad, pl.m_pad, Op::PP);
    LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
    combine_kernel<<<grid_for(a.n), 256, 0, st>>>(part, a.n, 1, pl.split, ks.dscale, a.f, 1, 0);
    return cuda_check(cudaGetLastError(), "applydiv");
}

template <class Real>
int div_run(const ApplyKArgs& a, Workspace& ws, cudaStream_t st) {
    return dispatch_kind_q(a.order, [&](auto kind, auto deg) {
        return dispatch_d(a.d, [&](auto D) {
            return div_impl<Real, decltype(kind)::value, decltype(deg)::value, decltype(D)::value>(a, ws, st);
        });
    });
}

template <class Real>
size_t div_ws(int64_t n, int64_t m, int d) {
    if (n <= 0 || m <= 0 || d < 1 || d > 3) return 0;
    ApplyKArgs a{nullptr, n, nullptr, m, nullptr, d, d, 1.0, 10, nullptr, 0};
    Workspace ws;
    div_run<Real>(a, ws, 0);
    return ws.off + 256;
}

template <class Real>
int div_entry(const ApplyKArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(applyk_validate(a));
    if (a.order == 0) {
        set_error("applydiv: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    if (a.n == 0) return LDDMM_OK;
    if (a.m == 0) return cuda_check(cudaMemsetAsync(a.f, 0, sizeof(double) * a.n, st), "applydiv memset");
    Workspace meas;
    div_run<Real>(a, meas, st);
    if (wsp == nullptr || meas.off > wsb) {
        set_error("applydiv: workspace too small: need %zu bytes, got %zu", meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return div_run<Real>(a, ws, st);
}

size_t applyk_f32c_scratch_bytes(int64_t n, int64_t m, int d, int dimb, int split_cap) {
    if (n <= 0 || m <= 0 || d < 1 || d > 3 || dimb < 1) return 0;
    ApplyKArgs a{nullptr, n, nullptr, m, nullptr, d, dimb, 1.0, 10, nullptr, split_cap};
    size_t best = 0;
    for (int order : {10, 3}) {  // Gaussian and Laplacian plans
        a.order = order;
        Workspace ws;
        applyk_run<float>(a, ws, 0);
        best = std::max(best, ws.off);
    }
    return best + 256;
}

int applyk_f32c_in_workspace(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                             int dimb, double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                             cudaStream_t stream, int split_cap) {
    ApplyKArgs a{x, n, y, m, beta, d, dimb, sigma, order, f, split_cap};
    return applyk_entry<float>(a, workspace, workspace_bytes, stream);
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_applyk_f32c_workspace(int64_t n, int64_t m, int d, int dimb) { return applyk_ws<float>(n, m, d, dimb); }
size_t lddmm_applyk_f64_workspace(int64_t n, int64_t m, int d, int dimb) { return applyk_ws<double>(n, m, d, dimb); }

int lddmm_applyk_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                      double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                      lddmm_stream_t stream) {
    ApplyKArgs a{x, n, y, m, beta, d, dimb, sigma, order, f, 0};
    return applyk_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_applyk_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                     double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                     lddmm_stream_t stream) {
    ApplyKArgs a{x, n, y, m, beta, d, dimb, sigma, order, f, 0};
    return applyk_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t lddmm_applykdifft_f32c_workspace(int64_t n, int64_t m, int na, int d, int dimb) {
    return difft_ws<float>(n, m, na, d, dimb);
}
size_t lddmm_applykdifft_f64_workspace(int64_t n, int64_t m, int na, int d, int dimb) {
    return difft_ws<double>(n, m, na, d, dimb);
}

int lddmm_applykdifft_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* a1,
                           const double* a2, int na, int d, int dimb, double sigma, int order, double* f,
                           void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    DiffKTArgs a{x, n, y, m, a1, a2, na, d, dimb, sigma, order, f};
    return difft_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_applykdifft_f64(const double* x, int64_t n, const double* y, int64_t m, const double* a1,
                          const double* a2, int na, int d, int dimb, double sigma, int order, double* f,
                          void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    DiffKTArgs a{x, n, y, m, a1, a2, na, d, dimb, sigma, order, f};
    return difft_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t lddmm_applydiv_f32c_workspace(int64_t n, int64_t m, int d) { return div_ws<float>(n, m, d); }
size_t lddmm_applydiv_f64_workspace(int64_t n, int64_t m, int d) { return div_ws<double>(n, m, d); }

int lddmm_applydiv_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* a, int d, double sigma,
                        int order, double* f, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    ApplyKArgs q{x, n, y, m, a, d, d, sigma, order, f, 0};
    return div_entry<float>(q, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_applydiv_f64(const double* x, int64_t n, const double* y, int64_t m, const double* a, int d, double sigma,
                       int order, double* f, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    ApplyKArgs q{x, n, y, m, a, d, d, sigma, order, f, 0};
    return div_entry<double>(q, workspace, workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
