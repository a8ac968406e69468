// C ABI for the first- and second-derivative kernel loops of
// py-lddmm/kernelFunctions.f90:116-496 (self-interaction: targets = sources = x):
//
//   applykdiff1     f_k =  sum_l K'  2 <dx, a1_k> a2_l                      (:116-172)
//   applykdiff2     f_k = -sum_l K'  2 <dx, a1_l> a2_l                      (:174-230)
//   applykdiff1and2 f_k =  sum_l K'  2 <dx, a1_k - a1_l> a2_l               (:233-290)
//   applykdiff11    f_k =  sum_l c (K'' 4 <dx, p_k> dx + K' 2 p_k)           (:293-359)
//   applykdiff12    f_k = -sum_l c (K'' 4 <dx, p_l> dx + K' 2 p_l)           (:361-428)
//   applykdiff11and12 f_k = sum_l c (K'' 4 <dx, dp> dx + K' 2 dp)            (:430-496)
//
// with dx = x_k - x_l, dp = p_k - p_l, c = <a1_k, a2_l>, and K' (c1_ table),
// K'' (c2_ table) the Fortran's first and second derivative factors.  The
// reference's 11 / 12 loops run over an undeclared `num_nodes_y`; the
// intended y = x is computed.  K'' needs Laplacian order >= 2 (the Fortran
// reads c2_(ord-1,.) out of bounds for orders 0 and 1): those orders are
// rejected, as order 0 is for the first-derivative loops.
//
// Same sweep as the kernel sums (tiled, chunked, deterministic combine) with
// FP32-compensated (_f32c) or FP64 (_f64) pair arithmetic on prescaled
// coordinates x' = scale x:  K' 2 dx = dscale F dx',  K'' 4 <dx,v> dx =
// d2scale G <dx',v> dx',  K' 2 = c1s F, with F = Q e, G = R e the polynomial
// times exponential factors (Gaussian: F = G = e).
#include <type_traits>

#include "host.h"
#include "internal.h"
#include "ops.cuh"
#include "pack.cuh"
#include "sweep.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

enum SecondMode : int { S_D1 = 1, S_D2 = 2, S_D12 = 3, S_11 = 11, S_12 = 12, S_1112 = 13 };

template <int MODE, int D>
struct SecondLayout {
    // target values: a1_k (D) [+ p_k (D)]; source values: a1_l / a2_l / p_l as needed
    static constexpr int TV = (MODE == S_D1 || MODE == S_D12 || MODE == S_12) ? D
                              : (MODE == S_11 || MODE == S_1112)          ? 2 * D
                                                                           : 0;
    static constexpr int SV = (MODE == S_D1 || MODE == S_11) ? D : 2 * D;
    static constexpr int NOUT = (MODE == S_11) ? D + 1 : (MODE == S_12 || MODE == S_1112) ? 2 * D : D;
    static constexpr bool SECOND = MODE >= S_11;
};

template <class Real>
struct SecondParams : KernelParamsBase<Real> {
    Real pr[3];  // K'' polynomial (prescaled)
};

// F (first-derivative factor) and G (second) from the prescaled squared distance
template <class Real, int KIND, int QDEG, int RDEG, bool SECOND>
LDDMM_D void kfactors(const Real* pq, const Real* pr, Real r2, Real& F, Real& G) {
    if constexpr (KIND == KGAUSS) {
        F = kdiff<Real, KIND, 0>(pq, r2);
        G = F;
    } else if constexpr (sizeof(Real) == 4) {
        const float u = sqrt_approx(r2);
        const float e = ex2(-u);
        F = (QDEG == 0 ? pq[0] : horner<QDEG>(pq, u)) * e;
        if constexpr (SECOND) G = (RDEG == 0 ? pr[0] : horner<RDEG>(pr, u)) * e;
        else G = 0.f;
    } else {
        const double u = sqrt(r2);
        if (u < kZeroThresh) {
            F = pq[0];
            G = SECOND ? pr[0] : 0.0;
        } else {
            const double e = exp(-1.0 * u);
            F = poly64<QDEG>(pq, u) * e;
            G = SECOND ? poly64<RDEG>(pr, u) * e : 0.0;
        }
    }
}

template <class Real_, int KIND, int QDEG, int RDEG, int D, int MODE>
struct OpSecond {
    using Real = Real_;
    using L = SecondLayout<MODE, D>;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = 128, R = 2, TILE = 128, FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int PW = Traits<Real>::PER_WORD;
    static constexpr int TVW = (L::TV + PW - 1) / PW;
    static constexpr int SVW = (L::SV + PW - 1) / PW;
    static constexpr int NT = PP + TVW;
    static constexpr int NS = PP + SVW;
    static constexpr int NOUT = L::NOUT;
    using Params = SecondParams<Real>;
    using Acc = typename AccFor<Real>::template type<NOUT>;
    struct Tgt {
        Real x[D];
        Real u[L::TV > 0 ? L::TV : 1];
    };
    struct Src {
        Real y[D];
        Real v[L::SV];
    };
    static LDDMM_D void load_target(const Params& P, long long row, Tgt& t) {
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, 0, t.x);
        if constexpr (L::TV > 0) load_vals<Real, L::TV>(P.tgt4, P.tgt_stride, row, PP, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) {
        load_vals_smem<Real, D, TILE>(S, j, 0, s.y);
        load_vals_smem<Real, L::SV, TILE>(S, j, PP, s.v);
    }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& acc) {
        Real dx[D], r2 = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            dx[j] = t.x[j] - s.y[j];
            r2 = j == 0 ? dx[j] * dx[j] : r2 + dx[j] * dx[j];
        }
        Real F, G;
        kfactors<Real, KIND, QDEG, RDEG, L::SECOND>(P.pq, P.pr, r2, F, G);
        if constexpr (MODE == S_D1 || MODE == S_D2 || MODE == S_D12) {
            // a1 of the <dx, .> product: target (D1), source (D2), difference (D12)
            Real dot = 0;
#pragma unroll
            for (int j = 0; j < D; ++j) {
                const Real a = MODE == S_D1 ? t.u[j] : MODE == S_D2 ? s.v[j] : t.u[j] - s.v[j];
                dot = j == 0 ? dx[0] * a : dot + dx[j] * a;
            }
            const Real g = F * dot;
            constexpr int OFF = MODE == S_D1 ? 0 : D;   // a2_l position in the source values
#pragma unroll
            for (int j = 0; j < D; ++j) acc.fma(j, g, s.v[OFF + j]);
        } else {
            Real c = 0, q = 0;
            Real w[D];  // p_k (11), p_l (12), p_k - p_l (11and12)
#pragma unroll
            for (int j = 0; j < D; ++j) {
                c = j == 0 ? t.u[0] * s.v[0] : c + t.u[j] * s.v[j];
                w[j] = MODE == S_11 ? t.u[D + j] : MODE == S_12 ? s.v[D + j] : t.u[D + j] - s.v[D + j];
                q = j == 0 ? dx[0] * w[0] : q + dx[j] * w[j];
            }
            const Real gq = G * c * q;
#pragma unroll
            for (int j = 0; j < D; ++j) acc.fma(j, gq, dx[j]);
            if constexpr (MODE == S_11) {
                acc.add(D, F * c);
            } else {
                const Real fc = F * c;
#pragma unroll
                for (int j = 0; j < D; ++j) acc.fma(D + j, fc, w[j]);
            }
        }
    }
};

// record i: prescaled position, then the values of up to two (n, d) arrays in
// slots [0, D) and [D, 2D)
template <class Real>
static __global__ void second_pack_kernel(const double* __restrict__ x, long long n, int d, double scale,
                                          const double* __restrict__ center, const double* __restrict__ v0,
                                          const double* __restrict__ v1, int D, float4* __restrict__ planes,
                                          long long stride, long long npad) {
    constexpr int PP = PointPlanes<Real>::N;
    constexpr int PW = Traits<Real>::PER_WORD;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        double pos[4] = {0, 0, 0, 0}, vals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (i < n)
            for (int j = 0; j < d; ++j) {
                pos[j] = (x[i * d + j] - center[j]) * scale;
                if (v0) vals[j] = v0[i * d + j];
                if (v1) vals[D + j] = v1[i * d + j];
            }
        if constexpr (PP == 1) {
            planes[i] = make_float4((float)pos[0], (float)pos[1], (float)pos[2], 0.f);
        } else {
            double2* o = reinterpret_cast<double2*>(planes);
            o[i] = make_double2(pos[0], pos[1]);
            o[stride + i] = make_double2(pos[2], 0.0);
        }
        const int nv = (v1 ? 2 : 1) * D;
        if (!v0) continue;
        for (int w = 0; w < (nv + PW - 1) / PW; ++w) {
            float4* dst = planes + (long long)(PP + w) * stride + i;
            if constexpr (PW == 4) {
                *dst = make_float4((float)vals[4 * w], (float)vals[4 * w + 1], (float)vals[4 * w + 2],
                                   (float)vals[4 * w + 3]);
            } else {
                *reinterpret_cast<double2*>(dst) = make_double2(vals[2 * w], vals[2 * w + 1]);
            }
        }
    }
}

// f_k from the chunk sums (fixed order), with the routine's constants
template <int MODE, int D>
static __global__ void second_combine_kernel(const double* __restrict__ part, long long n, int split, double dscale,
                                             double d2scale, double c1s, const double* __restrict__ p,
                                             double* __restrict__ f, int d) {
    using L = SecondLayout<MODE, D>;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double acc[L::NOUT];
        for (int c = 0; c < L::NOUT; ++c) acc[c] = 0.0;
        for (int k = 0; k < split; ++k) {
            const double* pk = part + ((long long)k * n + i) * L::NOUT;
            for (int c = 0; c < L::NOUT; ++c) acc[c] += pk[c];
        }
        for (int j = 0; j < d; ++j) {
            double v;
            if constexpr (MODE == S_D1 || MODE == S_D12) v = dscale * acc[j];
            else if constexpr (MODE == S_D2) v = -dscale * acc[j];
            else if constexpr (MODE == S_11) v = d2scale * acc[j] + c1s * acc[D] * p[i * d + j];
            else if constexpr (MODE == S_12) v = -(d2scale * acc[j] + c1s * acc[D + j]);
            else v = d2scale * acc[j] + c1s * acc[D + j];
            f[i * d + j] = v;
        }
    }
}

struct SecondArgs {
    const double* x;
    long long n;
    int d;
    const double* a1;
    const double* a2;
    const double* p;
    double sigma;
    int order;
    double* f;
};

template <class Real, int KIND, int QDEG, int RDEG, int D, int MODE>
int second_impl(const SecondArgs& a, Workspace& ws, cudaStream_t st) {
    using Op = OpSecond<Real, KIND, QDEG, RDEG, D, MODE>;
    using L = SecondLayout<MODE, D>;
    const SinglePlan pl = plan_single<Op>(a.n, a.n);
    float4* tgt = ws.take<float4>((size_t)Op::NT * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n * Op::NOUT);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    double Pp[5], Qq[4], Rr[3];
    laplacian_tables(a.order, Pp, Qq, Rr, false);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    const double Lg = 1.4426950408889634;
    double Lj = 1.0;
    for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
    for (int j = 0; j < 3; ++j) {
        P.pr[j] = (Real)(sizeof(Real) == 4 ? Rr[j] / Lj : Rr[j]);
        Lj *= Lg;
    }
    const double s2 = a.sigma * a.sigma;
    const double d2scale = 1.0 / (s2 * s2 * ks.scale * ks.scale);
    const double c1s = -1.0 / s2;
    // target values: a1_k [, p_k];  source values per mode
    const double* tv0 = L::TV > 0 ? a.a1 : nullptr;
    const double* tv1 = (MODE == S_11 || MODE == S_1112) ? a.p : nullptr;
    const double* sv0 = MODE == S_D1 ? a.a2 : MODE == S_D2 || MODE == S_D12 ? a.a1 : a.a2;
    const double* sv1 = MODE == S_D1 || MODE == S_11 ? nullptr : MODE == S_D2 || MODE == S_D12 ? a.a2 : a.p;
    launch_bbox_center(a.x, a.n, nullptr, 0, a.d, center, st);
    second_pack_kernel<Real><<<grid_for(pl.n_tpad), 256, 0, st>>>(a.x, a.n, a.d, ks.scale, center, tv0, tv1, D, tgt,
                                                                  pl.n_tpad, pl.n_tpad);
    second_pack_kernel<Real><<<grid_for(pl.m_pad), 256, 0, st>>>(a.x, a.n, a.d, ks.scale, center, sv0, sv1, D, src,
                                                                 pl.m_pad, pl.m_pad);
    LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
    second_combine_kernel<MODE, D><<<grid_for(a.n), 256, 0, st>>>(part, a.n, pl.split, ks.dscale, d2scale, c1s, a.p,
                                                                  a.f, a.d);
    return cuda_check(cudaGetLastError(), "applykdiff");
}

// Gaussian: (KGAUSS, 0, 0); Laplacian order o: Q degree o-1, R degree o-2
template <class F>
int dispatch_second(int order, F&& f) {
    switch (order) {
        case 1: return f(IC<KLAP>{}, IC<0>{}, IC<0>{});
        case 2: return f(IC<KLAP>{}, IC<1>{}, IC<0>{});
        case 3: return f(IC<KLAP>{}, IC<2>{}, IC<1>{});
        case 4: return f(IC<KLAP>{}, IC<3>{}, IC<2>{});
        default: return f(IC<KGAUSS>{}, IC<0>{}, IC<0>{});
    }
}

template <class Real, int MODE>
int second_run(const SecondArgs& a, Workspace& ws, cudaStream_t st) {
    return dispatch_second(a.order, [&](auto K, auto Q, auto Rd) {
        return dispatch_d(a.d, [&](auto D) {
            return second_impl<Real, decltype(K)::value, decltype(Q)::value, decltype(Rd)::value,
                               decltype(D)::value, MODE>(a, ws, st);
        });
    });
}

template <class Real, int MODE>
int second_entry(const SecondArgs& a, void* wsp, size_t wsb, cudaStream_t st, const char* who) {
    const bool second = MODE >= S_11;
    if (a.n < 0 || a.d < 1 || a.d > 3 || !(a.sigma > 0) || a.order < 0 || a.order == 0 ||
        (second && a.order >= 0 && a.order <= 1)) {
        set_error("%s: invalid arguments (n=%lld d=%d sigma=%g order=%d%s)", who, a.n, a.d, a.sigma, a.order,
                  second ? "; second derivatives need a Gaussian or a Laplacian of order >= 2" : "");
        return LDDMM_ERR_ARG;
    }
    if (a.n == 0) return LDDMM_OK;
    LDDMM_TRY(check_device_ptr(a.x, "x"));
    LDDMM_TRY(check_device_ptr(a.a1, "a1"));
    LDDMM_TRY(check_device_ptr(a.a2, "a2"));
    if (second) LDDMM_TRY(check_device_ptr(a.p, "p"));
    LDDMM_TRY(check_device_ptr(a.f, "f"));
    Workspace meas;
    LDDMM_TRY((second_run<Real, MODE>(a, meas, st)));
    if (wsp == nullptr || meas.off > wsb) {
        set_error("%s: workspace too small: need %zu bytes, got %zu", who, meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return second_run<Real, MODE>(a, ws, st);
}

template <class Real>
size_t second_workspace(int routine, long long n, int d, int order) {
    if (n < 1 || d < 1 || d > 3) return 0;
    SecondArgs a{nullptr, n, d, nullptr, nullptr, nullptr, 1.0, order, nullptr};
    Workspace ws;
    int rc = LDDMM_ERR_ARG;
    switch (routine) {
        case S_D1: rc = second_run<Real, S_D1>(a, ws, 0); break;
        case S_D2: rc = second_run<Real, S_D2>(a, ws, 0); break;
        case S_D12: rc = second_run<Real, S_D12>(a, ws, 0); break;
        case S_11: rc = second_run<Real, S_11>(a, ws, 0); break;
        case S_12: rc = second_run<Real, S_12>(a, ws, 0); break;
        case S_1112: rc = second_run<Real, S_1112>(a, ws, 0); break;
        default: return 0;
    }
    return rc == LDDMM_OK ? ws.off + 256 : 0;
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_applykdiffx_f32c_workspace(int routine, int64_t n, int d, int order) {
    return second_workspace<float>(routine, n, d, order);
}
size_t lddmm_applykdiffx_f64_workspace(int routine, int64_t n, int d, int order) {
    return second_workspace<double>(routine, n, d, order);
}

#define LDDMM_FIRST_ENTRY(NAME, SFX, REAL, MODE)                                                                  \
    int NAME##_##SFX(const double* x, int64_t n, int d, const double* a1, const double* a2, double sigma,          \
                     int order, double* f, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {       \
        SecondArgs a{x, n, d, a1, a2, nullptr, sigma, order, f};                                                    \
        return second_entry<REAL, MODE>(a, workspace, workspace_bytes, (cudaStream_t)stream, #NAME);              \
    }
#define LDDMM_SECOND_ENTRY(NAME, SFX, REAL, MODE)                                                                 \
    int NAME##_##SFX(const double* x, int64_t n, int d, const double* a1, const double* a2, const double* p,       \
                     double sigma, int order, double* f, void* workspace, size_t workspace_bytes,                  \
                     lddmm_stream_t stream) {                                                                      \
        SecondArgs a{x, n, d, a1, a2, p, sigma, order, f};                                                          \
        return second_entry<REAL, MODE>(a, workspace, workspace_bytes, (cudaStream_t)stream, #NAME);              \
    }

LDDMM_FIRST_ENTRY(lddmm_applykdiff1, f32c, float, S_D1)
LDDMM_FIRST_ENTRY(lddmm_applykdiff1, f64, double, S_D1)
LDDMM_FIRST_ENTRY(lddmm_applykdiff2, f32c, float, S_D2)
LDDMM_FIRST_ENTRY(lddmm_applykdiff2, f64, double, S_D2)
LDDMM_FIRST_ENTRY(lddmm_applykdiff1and2, f32c, float, S_D12)
LDDMM_FIRST_ENTRY(lddmm_applykdiff1and2, f64, double, S_D12)
LDDMM_SECOND_ENTRY(lddmm_applykdiff11, f32c, float, S_11)
LDDMM_SECOND_ENTRY(lddmm_applykdiff11, f64, double, S_11)
LDDMM_SECOND_ENTRY(lddmm_applykdiff12, f32c, float, S_12)
LDDMM_SECOND_ENTRY(lddmm_applykdiff12, f64, double, S_12)
LDDMM_SECOND_ENTRY(lddmm_applykdiff11and12, f32c, float, S_1112)
LDDMM_SECOND_ENTRY(lddmm_applykdiff11and12, f64, double, S_1112)

}  // extern "C"
