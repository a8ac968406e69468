// Data-attachment terms on surfaces (triangles) and curves (edges):
// current, measure and varifold norms and their vertex gradients.
//
// Reference: py-lddmm/surfaces.py:1009-1276 and curves.py:539-703.
//   cell geometry  : surfaces c = (x0+x1+x2)/3, s = (x1-x0) x (x2-x0) (surfaces.py:61-75)
//                    curves   c = (x0+x1)/2,    s = x1 - x0           (curves.py:58-75)
//   weights        : current s;  measure a = sqrt(|s|^2 + eps);  varifold (n = s/a, a)
//   value (Def)    : <S1, S1> - 2 <S1, S2>,  with Norm0(S) = <S, S>
//       current  : sum_kl K(c_k,c_l) <s_k, s_l>
//       measure  : sum_kl K(c_k,c_l) a_k a_l
//       varifold : sum_kl K(c_k,c_l) (1 + <n_k,n_l>^2) a_k a_l           (surfaces.py:1200-1221)
//   gradient       : per cell z1 = sum_l K w_l (signed sources: set 1 +, set 2 -),
//                    dz1 = fac * sum_l K' 2 (c_k - c_l) beta_kl, fac = 1/3 (surfaces), 1/2 (curves),
//                    then px[v] = 2 sum over the cells of v of (dz1 - e x z1) (surfaces, e the
//                    opposite edge of the corner, surfaces.py:1069-1089) or dz1 -/+ z1 (curves,
//                    curves.py:596-613).
//     varifold z1 = sum_l K a_l (2 <n_k,n_l> n_l - <n_k,n_l>^2 n_k + n_k)   (surfaces.py:1247-1252)
//
// One sweep per call: targets = cells of set 1, sources = cells of set 1 then of
// set 2 (target shape), both weighted per source.  No F x F array is formed.
#include "host.h"
#include "pack.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

enum DataNorm : int { NCURRENT = 0, NMEASURE = 1, NVARIFOLD = 2 };
enum DataMode : int { M_VARI_VALUE = 0, M_VARI_GRAD = 1, M_CUR_GRAD = 2, M_MEAS_GRAD = 3 };

// Gaussian K' uses the same exponential as K.
template <class Real, int KIND, int PDEG, int QDEG>
LDDMM_D void kboth(const Real* pk, const Real* pq, Real r2, Real& k, Real& f) {
    if constexpr (KIND == KGAUSS) {
        k = kval<Real, KIND, 0>(pk, r2);
        f = k;
    } else if constexpr (sizeof(Real) == 4) {
        const float u = sqrt_approx(r2);
        const float e = ex2(-u);
        k = (PDEG == 0 ? 1.f : horner<PDEG>(pk, u)) * e;
        f = (QDEG == 0 ? pq[0] : horner<QDEG>(pq, u)) * e;
    } else {
        const double u = sqrt(r2);
        if (u < kZeroThresh) {
            k = 1.0;
            f = pq[0];
        } else {
            const double e = exp(-1.0 * u);
            k = poly64<PDEG>(pk, u) * e;
            f = poly64<QDEG>(pq, u) * e;
        }
    }
}

template <int MODE, int D>
struct DataLayout {
    static constexpr int TV = (MODE == M_VARI_VALUE || MODE == M_VARI_GRAD) ? 3 : (MODE == M_CUR_GRAD ? D : 0);
    static constexpr int SV = (MODE == M_VARI_VALUE || MODE == M_VARI_GRAD) ? 4 : (MODE == M_CUR_GRAD ? D : 1);
    static constexpr int NOUT = MODE == M_VARI_VALUE ? 1
                                : MODE == M_VARI_GRAD ? 2 * D + 1
                                : MODE == M_CUR_GRAD  ? 2 * D
                                                      : D + 1;
};

template <class Real_, int KIND, int PDEG, int QDEG, int D, int MODE>
struct OpData {
    using Real = Real_;
    using L = DataLayout<MODE, D>;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = 128, R = 2, TILE = 128, FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int PW = Traits<Real>::PER_WORD;
    static constexpr int TVW = (L::TV + PW - 1) / PW;
    static constexpr int SVW = (L::SV + PW - 1) / PW;
    static constexpr int NT = PP + TVW;  // target planes
    static constexpr int NS = PP + SVW;  // source planes
    static constexpr int NOUT = L::NOUT;
    using Params = KernelParamsBase<Real>;
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
        if constexpr (MODE == M_VARI_VALUE) {
            const Real k = kval<Real, KIND, PDEG>(P.pk, r2);
            const Real dn = t.u[0] * s.v[0] + t.u[1] * s.v[1] + t.u[2] * s.v[2];
            acc.fma(0, k * s.v[3], (Real)1 + dn * dn);
        } else {
            Real k, f;
            kboth<Real, KIND, PDEG, QDEG>(P.pk, P.pq, r2, k, f);
            if constexpr (MODE == M_VARI_GRAD) {
                const Real dn = t.u[0] * s.v[0] + t.u[1] * s.v[1] + t.u[2] * s.v[2];
                const Real wk = k * s.v[3];
                const Real ca = 2 * dn * wk;
#pragma unroll
                for (int j = 0; j < D; ++j) acc.fma(j, ca, s.v[j]);
                acc.fma(D, wk, (Real)1 - dn * dn);
                const Real wf = f * s.v[3] * ((Real)1 + dn * dn);
#pragma unroll
                for (int j = 0; j < D; ++j) acc.fma(D + 1 + j, wf, dx[j]);
            } else if constexpr (MODE == M_CUR_GRAD) {
                Real dot = 0;
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    acc.fma(j, k, s.v[j]);
                    dot = j == 0 ? t.u[0] * s.v[0] : dot + t.u[j] * s.v[j];
                }
                const Real g = f * dot;
#pragma unroll
                for (int j = 0; j < D; ++j) acc.fma(D + j, g, dx[j]);
            } else {  // M_MEAS_GRAD
                acc.fma(0, k, s.v[0]);
                const Real g = f * s.v[0];
#pragma unroll
                for (int j = 0; j < D; ++j) acc.fma(1 + j, g, dx[j]);
            }
        }
    }
};

// ---- geometry -----------------------------------------------------------------
// centres (nc, d), vectors (nc, d) (surfels or tangents) of set 1; invalid cell
// indices give zero geometry (host code validates them before the call).
static __global__ void cell_geometry_kernel(int ncorner, const double* __restrict__ v, long long nv, int d,
                                            const int64_t* __restrict__ cells, long long nc, double* __restrict__ c,
                                            double* __restrict__ s) {
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nc;
         f += (long long)gridDim.x * blockDim.x) {
        long long id[3] = {0, 0, 0};
        bool ok = true;
        for (int q = 0; q < ncorner; ++q) {
            id[q] = cells[f * ncorner + q];
            ok = ok && id[q] >= 0 && id[q] < nv;
        }
        if (!ok) {
            for (int j = 0; j < d; ++j) c[f * d + j] = s[f * d + j] = 0.0;
            continue;
        }
        const double* x0 = v + id[0] * d;
        const double* x1 = v + id[1] * d;
        if (ncorner == 3) {
            const double* x2 = v + id[2] * d;
            for (int j = 0; j < 3; ++j) c[f * 3 + j] = (x0[j] + x1[j] + x2[j]) / 3;
            const double e1[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
            const double e2[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
            s[f * 3 + 0] = e1[1] * e2[2] - e1[2] * e2[1];
            s[f * 3 + 1] = e1[2] * e2[0] - e1[0] * e2[2];
            s[f * 3 + 2] = e1[0] * e2[1] - e1[1] * e2[0];
        } else {
            for (int j = 0; j < d; ++j) {
                c[f * d + j] = (x0[j] + x1[j]) / 2;
                s[f * d + j] = x1[j] - x0[j];
            }
        }
    }
}

LDDMM_D double vec_norm_eps(const double* s, int d, double eps) {
    double q = 0.0;
    for (int j = 0; j < d; ++j) q += s[j] * s[j];
    return sqrt(q + eps);
}

// Targets: set-1 cells.  Sources: set-1 cells (sign +1) then set-2 cells (sign2).
// Values per record follow DataLayout / OpApplyK:
//   norm current : target -, source s*sign              (value, OpApplyK DIMB = d)
//                  target s, source s*sign              (gradient)
//   norm measure : target -, source a*sign              (value and gradient)
//   norm varifold: target n, source (n, a*sign)         (value and gradient)
template <class Real>
static __global__ void dt_pack_kernel(int norm, int grad, const double* __restrict__ c1, const double* __restrict__ s1,
                                      long long n1, const double* __restrict__ c2, const double* __restrict__ s2,
                                      long long n2, int d, double eps1, double eps2, double sign2, double scale,
                                      const double* __restrict__ center, float4* tgt, long long tstride, int tplanes,
                                      int tslots, float4* src, long long sstride, int splanes, int sslots) {
    constexpr int PP = PointPlanes<Real>::N;
    const long long npad = tstride > sstride ? tstride : sstride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        for (int role = 0; role < 2; ++role) {
            const bool is_t = role == 0;
            const long long stride = is_t ? tstride : sstride;
            if (i >= stride) continue;
            float4* planes = is_t ? tgt : src;
            const int nplanes = is_t ? tplanes : splanes;
            const long long nrows = is_t ? n1 : n1 + n2;
            if (i >= nrows) {
                for (int p = 0; p < nplanes; ++p) planes[(long long)p * stride + i] = make_float4(0.f, 0.f, 0.f, 0.f);
                continue;
            }
            const bool first = i < n1;
            const double* c = first ? c1 + i * d : c2 + (i - n1) * d;
            const double* s = first ? s1 + i * d : s2 + (i - n1) * d;
            const double sign = (is_t || first) ? 1.0 : sign2;
            const double a = vec_norm_eps(s, d, first ? eps1 : eps2);
            double pos[4] = {0, 0, 0, 0};
            for (int j = 0; j < d; ++j) pos[j] = (c[j] - center[j]) * scale;
            if constexpr (sizeof(Real) == 4) {
                planes[i] = make_float4((float)pos[0], (float)pos[1], (float)pos[2], 0.f);
            } else {
                double2* o = reinterpret_cast<double2*>(planes);
                o[i] = make_double2(pos[0], pos[1]);
                o[stride + i] = make_double2(pos[2], 0.0);
            }
            double vals[4] = {0, 0, 0, 0};
            int nv = 0;
            if (norm == NVARIFOLD) {
                for (int j = 0; j < 3; ++j) vals[j] = s[j] / a;
                nv = 3;
                if (!is_t) {
                    vals[3] = a * sign;
                    nv = 4;
                }
            } else if (norm == NCURRENT) {
                if (!is_t || grad) {
                    for (int j = 0; j < d; ++j) vals[j] = s[j] * sign;
                    nv = d;
                }
            } else {
                if (!is_t) {
                    vals[0] = a * sign;
                    nv = 1;
                }
            }
            const int slots = is_t ? tslots : sslots;
            constexpr int PWv = Traits<Real>::PER_WORD;
            for (int w = 0; w < (slots + PWv - 1) / PWv; ++w) {
                Real q[PWv];
                for (int j = 0; j < PWv; ++j) q[j] = (w * PWv + j < nv) ? (Real)vals[w * PWv + j] : (Real)0;
                float4* dst = planes + (long long)(PP + w) * stride + i;
                if constexpr (sizeof(Real) == 4) *dst = make_float4(q[0], q[1], q[2], q[3]);
                else *reinterpret_cast<double2*>(dst) = make_double2(q[0], q[1]);
            }
        }
    }
}

constexpr int kDtThreads = 256;

LDDMM_D void dt_block_sum(double v, double* out) {
    __shared__ double red[kDtThreads];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = kDtThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// energy partial: sum_k w1_k . acc_k (current: s1 . z, measure: a1 z, varifold: a1 z)
static __global__ void dt_value_combine_kernel(int norm, const double* __restrict__ part, long long n1, int nout,
                                               int split, const double* __restrict__ s1, int d, double eps1,
                                               double* __restrict__ epart) {
    double e = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n1;
         i += (long long)gridDim.x * blockDim.x) {
        double z[4] = {0, 0, 0, 0};
        for (int c = 0; c < nout; ++c)
            for (int k = 0; k < split; ++k) z[c] += part[((long long)k * n1 + i) * nout + c];
        const double* s = s1 + i * d;
        if (norm == NCURRENT) {
            for (int j = 0; j < d; ++j) e += s[j] * z[j];
        } else {
            e += vec_norm_eps(s, d, eps1) * z[0];
        }
    }
    dt_block_sum(e, epart);
}

static __global__ void dt_finalize_kernel(const double* __restrict__ vals, long long count, double scale,
                                          double* __restrict__ out) {
    double v = 0.0;
    for (long long i = threadIdx.x; i < count; i += blockDim.x) v += vals[i];
    dt_block_sum(v, out);
    if (threadIdx.x == 0) out[0] = scale * out[0];
}

// per-cell z1, dz1 from the gradient sweep
static __global__ void dt_grad_combine_kernel(int norm, const double* __restrict__ part, long long n1, int nout,
                                              int split, const double* __restrict__ s1, int d, double eps1,
                                              double dzscale, double* __restrict__ z1, double* __restrict__ dz1) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n1;
         i += (long long)gridDim.x * blockDim.x) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < nout; ++c)
            for (int k = 0; k < split; ++k) acc[c] += part[((long long)k * n1 + i) * nout + c];
        const double* s = s1 + i * d;
        if (norm == NCURRENT) {
            for (int j = 0; j < d; ++j) {
                z1[i * d + j] = acc[j];
                dz1[i * d + j] = dzscale * acc[d + j];
            }
        } else if (norm == NMEASURE) {
            const double a = vec_norm_eps(s, d, eps1);
            for (int j = 0; j < d; ++j) {
                z1[i * d + j] = acc[0] * (s[j] / a);
                dz1[i * d + j] = dzscale * a * acc[1 + j];
            }
        } else {
            const double a = vec_norm_eps(s, d, eps1);
            for (int j = 0; j < d; ++j) {
                z1[i * d + j] = acc[j] + acc[d] * (s[j] / a);
                dz1[i * d + j] = dzscale * a * acc[d + 1 + j];
            }
        }
    }
}

// px[v] = 2 sum over (cell, corner) entries of v of the corner contribution.
static __global__ void dt_gather_kernel(int ncorner, const double* __restrict__ v, long long nv, int d,
                                        const int64_t* __restrict__ cells, long long nc,
                                        const int64_t* __restrict__ vptr, const int64_t* __restrict__ vidx,
                                        const double* __restrict__ z1, const double* __restrict__ dz1,
                                        double* __restrict__ px) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
         q += (long long)gridDim.x * blockDim.x) {
        double acc[3] = {0, 0, 0};
        const long long b = vptr[q], e = vptr[q + 1];
        for (long long k = b; k < e; ++k) {
            const long long code = vidx[k];
            if (code < 0 || code >= nc * ncorner) continue;
            const long long f = code / ncorner;
            const int corner = (int)(code - f * ncorner);
            const double* z = z1 + f * d;
            const double* dz = dz1 + f * d;
            if (ncorner == 3) {
                // opposite edge of the corner: x2-x1, x0-x2, x1-x0
                const int ia = (corner + 2) % 3, ib = (corner + 1) % 3;
                const long long va = cells[f * 3 + ia], vb = cells[f * 3 + ib];
                if (va < 0 || va >= nv || vb < 0 || vb >= nv) continue;
                double ed[3];
                for (int j = 0; j < 3; ++j) ed[j] = v[va * 3 + j] - v[vb * 3 + j];
                const double cr[3] = {ed[1] * z[2] - ed[2] * z[1], ed[2] * z[0] - ed[0] * z[2],
                                      ed[0] * z[1] - ed[1] * z[0]};
                for (int j = 0; j < 3; ++j) acc[j] += dz[j] - cr[j];
            } else {
                const double sgn = corner == 0 ? -1.0 : 1.0;
                for (int j = 0; j < d; ++j) acc[j] += dz[j] + sgn * z[j];
            }
        }
        for (int j = 0; j < d; ++j) px[q * d + j] = 2 * acc[j];
    }
}

struct DataArgs {
    int ncorner;  // 3 surfaces, 2 curves
    int norm;     // NCURRENT / NMEASURE / NVARIFOLD
    const double* v;
    long long nv;
    int d;
    const int64_t* cells;
    long long nc;
    const double* c2;
    const double* s2;
    long long nc2;
    double sigma;
    int order;
    double eps1, eps2;
    double* energy;
    const int64_t* vptr;
    const int64_t* vidx;
    double* px;
};

template <class Op, class Real>
int dt_sweep(const DataArgs& a, Workspace& ws, cudaStream_t st, int grad, double sign2, const double* c1,
             const double* s1, double*& part, SinglePlan& pl, const KScale& ks, const double* center) {
    pl = plan_single<Op>(a.nc, a.nc + a.nc2);
    float4* tgt = ws.take<float4>((size_t)Op::NT_ * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    part = ws.take<double>((size_t)pl.split * a.nc * Op::NOUT);
    if (ws.measuring()) return LDDMM_OK;
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
    dt_pack_kernel<Real><<<grid_for(std::max(pl.n_tpad, pl.m_pad)), 256, 0, st>>>(
        a.norm, grad, c1, s1, a.nc, a.c2, a.s2, a.nc2, a.d, a.eps1, a.eps2, sign2, ks.scale, center, tgt, pl.n_tpad,
        Op::NT_, Op::TSLOTS, src, pl.m_pad, Op::NS, Op::SSLOTS);
    return launch_single<Op>(pl, a.nc, P, part, st);
}

// Adapters giving OpApplyK / OpData a uniform plane description.
template <class Base, int TSLOTS_, int SSLOTS_, int NT>
struct DtOp : Base {
    static constexpr int NT_ = NT;
    static constexpr int TSLOTS = TSLOTS_;
    static constexpr int SSLOTS = SSLOTS_;
};

template <class Real, int KIND, int PDEG, int QDEG, int D>
int dt_impl(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    constexpr int PW = Traits<Real>::PER_WORD;
    constexpr int PP = PointPlanes<Real>::N;
    double* c1 = ws.take<double>((size_t)a.nc * a.d);
    double* s1 = ws.take<double>((size_t)a.nc * a.d);
    double* center = ws.take<double>(4);
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    const int nb = (int)std::min<long long>(1024, (a.nc + kDtThreads - 1) / kDtThreads);
    if (!ws.measuring()) {
        cell_geometry_kernel<<<grid_for(a.nc), 256, 0, st>>>(a.ncorner, a.v, a.nv, a.d, a.cells, a.nc, c1, s1);
        bbox_center_kernel<<<1, 256, 0, st>>>(c1, a.nc, a.c2, a.nc2, a.d, center);
    }
    if (a.energy != nullptr) {
        double* part = nullptr;
        SinglePlan pl{};
        double* epart = nullptr;
        int rc = LDDMM_OK;
        int nout = 1;
        if (a.norm == NVARIFOLD) {
            using Op = DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_VARI_VALUE>, 3, 4, PP + (3 + PW - 1) / PW>;
            rc = dt_sweep<Op, Real>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else if (a.norm == NCURRENT) {
            using Op = DtOp<OpApplyK<Real, KIND, PDEG, D, D>, 0, D, PP>;
            rc = dt_sweep<Op, Real>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else {
            using Op = DtOp<OpApplyK<Real, KIND, PDEG, D, 1>, 0, 1, PP>;
            rc = dt_sweep<Op, Real>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        }
        if (rc != LDDMM_OK) return rc;
        epart = ws.take<double>((size_t)nb);
        if (!ws.measuring()) {
            dt_value_combine_kernel<<<nb, kDtThreads, 0, st>>>(a.norm, part, a.nc, nout, pl.split, s1, a.d, a.eps1,
                                                               epart);
            dt_finalize_kernel<<<1, kDtThreads, 0, st>>>(epart, nb, 1.0, a.energy);
        }
    }
    if (a.px != nullptr) {
        double* part = nullptr;
        SinglePlan pl{};
        int rc = LDDMM_OK;
        int nout = 1;
        if (a.norm == NVARIFOLD) {
            using Op = DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_VARI_GRAD>, 3, 4, PP + (3 + PW - 1) / PW>;
            rc = dt_sweep<Op, Real>(a, ws, st, 1, -1.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else if (a.norm == NCURRENT) {
            using Op = DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_CUR_GRAD>, D, D, PP + (D + PW - 1) / PW>;
            rc = dt_sweep<Op, Real>(a, ws, st, 1, -1.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else {
            using Op = DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_MEAS_GRAD>, 0, 1, PP>;
            rc = dt_sweep<Op, Real>(a, ws, st, 1, -1.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        }
        if (rc != LDDMM_OK) return rc;
        double* z1 = ws.take<double>((size_t)a.nc * a.d);
        double* dz1 = ws.take<double>((size_t)a.nc * a.d);
        if (!ws.measuring()) {
            const double fac = a.ncorner == 3 ? 1.0 / 3.0 : 0.5;
            dt_grad_combine_kernel<<<grid_for(a.nc), 256, 0, st>>>(a.norm, part, a.nc, nout, pl.split, s1, a.d,
                                                                   a.eps1, fac * ks.dscale, z1, dz1);
            dt_gather_kernel<<<grid_for(a.nv), 256, 0, st>>>(a.ncorner, a.v, a.nv, a.d, a.cells, a.nc, a.vptr,
                                                             a.vidx, z1, dz1, a.px);
        }
    }
    if (ws.measuring()) return LDDMM_OK;
    return cuda_check(cudaGetLastError(), "dataterm");
}

template <class Real>
int dt_run(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    auto go = [&](auto kind, auto pdeg, auto qdeg) {
        return dispatch_d(a.d, [&](auto D) {
            return dt_impl<Real, decltype(kind)::value, decltype(pdeg)::value, decltype(qdeg)::value,
                           decltype(D)::value>(a, ws, st);
        });
    };
    switch (a.order) {
        case 0: return go(IC<KLAP>{}, IC<0>{}, IC<0>{});
        case 1: return go(IC<KLAP>{}, IC<1>{}, IC<0>{});
        case 2: return go(IC<KLAP>{}, IC<2>{}, IC<1>{});
        case 3: return go(IC<KLAP>{}, IC<3>{}, IC<2>{});
        case 4: return go(IC<KLAP>{}, IC<4>{}, IC<3>{});
        default: return go(IC<KGAUSS>{}, IC<0>{}, IC<0>{});
    }
}

static int dt_validate(const DataArgs& a) {
    if ((a.ncorner != 2 && a.ncorner != 3) || a.norm < 0 || a.norm > 2 || a.nv < 1 || a.nc < 1 || a.nc2 < 0 ||
        a.d < 2 || a.d > 3 || !(a.sigma > 0) || a.order < 0 || a.eps1 < 0 || a.eps2 < 0 ||
        a.nv > (1LL << 30) || a.nc > (1LL << 30) || a.nc2 > (1LL << 30)) {
        set_error("dataterm: invalid arguments, d must be 2 or 3 (cells of %d vertices, norm=%d nv=%lld nc=%lld nc2=%lld d=%d "
                  "sigma=%g order=%d)", a.ncorner, a.norm, a.nv, a.nc, a.nc2, a.d, a.sigma, a.order);
        return LDDMM_ERR_ARG;
    }
    if (a.ncorner == 3 && a.d != 3) {
        set_error("dataterm: surfaces need d = 3");
        return LDDMM_ERR_ARG;
    }
    if (a.norm == NVARIFOLD && a.ncorner != 3) {
        set_error("dataterm: the varifold norm is defined for surfaces only (as in the reference)");
        return LDDMM_ERR_UNSUPPORTED;
    }
    if (a.px != nullptr && a.order == 0) {
        set_error("dataterm: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    if (a.energy == nullptr && a.px == nullptr) {
        set_error("dataterm: nothing requested (energy and px are both NULL)");
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(a.v, "vertices"));
    LDDMM_TRY(check_device_ptr(a.cells, "cells"));
    if (a.nc2 > 0) {
        LDDMM_TRY(check_device_ptr(a.c2, "target centers"));
        LDDMM_TRY(check_device_ptr(a.s2, "target vectors"));
    }
    if (a.energy) LDDMM_TRY(check_device_ptr(a.energy, "energy"));
    if (a.px) {
        LDDMM_TRY(check_device_ptr(a.px, "px"));
        LDDMM_TRY(check_device_ptr(a.vptr, "vertex_ptr"));
        LDDMM_TRY(check_device_ptr(a.vidx, "vertex_idx"));
    }
    return LDDMM_OK;
}

template <class Real>
size_t dt_ws(int ncorner, int norm, int64_t nv, int d, int64_t nc, int64_t nc2, int order, int want_energy,
             int want_grad) {
    DataArgs a{};
    a.ncorner = ncorner;
    a.norm = norm;
    a.nv = nv;
    a.d = d;
    a.nc = nc;
    a.nc2 = nc2;
    a.sigma = 1.0;
    a.order = order;
    a.energy = want_energy ? reinterpret_cast<double*>(16) : nullptr;
    a.px = want_grad ? reinterpret_cast<double*>(16) : nullptr;
    if (ncorner != 2 && ncorner != 3) return 0;
    if (nv < 1 || nc < 1 || nc2 < 0 || d < 2 || d > 3 || norm < 0 || norm > 2) return 0;
    Workspace ws;
    if (dt_run<Real>(a, ws, 0) != LDDMM_OK) return 0;
    return ws.off + 256;
}

template <class Real>
int dt_entry(const DataArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(dt_validate(a));
    Workspace meas;
    LDDMM_TRY(dt_run<Real>(a, meas, st));
    if (wsp == nullptr || meas.off > wsb) {
        set_error("dataterm: workspace too small: need %zu bytes, got %zu", meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return dt_run<Real>(a, ws, st);
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_dataterm_f32c_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2, int order,
                                     int want_energy, int want_grad) {
    return dt_ws<float>(cell_size, norm, nv, d, nc, nc2, order, want_energy, want_grad);
}
size_t lddmm_dataterm_f64_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2, int order,
                                    int want_energy, int want_grad) {
    return dt_ws<double>(cell_size, norm, nv, d, nc, nc2, order, want_energy, want_grad);
}

#define DT_ARGS                                                                                                 \
    DataArgs a{cell_size, norm,  vertices, nv,  d,          cells,      nc,       tgt_centers, tgt_vectors, nc2, \
               sigma,     order, eps1,     eps2, energy,    vertex_ptr, vertex_idx, px}

int lddmm_dataterm_f32c(int cell_size, int norm, const double* vertices, int64_t nv, int d, const int64_t* cells,
                        int64_t nc, const double* tgt_centers, const double* tgt_vectors, int64_t nc2, double sigma,
                        int order, double eps1, double eps2, double* energy, const int64_t* vertex_ptr,
                        const int64_t* vertex_idx, double* px, void* workspace, size_t workspace_bytes,
                        lddmm_stream_t stream) {
    DT_ARGS;
    return dt_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_dataterm_f64(int cell_size, int norm, const double* vertices, int64_t nv, int d, const int64_t* cells,
                       int64_t nc, const double* tgt_centers, const double* tgt_vectors, int64_t nc2, double sigma,
                       int order, double eps1, double eps2, double* energy, const int64_t* vertex_ptr,
                       const int64_t* vertex_idx, double* px, void* workspace, size_t workspace_bytes,
                       lddmm_stream_t stream) {
    DT_ARGS;
    return dt_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
