// Data-term operators and helper kernels shared by dataterms.cu (single
// problem) and ragged.cu (many requests per launch).  Formulas and reference
// lines: see dataterms.cu.
#pragma once
#include <type_traits>

#include "host.h"
#include "ops2.cuh"
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

template <class Real_, int KIND, int PDEG, int QDEG, int D, int MODE, bool SMALL = false>
struct OpData {
    using Real = Real_;
    using L = DataLayout<MODE, D>;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = SMALL ? 32 : 128, R = 2, TILE = SMALL ? 32 : 128, FOLD = F32 ? 32 : TILE;
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

// Packed-pair FP32 varifold VALUE operator (two targets per thread slot, see
// ops2.cuh): the per-pair arithmetic of OpData<float, ..., M_VARI_VALUE>
//   acc += K(c_k, c_l) (1 + <n_k, n_l>^2) w_l
// with sources stored as duplicated records [y0 y1 y2 n0 n1 n2 w] (4 words)
// and targets in the standard planes (pos word, normal word).  d = 3 only.
template <int KIND, int PDEG>
struct OpVariValue2 {
    using Real = float;
    static constexpr bool F32 = true;
    static constexpr bool DUP = true;
    static constexpr int TPS = 2;
    static constexpr int BLOCK = 128, R = 4, TILE = 128, FOLD = 32;
    static constexpr int PP = 1;
    static constexpr int NV = 7;
    static constexpr int NS = (NV + 1) / 2;
    static constexpr int NOUT = 1;
    using Params = KernelParams2;
    using Acc = AccF32C2<1>;
    struct Tgt {
        f2 x[3];
        f2 u[3];
    };
    struct Src {
        f2 val[NV];
    };
    static LDDMM_D void load_target(const Params& P, long long ra, long long rb, Tgt& t) {
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 0, t.x);
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 1, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) { load_dup_source<NV, TILE>(S, j, s.val); }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        f2 r2;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const f2 dj = sub2(t.x[j], s.val[j]);
            r2 = j == 0 ? mul2(dj, dj) : fma2(dj, dj, r2);
        }
        const f2 k = kval2<KIND, PDEG>(P.pkd, r2);
        const f2 dn = fma2(t.u[2], s.val[5], fma2(t.u[1], s.val[4], mul2(t.u[0], s.val[3])));
        const f2 q = fma2(dn, dn, splat2(1.f));
        a.fma(0, mul2(k, s.val[6]), q);
    }
};

// Packed-pair FP32 varifold GRADIENT operator: the arithmetic of
// OpData<float, ..., M_VARI_GRAD> for two target cells per slot (sources as in
// OpVariValue2, weights carrying the -1 of the target shape):
//   acc[0..3) += 2 <n_k,n_l> K w_l n_l,  acc[3] += K w_l (1 - <n_k,n_l>^2),
//   acc[4..7) += K' w_l (1 + <n_k,n_l>^2) (c_k - c_l)'
// 21 packed instructions per slot and source (Gaussian): acc[0..3) is summed
// without its factor 2 (restored exactly by out_scale when written), and
// 1 - <n,n'>^2 is formed as 2 - (1 + <n,n'>^2) from the factor the K' part needs.
// Two packed slots per thread (R = 4): each 4-word source record read from
// shared memory serves four target cells (11.6% faster than one slot at
// F = 100k, 200k sources).
template <int KIND, int PDEG, int QDEG>
struct OpVariGrad2 {
    using Real = float;
    static constexpr bool F32 = true;
    static constexpr bool DUP = true;
    static constexpr int TPS = 2;
    static constexpr int BLOCK = 128, R = 4, TILE = 128, FOLD = 32;
    static constexpr int PP = 1;
    static constexpr int NV = 7;
    static constexpr int NS = (NV + 1) / 2;
    static constexpr int NOUT = 7;
    using Params = KernelParams2;
    using Acc = AccF32C2<NOUT>;
    struct Tgt {
        f2 x[3];
        f2 u[3];
    };
    struct Src {
        f2 val[NV];
    };
    static LDDMM_D void load_target(const Params& P, long long ra, long long rb, Tgt& t) {
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 0, t.x);
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 1, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) { load_dup_source<NV, TILE>(S, j, s.val); }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        f2 dx[3], r2;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            dx[j] = sub2(t.x[j], s.val[j]);
            r2 = j == 0 ? mul2(dx[j], dx[j]) : fma2(dx[j], dx[j], r2);
        }
        f2 k, f;
        if constexpr (KIND == KGAUSS) {
            k = kval2<KIND, PDEG>(P.pkd, r2);
            f = k;
        } else {
            const f2 u = sqrt2(r2);
            const f2 e = ex2neg2(u);
            k = PDEG == 0 ? e : mul2(horner2<PDEG>(P.pkd, u), e);
            f = QDEG == 0 ? mul2(f2{P.pqd[0]}, e) : mul2(horner2<QDEG>(P.pqd, u), e);
        }
        const f2 dn = fma2(t.u[2], s.val[5], fma2(t.u[1], s.val[4], mul2(t.u[0], s.val[3])));
        const f2 wk = mul2(k, s.val[6]);
        const f2 ca = mul2(dn, wk);                       // half of 2 <n,n'> K w
#pragma unroll
        for (int j = 0; j < 3; ++j) a.fma(j, ca, s.val[3 + j]);
        const f2 q1 = fma2(dn, dn, splat2(1.f));          // 1 + <n,n'>^2
        a.fma(3, wk, sub2(splat2(2.f), q1));              // 1 - <n,n'>^2
        const f2 wf = mul2(KIND == KGAUSS ? wk : mul2(f, s.val[6]), q1);
#pragma unroll
        for (int j = 0; j < 3; ++j) a.fma(4 + j, wf, dx[j]);
    }
    static LDDMM_D double out_scale(int c) { return c < 3 ? 2.0 : 1.0; }
};

// Packed-pair FP32 current GRADIENT operator (OpData<float, ..., M_CUR_GRAD>,
// d = 3): sources [y0 y1 y2 s0 s1 s2] duplicated, targets (pos, s_k):
//   acc[0..3) += K s_l,  acc[3..6) += K' <s_k, s_l> (c_k - c_l)'
template <int KIND, int PDEG, int QDEG>
struct OpCurGrad2 {
    using Real = float;
    static constexpr bool F32 = true;
    static constexpr bool DUP = true;
    static constexpr int TPS = 2;
    static constexpr int BLOCK = 128, R = 2, TILE = 128, FOLD = 32;
    static constexpr int PP = 1;
    static constexpr int NV = 6;
    static constexpr int NS = (NV + 1) / 2;
    static constexpr int NOUT = 6;
    using Params = KernelParams2;
    using Acc = AccF32C2<NOUT>;
    struct Tgt {
        f2 x[3];
        f2 u[3];
    };
    struct Src {
        f2 val[NV];
    };
    static LDDMM_D void load_target(const Params& P, long long ra, long long rb, Tgt& t) {
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 0, t.x);
        load_target_pair<3>(P.tgt4, P.tgt_stride, ra, rb, 1, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) { load_dup_source<NV, TILE>(S, j, s.val); }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        f2 dx[3], r2;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            dx[j] = sub2(t.x[j], s.val[j]);
            r2 = j == 0 ? mul2(dx[j], dx[j]) : fma2(dx[j], dx[j], r2);
        }
        f2 k, f;
        if constexpr (KIND == KGAUSS) {
            k = kval2<KIND, PDEG>(P.pkd, r2);
            f = k;
        } else {
            const f2 u = sqrt2(r2);
            const f2 e = ex2neg2(u);
            k = PDEG == 0 ? e : mul2(horner2<PDEG>(P.pkd, u), e);
            f = QDEG == 0 ? mul2(f2{P.pqd[0]}, e) : mul2(horner2<QDEG>(P.pqd, u), e);
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) a.fma(j, k, s.val[3 + j]);
        const f2 dot = fma2(t.u[2], s.val[5], fma2(t.u[1], s.val[4], mul2(t.u[0], s.val[3])));
        const f2 g = mul2(f, dot);
#pragma unroll
        for (int j = 0; j < 3; ++j) a.fma(3 + j, g, dx[j]);
    }
};

// Operators with duplicated source records (DUP) take duplicated polynomial
// coefficients and a duplicated source layout from the pack.
template <class Op, class = void>
struct op_dup : std::false_type {};
template <class Op>
struct op_dup<Op, std::void_t<decltype(Op::DUP)>> : std::bool_constant<Op::DUP> {};

template <class Op, class Real>
inline void set_data_poly(typename Op::Params& P, const KScale& ks) {
    if constexpr (op_dup<Op>::value) {
        for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks.pk[j]);
        for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks.pq[j]);
    } else {
        for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
        for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
    }
}

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

// One packed record of a data-term sweep (row i of `planes`, stride words per
// plane): the prescaled centre, then the values of the norm:
//   norm current : target -, source s*sign              (value, OpApplyK DIMB = d)
//                  target s, source s*sign              (gradient)
//   norm measure : target -, source a*sign              (value and gradient)
//   norm varifold: target n, source (n, a*sign)         (value and gradient)
// c == nullptr writes a zero (padding) record of nplanes planes.
template <class Real>
LDDMM_D void dt_pack_record(int norm, int grad, bool is_t, const double* c, const double* s, int d, double eps,
                            double sign, double scale, const double* center, float4* planes, long long stride,
                            long long i, int nplanes, int slots, bool dup = false) {
    constexpr int PP = PointPlanes<Real>::N;
    if (c == nullptr) {
        for (int p = 0; p < nplanes; ++p) planes[(long long)p * stride + i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const double a = vec_norm_eps(s, d, eps);
    double pos[4] = {0, 0, 0, 0};
    for (int j = 0; j < d; ++j) pos[j] = (c[j] - center[j]) * scale;
    if (sizeof(Real) == 4 && dup) {
        // duplicated source record [pos0 pos1 pos2 vals...], two values per word (see ops2.cuh)
        double vals[4] = {0, 0, 0, 0};
        if (norm == NVARIFOLD) {
            for (int j = 0; j < 3; ++j) vals[j] = s[j] / a;
            vals[3] = a * sign;
        } else if (norm == NCURRENT) {
            for (int j = 0; j < d; ++j) vals[j] = s[j] * sign;
        } else {
            vals[0] = a * sign;
        }
        float q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < 3; ++j) q[j] = (float)pos[j];
        for (int j = 0; j < slots && j < 4; ++j) q[3 + j] = (float)vals[j];
        for (int w = 0; w < nplanes; ++w)
            planes[(long long)w * stride + i] = make_float4(q[2 * w], q[2 * w], q[2 * w + 1], q[2 * w + 1]);
        return;
    }
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
    constexpr int PWv = Traits<Real>::PER_WORD;
    for (int w = 0; w < (slots + PWv - 1) / PWv; ++w) {
        Real q[PWv];
        for (int j = 0; j < PWv; ++j) q[j] = (w * PWv + j < nv) ? (Real)vals[w * PWv + j] : (Real)0;
        float4* dst = planes + (long long)(PP + w) * stride + i;
        if constexpr (sizeof(Real) == 4) *dst = make_float4(q[0], q[1], q[2], q[3]);
        else *reinterpret_cast<double2*>(dst) = make_double2(q[0], q[1]);
    }
}

// Targets: set-1 cells.  Sources: set-1 cells (sign +1) then set-2 cells (sign2).
template <class Real>
static __global__ void dt_pack_kernel(int norm, int grad, const double* __restrict__ c1, const double* __restrict__ s1,
                                      long long n1, const double* __restrict__ c2, const double* __restrict__ s2,
                                      long long n2, int d, double eps1, double eps2, double sign2, double scale,
                                      const double* __restrict__ center, float4* tgt, long long tstride, int tplanes,
                                      int tslots, float4* src, long long sstride, int splanes, int sslots,
                                      int dup = 0, long long n1s = -1) {
    // set-2 sources start at row n1s (n1 rounded up to a tile for symmetric sweeps)
    if (n1s < 0) n1s = n1;
    const long long npad = tstride > sstride ? tstride : sstride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < tstride)
            dt_pack_record<Real>(norm, grad, true, i < n1 ? c1 + i * d : nullptr, i < n1 ? s1 + i * d : nullptr, d,
                                 eps1, 1.0, scale, center, tgt, tstride, i, tplanes, tslots);
        if (i < sstride) {
            const bool first = i < n1, second = i >= n1s && i < n1s + n2;
            const double* c = first ? c1 + i * d : (second ? c2 + (i - n1s) * d : nullptr);
            const double* sv = first ? s1 + i * d : (second ? s2 + (i - n1s) * d : nullptr);
            dt_pack_record<Real>(norm, grad, false, c, sv, d, first ? eps1 : eps2, first ? 1.0 : sign2, scale, center,
                                 src, sstride, i, splanes, sslots, dup != 0);
        }
    }
}

// per-cell z1, dz1 of row i from the chunk sums (see dt_grad_combine_kernel)
LDDMM_D void dt_grad_row(int norm, const double* acc, const double* s, int d, double eps1, double dzscale, double* z1,
                         double* dz1) {
    if (norm == NCURRENT) {
        for (int j = 0; j < d; ++j) {
            z1[j] = acc[j];
            dz1[j] = dzscale * acc[d + j];
        }
    } else if (norm == NMEASURE) {
        const double a = vec_norm_eps(s, d, eps1);
        for (int j = 0; j < d; ++j) {
            z1[j] = acc[0] * (s[j] / a);
            dz1[j] = dzscale * a * acc[1 + j];
        }
    } else {
        const double a = vec_norm_eps(s, d, eps1);
        for (int j = 0; j < d; ++j) {
            z1[j] = acc[j] + acc[d] * (s[j] / a);
            dz1[j] = dzscale * a * acc[d + 1 + j];
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
        dt_grad_row(norm, acc, s1 + i * d, d, eps1, dzscale, z1 + i * d, dz1 + i * d);
    }
}

// px[q] = 2 sum over the (cell, corner) entries of vertex q of the corner contribution.
// L2ONLY: z1 / dz1 were written by other CTAs of the same launch (loads bypass L1).
template <bool L2ONLY = false>
LDDMM_D void dt_gather_vertex(long long q, int ncorner, const double* __restrict__ v, long long nv, int d,
                              const int64_t* __restrict__ cells, long long nc, const int64_t* __restrict__ vptr,
                              const int64_t* __restrict__ vidx, const double* z1, const double* dz1,
                              double* __restrict__ px) {
    double acc[3] = {0, 0, 0};
    const long long b = vptr[q], e = vptr[q + 1];
    for (long long k = b; k < e; ++k) {
        const long long code = vidx[k];
        if (code < 0 || code >= nc * ncorner) continue;
        const long long f = code / ncorner;
        const int corner = (int)(code - f * ncorner);
        double z[3] = {0, 0, 0}, dz[3] = {0, 0, 0};
        for (int j = 0; j < d; ++j) {
            z[j] = L2ONLY ? __ldcg(z1 + f * d + j) : z1[f * d + j];
            dz[j] = L2ONLY ? __ldcg(dz1 + f * d + j) : dz1[f * d + j];
        }
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

static __global__ void dt_gather_kernel(int ncorner, const double* __restrict__ v, long long nv, int d,
                                        const int64_t* __restrict__ cells, long long nc,
                                        const int64_t* __restrict__ vptr, const int64_t* __restrict__ vidx,
                                        const double* __restrict__ z1, const double* __restrict__ dz1,
                                        double* __restrict__ px) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
         q += (long long)gridDim.x * blockDim.x)
        dt_gather_vertex(q, ncorner, v, nv, d, cells, nc, vptr, vidx, z1, dz1, px);
}


}  // namespace lddmm
