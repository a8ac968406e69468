// Pair operators plugged into sweep_kernel (sweep.cuh).
//
//   OpApplyK<Real, KIND, DEG, D, DIMB>   f_k = sum_l K(x_k,y_l) beta_l
//       py-lddmm/kernelFunctions.f90:1-54 (applyk)
//   OpDiffKT<Real, KIND, DEG, D, W>      f_k = sum_l K'(x_k,y_l) 2(x_k-y_l) <u_k, v_l>
//       py-lddmm/kernelFunctions.f90:56-114 (applykdifft), with
//       u_k = a1[:,k,:], v_l = a2[:,l,:] flattened to W = na*dimb entries.
//
// Packed layouts (all planes are arrays of 16-byte words, one word per record):
//   FP32 points : plane 0 = (x', y', z', 0) float4
//   FP32 weights: plane 1.. = 4 floats per plane
//   FP64 points : planes 0,1 = (x', y') (z', 0) double2 words
//   FP64 weights: 2 doubles per plane
#pragma once
#include "kfun.cuh"
#include "sweep.cuh"

namespace lddmm {

template <class Real>
struct Traits;
template <>
struct Traits<float> {
    static constexpr int PER_WORD = 4;  // values per 16-byte word
};
template <>
struct Traits<double> {
    static constexpr int PER_WORD = 2;
};

template <class Real>
LDDMM_D Real word_get(const float4* w, int i) {
    if constexpr (sizeof(Real) == 4) {
        const float* f = reinterpret_cast<const float*>(w);
        return f[i];
    } else {
        const double* f = reinterpret_cast<const double*>(w);
        return f[i];
    }
}

// Reads `n` consecutive values starting at value index 0 of a record that is
// spread over planes: value i lives in plane (first_plane + i / PER_WORD).
template <class Real, int N>
LDDMM_D void load_vals(const float4* base, long long stride, long long row, int first_plane, Real* out) {
    constexpr int PW = Traits<Real>::PER_WORD;
#pragma unroll
    for (int w = 0; w < (N + PW - 1) / PW; ++w) {
        const float4 word = base[(long long)(first_plane + w) * stride + row];
#pragma unroll
        for (int i = 0; i < PW; ++i)
            if (w * PW + i < N) out[w * PW + i] = word_get<Real>(&word, i);
    }
}

// smem version: plane p of record j at S[p*TILE + j]
template <class Real, int N, int TILE>
LDDMM_D void load_vals_smem(const float4* S, int j, int first_plane, Real* out) {
    constexpr int PW = Traits<Real>::PER_WORD;
#pragma unroll
    for (int w = 0; w < (N + PW - 1) / PW; ++w) {
        const float4 word = S[(first_plane + w) * TILE + j];
#pragma unroll
        for (int i = 0; i < PW; ++i)
            if (w * PW + i < N) out[w * PW + i] = word_get<Real>(&word, i);
    }
}

template <class Real>
struct AccFor;
template <>
struct AccFor<float> {
    template <int N>
    using type = AccF32C<N>;
};
template <>
struct AccFor<double> {
    template <int N>
    using type = AccF64<N>;
};

template <class Real, int KIND, int DEG>
LDDMM_D Real kval(const Real* pk, Real r2) {
    if constexpr (sizeof(Real) == 4) return kval32<KIND, DEG>(pk, r2);
    else return kval64<KIND, DEG>(pk, r2);
}
template <class Real, int KIND, int DEG>
LDDMM_D Real kdiff(const Real* pq, Real r2) {
    if constexpr (sizeof(Real) == 4) return kdiff32<KIND, DEG>(pq, r2);
    else return kdiff64<KIND, DEG>(pq, r2);
}

template <class Real>
struct KernelParamsBase {
    const float4* src4;      // source planes
    long long src_stride;    // words per source plane
    const float4* tgt4;      // target planes
    long long tgt_stride;    // words per target plane
    Real pk[5];              // K polynomial (prescaled), Laplacian only
    Real pq[4];              // K' polynomial (prescaled), Laplacian only
};

// Point planes per record: FP32 one float4, FP64 two double2 words.
template <class Real>
struct PointPlanes {
    static constexpr int N = (sizeof(Real) == 4) ? 1 : 2;
};

// ---------------------------------------------------------------------------
// f_k = sum_l K(x_k, y_l) beta_l
// ---------------------------------------------------------------------------
// SMALL: 32-thread blocks and 32-record tiles for a few thousand targets or
// fewer (see OpApplyK2 in ops2.cuh)
template <class Real_, int KIND, int DEG, int D, int DIMB, bool SMALL = false>
struct OpApplyK {
    using Real = Real_;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = SMALL ? 32 : 128;
    static constexpr int R = (F32 && !SMALL) ? 4 : 2;
    static constexpr int TILE = SMALL ? 32 : 128;
    static constexpr int FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int WP = (DIMB + Traits<Real>::PER_WORD - 1) / Traits<Real>::PER_WORD;
    static constexpr int NS = PP + WP;
    static constexpr int NOUT = DIMB;
    using Params = KernelParamsBase<Real>;
    using Acc = typename AccFor<Real>::template type<DIMB>;
    struct Tgt {
        Real x[D];
    };
    struct Src {
        Real y[D];
        Real b[DIMB];
    };
    static LDDMM_D void load_target(const Params& P, long long row, Tgt& t) {
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, 0, t.x);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) {
        load_vals_smem<Real, D, TILE>(S, j, 0, s.y);
        load_vals_smem<Real, DIMB, TILE>(S, j, PP, s.b);
    }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        Real r2 = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const Real dj = t.x[j] - s.y[j];
            r2 = j == 0 ? dj * dj : r2 + dj * dj;
        }
        const Real k = kval<Real, KIND, DEG>(P.pk, r2);
#pragma unroll
        for (int c = 0; c < DIMB; ++c) a.fma(c, k, s.b[c]);
    }
};

// ---------------------------------------------------------------------------
// f_k = sum_l K'(x_k,y_l) 2 (x_k - y_l) <u_k, v_l>     (up to the combine scale)
// ---------------------------------------------------------------------------
template <class Real_, int KIND, int DEG, int D, int W, bool SMALL = false>
struct OpDiffKT {
    using Real = Real_;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = SMALL ? 32 : 128;
    static constexpr int R = 2;
    static constexpr int TILE = SMALL ? 32 : 128;
    static constexpr int FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int WP = (W + Traits<Real>::PER_WORD - 1) / Traits<Real>::PER_WORD;
    static constexpr int NS = PP + WP;
    static constexpr int NOUT = D;
    using Params = KernelParamsBase<Real>;
    using Acc = typename AccFor<Real>::template type<D>;
    struct Tgt {
        Real x[D];
        Real u[W];
    };
    struct Src {
        Real y[D];
        Real v[W];
    };
    static LDDMM_D void load_target(const Params& P, long long row, Tgt& t) {
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, 0, t.x);
        load_vals<Real, W>(P.tgt4, P.tgt_stride, row, PP, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) {
        load_vals_smem<Real, D, TILE>(S, j, 0, s.y);
        load_vals_smem<Real, W, TILE>(S, j, PP, s.v);
    }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        Real dx[D];
        Real r2 = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            dx[j] = t.x[j] - s.y[j];
            r2 = j == 0 ? dx[j] * dx[j] : r2 + dx[j] * dx[j];
        }
        Real dot = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) dot = w == 0 ? t.u[0] * s.v[0] : dot + t.u[w] * s.v[w];
        const Real g = kdiff<Real, KIND, DEG>(P.pq, r2) * dot;
#pragma unroll
        for (int j = 0; j < D; ++j) a.fma(j, g, dx[j]);
    }
};

// ---------------------------------------------------------------------------
// div_k = sum_l K'(x_k,y_l) 2 <x_k - y_l, a_l>      (up to the combine scale)
// py-lddmm/kernelFunctions.py:510-530 (applyDivergence)
// ---------------------------------------------------------------------------
template <class Real_, int KIND, int DEG, int D>
struct OpDivergence {
    using Real = Real_;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = 128;
    static constexpr int R = 4;
    static constexpr int TILE = 128;
    static constexpr int FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int WP = (D + Traits<Real>::PER_WORD - 1) / Traits<Real>::PER_WORD;
    static constexpr int NS = PP + WP;
    static constexpr int NOUT = 1;
    using Params = KernelParamsBase<Real>;
    using Acc = typename AccFor<Real>::template type<1>;
    struct Tgt {
        Real x[D];
    };
    struct Src {
        Real y[D];
        Real a[D];
    };
    static LDDMM_D void load_target(const Params& P, long long row, Tgt& t) {
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, 0, t.x);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) {
        load_vals_smem<Real, D, TILE>(S, j, 0, s.y);
        load_vals_smem<Real, D, TILE>(S, j, PP, s.a);
    }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& acc) {
        Real r2 = 0, dot = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const Real dj = t.x[j] - s.y[j];
            r2 = j == 0 ? dj * dj : r2 + dj * dj;
            dot = j == 0 ? dj * s.a[j] : dot + dj * s.a[j];
        }
        acc.fma(0, kdiff<Real, KIND, DEG>(P.pq, r2), dot);
    }
};

}  // namespace lddmm
