// Packed-pair (two targets per thread slot) FP32 operators for sweep_kernel.
//
//   OpApplyK2<KIND, DEG, D, DIMB>  f_k = sum_l K(x_k,y_l) beta_l        (kernelFunctions.f90:1-54)
//   OpDiffKT2<KIND, DEG, D, W>     f_k = sum_l K'(x_k,y_l) 2(x_k-y_l) <u_k,v_l>  (kernelFunctions.f90:56-114)
//
// Same arithmetic as OpApplyK / OpDiffKT<float> (ops.cuh), evaluated for two
// targets at once with `f32x2` instructions.  Layouts:
//   targets : the standard planes (pos word, then values 4 per word);
//   sources : "duplicated" records, the value list [y_0..y_{D-1}, v_0..v_{V-1}]
//             with every value stored twice, two values per 16-byte word
//             (v_a, v_a, v_b, v_b), so one shared-memory load yields two packed
//             operands ready for the f32x2 instructions.
#pragma once
#include <cstring>

#include "f32x2.cuh"
#include "ops.cuh"
#include "pack.cuh"

namespace lddmm {

struct KernelParams2 {
    const float4* src4;
    long long src_stride;
    const float4* tgt4;
    long long tgt_stride;
    unsigned long long pkd[5];  // K polynomial, each coefficient duplicated as an f32x2 pair
    unsigned long long pqd[4];  // K' polynomial, duplicated
};

// Source records with duplicated values: NV values -> (NV + 1) / 2 words.
template <int NV, int TILE>
LDDMM_D void load_dup_source(const float4* S, int j, f2* val) {
#pragma unroll
    for (int w = 0; w < (NV + 1) / 2; ++w) {
        const float4 word = S[w * TILE + j];
        val[2 * w] = word_lo(word);
        if (2 * w + 1 < NV) val[2 * w + 1] = word_hi(word);
    }
}

// Two target rows (standard planes), N values from first_plane, packed lane-wise.
template <int N>
LDDMM_D void load_target_pair(const float4* base, long long stride, long long ra, long long rb, int first_plane,
                              f2* out) {
#pragma unroll
    for (int w = 0; w < (N + 3) / 4; ++w) {
        const float4 a = base[(long long)(first_plane + w) * stride + ra];
        const float4 b = base[(long long)(first_plane + w) * stride + rb];
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (w * 4 + i < N) out[w * 4 + i] = pk2(av[i], bv[i]);
    }
}

template <int KIND, int DEG>
LDDMM_D f2 kval2(const unsigned long long* pkd, f2 r2) {
    if constexpr (KIND == KGAUSS) {
        return ex2neg2(r2);
    } else {
        const f2 u = sqrt2(r2);
        const f2 e = ex2neg2(u);
        if constexpr (DEG == 0) return e;
        else return mul2(horner2<DEG>(pkd, u), e);
    }
}

template <int KIND, int QDEG>
LDDMM_D f2 kdiff2(const unsigned long long* pqd, f2 r2) {
    if constexpr (KIND == KGAUSS) {
        return ex2neg2(r2);
    } else {
        const f2 u = sqrt2(r2);
        const f2 e = ex2neg2(u);
        if constexpr (QDEG == 0) return mul2(f2{pqd[0]}, e);
        else return mul2(horner2<QDEG>(pqd, u), e);
    }
}

// SMALL: tile shape for a few thousand targets or fewer (64 targets per
// 32-thread block, 32-source tiles), so that the (target block, source chunk)
// items spread over the SMs instead of filling one or two 512-target blocks.
template <int KIND, int DEG, int D, int DIMB, bool SMALL = false>
struct OpApplyK2 {
    using Real = float;
    static constexpr bool F32 = true;
    static constexpr bool DUP = true;
    static constexpr int TPS = 2;
    static constexpr int BLOCK = SMALL ? 32 : 128, R = SMALL ? 2 : 4, TILE = SMALL ? 32 : 128, FOLD = 32;
    static constexpr int PP = 1;            // target planes: pos
    static constexpr int NV = D + DIMB;     // source values
    static constexpr int NS = (NV + 1) / 2; // source words (duplicated values)
    static constexpr int NOUT = DIMB;
    using Params = KernelParams2;
    using Acc = AccF32C2<DIMB>;
    struct Tgt {
        f2 x[D];
    };
    struct Src {
        f2 val[NV];
    };
    static LDDMM_D void load_target(const Params& P, long long ra, long long rb, Tgt& t) {
        load_target_pair<D>(P.tgt4, P.tgt_stride, ra, rb, 0, t.x);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) { load_dup_source<NV, TILE>(S, j, s.val); }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        f2 r2;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const f2 dj = sub2(t.x[j], s.val[j]);
            r2 = j == 0 ? mul2(dj, dj) : fma2(dj, dj, r2);
        }
        const f2 k = kval2<KIND, DEG>(P.pkd, r2);
#pragma unroll
        for (int c = 0; c < DIMB; ++c) a.fma(c, k, s.val[D + c]);
    }
};

template <int KIND, int DEG, int D, int W, bool SMALL = false>
struct OpDiffKT2 {
    using Real = float;
    static constexpr bool F32 = true;
    static constexpr bool DUP = true;
    static constexpr int TPS = 2;
    static constexpr int BLOCK = SMALL ? 32 : 128, R = SMALL ? 2 : 4, TILE = SMALL ? 32 : 128, FOLD = 32;
    static constexpr int PP = 1;
    static constexpr int NV = D + W;
    static constexpr int NS = (NV + 1) / 2;
    static constexpr int NT = 1 + (W + 3) / 4;  // target planes: pos, u values
    static constexpr int NOUT = D;
    using Params = KernelParams2;
    using Acc = AccF32C2<D>;
    struct Tgt {
        f2 x[D];
        f2 u[W];
    };
    struct Src {
        f2 val[NV];
    };
    static LDDMM_D void load_target(const Params& P, long long ra, long long rb, Tgt& t) {
        load_target_pair<D>(P.tgt4, P.tgt_stride, ra, rb, 0, t.x);
        load_target_pair<W>(P.tgt4, P.tgt_stride, ra, rb, 1, t.u);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) { load_dup_source<NV, TILE>(S, j, s.val); }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& a) {
        f2 dx[D], r2;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            dx[j] = sub2(t.x[j], s.val[j]);
            r2 = j == 0 ? mul2(dx[j], dx[j]) : fma2(dx[j], dx[j], r2);
        }
        f2 dot = mul2(t.u[0], s.val[D]);
#pragma unroll
        for (int w = 1; w < W; ++w) dot = fma2(t.u[w], s.val[D + w], dot);
        const f2 g = mul2(kdiff2<KIND, DEG>(P.pqd, r2), dot);
#pragma unroll
        for (int j = 0; j < D; ++j) a.fma(j, g, dx[j]);
    }
};

// Host: duplicated polynomial coefficients for KernelParams2.
inline unsigned long long dup_coeff(double c) {
    const float f = (float)c;
    unsigned int u;
    memcpy(&u, &f, 4);
    return ((unsigned long long)u << 32) | (unsigned long long)u;
}

// Packs sources into duplicated records: values [ (x_i - c) * s (D of them, zero
// beyond d), gather values (V of them, zero beyond g.nvals) ], rows >= n zero.
static __global__ void pack_dup_kernel(const double* __restrict__ x, long long n, int d, double scale,
                                       const double* __restrict__ center, const Gather g, int D, int V,
                                       float4* __restrict__ out, long long stride, long long n_pad) {
    const int nv = D + V;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_pad;
         i += (long long)gridDim.x * blockDim.x) {
        float v[16];
        for (int q = 0; q < nv && q < 16; ++q) v[q] = 0.f;
        if (i < n) {
            for (int j = 0; j < d && j < D; ++j) v[j] = (float)((x[i * d + j] - (center ? center[j] : 0.0)) * scale);
            for (int q = 0; q < V && q < g.nvals; ++q) v[D + q] = (float)(g.src[i * g.row_stride + g.off[q]] * g.mult);
        }
        for (int w = 0; w < (nv + 1) / 2; ++w) {
            const float a = v[2 * w], b = (2 * w + 1 < nv) ? v[2 * w + 1] : 0.f;
            out[(long long)w * stride + i] = make_float4(a, a, b, b);
        }
    }
}

}  // namespace lddmm
