// Kernel functions K (value) and K' (first derivative factor) on prescaled
// coordinates, for the FP32 compensated path and the FP64 path.
//
// Reference: py-lddmm/kernelFunctions.f90 -- Gaussian (`ord > 4`):
//   K = exp(-u/2), K' = -exp(-u/2)/(2 s^2), u = |x-y|^2/s^2        (:33-40, :94-100)
// Laplacian of order p (0..4):
//   K = P_p(u) e^-u, K' = -Q_p(u) e^-u / (2 s^2), u = |x-y|/s          (:41-47, :101-107)
// with the polynomial tables c_ (P) and c1_ (Q).  Constant factors
// (-1/(2 s^2), the 2 of the gradient and the coordinate prescale) are applied
// once per target in the combine step, not per pair.
//
// FP32 prescaling (done when points are packed):
//   Gaussian:  x' = x * sqrt(log2(e)/2)/s  ->  K  = 2^(-|x'-y'|^2)
//   Laplacian: x' = x * log2(e)/s          ->  u' = |x'-y'| = log2(e) u,
//              e^-u = 2^(-u'), polynomials rewritten in u' (c_j / log2(e)^j).
// The Fortran zero-distance branch (K = 1 when u < 1e-8) is a no-op in FP32:
// 2^(-t) for 0 <= t < 1.5e-8 rounds to 1.0f, and so does P(u)e^-u.
//
// FP64: x' = x/s, u = |x'-y'|^2 (Gaussian) or |x'-y'| (Laplacian), exp() from
// the CUDA math library, and the zero-distance branch kept as in the Fortran.
#pragma once
#include "common.cuh"

namespace lddmm {

// Polynomial in Horner form, DEG is the polynomial degree (coefficients c[0..DEG]).
template <int DEG>
LDDMM_D float horner(const float* c, float u) {
    float p = c[DEG];
#pragma unroll
    for (int j = DEG - 1; j >= 0; --j) p = fmaf(p, u, c[j]);
    return p;
}

// FP32 kernel value from the prescaled squared distance.
template <int KIND, int PDEG>
LDDMM_D float kval32(const float* pk, float r2) {
    if constexpr (KIND == KGAUSS) {
        return ex2(-r2);
    } else {
        const float u = sqrt_approx(r2);
        const float e = ex2(-u);
        if constexpr (PDEG == 0) return e;
        else return horner<PDEG>(pk, u) * e;
    }
}

// FP32 derivative factor: returns F with K'(x,y) 2 (x-y) = scale * F * (x'-y').
template <int KIND, int QDEG>
LDDMM_D float kdiff32(const float* pq, float r2) {
    if constexpr (KIND == KGAUSS) {
        return ex2(-r2);
    } else {
        const float u = sqrt_approx(r2);
        const float e = ex2(-u);
        if constexpr (QDEG == 0) return pq[0] * e;
        else return horner<QDEG>(pq, u) * e;
    }
}

// FP64 monomial-sum polynomial, evaluated like the Fortran expression
// c0 + c1*u + c2*u**2 + ... (left-to-right).
template <int DEG>
LDDMM_D double poly64(const double* c, double u) {
    double s = c[0];
    double up = 1.0;
#pragma unroll
    for (int j = 1; j <= DEG; ++j) {
        up = up * u;
        s = s + c[j] * up;
    }
    return s;
}

template <int KIND, int PDEG>
LDDMM_D double kval64(const double* pk, double r2) {
    if constexpr (KIND == KGAUSS) {
        if (r2 < kZeroThresh) return 1.0;
        return exp(-0.5 * r2);
    } else {
        const double u = sqrt(r2);
        if (u < kZeroThresh) return 1.0;
        return poly64<PDEG>(pk, u) * exp(-1.0 * u);
    }
}

template <int KIND, int QDEG>
LDDMM_D double kdiff64(const double* pq, double r2) {
    if constexpr (KIND == KGAUSS) {
        if (r2 < kZeroThresh) return 1.0;
        return exp(-0.5 * r2);
    } else {
        const double u = sqrt(r2);
        if (u < kZeroThresh) return pq[0];
        return poly64<QDEG>(pq, u) * exp(-1.0 * u);
    }
}

}  // namespace lddmm
