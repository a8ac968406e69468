// Packed two-lane FP32 arithmetic (sm_100a `add/sub/mul/fma.rn.f32x2`).
//
// One instruction computes two independent FP32 operations, so a thread that
// evaluates two target-source pairs at once spends half the issue slots on the
// FP32 part of the pair math (the FMA pipe still executes 2 lanes of work per
// packed instruction).  A value `f2` is a 64-bit register pair (lo, hi).
#pragma once
#include "common.cuh"

namespace lddmm {

struct f2 {
    unsigned long long v;
};

LDDMM_D f2 pk2(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
    return r;
}
LDDMM_D void upk2(f2 a, float& lo, float& hi) { asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v)); }
LDDMM_D f2 add2(f2 a, f2 b) {
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
LDDMM_D f2 sub2(f2 a, f2 b) {
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
LDDMM_D f2 mul2(f2 a, f2 b) {
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
LDDMM_D f2 fma2(f2 a, f2 b, f2 c) {
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
LDDMM_D f2 splat2(float a) { return pk2(a, a); }

// 2^(-x) lane by lane on the MUFU
LDDMM_D f2 ex2neg2(f2 x) {
    float a, b;
    upk2(x, a, b);
    return pk2(ex2(-a), ex2(-b));
}
LDDMM_D f2 sqrt2(f2 x) {
    float a, b;
    upk2(x, a, b);
    return pk2(sqrt_approx(a), sqrt_approx(b));
}

// The two halves of a 16-byte word as packed pairs: (x, y) and (z, w).
LDDMM_D f2 word_lo(const float4& w) { return pk2(w.x, w.y); }
LDDMM_D f2 word_hi(const float4& w) { return pk2(w.z, w.w); }

// Packed accumulator for two targets: FP32 partials over FOLD sources folded
// into TwoSum-compensated (sum, error) pairs, lane by lane.
template <int N>
struct AccF32C2 {
    f2 p[N], s[N], e[N];
    LDDMM_D void zero() {
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] = e[c] = splat2(0.f);
    }
    LDDMM_D void begin_fold() {
#pragma unroll
        for (int c = 0; c < N; ++c) p[c] = splat2(0.f);
    }
    LDDMM_D void end_fold() {
#pragma unroll
        for (int c = 0; c < N; ++c) {
            const f2 t = add2(s[c], p[c]);
            const f2 bp = sub2(t, s[c]);
            const f2 err = add2(sub2(s[c], sub2(t, bp)), sub2(p[c], bp));
            s[c] = t;
            e[c] = add2(e[c], err);
        }
    }
    LDDMM_D void end_fold_w(float w) {
#pragma unroll
        for (int c = 0; c < N; ++c) p[c] = mul2(p[c], splat2(w));
        end_fold();
    }
    LDDMM_D void fma(int c, f2 a, f2 b) { p[c] = fma2(a, b, p[c]); }
    LDDMM_D double value(int c, int lane) const {
        float s0, s1, e0, e1;
        upk2(s[c], s0, s1);
        upk2(e[c], e0, e1);
        return lane == 0 ? (double)s0 + (double)e0 : (double)s1 + (double)e1;
    }
};

// Horner on packed lanes; c holds each coefficient duplicated as a pair.
template <int DEG>
LDDMM_D f2 horner2(const unsigned long long* c, f2 u) {
    f2 p{c[DEG]};
#pragma unroll
    for (int j = DEG - 1; j >= 0; --j) p = fma2(p, u, f2{c[j]});
    return p;
}

}  // namespace lddmm
