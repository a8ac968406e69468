// Host-side planning, launching and template dispatch for sweep_kernel.
#pragma once
#include <cmath>
#include <type_traits>

#include "host.h"
#include "ops.cuh"
#include "sweep.cuh"

namespace lddmm {

template <int V>
using IC = std::integral_constant<int, V>;

// Nominal resident blocks of a sweep on the whole device (8 per SM for every
// operator, so plans and workspaces do not depend on register allocation).
template <class Op>
int sweep_slots() {
    return 8 * device_info().sms;
}

// Problems with at most this many targets use the SMALL tile shape of the
// packed operators that have one (more, smaller items: the large shape would
// leave most SMs idle).
#ifndef LDDMM_SMALL_TARGETS
#define LDDMM_SMALL_TARGETS 4096
#endif
constexpr long long kSmallTargets = LDDMM_SMALL_TARGETS;

struct SinglePlan {
    long long n_tpad, m_pad;
    int n_tb, n_src_tiles, split;
};

template <class Op>
SinglePlan plan_single(long long n, long long m, int split_cap = 0) {
    SinglePlan p;
    const long long per_block = (long long)Op::BLOCK * Op::R;
    p.n_tb = (int)((n + per_block - 1) / per_block);
    p.n_tpad = (long long)std::max(p.n_tb, 1) * per_block;
    p.n_src_tiles = (int)((m + Op::TILE - 1) / Op::TILE);
    p.m_pad = (long long)std::max(p.n_src_tiles, 1) * Op::TILE;
    p.split = choose_split(p.n_tb, p.n_src_tiles, sweep_slots<Op>());
    if (split_cap > 0 && p.split > split_cap) p.split = split_cap;
    return p;
}

// SYM: symmetric sweep over sym_tiles own source tiles (see sweep_kernel<Op, true>)
template <class Op, bool SYM = false>
int launch_single(const SinglePlan& pl, long long n, const typename Op::Params& P, double* part, cudaStream_t st,
                  int sym_tiles = 0) {
    SweepGrid g{};
    g.seg0.n_tgt = (int)n;
    g.seg0.n_src_tiles = pl.n_src_tiles;
    g.seg0.n_tb = pl.n_tb;
    g.seg0.split = pl.split;
    g.seg0.sym_tiles = sym_tiles;
    g.nseg = 0;
    g.n_items = pl.n_tb * pl.split;
    if (g.n_items <= 0) return LDDMM_OK;
    sweep_kernel<Op, SYM><<<g.n_items, Op::BLOCK, 0, st>>>(g, P, part);
    return cuda_check(cudaGetLastError(), "sweep launch");
}

// Kernel-dependent prescale of the coordinates, rescaled polynomials, and the
// constant of the derivative sums (see kfun.cuh).
struct KScale {
    double scale;   // coordinate multiplier used when packing
    double pk[5];   // K polynomial in the prescaled variable
    double pq[4];   // K' polynomial in the prescaled variable
    double dscale;  // sum_l K' 2 (x-y) <u,v> = dscale * sum_l F (x'-y') <u,v>
};

template <class Real>
KScale kernel_scale(int kind, int order, double sigma, bool exact_tables = false) {
    KScale k{};
    double P[5], Q[4], Rr[3];
    laplacian_tables(order, P, Q, Rr, exact_tables);
    const double L = 1.4426950408889634;  // log2(e)
    if (sizeof(Real) == 4) {
        k.scale = (kind == KGAUSS) ? std::sqrt(0.5 * L) / sigma : L / sigma;
        double Lj = 1.0;
        for (int j = 0; j < 5; ++j) {
            k.pk[j] = P[j] / Lj;
            if (j < 4) k.pq[j] = Q[j] / Lj;
            Lj *= L;
        }
    } else {
        k.scale = 1.0 / sigma;
        for (int j = 0; j < 5; ++j) k.pk[j] = P[j];
        for (int j = 0; j < 4; ++j) k.pq[j] = Q[j];
    }
    k.dscale = -1.0 / (sigma * sigma * k.scale);
    return k;
}

// order > 4: Gaussian; otherwise Laplacian with polynomial degree = order (K)
template <class F>
int dispatch_kind_p(int order, F&& f) {
    switch (order) {
        case 0: return f(IC<KLAP>{}, IC<0>{});
        case 1: return f(IC<KLAP>{}, IC<1>{});
        case 2: return f(IC<KLAP>{}, IC<2>{});
        case 3: return f(IC<KLAP>{}, IC<3>{});
        case 4: return f(IC<KLAP>{}, IC<4>{});
        default: return f(IC<KGAUSS>{}, IC<0>{});
    }
}

// derivative: polynomial degree = order - 1 (order 0 is rejected earlier)
template <class F>
int dispatch_kind_q(int order, F&& f) {
    switch (order) {
        case 1: return f(IC<KLAP>{}, IC<0>{});
        case 2: return f(IC<KLAP>{}, IC<1>{});
        case 3: return f(IC<KLAP>{}, IC<2>{});
        case 4: return f(IC<KLAP>{}, IC<3>{});
        default: return f(IC<KGAUSS>{}, IC<0>{});
    }
}

template <class F>
int dispatch_d(int d, F&& f) {
    if (d <= 2) return f(IC<2>{});
    return f(IC<3>{});
}

template <class F>
int dispatch_dimb(int b, F&& f) {
    switch (b) {
        case 1: return f(IC<1>{});
        case 2: return f(IC<2>{});
        case 3: return f(IC<3>{});
        default: return f(IC<4>{});
    }
}

// inner-product widths built: 1,2,3,4,6,8,9,12 (others padded with zeros)
template <class F>
int dispatch_w(int w, F&& f) {
    if (w <= 1) return f(IC<1>{});
    if (w <= 2) return f(IC<2>{});
    if (w <= 3) return f(IC<3>{});
    if (w <= 4) return f(IC<4>{});
    if (w <= 6) return f(IC<6>{});
    if (w <= 8) return f(IC<8>{});
    if (w <= 9) return f(IC<9>{});
    return f(IC<12>{});
}


}  // namespace lddmm
