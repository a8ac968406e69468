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
#include <type_traits>

#include "dataterm_fused.cuh"
#include "dataterm_ops.cuh"
#include "host.h"
#include "pack.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

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
    // batched values: vertex sets v + b vstride (b < nbatch) into energy[b]
    int nbatch = 1;
    long long vstride = 0;
};

// SYM (values): the cell-cell self part is evaluated once per unordered pair
// (sweep_kernel<Op, true>); the target cells then start at a tile boundary.
template <class Op, class Real, bool SYM = false>
int dt_sweep(const DataArgs& a, Workspace& ws, cudaStream_t st, int grad, double sign2, const double* c1,
             const double* s1, double*& part, SinglePlan& pl, const KScale& ks, const double* center) {
    const long long n1s = SYM ? (a.nc + Op::TILE - 1) / Op::TILE * Op::TILE : a.nc;
    pl = plan_single<Op>(a.nc, n1s + a.nc2);
    float4* tgt = ws.take<float4>((size_t)Op::NT_ * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    part = ws.take<double>((size_t)pl.split * a.nc * Op::NOUT);
    if (ws.measuring()) return LDDMM_OK;
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    set_data_poly<Op, Real>(P, ks);
    dt_pack_kernel<Real><<<grid_for(std::max(pl.n_tpad, pl.m_pad)), 256, 0, st>>>(
        a.norm, grad, c1, s1, a.nc, a.c2, a.s2, a.nc2, a.d, a.eps1, a.eps2, sign2, ks.scale, center, tgt, pl.n_tpad,
        Op::NT_, Op::TSLOTS, src, pl.m_pad, Op::NS, Op::SSLOTS, op_dup<Op>::value ? 1 : 0, n1s);
    return launch_single<Op, SYM>(pl, a.nc, P, part, st, (int)(n1s / Op::TILE));
}

// Adapters giving OpApplyK / OpData a uniform plane description.
template <class Base, int TSLOTS_, int SSLOTS_, int NT>
struct DtOp : Base {
    static constexpr int NT_ = NT;
    static constexpr int TSLOTS = TSLOTS_;
    static constexpr int SSLOTS = SSLOTS_;
};

// SMALL: the small tile shape for the unpacked operators (few target cells);
// the packed FP32 surface operators keep their shape.
template <class Real, int KIND, int PDEG, int QDEG, int D, bool SMALL = false>
int dt_impl(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    constexpr int PW = Traits<Real>::PER_WORD;
    constexpr int PP = PointPlanes<Real>::N;
    double* c1 = ws.take<double>((size_t)a.nc * a.d);
    double* s1 = ws.take<double>((size_t)a.nc * a.d);
    double* center = ws.take<double>(kCenterWords);
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    const int nb = (int)std::min<long long>(1024, (a.nc + kDtThreads - 1) / kDtThreads);
    if (!ws.measuring()) {
        cell_geometry_kernel<<<grid_for(a.nc), 256, 0, st>>>(a.ncorner, a.v, a.nv, a.d, a.cells, a.nc, c1, s1);
        launch_bbox_center(c1, a.nc, a.c2, a.nc2, a.d, center, st);
    }
    if (a.energy != nullptr) {
        double* part = nullptr;
        SinglePlan pl{};
        double* epart = nullptr;
        int rc = LDDMM_OK;
        int nout = 1;
        if (a.norm == NVARIFOLD) {
            // FP32: packed-pair operator (two targets per slot, duplicated sources)
            using Op = std::conditional_t<(sizeof(Real) == 4 && D == 3), DtOp<OpVariValue2<KIND, PDEG>, 3, 4, 2>,
                                          DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_VARI_VALUE, SMALL>, 3, 4,
                                               PP + (3 + PW - 1) / PW>>;
            rc = dt_sweep<Op, Real, true>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else if (a.norm == NCURRENT) {
            using Op = DtOp<OpApplyK<Real, KIND, PDEG, D, D, SMALL>, 0, D, PP>;
            rc = dt_sweep<Op, Real, true>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else {
            using Op = DtOp<OpApplyK<Real, KIND, PDEG, D, 1, SMALL>, 0, 1, PP>;
            rc = dt_sweep<Op, Real, true>(a, ws, st, 0, -2.0, c1, s1, part, pl, ks, center);
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
        constexpr bool PACK = sizeof(Real) == 4 && D == 3;   // FP32 surfaces: packed-pair operators
        if (a.norm == NVARIFOLD) {
            using Op = std::conditional_t<PACK, DtOp<OpVariGrad2<KIND, PDEG, QDEG>, 3, 4, 2>,
                                          DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_VARI_GRAD, SMALL>, 3, 4,
                                               PP + (3 + PW - 1) / PW>>;
            rc = dt_sweep<Op, Real>(a, ws, st, 1, -1.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else if (a.norm == NCURRENT) {
            using Op = std::conditional_t<PACK, DtOp<OpCurGrad2<KIND, PDEG, QDEG>, D, D, 2>,
                                          DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_CUR_GRAD, SMALL>, D, D,
                                               PP + (D + PW - 1) / PW>>;
            rc = dt_sweep<Op, Real>(a, ws, st, 1, -1.0, c1, s1, part, pl, ks, center);
            nout = Op::NOUT;
        } else {
            using Op = DtOp<OpData<Real, KIND, PDEG, QDEG, D, M_MEAS_GRAD, SMALL>, 0, 1, PP>;
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

// Values alone of small shapes (dataterm_fused.cuh limits): one cluster launch.
template <class Real, int KIND, int PDEG, int D>
int dt_value_fused(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    const FusedShape fs = fused_shape(a.nc);
    double* epart = ws.take<double>((size_t)kFusedMaxCluster * a.nbatch);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    FusedCoef cf{};
    for (int j = 0; j < 5; ++j) cf.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) cf.pq[j] = ks.pq[j];
    const long long total = a.nc + a.nc2;
    return launch_fused(dt_value_fused_kernel<Real, KIND, PDEG, D>, fs, a.nbatch, dt_fused_smem<Real>(total),
                        dt_fused_smem<Real>(DtTile<Real>::N), st, a.ncorner, a.norm, a.v, (long long)a.nv, a.cells,
                        (long long)a.nc, a.c2, a.s2, (long long)a.nc2, a.eps1, a.eps2, ks.scale, cf, fs, epart,
                        a.energy, a.vstride, dt_fused_tile<Real>(total));
}

// Gradient (and value, if asked) of small shapes: one cluster launch each (dataterm_fused.cuh).
template <class Real, int KIND, int PDEG, int QDEG, int D>
int dt_grad_fused(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    if (a.energy != nullptr) LDDMM_TRY((dt_value_fused<Real, KIND, PDEG, D>(a, ws, st)));
    const FusedShape fs = fused_shape(a.nc);
    double* z1 = ws.take<double>((size_t)a.nc * a.d);
    double* dz1 = ws.take<double>((size_t)a.nc * a.d);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    FusedCoef cf{};
    for (int j = 0; j < 5; ++j) cf.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) cf.pq[j] = ks.pq[j];
    const double fac = a.ncorner == 3 ? 1.0 / 3.0 : 0.5;
    const int tile = dt_fused_tile<Real>(a.nc + a.nc2);
    return launch_fused(dt_grad_fused_kernel<Real, KIND, PDEG, QDEG, D>, fs, 1, dt_grad_fused_smem<Real>(tile),
                        dt_grad_fused_smem<Real>(DtTile<Real>::N), st, a.ncorner, a.norm, a.v, (long long)a.nv,
                        a.cells, (long long)a.nc, a.c2, a.s2, (long long)a.nc2, a.eps1, a.eps2, ks.scale,
                        fac * ks.dscale, cf, fs, tile, a.vptr, a.vidx, z1, dz1, a.px);
}

int dt_value_resident_clusters(long long nc, long long nc2, int d, int fp64) {
    const FusedShape fs = fused_shape(nc);
    auto go = [&](auto D) {
        constexpr int D_ = decltype(D)::value;
        return fp64 ? fused_resident_clusters(dt_value_fused_kernel<double, KGAUSS, 0, D_>, fs,
                                              dt_fused_smem<double>(nc + nc2), dt_fused_smem<double>(DtTile<double>::N))
                    : fused_resident_clusters(dt_value_fused_kernel<float, KGAUSS, 0, D_>, fs,
                                              dt_fused_smem<float>(nc + nc2), dt_fused_smem<float>(DtTile<float>::N));
    };
    return d == 2 ? go(IC<2>{}) : go(IC<3>{});
}

template <class Real>
int dt_run(const DataArgs& a, Workspace& ws, cudaStream_t st) {
    const bool fused = a.px == nullptr && a.energy != nullptr && dt_fused_fits(a.nc, a.nc2);
    if (a.nbatch > 1 && !fused) {
        // general path: the vertex sets one after the other, each on the same workspace
        const size_t off0 = ws.off;
        size_t top = off0;
        for (int b = 0; b < a.nbatch; ++b) {
            DataArgs q = a;
            q.nbatch = 1;
            q.v = a.v ? a.v + (long long)b * a.vstride : nullptr;
            q.energy = a.energy ? a.energy + b : nullptr;
            ws.off = off0;
            LDDMM_TRY(dt_run<Real>(q, ws, st));
            top = std::max(top, ws.off);
        }
        ws.off = top;
        return LDDMM_OK;
    }
    auto go = [&](auto kind, auto pdeg, auto qdeg) {
        return dispatch_d(a.d, [&](auto D) {
            constexpr int K_ = decltype(kind)::value, P_ = decltype(pdeg)::value, Q_ = decltype(qdeg)::value,
                          D_ = decltype(D)::value;
            if (fused && a.d == D_) return dt_value_fused<Real, K_, P_, D_>(a, ws, st);
            if (a.px != nullptr && a.nbatch == 1 && dt_fused_fits(a.nc, a.nc2) && a.d == D_)
                return dt_grad_fused<Real, K_, P_, Q_, D_>(a, ws, st);
            if (a.nc <= kSmallTargets) return dt_impl<Real, K_, P_, Q_, D_, true>(a, ws, st);
            return dt_impl<Real, K_, P_, Q_, D_>(a, ws, st);
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
    if (a.nbatch < 1 || a.nbatch > (1 << 12) || (a.nbatch > 1 && (a.px != nullptr || a.vstride < a.nv * a.d))) {
        set_error("dataterm: a batch needs 1 <= nbatch <= 4096, values only and vertex_stride >= nv * d "
                  "(nbatch=%d vertex_stride=%lld)", a.nbatch, a.vstride);
        return LDDMM_ERR_ARG;
    }
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
             int want_grad, int nbatch = 1) {
    if (nbatch < 1 || nbatch > (1 << 12) || (nbatch > 1 && (want_grad || !want_energy))) return 0;
    DataArgs a{};
    a.nbatch = nbatch;
    a.vstride = nv * d;
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

size_t lddmm_dataterm_value_batch_f32c_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2,
                                                 int order, int nbatch) {
    return dt_ws<float>(cell_size, norm, nv, d, nc, nc2, order, 1, 0, nbatch);
}
size_t lddmm_dataterm_value_batch_f64_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2,
                                                int order, int nbatch) {
    return dt_ws<double>(cell_size, norm, nv, d, nc, nc2, order, 1, 0, nbatch);
}

#define DT_BATCH_ARGS                                                                                           \
    DataArgs a{cell_size, norm,  vertices, nv,   d,      cells,   nc,     tgt_centers, tgt_vectors, nc2, \
               sigma,     order, eps1,     eps2, energy, nullptr, nullptr, nullptr};                      \
    a.nbatch = nbatch;                                                                                  \
    a.vstride = vertex_stride

int lddmm_dataterm_value_batch_f32c(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                    const int64_t* cells, int64_t nc, const double* tgt_centers,
                                    const double* tgt_vectors, int64_t nc2, double sigma, int order, double eps1,
                                    double eps2, int nbatch, int64_t vertex_stride, double* energy, void* workspace,
                                    size_t workspace_bytes, lddmm_stream_t stream) {
    DT_BATCH_ARGS;
    return dt_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_dataterm_value_batch_f64(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                   const int64_t* cells, int64_t nc, const double* tgt_centers,
                                   const double* tgt_vectors, int64_t nc2, double sigma, int order, double eps1,
                                   double eps2, int nbatch, int64_t vertex_stride, double* energy, void* workspace,
                                   size_t workspace_bytes, lddmm_stream_t stream) {
    DT_BATCH_ARGS;
    return dt_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
