// Geodesic shooting and its Hamiltonian adjoint, fused per time step.
//
//   lddmm_shoot_*    : landmarkDirectEvolutionEuler (py-lddmm/pointEvolution.py:666-730)
//                      x_{t+1} = x_t + dt K(x_t, x_t) a_t, dt = 1/T, plus the
//                      regularisation energy sum_t rw dt <a_t, K(x_t) a_t> of
//                      objectiveFunDef (surfaceMatching.py:205-212), computed
//                      from the same kernel sums.
//   lddmm_covector_* : landmarkHamiltonianCovector / Gradient (pointEvolution.py:735-817)
//                      p_t = p_{t+1} + dt applyDiffKT(x_t, [p, a, -2 rw a], [a, p, a]),
//                      dat_t = 2 rw a_t - p_{t+1}.
//   lddmm_epdiff_*   : landmarkEPDiff (pointEvolution.py:599-658).
//
// The 3-momentum inner product of the adjoint is rewritten as
//   <p_k,a_l> + <a_k,p_l> - 2 rw <a_k,a_l> = <p_k - 2 rw a_k, a_l> + <a_k, p_l>,
// a 2d-wide dot (u_k = (p_k - 2 rw a_k, a_k), v_l = (a_l, p_l)).
//
// One time step = one sweep over (target block, source chunk) items + one
// combine kernel that adds the chunks in a fixed order, applies the Euler (or
// adjoint) update in FP64, writes the packed planes of the next step and the
// step's energy partials (one per combine block; the grid size depends only on
// n, so the reduction order is fixed).
#include "dataterm_fused.cuh"
#include "fused_small.cuh"
#include "host.h"
#include "ops2.cuh"
#include "pack.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

constexpr int kCombineThreads = 256;
constexpr int kMaxBatch = 1 << 12;   // trial step sizes per batched call

inline int combine_blocks(long long n) { return (int)std::min<long long>(1024, (n + kCombineThreads - 1) / kCombineThreads); }

// the packing frame: (v - c) * s, c the bounding-box centre of the initial points
template <class Real>
LDDMM_D void store_point(float4* planes, long long stride, long long i, const double* v, int d, double s,
                         const double* c) {
    double q[4] = {0, 0, 0, 0};
    for (int j = 0; j < d; ++j) q[j] = (v[j] - c[j]) * s;
    if constexpr (sizeof(Real) == 4) {
        planes[i] = make_float4((float)q[0], (float)q[1], (float)q[2], 0.f);
    } else {
        double2* o = reinterpret_cast<double2*>(planes);
        o[i] = make_double2(q[0], q[1]);
        o[stride + i] = make_double2(q[2], 0.0);
    }
}

// values v[0..nv) into planes first_plane.. of record i
template <class Real>
LDDMM_D void store_vals(float4* planes, long long stride, long long i, int first_plane, const double* v, int nv,
                        int nslots) {
    constexpr int PW = Traits<Real>::PER_WORD;
    for (int w = 0; w < (nslots + PW - 1) / PW; ++w) {
        Real q[PW];
        for (int j = 0; j < PW; ++j) q[j] = (w * PW + j < nv) ? (Real)v[w * PW + j] : (Real)0;
        float4* dst = planes + (long long)(first_plane + w) * stride + i;
        if constexpr (sizeof(Real) == 4) *dst = make_float4(q[0], q[1], q[2], q[3]);
        else *reinterpret_cast<double2*>(dst) = make_double2(q[0], q[1]);
    }
}

template <class Real>
LDDMM_D void zero_record(float4* planes, long long stride, long long i, int nplanes) {
    for (int p = 0; p < nplanes; ++p) planes[(long long)p * stride + i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Duplicated source record (packed-pair FP32 operators, ops2.cuh): values
// [(x - c) * s for D coordinates, vals[0..nv) padded to V], each value twice.
LDDMM_D void store_dup(float4* planes, long long stride, long long i, const double* x, int d, int D, double s,
                       const double* c, const double* vals, int nv, int V) {
    float v[16];
    const int NV = D + V;
    for (int q = 0; q < NV; ++q) v[q] = 0.f;
    for (int j = 0; j < d; ++j) v[j] = (float)((x[j] - c[j]) * s);
    for (int q = 0; q < nv && q < V; ++q) v[D + q] = (float)vals[q];
    for (int w = 0; w < (NV + 1) / 2; ++w) {
        const float a = v[2 * w], b = (2 * w + 1 < NV) ? v[2 * w + 1] : 0.f;
        planes[(long long)w * stride + i] = make_float4(a, a, b, b);
    }
}

// block-level FP64 sum with a fixed tree; thread 0 writes out[blockIdx.x]
LDDMM_D void block_sum_store(double v, double* out) {
    __shared__ double red[kCombineThreads];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = kCombineThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// kernel polynomials into either parameter block
inline void set_poly(KernelParamsBase<double>& P, const KScale& ks) {
    for (int j = 0; j < 5; ++j) P.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = ks.pq[j];
}
inline void set_poly(KernelParamsBase<float>& P, const KScale& ks) {
    for (int j = 0; j < 5; ++j) P.pk[j] = (float)ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = (float)ks.pq[j];
}
inline void set_poly(KernelParams2& P, const KScale& ks) {
    for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks.pk[j]);
    for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks.pq[j]);
}

// ---- shooting ---------------------------------------------------------------
// Packs step-0 planes: targets (pos) and sources (pos, a).
template <class Real, bool DUP>
static __global__ void shoot_pack_kernel(const double* __restrict__ x, const double* __restrict__ a, long long n,
                                         int d, double s, const double* __restrict__ c, float4* tgt,
                                         long long tstride, float4* src, long long sstride, int pp, int nslots,
                                         int ns) {
    const long long npad = tstride > sstride ? tstride : sstride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n) {
            if (i < tstride) store_point<Real>(tgt, tstride, i, x + i * d, d, s, c);
            if (i < sstride) {
                if constexpr (DUP) {
                    store_dup(src, sstride, i, x + i * d, d, nslots, s, c, a + i * d, d, nslots);
                } else {
                    store_point<Real>(src, sstride, i, x + i * d, d, s, c);
                    store_vals<Real>(src, sstride, i, pp, a + i * d, d, nslots);
                }
            }
        } else {
            if (i < tstride) zero_record<Real>(tgt, tstride, i, pp);
            if (i < sstride) zero_record<Real>(src, sstride, i, ns);
        }
    }
}

// v = sum of chunks; x1 = x0 + dt v; energy partial <a, v>; pack next step.
template <class Real, bool DUP>
static __global__ void shoot_combine_kernel(const double* __restrict__ part, long long n, int d, int dout,
                                            int split, double dt, const double* __restrict__ x0,
                                            const double* __restrict__ a0, double* __restrict__ x1,
                                            const double* __restrict__ a1, double s, const double* __restrict__ c,
                                            float4* tgt, long long tstride, float4* src, long long sstride, int pp,
                                            int nslots, double* __restrict__ epart) {
    double e = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double xn[4];
        for (int j = 0; j < d; ++j) {
            double v = 0.0;
            for (int k = 0; k < split; ++k) v += part[((long long)k * n + i) * dout + j];
            e += a0[i * d + j] * v;
            xn[j] = x0[i * d + j] + dt * v;
            x1[i * d + j] = xn[j];
        }
        if (a1 != nullptr) {
            store_point<Real>(tgt, tstride, i, xn, d, s, c);
            if constexpr (DUP) {
                store_dup(src, sstride, i, xn, d, nslots, s, c, a1 + i * d, d, nslots);
            } else {
                store_point<Real>(src, sstride, i, xn, d, s, c);
                store_vals<Real>(src, sstride, i, pp, a1 + i * d, d, nslots);
            }
        }
    }
    block_sum_store(e, epart);
}

// out = scale * sum(vals[0..count)) in a fixed order (single block)
static __global__ void finalize_sum_kernel(const double* __restrict__ vals, long long count, double scale,
                                           double* __restrict__ out) {
    double v = 0.0;
    for (long long i = threadIdx.x; i < count; i += blockDim.x) v += vals[i];
    block_sum_store(v, out);
    if (threadIdx.x == 0) out[0] = scale * out[0];
}

struct ShootArgs {
    const double* x0;
    long long n;
    int d;
    const double* at;
    int T;
    double dt;  // Euler step; <= 0 means 1/T
    double sigma;
    int order;
    double rw;
    double* xt;
    double* energy;
    // optional search direction: the shot's momenta are at - (*eps) dir, written to at_try
    const double* dir = nullptr;
    const double* eps = nullptr;
    double* at_try = nullptr;
    // batched trial steps: nbatch step sizes eps[0..nbatch), outputs at_try, xt, energy stacked per candidate
    int nbatch = 1;
};

// at_try = at - (*eps) dir, rounded as two FP64 operations (the trial step of a line search)
static __global__ void trial_momenta_kernel(const double* __restrict__ at, const double* __restrict__ dir,
                                            const double* __restrict__ eps, long long count,
                                            double* __restrict__ at_try) {
    const double e = *eps;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        at_try[i] = __dsub_rn(at[i], __dmul_rn(e, dir[i]));
}

template <class Real, int KIND, int DEG, int D, bool SMALL = false>
int shoot_impl(const ShootArgs& a, Workspace& ws, cudaStream_t st) {
    constexpr bool DUP = sizeof(Real) == 4;  // FP32: packed-pair operator with duplicated sources
    using Op = std::conditional_t<DUP, OpApplyK2<KIND, DEG, D, D, SMALL>, OpApplyK<Real, KIND, DEG, D, D, SMALL>>;
    const SinglePlan pl = plan_single<Op>(a.n, a.n);
    float4* tgt = ws.take<float4>((size_t)Op::PP * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n * D);
    const int nb = combine_blocks(a.n);
    double* epart = ws.take<double>((size_t)a.T * nb);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    set_poly(P, ks);
    const long long N = a.n * a.d;
    LDDMM_TRY(cuda_check(cudaMemcpyAsync(a.xt, a.x0, sizeof(double) * N, cudaMemcpyDeviceToDevice, st), "shoot copy"));
    launch_bbox_center(a.x0, a.n, nullptr, 0, a.d, center, st);
    shoot_pack_kernel<Real, DUP><<<grid_for(std::max(pl.n_tpad, pl.m_pad)), 256, 0, st>>>(
        a.x0, a.at, a.n, a.d, ks.scale, center, tgt, pl.n_tpad, src, pl.m_pad, Op::PP, D, Op::NS);
    const double dt = a.dt > 0 ? a.dt : 1.0 / a.T;
    for (int t = 0; t < a.T; ++t) {
        LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
        shoot_combine_kernel<Real, DUP><<<nb, kCombineThreads, 0, st>>>(
            part, a.n, a.d, D, pl.split, dt, a.xt + t * N, a.at + t * N, a.xt + (t + 1) * N,
            t + 1 < a.T ? a.at + (t + 1) * N : nullptr, ks.scale, center, tgt, pl.n_tpad, src, pl.m_pad, Op::PP,
            D, epart + (long long)t * nb);
    }
    if (a.energy != nullptr)
        finalize_sum_kernel<<<1, kCombineThreads, 0, st>>>(epart, (long long)a.T * nb, a.rw * dt, a.energy);
    return cuda_check(cudaGetLastError(), "shoot");
}

// n <= kFusedMaxPoints (and d >= 2): all T steps in one cluster launch (fused_small.cuh)
template <class Real, int KIND, int DEG, int D>
int shoot_fused(const ShootArgs& a, Workspace& ws, cudaStream_t st) {
    const FusedShape fs = fused_shape(a.n);
    double* epart = ws.take<double>((size_t)kFusedMaxCluster * a.nbatch);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    FusedCoef cf{};
    for (int j = 0; j < 5; ++j) cf.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) cf.pq[j] = ks.pq[j];
    const double dt = a.dt > 0 ? a.dt : 1.0 / a.T;
    return launch_fused(shoot_fused_kernel<Real, KIND, DEG, D>, fs, a.nbatch, fused_dyn_smem<Real>(a.n, D),
                        fused_dyn_smem<Real>(kFusedMaxPoints, 3), st, a.x0, a.at,
                        (long long)a.n, a.T, dt, ks.scale, cf, a.rw, fs, a.xt, a.energy, epart, a.dir, a.eps,
                        a.at_try);
}

template <class Real>
int shoot_run(const ShootArgs& a0, Workspace& ws, cudaStream_t st) {
    ShootArgs a = a0;
    const bool fused = a.n <= kFusedMaxPoints && a.d >= 2;
    if (a.nbatch > 1 && !fused) {
        // general path: the candidates one after the other, each on the same workspace
        const long long N = a.n * a.d;
        const size_t off0 = ws.off;
        size_t top = off0;
        for (int b = 0; b < a.nbatch; ++b) {
            ShootArgs q = a;
            q.nbatch = 1;
            q.eps = a.eps ? a.eps + b : nullptr;
            q.at_try = a.at_try ? a.at_try + (long long)b * a.T * N : nullptr;
            q.xt = a.xt ? a.xt + (long long)b * (a.T + 1) * N : nullptr;
            q.energy = a.energy ? a.energy + b : nullptr;
            ws.off = off0;
            LDDMM_TRY(shoot_run<Real>(q, ws, st));
            top = std::max(top, ws.off);
        }
        ws.off = top;
        return LDDMM_OK;
    }
    if (a.dir != nullptr && !fused) {
        // general path: form the trial momenta, then shoot them
        if (!ws.measuring()) {
            const long long cnt = (long long)a.T * a.n * a.d;
            trial_momenta_kernel<<<grid_for(cnt), 256, 0, st>>>(a.at, a.dir, a.eps, cnt, a.at_try);
        }
        a.at = a.at_try;
        a.dir = nullptr;
    }
    return dispatch_kind_p(a.order, [&](auto kind, auto deg) {
        return dispatch_d(a.d, [&](auto D) {
            constexpr int K_ = decltype(kind)::value, P_ = decltype(deg)::value, D_ = decltype(D)::value;
            if (a.n <= kFusedMaxPoints && a.d == D_) return shoot_fused<Real, K_, P_, D_>(a, ws, st);
            if (a.n <= kSmallTargets) return shoot_impl<Real, K_, P_, D_, true>(a, ws, st);
            return shoot_impl<Real, K_, P_, D_>(a, ws, st);
        });
    });
}

// ---- covector ---------------------------------------------------------------
// planes of step t: targets (pos, u = (p - 2 rw a, a)), sources (pos, v = (a, p))
template <class Real, bool DUP>
LDDMM_D void cov_store(float4* tgt, long long tstride, float4* src, long long sstride, long long i, int pp,
                       const double* x, const double* a, const double* p, int d, double s, const double* c,
                       double rw, int tw) {
    double u[8], v[8];
    for (int j = 0; j < d; ++j) {
        u[j] = p[j] - 2.0 * rw * a[j];
        u[d + j] = a[j];
        v[j] = a[j];
        v[d + j] = p[j];
    }
    if (i < tstride) {
        store_point<Real>(tgt, tstride, i, x, d, s, c);
        store_vals<Real>(tgt, tstride, i, pp, u, 2 * d, tw);
    }
    if (i < sstride) {
        if constexpr (DUP) {
            store_dup(src, sstride, i, x, d, tw / 2, s, c, v, 2 * d, tw);
        } else {
            store_point<Real>(src, sstride, i, x, d, s, c);
            store_vals<Real>(src, sstride, i, pp, v, 2 * d, tw);
        }
    }
}

template <class Real, bool DUP>
static __global__ void cov_pack_kernel(const double* __restrict__ x, const double* __restrict__ a,
                                       const double* __restrict__ p, long long n, int d, double s,
                                       const double* __restrict__ c, double rw, float4* tgt, long long tstride,
                                       float4* src, long long sstride, int pp, int tplanes, int nplanes, int tw) {
    const long long npad = tstride > sstride ? tstride : sstride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n) {
            cov_store<Real, DUP>(tgt, tstride, src, sstride, i, pp, x + i * d, a + i * d, p + i * d, d, s, c, rw, tw);
        } else {
            if (i < tstride) zero_record<Real>(tgt, tstride, i, tplanes);
            if (i < sstride) zero_record<Real>(src, sstride, i, nplanes);
        }
    }
}

// p_t = p_{t+1} + dt * dscale * sum(chunks); dat_t = 2 rw a_t - p_{t+1}; pack step t-1.
template <class Real, bool DUP>
static __global__ void cov_combine_kernel(const double* __restrict__ part, long long n, int d, int dout, int split,
                                          double dt, double dscale, double rw, const double* __restrict__ p_next,
                                          const double* __restrict__ a_t, double* __restrict__ p_t,
                                          double* __restrict__ dat_t, const double* __restrict__ x_prev,
                                          const double* __restrict__ a_prev, double s, const double* __restrict__ c,
                                          float4* tgt, long long tstride, float4* src, long long sstride, int pp,
                                          int tw) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double pn[4];
        for (int j = 0; j < d; ++j) {
            double f = 0.0;
            for (int k = 0; k < split; ++k) f += part[((long long)k * n + i) * dout + j];
            const double pj = p_next[i * d + j];
            pn[j] = pj + dt * (dscale * f);
            p_t[i * d + j] = pn[j];
            if (dat_t != nullptr) dat_t[i * d + j] = 2.0 * rw * a_t[i * d + j] - pj;
        }
        if (x_prev != nullptr)
            cov_store<Real, DUP>(tgt, tstride, src, sstride, i, pp, x_prev + i * d, a_prev + i * d, pn, d, s, c, rw,
                                 tw);
    }
}

struct CovArgs {
    const double* xt;
    long long n;
    int d;
    const double* at;
    int T;
    double dt;  // Euler step; <= 0 means 1/T
    const double* px1;
    double sigma;
    int order;
    double rw;
    double* pxt;
    double* dat;
};

template <class Real, int KIND, int DEG, int D, bool SMALL = false>
int cov_impl(const CovArgs& a, Workspace& ws, cudaStream_t st) {
    constexpr int W = 2 * D;
    constexpr bool DUP = sizeof(Real) == 4;  // FP32: packed-pair operator with duplicated sources
    using Op = std::conditional_t<DUP, OpDiffKT2<KIND, DEG, D, W, SMALL>, OpDiffKT<Real, KIND, DEG, D, W, SMALL>>;
    constexpr int NT = DUP ? 1 + (W + 3) / 4 : Op::NS;  // target planes (standard layout)
    const SinglePlan pl = plan_single<Op>(a.n, a.n);
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
    set_poly(P, ks);
    const long long N = a.n * a.d;
    const double dt = a.dt > 0 ? a.dt : 1.0 / a.T;
    LDDMM_TRY(cuda_check(cudaMemcpyAsync(a.pxt + (long long)a.T * N, a.px1, sizeof(double) * N,
                                         cudaMemcpyDeviceToDevice, st), "covector copy"));
    const int T = a.T;
    launch_bbox_center(a.xt, a.n, nullptr, 0, a.d, center, st);
    cov_pack_kernel<Real, DUP><<<grid_for(std::max(pl.n_tpad, pl.m_pad)), 256, 0, st>>>(
        a.xt + (long long)(T - 1) * N, a.at + (long long)(T - 1) * N, a.px1, a.n, a.d, ks.scale, center, a.rw,
        tgt, pl.n_tpad, src, pl.m_pad, Op::PP, NT, Op::NS, W);
    const int nb = combine_blocks(a.n);
    for (int t = T - 1; t >= 0; --t) {
        LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
        cov_combine_kernel<Real, DUP><<<nb, kCombineThreads, 0, st>>>(
            part, a.n, a.d, D, pl.split, dt, ks.dscale, a.rw, a.pxt + (long long)(t + 1) * N,
            a.at + (long long)t * N, a.pxt + (long long)t * N, a.dat ? a.dat + (long long)t * N : nullptr,
            t > 0 ? a.xt + (long long)(t - 1) * N : nullptr, t > 0 ? a.at + (long long)(t - 1) * N : nullptr,
            ks.scale, center, tgt, pl.n_tpad, src, pl.m_pad, Op::PP, W);
    }
    return cuda_check(cudaGetLastError(), "covector");
}

template <class Real, int KIND, int QDEG, int D>
int cov_fused(const CovArgs& a, Workspace& ws, cudaStream_t st) {
    const FusedShape fs = fused_shape(a.n);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    FusedCoef cf{};
    for (int j = 0; j < 5; ++j) cf.pk[j] = ks.pk[j];
    for (int j = 0; j < 4; ++j) cf.pq[j] = ks.pq[j];
    const double dt = a.dt > 0 ? a.dt : 1.0 / a.T;
    return launch_fused(cov_fused_kernel<Real, KIND, QDEG, D>, fs, 1, fused_dyn_smem<Real>(a.n, D),
                        fused_dyn_smem<Real>(kFusedMaxPoints, 3), st, a.xt, a.at,
                        a.px1, (long long)a.n, a.T, dt, ks.scale, ks.dscale, cf, a.rw, fs, a.pxt, a.dat);
}

template <class Real>
int cov_run(const CovArgs& a, Workspace& ws, cudaStream_t st) {
    return dispatch_kind_q(a.order, [&](auto kind, auto deg) {
        return dispatch_d(a.d, [&](auto D) {
            constexpr int K_ = decltype(kind)::value, Q_ = decltype(deg)::value, D_ = decltype(D)::value;
            if (a.n <= kFusedMaxPoints && a.d == D_) return cov_fused<Real, K_, Q_, D_>(a, ws, st);
            if (a.n <= kSmallTargets) return cov_impl<Real, K_, Q_, D_, true>(a, ws, st);
            return cov_impl<Real, K_, Q_, D_>(a, ws, st);
        });
    });
}

// ---- EPDiff -------------------------------------------------------------------
// x_{k+1} = x_k + dt K a_k ; a_{k+1} = a_k - dt applyDiffKT(x_k, [a_k], [a_k]).
// Two sums over the same pairs, computed by one operator.
template <class Real_, int KIND, int PDEG, int QDEG, int D>
struct OpEPDiff {
    using Real = Real_;
    static constexpr bool F32 = sizeof(Real) == 4;
    static constexpr int TPS = 1;
    static constexpr int BLOCK = 128, R = 2, TILE = 128, FOLD = F32 ? 32 : TILE;
    static constexpr int PP = PointPlanes<Real>::N;
    static constexpr int WP = (D + Traits<Real>::PER_WORD - 1) / Traits<Real>::PER_WORD;
    static constexpr int NS = PP + WP;
    static constexpr int NOUT = 2 * D;
    using Params = KernelParamsBase<Real>;
    using Acc = typename AccFor<Real>::template type<2 * D>;
    struct Tgt {
        Real x[D];
        Real a[D];
    };
    struct Src {
        Real y[D];
        Real a[D];
    };
    static LDDMM_D void load_target(const Params& P, long long row, Tgt& t) {
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, 0, t.x);
        load_vals<Real, D>(P.tgt4, P.tgt_stride, row, PP, t.a);
    }
    static LDDMM_D void load_source(const float4* S, int j, Src& s) {
        load_vals_smem<Real, D, TILE>(S, j, 0, s.y);
        load_vals_smem<Real, D, TILE>(S, j, PP, s.a);
    }
    static LDDMM_D void pair(const Params& P, const Tgt& t, const Src& s, Acc& acc) {
        Real dx[D], r2 = 0, dot = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            dx[j] = t.x[j] - s.y[j];
            r2 = j == 0 ? dx[j] * dx[j] : r2 + dx[j] * dx[j];
            dot = j == 0 ? t.a[j] * s.a[j] : dot + t.a[j] * s.a[j];
        }
        const Real k = kval<Real, KIND, PDEG>(P.pk, r2);
        const Real g = kdiff<Real, KIND, QDEG>(P.pq, r2) * dot;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            acc.fma(j, k, s.a[j]);
            acc.fma(D + j, g, dx[j]);
        }
    }
};

template <class Real>
static __global__ void epd_pack_kernel(const double* __restrict__ x, const double* __restrict__ a, long long n,
                                       int d, double s, const double* __restrict__ c, float4* tgt, long long tstride,
                                       float4* src, long long sstride, int pp, int nslots, int ns) {
    const long long npad = tstride > sstride ? tstride : sstride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npad;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n) {
            if (i < tstride) {
                store_point<Real>(tgt, tstride, i, x + i * d, d, s, c);
                store_vals<Real>(tgt, tstride, i, pp, a + i * d, d, nslots);
            }
            if (i < sstride) {
                store_point<Real>(src, sstride, i, x + i * d, d, s, c);
                store_vals<Real>(src, sstride, i, pp, a + i * d, d, nslots);
            }
        } else {
            if (i < tstride) zero_record<Real>(tgt, tstride, i, ns);
            if (i < sstride) zero_record<Real>(src, sstride, i, ns);
        }
    }
}

template <class Real>
static __global__ void epd_combine_kernel(const double* __restrict__ part, long long n, int d, int dout, int split,
                                          double dt, double dscale, const double* __restrict__ x0,
                                          const double* __restrict__ a0, double* __restrict__ x1,
                                          double* __restrict__ a1) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        for (int j = 0; j < d; ++j) {
            double v = 0.0, g = 0.0;
            for (int k = 0; k < split; ++k) {
                v += part[((long long)k * n + i) * dout + j];
                g += part[((long long)k * n + i) * dout + dout / 2 + j];
            }
            x1[i * d + j] = x0[i * d + j] + dt * v;
            if (a1 != nullptr) a1[i * d + j] = a0[i * d + j] - dt * (dscale * g);
        }
    }
}

struct EPDArgs {
    const double* x0;
    long long n;
    int d;
    const double* a0;
    int T;
    double sigma;
    int order;
    double* xt;
    double* at;
};

template <class Real, int KIND, int PDEG, int QDEG, int D>
int epd_impl(const EPDArgs& a, Workspace& ws, cudaStream_t st) {
    using Op = OpEPDiff<Real, KIND, PDEG, QDEG, D>;
    const SinglePlan pl = plan_single<Op>(a.n, a.n);
    float4* tgt = ws.take<float4>((size_t)Op::NS * pl.n_tpad);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.m_pad);
    double* part = ws.take<double>((size_t)pl.split * a.n * Op::NOUT);
    double* center = ws.take<double>(kCenterWords);
    if (ws.measuring()) return LDDMM_OK;
    const KScale ks = kernel_scale<Real>(KIND, a.order, a.sigma);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.m_pad;
    P.tgt4 = tgt;
    P.tgt_stride = pl.n_tpad;
    for (int j = 0; j < 5; ++j) P.pk[j] = (Real)ks.pk[j];
    for (int j = 0; j < 4; ++j) P.pq[j] = (Real)ks.pq[j];
    const long long N = a.n * a.d;
    const double dt = 1.0 / a.T;
    LDDMM_TRY(cuda_check(cudaMemcpyAsync(a.xt, a.x0, sizeof(double) * N, cudaMemcpyDeviceToDevice, st), "epdiff"));
    LDDMM_TRY(cuda_check(cudaMemcpyAsync(a.at, a.a0, sizeof(double) * N, cudaMemcpyDeviceToDevice, st), "epdiff"));
    const int nb = combine_blocks(a.n);
    launch_bbox_center(a.x0, a.n, nullptr, 0, a.d, center, st);
    for (int t = 0; t < a.T; ++t) {
        epd_pack_kernel<Real><<<grid_for(std::max(pl.n_tpad, pl.m_pad)), 256, 0, st>>>(
            a.xt + t * N, a.at + t * N, a.n, a.d, ks.scale, center, tgt, pl.n_tpad, src, pl.m_pad, Op::PP, D,
            Op::NS);
        LDDMM_TRY(launch_single<Op>(pl, a.n, P, part, st));
        epd_combine_kernel<Real><<<nb, kCombineThreads, 0, st>>>(part, a.n, a.d, Op::NOUT, pl.split, dt, ks.dscale,
                                                                 a.xt + t * N, a.at + t * N, a.xt + (t + 1) * N,
                                                                 t + 1 < a.T ? a.at + (t + 1) * N : nullptr);
    }
    return cuda_check(cudaGetLastError(), "epdiff");
}

template <class Real>
int epd_run(const EPDArgs& a, Workspace& ws, cudaStream_t st) {
    if (a.order == 0) {
        set_error("epdiff: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    auto go = [&](auto kind, auto pdeg, auto qdeg) {
        return dispatch_d(a.d, [&](auto D) {
            return epd_impl<Real, decltype(kind)::value, decltype(pdeg)::value, decltype(qdeg)::value,
                            decltype(D)::value>(a, ws, st);
        });
    };
    switch (a.order) {
        case 1: return go(IC<KLAP>{}, IC<1>{}, IC<0>{});
        case 2: return go(IC<KLAP>{}, IC<2>{}, IC<1>{});
        case 3: return go(IC<KLAP>{}, IC<3>{}, IC<2>{});
        case 4: return go(IC<KLAP>{}, IC<4>{}, IC<3>{});
        default: return go(IC<KGAUSS>{}, IC<0>{}, IC<0>{});
    }
}

// ---- entry helpers --------------------------------------------------------------
static int basic_validate(long long n, int d, int T, double sigma, int order, const char* who) {
    if (n < 1 || n > (1LL << 30) || d < 1 || d > 3 || T < 1 || T > 100000 || !(sigma > 0) || order < 0) {
        set_error("%s: invalid arguments (n=%lld d=%d T=%d sigma=%g order=%d); d must be 1..3", who, n, d, T, sigma,
                  order);
        return LDDMM_ERR_ARG;
    }
    return LDDMM_OK;
}

template <class Run, class Args>
int run_with_workspace(Run run, const Args& a, void* wsp, size_t wsb, cudaStream_t st, const char* who) {
    Workspace meas;
    LDDMM_TRY(run(a, meas, st));
    if (wsp == nullptr || meas.off > wsb) {
        set_error("%s: workspace too small: need %zu bytes, got %zu", who, meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return run(a, ws, st);
}

template <class Real>
size_t shoot_ws(int64_t n, int d, int T, int nbatch = 1) {
    if (basic_validate(n, d, T, 1.0, 10, "shoot") != LDDMM_OK) return 0;
    if (nbatch < 1 || nbatch > kMaxBatch) return 0;
    ShootArgs a{};
    a.n = n;
    a.d = d;
    a.T = T;
    a.sigma = 1.0;
    a.order = 10;
    a.nbatch = nbatch;
    Workspace ws;
    size_t best = 0;
    for (int order : {10, 3}) {  // the Laplacian and Gaussian plans may differ
        a.order = order;
        ws = Workspace();
        shoot_run<Real>(a, ws, 0);
        best = std::max(best, ws.off);
    }
    return best + 256;
}

template <class Real>
int shoot_entry(const ShootArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(basic_validate(a.n, a.d, a.T, a.sigma, a.order, "shoot"));
    LDDMM_TRY(check_device_ptr(a.x0, "x0"));
    LDDMM_TRY(check_device_ptr(a.at, "at"));
    LDDMM_TRY(check_device_ptr(a.xt, "xt"));
    if (a.energy) LDDMM_TRY(check_device_ptr(a.energy, "energy"));
    if (a.dir != nullptr || a.eps != nullptr || a.at_try != nullptr || a.nbatch != 1) {
        if (a.nbatch < 1 || a.nbatch > kMaxBatch) {
            set_error("shoot: nbatch must be in [1, %d] (got %d)", kMaxBatch, a.nbatch);
            return LDDMM_ERR_ARG;
        }
        LDDMM_TRY(check_device_ptr(a.dir, "dir"));
        LDDMM_TRY(check_device_ptr(a.eps, "eps"));
        LDDMM_TRY(check_device_ptr(a.at_try, "at_try"));
    }
    return run_with_workspace([](const ShootArgs& q, Workspace& w, cudaStream_t s) { return shoot_run<Real>(q, w, s); },
                              a, wsp, wsb, st, "shoot");
}

template <class Real>
size_t cov_ws(int64_t n, int d, int T) {
    if (basic_validate(n, d, T, 1.0, 10, "covector") != LDDMM_OK) return 0;
    CovArgs a{};
    a.n = n;
    a.d = d;
    a.T = T;
    a.sigma = 1.0;
    size_t best = 0;
    for (int order : {10, 3}) {
        a.order = order;
        Workspace ws;
        cov_run<Real>(a, ws, 0);
        best = std::max(best, ws.off);
    }
    return best + 256;
}

template <class Real>
int cov_entry(const CovArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(basic_validate(a.n, a.d, a.T, a.sigma, a.order, "covector"));
    if (a.order == 0) {
        set_error("covector: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(a.xt, "xt"));
    LDDMM_TRY(check_device_ptr(a.at, "at"));
    LDDMM_TRY(check_device_ptr(a.px1, "px1"));
    LDDMM_TRY(check_device_ptr(a.pxt, "pxt"));
    if (a.dat) LDDMM_TRY(check_device_ptr(a.dat, "dat"));
    return run_with_workspace([](const CovArgs& q, Workspace& w, cudaStream_t s) { return cov_run<Real>(q, w, s); },
                              a, wsp, wsb, st, "covector");
}

template <class Real>
size_t epd_ws(int64_t n, int d, int T) {
    if (basic_validate(n, d, T, 1.0, 10, "epdiff") != LDDMM_OK) return 0;
    EPDArgs a{};
    a.n = n;
    a.d = d;
    a.T = T;
    a.sigma = 1.0;
    size_t best = 0;
    for (int order : {10, 3}) {
        a.order = order;
        Workspace ws;
        epd_run<Real>(a, ws, 0);
        best = std::max(best, ws.off);
    }
    return best + 256;
}

template <class Real>
int epd_entry(const EPDArgs& a, void* wsp, size_t wsb, cudaStream_t st) {
    LDDMM_TRY(basic_validate(a.n, a.d, a.T, a.sigma, a.order, "epdiff"));
    LDDMM_TRY(check_device_ptr(a.x0, "x0"));
    LDDMM_TRY(check_device_ptr(a.a0, "a0"));
    LDDMM_TRY(check_device_ptr(a.xt, "xt"));
    LDDMM_TRY(check_device_ptr(a.at, "at"));
    return run_with_workspace([](const EPDArgs& q, Workspace& w, cudaStream_t s) { return epd_run<Real>(q, w, s); },
                              a, wsp, wsb, st, "epdiff");
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_shoot_f32c_workspace(int64_t n, int d, int T) { return shoot_ws<float>(n, d, T); }
size_t lddmm_shoot_f64_workspace(int64_t n, int d, int T) { return shoot_ws<double>(n, d, T); }

int lddmm_shoot_f32c(const double* x0, int64_t n, int d, const double* at, int T, double dt, double sigma,
                     int order, double regweight, double* xt, double* energy, void* workspace,
                     size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    return shoot_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_shoot_f64(const double* x0, int64_t n, int d, const double* at, int T, double dt, double sigma,
                    int order, double regweight, double* xt, double* energy, void* workspace,
                    size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    return shoot_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_shoot_along_f32c(const double* x0, int64_t n, int d, const double* at, const double* dir, const double* eps,
                           int T, double dt, double sigma, int order, double regweight, double* at_try, double* xt,
                           double* energy, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    a.dir = dir;
    a.eps = eps;
    a.at_try = at_try;
    return shoot_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_shoot_along_f64(const double* x0, int64_t n, int d, const double* at, const double* dir, const double* eps,
                          int T, double dt, double sigma, int order, double regweight, double* at_try, double* xt,
                          double* energy, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    a.dir = dir;
    a.eps = eps;
    a.at_try = at_try;
    return shoot_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t lddmm_shoot_along_batch_f32c_workspace(int64_t n, int d, int T, int nbatch) {
    return shoot_ws<float>(n, d, T, nbatch);
}
size_t lddmm_shoot_along_batch_f64_workspace(int64_t n, int d, int T, int nbatch) {
    return shoot_ws<double>(n, d, T, nbatch);
}

int lddmm_shoot_along_batch_f32c(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                 const double* eps, int nbatch, int T, double dt, double sigma, int order,
                                 double regweight, double* at_try, double* xt, double* energy, void* workspace,
                                 size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    a.dir = dir;
    a.eps = eps;
    a.at_try = at_try;
    a.nbatch = nbatch;
    return shoot_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_shoot_along_batch_f64(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                const double* eps, int nbatch, int T, double dt, double sigma, int order,
                                double regweight, double* at_try, double* xt, double* energy, void* workspace,
                                size_t workspace_bytes, lddmm_stream_t stream) {
    ShootArgs a{x0, n, d, at, T, dt, sigma, order, regweight, xt, energy};
    a.dir = dir;
    a.eps = eps;
    a.at_try = at_try;
    a.nbatch = nbatch;
    return shoot_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_trial_batch_size(int64_t n, int d, int64_t nc, int64_t nc2, int shot_fp64, int value_fp64) {
    if (n < 1 || d < 2 || d > 3 || n > kFusedMaxPoints || !dt_fused_fits(nc, nc2)) return 1;
    // clusters of the batched shot and value kernels resident at once (the Gaussian
    // instances stand for the kernel family)
    auto shot = [&](auto D) {
        constexpr int D_ = decltype(D)::value;
        const FusedShape fs = fused_shape(n);
        return shot_fp64 ? fused_resident_clusters(shoot_fused_kernel<double, KGAUSS, 0, D_>, fs,
                                                   fused_dyn_smem<double>(n, D_), fused_dyn_smem<double>(kFusedMaxPoints, 3))
                         : fused_resident_clusters(shoot_fused_kernel<float, KGAUSS, 0, D_>, fs,
                                                   fused_dyn_smem<float>(n, D_), fused_dyn_smem<float>(kFusedMaxPoints, 3));
    };
    const int c = std::min(d == 2 ? shot(IC<2>{}) : shot(IC<3>{}), dt_value_resident_clusters(nc, nc2, d, value_fp64));
    return std::max(1, std::min(kTrialBatch, c));
}

size_t lddmm_covector_f32c_workspace(int64_t n, int d, int T) { return cov_ws<float>(n, d, T); }
size_t lddmm_covector_f64_workspace(int64_t n, int d, int T) { return cov_ws<double>(n, d, T); }

int lddmm_covector_f32c(const double* xt, int64_t n, int d, const double* at, int T, double dt, const double* px1,
                        double sigma, int order, double regweight, double* pxt, double* dat, void* workspace,
                        size_t workspace_bytes, lddmm_stream_t stream) {
    CovArgs a{xt, n, d, at, T, dt, px1, sigma, order, regweight, pxt, dat};
    return cov_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_covector_f64(const double* xt, int64_t n, int d, const double* at, int T, double dt, const double* px1,
                       double sigma, int order, double regweight, double* pxt, double* dat, void* workspace,
                       size_t workspace_bytes, lddmm_stream_t stream) {
    CovArgs a{xt, n, d, at, T, dt, px1, sigma, order, regweight, pxt, dat};
    return cov_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t lddmm_epdiff_f32c_workspace(int64_t n, int d, int T) { return epd_ws<float>(n, d, T); }
size_t lddmm_epdiff_f64_workspace(int64_t n, int d, int T) { return epd_ws<double>(n, d, T); }

int lddmm_epdiff_f32c(const double* x0, int64_t n, int d, const double* a0, int T, double sigma, int order,
                      double* xt, double* at, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    EPDArgs a{x0, n, d, a0, T, sigma, order, xt, at};
    return epd_entry<float>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

int lddmm_epdiff_f64(const double* x0, int64_t n, int d, const double* a0, int T, double sigma, int order,
                     double* xt, double* at, void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    EPDArgs a{x0, n, d, a0, T, sigma, order, xt, at};
    return epd_entry<double>(a, workspace, workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
