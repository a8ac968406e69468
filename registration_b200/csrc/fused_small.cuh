// Single-launch geodesic shooting and Hamiltonian adjoint for small point sets.
//
// For n <= kFusedMaxPoints the T Euler steps of landmarkDirectEvolutionEuler
// (py-lddmm/pointEvolution.py:666-730) and the T backward steps of
// landmarkHamiltonianCovector (pointEvolution.py:735-765) each run as ONE
// kernel on one thread-block cluster of C <= 8 CTAs instead of a sweep and a
// combine launch per step (plus bounding-box and pack launches): at a few
// hundred points every launch is a few microseconds of mostly idle GPU.
// Beyond about 512 points the n^2 pair sums of a step keep the cluster's 8
// SMs busy for longer than the general path's launches over all SMs take
// (measured on B200 at T = 10: 59 vs 82 us per shot at 512 points, 120 vs
// 89 us at 768), so the limit is 512.
//
// Work split: C = min(8, ceil(n / 32)) CTAs; CTA r of the cluster owns the
// targets [r*nc, (r+1)*nc), nc = ceil(n / C) <= 64.  Its 512 threads are tpt
// target slots (tpt = the next power of two >= nc) times S = 512 / tpt source
// groups; group g sums the sources [g*n/S, (g+1)*n/S) of its target (FP32
// partials over 32 sources folded into TwoSum pairs, or plain FP64), and the
// S group sums of a target are added in group order in FP64.  Every result is
// a function of the shape and the data only (no atomics), so repeated calls
// are bit-identical.
//
// Step t: every CTA sums over the n source records (position in the packing
// frame, weights) of the step held in its shared memory; the slot-0 thread of
// each target applies the FP64 update, stores the next state row in global
// memory (the output) and writes the target's next-step record into the
// shared memory of every CTA of the cluster (distributed shared memory,
// double-buffered).  A cluster barrier (arrive.release / wait.acquire) per
// step orders those writes.  The packing frame is the centre of the bounding
// box of the initial points (min / max exact in FP64, computed by every CTA
// over all points, so every CTA uses the same centre).
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "host.h"
#include "kfun.cuh"
#include "sweep.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

#ifndef LDDMM_FUSED_THREADS
#define LDDMM_FUSED_THREADS 512
#endif
#ifndef LDDMM_FUSED_UNROLL
#define LDDMM_FUSED_UNROLL 1
#endif
constexpr int kFusedThreads = LDDMM_FUSED_THREADS;
constexpr int kFusedUnroll = LDDMM_FUSED_UNROLL;   // inner source loop
#ifndef LDDMM_FUSED_MAX_POINTS
#define LDDMM_FUSED_MAX_POINTS 512
#endif
constexpr long long kFusedMaxPoints = LDDMM_FUSED_MAX_POINTS;
constexpr int kFusedMaxCluster = 8;
// targets per CTA before the cluster grows: every CTA of a full cluster then
// owns <= 64 targets, each target spread over >= 8 source groups
#ifndef LDDMM_FUSED_TPC
#define LDDMM_FUSED_TPC 32
#endif
constexpr int kFusedTargetsPerCta = LDDMM_FUSED_TPC;

struct FusedShape {
    int C;    // CTAs in the cluster
    int nc;   // targets per CTA
    int tpt;  // target slots per CTA (power of two >= nc)
    int S;    // source groups
};

inline FusedShape fused_shape(long long n) {
    FusedShape f;
    f.C = (int)std::max(1LL, std::min<long long>(kFusedMaxCluster, (n + kFusedTargetsPerCta - 1) / kFusedTargetsPerCta));
    f.nc = (int)((n + f.C - 1) / f.C);
    f.tpt = 1;
    while (f.tpt < f.nc) f.tpt <<= 1;
    f.S = kFusedThreads / f.tpt;
    return f;
}

LDDMM_D unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
LDDMM_D unsigned cluster_size() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// All threads of every CTA of the cluster: prior memory operations (global and
// shared) are visible to the cluster after the wait.
LDDMM_D void cluster_sync_acq_rel() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// FP64 loads of state written by other CTAs of the cluster in this launch: L2 only.
LDDMM_D double ldcg(const double* p) { return __ldcg(p); }

// Centre of the bounding box of x[0..n) (d coordinates) into c[0..3); block-wide,
// `scratch` holds 2 * 3 * kFusedThreads doubles.
LDDMM_D void fused_bbox_center(const double* x, long long n, int d, double* scratch, double* c) {
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool any = false;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        for (int j = 0; j < d; ++j) {
            const double v = x[i * d + j];
            lo[j] = any ? fmin(lo[j], v) : v;
            hi[j] = any ? fmax(hi[j], v) : v;
        }
        any = true;
    }
    for (int j = 0; j < 3; ++j) {
        scratch[(2 * j) * kFusedThreads + threadIdx.x] = any ? lo[j] : INFINITY;
        scratch[(2 * j + 1) * kFusedThreads + threadIdx.x] = any ? hi[j] : -INFINITY;
    }
    __syncthreads();
    for (int s = kFusedThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int j = 0; j < 3; ++j) {
                double* L = scratch + (2 * j) * kFusedThreads;
                double* H = scratch + (2 * j + 1) * kFusedThreads;
                L[threadIdx.x] = fmin(L[threadIdx.x], L[threadIdx.x + s]);
                H[threadIdx.x] = fmax(H[threadIdx.x], H[threadIdx.x + s]);
            }
        }
        __syncthreads();
    }
    for (int j = 0; j < 3; ++j)
        c[j] = j < d ? 0.5 * (scratch[(2 * j) * kFusedThreads] + scratch[(2 * j + 1) * kFusedThreads]) : 0.0;
    __syncthreads();
}

// FP64 block sum with a fixed tree (thread 0 gets the total); scratch >= kFusedThreads doubles.
LDDMM_D double fused_block_sum(double v, double* scratch) {
    scratch[threadIdx.x] = v;
    __syncthreads();
    for (int s = kFusedThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) scratch[threadIdx.x] += scratch[threadIdx.x + s];
        __syncthreads();
    }
    const double r = scratch[0];
    __syncthreads();
    return r;
}

template <class Real>
struct FusedRec;  // one packed record: position and up to 8 values
template <>
struct FusedRec<float> {
    float4 p, v0, v1;
};
template <>
struct FusedRec<double> {
    double4a p, v0, v1;
};

template <class Real>
LDDMM_D void fused_store(FusedRec<Real>& r, const double* pos, int d, double s, const double* c, const double* v,
                         int nv) {
    Real q[4] = {0, 0, 0, 0}, w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < d; ++j) q[j] = (Real)((pos[j] - c[j]) * s);
    for (int j = 0; j < nv; ++j) w[j] = (Real)v[j];
    if constexpr (sizeof(Real) == 4) {
        r.p = make_float4(q[0], q[1], q[2], 0.f);
        r.v0 = make_float4(w[0], w[1], w[2], w[3]);
        r.v1 = make_float4(w[4], w[5], w[6], w[7]);
    } else {
        r.p = double4a{q[0], q[1], q[2], 0.0};
        r.v0 = double4a{w[0], w[1], w[2], w[3]};
        r.v1 = double4a{w[4], w[5], w[6], w[7]};
    }
}

template <class Real>
LDDMM_D void fused_pos(const FusedRec<Real>& r, Real* x) {
    x[0] = r.p.x;
    x[1] = r.p.y;
    x[2] = r.p.z;
}
template <class Real>
LDDMM_D void fused_vals(const FusedRec<Real>& r, Real* v) {
    v[0] = r.v0.x;
    v[1] = r.v0.y;
    v[2] = r.v0.z;
    v[3] = r.v0.w;
    v[4] = r.v1.x;
    v[5] = r.v1.y;
}

template <class Real, int KIND, int DEG>
LDDMM_D Real fused_k(const Real* pk, Real r2) {
    if constexpr (sizeof(Real) == 4) return kval32<KIND, DEG>(pk, r2);
    else return kval64<KIND, DEG>(pk, r2);
}
template <class Real, int KIND, int QDEG>
LDDMM_D Real fused_kd(const Real* pq, Real r2) {
    if constexpr (sizeof(Real) == 4) return kdiff32<KIND, QDEG>(pq, r2);
    else return kdiff64<KIND, QDEG>(pq, r2);
}

template <class Real, int N>
using FusedAcc = std::conditional_t<sizeof(Real) == 4, AccF32C<N>, AccF64<N>>;

struct FusedCoef {
    double pk[5];
    double pq[4];
};

// The record `r` into the same slot `slot` of every CTA's shared memory
// (distributed shared memory of the cluster), 16 bytes at a time.
template <class Real>
LDDMM_D void fused_broadcast(const FusedRec<Real>& r, FusedRec<Real>* slot, int C) {
    constexpr int W = sizeof(FusedRec<Real>) / 16;
    const uint4* src = reinterpret_cast<const uint4*>(&r);
    const unsigned laddr = (unsigned)__cvta_generic_to_shared(slot);
    for (int q = 0; q < C; ++q) {
        unsigned raddr;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(raddr) : "r"(laddr), "r"(q));
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint4 v = src[w];
            asm volatile("st.shared::cluster.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(raddr + 16 * w), "r"(v.x),
                         "r"(v.y), "r"(v.z), "r"(v.w)
                         : "memory");
        }
    }
}

// ---- shooting: xt[t+1] = xt[t] + dt K(xt[t]) at[t]; energy = rw dt sum_t <at[t], K at[t]> ----
// Source records are double-buffered: step t reads buffer t & 1, and the owner
// of each target writes its step-(t+1) record into buffer (t+1) & 1 of every
// CTA; the cluster barrier at the end of step t orders those writes before the
// reads of step t+1 and after every read of step t-1.
// Momentum of the shot: at[i], or, with a search direction, at[i] - eps dir[i] (the
// trial step of a line search), rounded as the two separate FP64 operations.
LDDMM_D double shot_momentum(const double* at, const double* dir, double eps, long long i) {
    return dir == nullptr ? at[i] : __dsub_rn(at[i], __dmul_rn(eps, dir[i]));
}

template <class Real, int KIND, int DEG, int D>
__global__ void __launch_bounds__(kFusedThreads) shoot_fused_kernel(const double* __restrict__ x0,
                                                                    const double* __restrict__ at, long long n,
                                                                    int T, double dt, double scale, FusedCoef cf,
                                                                    double rw, FusedShape fs, double* xt,
                                                                    double* energy, double* epart,
                                                                    const double* __restrict__ dir,
                                                                    const double* __restrict__ epsp,
                                                                    double* at_try) {
    extern __shared__ __align__(32) unsigned char fused_smem[];
    FusedRec<Real>* rec0 = reinterpret_cast<FusedRec<Real>*>(fused_smem);
    FusedRec<Real>* rec1 = rec0 + n;
    double* red = reinterpret_cast<double*>(fused_smem + 2 * sizeof(FusedRec<Real>) * n);
    double* scratch = red + kFusedThreads * D;
    const int rank = (int)cluster_rank();
    const int tid = threadIdx.x;
    const int local = tid % fs.tpt, g = tid / fs.tpt;
    const long long k = (long long)rank * fs.nc + local;
    const bool owner = local < fs.nc && k < n;
    const long long j0 = g * n / fs.S, j1 = (g + 1) * n / fs.S;
    const long long N = n * D;
    // batched trial steps: cluster b shoots at - eps[b] dir into slot b of the outputs
    const long long b = blockIdx.x / fs.C;
    xt += b * (T + 1) * N;
    epart += b * kFusedMaxCluster;
    if (energy != nullptr) energy += b;
    if (at_try != nullptr) at_try += b * T * N;
    Real pk[5];
    for (int j = 0; j < 5; ++j) pk[j] = (Real)cf.pk[j];
    double c[3];
    fused_bbox_center(x0, n, D, scratch, c);
    const double eps = dir != nullptr ? epsp[b] : 0.0;
    for (long long i = tid; i < n; i += kFusedThreads) {
        double a0[3];
        for (int j = 0; j < D; ++j) a0[j] = shot_momentum(at, dir, eps, i * D + j);
        fused_store<Real>(rec0[i], x0 + i * D, D, scale, c, a0, D);
    }
    double xk64[3] = {0, 0, 0};
    if (owner && g == 0)
        for (int j = 0; j < D; ++j) xk64[j] = x0[k * D + j];
    // every CTA's buffer 0 is complete before any CTA's owners overwrite its buffer 1
    cluster_sync_acq_rel();
    double e_acc = 0.0;
    for (int t = 0; t < T; ++t) {
        const FusedRec<Real>* rec = (t & 1) ? rec1 : rec0;
        FusedRec<Real>* nxt = (t & 1) ? rec0 : rec1;
        // slot 0: store the row x_t of the output (off the critical path: the next cluster
        // barrier's release is a step away) and prefetch the momenta the update needs
        double a_now[3] = {0, 0, 0}, a_next[3] = {0, 0, 0};
        if (owner && g == 0) {
            for (int j = 0; j < D; ++j) {
                xt[(long long)t * N + k * D + j] = xk64[j];
                a_now[j] = shot_momentum(at, dir, eps, (long long)t * N + k * D + j);
                if (t + 1 < T) a_next[j] = shot_momentum(at, dir, eps, (long long)(t + 1) * N + k * D + j);
                if (at_try != nullptr) at_try[(long long)t * N + k * D + j] = a_now[j];
            }
        }
        if (owner) {
            Real xk[3];
            fused_pos<Real>(rec[k], xk);
            FusedAcc<Real, D> acc;
            acc.zero();
            constexpr int FOLD = sizeof(Real) == 4 ? 32 : 1 << 30;
            for (long long jb = j0; jb < j1; jb += FOLD) {
                acc.begin_fold();
                const long long je = jb + FOLD < j1 ? jb + FOLD : j1;
#pragma unroll kFusedUnroll
                for (long long j = jb; j < je; ++j) {
                    Real y[3], w[6];
                    fused_pos<Real>(rec[j], y);
                    fused_vals<Real>(rec[j], w);
                    Real r2 = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        const Real dq = xk[q] - y[q];
                        r2 = q == 0 ? dq * dq : r2 + dq * dq;
                    }
                    const Real kv = fused_k<Real, KIND, DEG>(pk, r2);
#pragma unroll
                    for (int q = 0; q < D; ++q) acc.fma(q, kv, w[q]);
                }
                acc.end_fold();
            }
#pragma unroll
            for (int q = 0; q < D; ++q) red[(g * fs.tpt + local) * D + q] = acc.value(q);
        }
        __syncthreads();
        if (owner && g == 0) {
            for (int q = 0; q < D; ++q) {
                double v = 0.0;
                for (int gg = 0; gg < fs.S; ++gg) v += red[(gg * fs.tpt + local) * D + q];
                e_acc += a_now[q] * v;
                xk64[q] = xk64[q] + dt * v;
            }
            if (t + 1 < T) {
                FusedRec<Real> r;
                fused_store<Real>(r, xk64, D, scale, c, a_next, D);
                fused_broadcast<Real>(r, nxt + k, fs.C);
            }
        }
        cluster_sync_acq_rel();
    }
    if (owner && g == 0)
        for (int j = 0; j < D; ++j) xt[(long long)T * N + k * D + j] = xk64[j];
    if (energy != nullptr) {
        const double e = fused_block_sum(e_acc, scratch);
        if (tid == 0) __stcg(epart + rank, e);
        cluster_sync_acq_rel();
        if (rank == 0 && tid == 0) {
            double sum = 0.0;
            for (int r = 0; r < fs.C; ++r) sum += __ldcg(epart + r);
            energy[0] = rw * dt * sum;
        }
    }
}

// ---- adjoint: pxt[T] = px1; pxt[t] = pxt[t+1] + dt dscale sum_l F(x_k, x_l) (x'_k - x'_l) <u_k, v_l>,
//      u = (p - 2 rw a, a), v = (a, p) with p = pxt[t+1], a = at[t]; dat[t] = 2 rw at[t] - pxt[t+1] ----
// Records of step t: position x_t, values (a_t, p_{t+1}); double-buffered as in the shot.
template <class Real, int KIND, int QDEG, int D>
__global__ void __launch_bounds__(kFusedThreads) cov_fused_kernel(const double* __restrict__ xt,
                                                                  const double* __restrict__ at,
                                                                  const double* __restrict__ px1, long long n, int T,
                                                                  double dt, double scale, double dscale,
                                                                  FusedCoef cf, double rw, FusedShape fs, double* pxt,
                                                                  double* dat) {
    extern __shared__ __align__(32) unsigned char fused_smem[];
    FusedRec<Real>* rec0 = reinterpret_cast<FusedRec<Real>*>(fused_smem);
    FusedRec<Real>* rec1 = rec0 + n;
    double* red = reinterpret_cast<double*>(fused_smem + 2 * sizeof(FusedRec<Real>) * n);
    double* scratch = red + kFusedThreads * D;
    const int rank = (int)cluster_rank();
    const int tid = threadIdx.x;
    const int local = tid % fs.tpt, g = tid / fs.tpt;
    const long long k = (long long)rank * fs.nc + local;
    const bool owner = local < fs.nc && k < n;
    const long long j0 = g * n / fs.S, j1 = (g + 1) * n / fs.S;
    Real pq[4];
    for (int j = 0; j < 4; ++j) pq[j] = (Real)cf.pq[j];
    double c[3];
    fused_bbox_center(xt, n, D, scratch, c);   // frame of the trajectory's first step
    const long long N = n * D;
    {
        const double* xs = xt + (long long)(T - 1) * N;
        const double* as = at + (long long)(T - 1) * N;
        for (long long i = tid; i < n; i += kFusedThreads) {
            double v[6];
            for (int j = 0; j < D; ++j) {
                v[j] = as[i * D + j];
                v[D + j] = px1[i * D + j];
            }
            fused_store<Real>(rec0[i], xs + i * D, D, scale, c, v, 2 * D);
        }
    }
    // p_{t+1} of this CTA's targets in FP64, shared by their source groups
    double* pown = scratch;   // fs.tpt * 3 doubles (the bounding-box scratch is free again)
    double pn[3] = {0, 0, 0};   // slot 0: the target's p_{t+1}
    if (owner && g == 0)
        for (int j = 0; j < D; ++j) {
            pn[j] = px1[k * D + j];
            pxt[(long long)T * N + k * D + j] = pn[j];
            pown[local * 3 + j] = pn[j];
        }
    cluster_sync_acq_rel();
    // slot 0 stores step t's rows of pxt and dat at the start of step t - 1 (off the
    // critical path: the release of the next cluster barrier is a step away)
    int pend = -1;
    double pend_p[3] = {0, 0, 0}, pend_d[3] = {0, 0, 0};
    auto flush = [&]() {
        if (pend >= 0)
            for (int q = 0; q < D; ++q) {
                pxt[(long long)pend * N + k * D + q] = pend_p[q];
                if (dat != nullptr) dat[(long long)pend * N + k * D + q] = pend_d[q];
            }
        pend = -1;
    };
    int b = 0;
    for (int t = T - 1; t >= 0; --t, b ^= 1) {
        const FusedRec<Real>* rec = b ? rec1 : rec0;
        FusedRec<Real>* nxt = b ? rec0 : rec1;
        const double* as = at + (long long)t * N;
        if (owner && g == 0) flush();
        if (owner) {
            Real xk[3], u[6];
            fused_pos<Real>(rec[k], xk);
            // u_k = (p - 2 rw a, a) in FP64, then rounded
            for (int j = 0; j < D; ++j) {
                const double aj = as[k * D + j];
                u[j] = (Real)(pown[local * 3 + j] - 2.0 * rw * aj);
                u[D + j] = (Real)aj;
            }
            FusedAcc<Real, D> acc;
            acc.zero();
            constexpr int FOLD = sizeof(Real) == 4 ? 32 : 1 << 30;
            for (long long jb = j0; jb < j1; jb += FOLD) {
                acc.begin_fold();
                const long long je = jb + FOLD < j1 ? jb + FOLD : j1;
#pragma unroll kFusedUnroll
                for (long long j = jb; j < je; ++j) {
                    Real y[3], w[6], dx[3];
                    fused_pos<Real>(rec[j], y);
                    fused_vals<Real>(rec[j], w);
                    Real r2 = 0, dot = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        dx[q] = xk[q] - y[q];
                        r2 = q == 0 ? dx[q] * dx[q] : r2 + dx[q] * dx[q];
                    }
#pragma unroll
                    for (int q = 0; q < 2 * D; ++q) dot = q == 0 ? u[0] * w[0] : dot + u[q] * w[q];
                    const Real gv = fused_kd<Real, KIND, QDEG>(pq, r2) * dot;
#pragma unroll
                    for (int q = 0; q < D; ++q) acc.fma(q, gv, dx[q]);
                }
                acc.end_fold();
            }
#pragma unroll
            for (int q = 0; q < D; ++q) red[(g * fs.tpt + local) * D + q] = acc.value(q);
        }
        __syncthreads();
        if (owner && g == 0) {
            double pc[3];
            for (int q = 0; q < D; ++q) {
                double f = 0.0;
                for (int gg = 0; gg < fs.S; ++gg) f += red[(gg * fs.tpt + local) * D + q];
                pc[q] = pn[q] + dt * (dscale * f);
            }
            if (t > 0) {
                double v[6];
                for (int j = 0; j < D; ++j) {
                    v[j] = as[-N + k * D + j];
                    v[D + j] = pc[j];
                }
                FusedRec<Real> r;
                fused_store<Real>(r, xt + (long long)(t - 1) * N + k * D, D, scale, c, v, 2 * D);
                fused_broadcast<Real>(r, nxt + k, fs.C);
            }
            for (int q = 0; q < D; ++q) {
                pend_d[q] = 2.0 * rw * as[k * D + q] - pn[q];
                pend_p[q] = pc[q];
                pown[local * 3 + q] = pc[q];
                pn[q] = pc[q];
            }
            pend = t;
        }
        cluster_sync_acq_rel();
    }
    if (owner && g == 0) flush();
}

template <class Real>
inline size_t fused_dyn_smem(long long n, int D) {
    return 2 * sizeof(FusedRec<Real>) * (size_t)n + sizeof(double) * kFusedThreads * (size_t)D +
           sizeof(double) * 6 * kFusedThreads;
}

// Launches `kernel` on `nbatch` clusters of fs.C CTAs (cluster b works on
// problem b of a batch) with `smem` bytes of dynamic shared memory
// (`max_smem`: the kernel's opt-in limit, at least smem).
// The shared-memory opt-in of a fused kernel, once per (device, kernel).
template <class Kern>
int fused_prepare(Kern kernel, size_t max_smem) {
    static std::mutex mu;
    static std::set<std::pair<int, const void*>> done;
    int dev = 0;
    LDDMM_TRY(cuda_check(cudaGetDevice(&dev), "fused: cudaGetDevice"));
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(dev, reinterpret_cast<const void*>(kernel));
    if (done.count(key) == 0) {
        LDDMM_TRY(cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem),
                             "fused kernel attribute"));
        done.insert(key);
    }
    return LDDMM_OK;
}

// cluster launch configuration: nbatch clusters of fs.C CTAs; attr must outlive cfg
inline cudaLaunchConfig_t fused_config(const FusedShape& fs, int nbatch, size_t smem, cudaStream_t st,
                                       cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(fs.C * nbatch, 1, 1);
    cfg.blockDim = dim3(kFusedThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = fs.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <class Kern, class... Args>
int launch_fused(Kern kernel, const FusedShape& fs, int nbatch, size_t smem, size_t max_smem, cudaStream_t st,
                 Args... args) {
    LDDMM_TRY(fused_prepare(kernel, max_smem));
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = fused_config(fs, nbatch, smem, st, attr);
    return cuda_check(cudaLaunchKernelEx(&cfg, kernel, args...), "fused launch");
}

// How many clusters of `kernel` (fs.C CTAs, smem bytes each) are resident on the device at once
// (0 on error).
template <class Kern>
int fused_resident_clusters(Kern kernel, const FusedShape& fs, size_t smem, size_t max_smem) {
    if (fused_prepare(kernel, max_smem) != LDDMM_OK) return 0;
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = fused_config(fs, 1, smem, 0, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return clusters;
}

}  // namespace lddmm
