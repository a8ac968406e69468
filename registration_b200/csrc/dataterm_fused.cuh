// Single-launch data-term value for small shapes (at most kFusedMaxCells cells,
// and at most kFusedMaxCells * 2 kFusedMaxCells cell pairs: beyond that the
// pair sums keep the cluster's SMs busy for longer than the general path's
// launches over all SMs take; measured crossover about 512 cells per shape).
//
// NormDef (or Norm0 with no target cells) of the current / measure / varifold
// data terms (py-lddmm/surfaces.py:1009-1221, curves.py:539-650) in one
// kernel on one thread-block cluster (fused_small.cuh) instead of the cell
// geometry, bounding-box, pack, sweep, combine and finalize launches of the
// general path: the line search of a small curve or surface evaluates it a
// dozen times per iteration.
//
//   phase 1: every CTA computes the centres c of all S1 cells (from the
//            vertices) and S2 cells and takes the centre of their bounding box
//            as the packing frame (exact min / max: the same in every CTA);
//   phase 2: targets are the CTA's own S1 cells, with vector s (surfel or
//            tangent) and weight a = sqrt(|s|^2 + eps1);
//   phase 3: sources (S1 cells with sign +1, then S2 cells with sign -2) are
//            staged through shared memory in tiles; per target
//              current  z = sum_l K(c_k, c_l) <s_k, sign_l s_l>
//              measure  z = sum_l K(c_k, c_l) sign_l a_l
//              varifold z = sum_l K(c_k, c_l) (1 + <n_k, n_l>^2) sign_l a_l
//            (FP32 partials over 32 sources folded into TwoSum pairs, or
//            FP64), the source groups added in order in FP64;
//   phase 4: energy = sum_k w_k z_k (w = 1 current, a_k otherwise), a fixed
//            block tree per CTA, then the CTA partials in rank order.
#pragma once
#include "dataterm_ops.cuh"
#include "fused_small.cuh"

namespace lddmm {

#ifndef LDDMM_FUSED_MAX_CELLS
#define LDDMM_FUSED_MAX_CELLS 512
#endif
constexpr long long kFusedMaxCells = LDDMM_FUSED_MAX_CELLS;

// a value of nc own cells against nc2 target cells runs as one cluster launch
inline bool dt_fused_fits(long long nc, long long nc2) {
    return nc >= 1 && nc <= kFusedMaxCells && nc2 >= 0 && nc * (nc + nc2) <= 2 * kFusedMaxCells * kFusedMaxCells;
}

// step sizes of one batched trial-step launch at most (one cluster each): the
// clusters of a batch run side by side on the SMs that one cluster leaves idle
// (at 256 points, 24 clusters of 8 CTAs take the time of one)
constexpr int kTrialBatch = 24;

// clusters of the single-launch value kernel (Gaussian instance) for nc own and
// nc2 target cells that are resident at once (defined with the kernel's launches)
int dt_value_resident_clusters(long long nc, long long nc2, int d, int fp64);

template <class Real>
struct DtTile {
    static constexpr int N = sizeof(Real) == 4 ? 2048 : 1024;   // records per shared-memory tile
};

template <class Real>
LDDMM_D void dt_fused_record(FusedRec<Real>& r, const double* c, const double* s, int d, double eps, double sign,
                             int norm, double scale, const double* ctr) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double q = 0.0;
    for (int j = 0; j < d; ++j) q += s[j] * s[j];
    const double a = sqrt(q + eps);
    if (norm == NCURRENT) {
        for (int j = 0; j < d; ++j) v[j] = sign * s[j];
    } else if (norm == NMEASURE) {
        v[0] = sign * a;
    } else {
        for (int j = 0; j < 3; ++j) v[j] = s[j] / a;
        v[3] = sign * a;
    }
    fused_store<Real>(r, c, d, scale, ctr, v, 4);
}

// Centre c and vector s of cell l: l < nc a cell of S1 (from the vertices;
// invalid vertex indices give zero geometry), else target cell l - nc of S2.
template <int D>
LDDMM_D void dt_fused_cell(long long l, int ncorner, const double* v, long long nv, const int64_t* cells, long long nc,
                           const double* c2, const double* s2, double* c, double* s) {
    for (int j = 0; j < 3; ++j) c[j] = s[j] = 0.0;
    if (l >= nc) {
        for (int j = 0; j < D; ++j) {
            c[j] = c2[(l - nc) * D + j];
            s[j] = s2[(l - nc) * D + j];
        }
        return;
    }
    long long id[3] = {0, 0, 0};
    for (int q = 0; q < ncorner; ++q) {
        id[q] = cells[l * ncorner + q];
        if (id[q] < 0 || id[q] >= nv) return;
    }
    const double* x0 = v + id[0] * D;
    const double* x1 = v + id[1] * D;
    if (ncorner == 3) {
        const double* x2 = v + id[2] * D;
        for (int j = 0; j < 3; ++j) c[j] = (x0[j] + x1[j] + x2[j]) / 3;
        const double e1[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
        const double e2[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
        s[0] = e1[1] * e2[2] - e1[2] * e2[1];
        s[1] = e1[2] * e2[0] - e1[0] * e2[2];
        s[2] = e1[0] * e2[1] - e1[1] * e2[0];
    } else {
        for (int j = 0; j < D; ++j) {
            c[j] = (x0[j] + x1[j]) / 2;
            s[j] = x1[j] - x0[j];
        }
    }
}

// Packing frame of a data term: the centre of the bounding box of all cell
// centres of S1 (from the vertices) and S2 (exact min / max, the same in every
// CTA); block-wide, `scratch` holds 6 * kFusedThreads doubles.
template <int D>
LDDMM_D void dt_fused_frame(int ncorner, const double* v, long long nv, const int64_t* cells, long long nc,
                            const double* c2, const double* s2, long long nc2, double* scratch, double* ctr) {
    const int tid = threadIdx.x;
    const long long total = nc + nc2;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool any = false;
    for (long long l = tid; l < total; l += kFusedThreads) {
        double c[3], sv[3];
        dt_fused_cell<D>(l, ncorner, v, nv, cells, nc, c2, s2, c, sv);
        for (int j = 0; j < D; ++j) {
            lo[j] = any ? fmin(lo[j], c[j]) : c[j];
            hi[j] = any ? fmax(hi[j], c[j]) : c[j];
        }
        any = true;
    }
    for (int j = 0; j < 3; ++j) {
        scratch[(2 * j) * kFusedThreads + tid] = any ? lo[j] : INFINITY;
        scratch[(2 * j + 1) * kFusedThreads + tid] = any ? hi[j] : -INFINITY;
    }
    __syncthreads();
    for (int sh = kFusedThreads / 2; sh > 0; sh >>= 1) {
        if (tid < sh)
            for (int j = 0; j < 3; ++j) {
                double* L = scratch + (2 * j) * kFusedThreads;
                double* H = scratch + (2 * j + 1) * kFusedThreads;
                L[tid] = fmin(L[tid], L[tid + sh]);
                H[tid] = fmax(H[tid], H[tid + sh]);
            }
        __syncthreads();
    }
    for (int j = 0; j < 3; ++j)
        ctr[j] = j < D ? 0.5 * (scratch[(2 * j) * kFusedThreads] + scratch[(2 * j + 1) * kFusedThreads]) : 0.0;
    __syncthreads();
}

// Every CTA computes the cell geometry it needs itself (a few cached loads per
// cell), so the only cluster barrier is the one of the final energy sum.
template <class Real, int KIND, int PDEG, int D>
__global__ void __launch_bounds__(kFusedThreads)
    dt_value_fused_kernel(int ncorner, int norm, const double* __restrict__ v, long long nv,
                          const int64_t* __restrict__ cells, long long nc, const double* __restrict__ c2,
                          const double* __restrict__ s2, long long nc2, double eps1, double eps2, double scale,
                          FusedCoef cf, FusedShape fs, double* epart, double* energy, long long vstride,
                          int tile) {
    extern __shared__ __align__(32) unsigned char fused_smem[];
    FusedRec<Real>* rec = reinterpret_cast<FusedRec<Real>*>(fused_smem);
    double* red = reinterpret_cast<double*>(fused_smem + sizeof(FusedRec<Real>) * tile);
    double* scratch = red + kFusedThreads;
    const int rank = (int)cluster_rank();
    const int tid = threadIdx.x;
    const int local = tid % fs.tpt, g = tid / fs.tpt;
    const long long k = (long long)rank * fs.nc + local;
    const bool owner = local < fs.nc && k < nc;
    // batched values: cluster b evaluates the vertex set v + b vstride into energy[b]
    const long long b = blockIdx.x / fs.C;
    v += b * vstride;
    energy += b;
    epart += b * kFusedMaxCluster;
    Real pk[5];
    for (int j = 0; j < 5; ++j) pk[j] = (Real)cf.pk[j];
    const long long total = nc + nc2;
    double ctr[3];
    dt_fused_frame<D>(ncorner, v, nv, cells, nc, c2, s2, nc2, scratch, ctr);
    // the target cell of this thread
    Real xk[3] = {0, 0, 0}, uk[3] = {0, 0, 0};
    double wk = 0.0;
    if (owner) {
        double ck[3], sk[3], q = 0.0;
        dt_fused_cell<D>(k, ncorner, v, nv, cells, nc, c2, s2, ck, sk);
        for (int j = 0; j < D; ++j) {
            xk[j] = (Real)((ck[j] - ctr[j]) * scale);
            q += sk[j] * sk[j];
        }
        const double ak = sqrt(q + eps1);
        if (norm == NCURRENT) {
            for (int j = 0; j < D; ++j) uk[j] = (Real)sk[j];
            wk = 1.0;
        } else {
            for (int j = 0; j < 3; ++j) uk[j] = (Real)(sk[j] / ak);
            wk = ak;
        }
    }
    // sources in tiles: S1 cells (sign +1), then S2 cells (sign -2)
    FusedAcc<Real, 1> acc;
    acc.zero();
    constexpr int FOLD = sizeof(Real) == 4 ? 32 : 1 << 30;
    for (long long t0 = 0; t0 < total; t0 += tile) {
        const int len = (int)(total - t0 < tile ? total - t0 : tile);
        for (int i = tid; i < len; i += kFusedThreads) {
            const long long l = t0 + i;
            double c[3], sv[3];
            dt_fused_cell<D>(l, ncorner, v, nv, cells, nc, c2, s2, c, sv);
            dt_fused_record<Real>(rec[i], c, sv, D, l < nc ? eps1 : eps2, l < nc ? 1.0 : -2.0, norm, scale, ctr);
        }
        __syncthreads();
        if (owner) {
            const int jb0 = (int)((long long)g * len / fs.S), je0 = (int)((long long)(g + 1) * len / fs.S);
            for (int jb = jb0; jb < je0; jb += FOLD) {
                acc.begin_fold();
                const int je = jb + FOLD < je0 ? jb + FOLD : je0;
#pragma unroll kFusedUnroll
                for (int j = jb; j < je; ++j) {
                    Real y[3], w[6];
                    fused_pos<Real>(rec[j], y);
                    fused_vals<Real>(rec[j], w);
                    Real r2 = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        const Real dq = xk[q] - y[q];
                        r2 = q == 0 ? dq * dq : r2 + dq * dq;
                    }
                    const Real kv = fused_k<Real, KIND, PDEG>(pk, r2);
                    Real term;
                    if (norm == NCURRENT) {
                        Real dot = 0;
#pragma unroll
                        for (int q = 0; q < D; ++q) dot = q == 0 ? uk[0] * w[0] : dot + uk[q] * w[q];
                        term = dot;
                    } else if (norm == NMEASURE) {
                        term = w[0];
                    } else {
                        const Real dn = uk[0] * w[0] + uk[1] * w[1] + uk[2] * w[2];
                        term = ((Real)1 + dn * dn) * w[3];
                    }
                    acc.fma(0, kv, term);
                }
                acc.end_fold();
            }
        }
        __syncthreads();
    }
    // energy = sum_k w_k z_k: source groups in order, a fixed block tree, the CTAs in rank order
    if (owner) red[g * fs.tpt + local] = acc.value(0);
    __syncthreads();
    double e = 0.0;
    if (owner && g == 0) {
        double z = 0.0;
        for (int gg = 0; gg < fs.S; ++gg) z += red[gg * fs.tpt + local];
        e = wk * z;
    }
    e = fused_block_sum(e, scratch);
    if (tid == 0) __stcg(epart + rank, e);
    cluster_sync_acq_rel();
    if (rank == 0 && tid == 0) {
        double sum = 0.0;
        for (int r = 0; r < fs.C; ++r) sum += __ldcg(epart + r);
        energy[0] = sum;
    }
}

// Single-launch data-term GRADIENT (NormGradient, surfaces.py:1069-1087,
// 1150-1182, 1228-1276; curves.py:594-650) for small shapes: the pair sums of
// the general path's gradient sweep (targets: the S1 cells, sources: S1 with
// sign +1 and S2 with sign -1) for each CTA's own cells, the per-cell z1 / dz1
// (dt_grad_row) into global memory, one cluster barrier, then the vertex
// gather of each CTA's share of the vertices (dt_gather_vertex).
constexpr int kDtGradOut = 7;   // accumulators: 2 d + 1 at most

template <class Real, int KIND, int PDEG, int QDEG, int D>
__global__ void __launch_bounds__(kFusedThreads)
    dt_grad_fused_kernel(int ncorner, int norm, const double* __restrict__ v, long long nv,
                         const int64_t* __restrict__ cells, long long nc, const double* __restrict__ c2,
                         const double* __restrict__ s2, long long nc2, double eps1, double eps2, double scale,
                         double dzscale, FusedCoef cf, FusedShape fs, int tile, const int64_t* __restrict__ vptr,
                         const int64_t* __restrict__ vidx, double* z1, double* dz1, double* __restrict__ px) {
    extern __shared__ __align__(32) unsigned char fused_smem[];
    FusedRec<Real>* rec = reinterpret_cast<FusedRec<Real>*>(fused_smem);
    double* red = reinterpret_cast<double*>(fused_smem + sizeof(FusedRec<Real>) * tile);
    double* scratch = red + kFusedThreads * kDtGradOut;
    const int rank = (int)cluster_rank();
    const int tid = threadIdx.x;
    const int local = tid % fs.tpt, g = tid / fs.tpt;
    const long long k = (long long)rank * fs.nc + local;
    const bool owner = local < fs.nc && k < nc;
    Real pk[5], pq[4];
    for (int j = 0; j < 5; ++j) pk[j] = (Real)cf.pk[j];
    for (int j = 0; j < 4; ++j) pq[j] = (Real)cf.pq[j];
    const long long total = nc + nc2;
    double ctr[3];
    dt_fused_frame<D>(ncorner, v, nv, cells, nc, c2, s2, nc2, scratch, ctr);
    // the target cell of this thread: position, and s (current) or n = s / a (varifold)
    Real xk[3] = {0, 0, 0}, uk[3] = {0, 0, 0};
    double sk[3] = {0, 0, 0};
    if (owner) {
        double ck[3], q = 0.0;
        dt_fused_cell<D>(k, ncorner, v, nv, cells, nc, c2, s2, ck, sk);
        for (int j = 0; j < D; ++j) {
            xk[j] = (Real)((ck[j] - ctr[j]) * scale);
            q += sk[j] * sk[j];
        }
        const double ak = sqrt(q + eps1);
        for (int j = 0; j < 3; ++j) uk[j] = (Real)(norm == NCURRENT ? sk[j] : sk[j] / ak);
    }
    FusedAcc<Real, kDtGradOut> acc;
    acc.zero();
    constexpr int FOLD = sizeof(Real) == 4 ? 32 : 1 << 30;
    for (long long t0 = 0; t0 < total; t0 += tile) {
        const int len = (int)(total - t0 < tile ? total - t0 : tile);
        for (int i = tid; i < len; i += kFusedThreads) {
            const long long l = t0 + i;
            double c[3], sv[3];
            dt_fused_cell<D>(l, ncorner, v, nv, cells, nc, c2, s2, c, sv);
            dt_fused_record<Real>(rec[i], c, sv, D, l < nc ? eps1 : eps2, l < nc ? 1.0 : -1.0, norm, scale, ctr);
        }
        __syncthreads();
        if (owner) {
            const int jb0 = (int)((long long)g * len / fs.S), je0 = (int)((long long)(g + 1) * len / fs.S);
            for (int jb = jb0; jb < je0; jb += FOLD) {
                acc.begin_fold();
                const int je = jb + FOLD < je0 ? jb + FOLD : je0;
                for (int j = jb; j < je; ++j) {
                    Real y[3], w[6], dx[3];
                    fused_pos<Real>(rec[j], y);
                    fused_vals<Real>(rec[j], w);
                    Real r2 = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        dx[q] = xk[q] - y[q];
                        r2 = q == 0 ? dx[q] * dx[q] : r2 + dx[q] * dx[q];
                    }
                    Real kv, fv;
                    kboth<Real, KIND, PDEG, QDEG>(pk, pq, r2, kv, fv);
                    if (norm == NVARIFOLD) {
                        const Real dn = uk[0] * w[0] + uk[1] * w[1] + uk[2] * w[2];
                        const Real wk = kv * w[3];
                        const Real ca = 2 * dn * wk;
#pragma unroll
                        for (int q = 0; q < D; ++q) acc.fma(q, ca, w[q]);
                        acc.fma(D, wk, (Real)1 - dn * dn);
                        const Real wf = fv * w[3] * ((Real)1 + dn * dn);
#pragma unroll
                        for (int q = 0; q < D; ++q) acc.fma(D + 1 + q, wf, dx[q]);
                    } else if (norm == NCURRENT) {
                        Real dot = 0;
#pragma unroll
                        for (int q = 0; q < D; ++q) {
                            acc.fma(q, kv, w[q]);
                            dot = q == 0 ? uk[0] * w[0] : dot + uk[q] * w[q];
                        }
                        const Real gq = fv * dot;
#pragma unroll
                        for (int q = 0; q < D; ++q) acc.fma(D + q, gq, dx[q]);
                    } else {
                        acc.fma(0, kv, w[0]);
                        const Real gq = fv * w[0];
#pragma unroll
                        for (int q = 0; q < D; ++q) acc.fma(1 + q, gq, dx[q]);
                    }
                }
                acc.end_fold();
            }
        }
        __syncthreads();
    }
    // z1 / dz1 of the target cell: source groups in order, in FP64
    if (owner)
#pragma unroll
        for (int c = 0; c < kDtGradOut; ++c) red[(g * fs.tpt + local) * kDtGradOut + c] = acc.value(c);
    __syncthreads();
    if (owner && g == 0) {
        double a[kDtGradOut];
        for (int c = 0; c < kDtGradOut; ++c) {
            a[c] = 0.0;
            for (int gg = 0; gg < fs.S; ++gg) a[c] += red[(gg * fs.tpt + local) * kDtGradOut + c];
        }
        double z[3], dz[3];
        dt_grad_row(norm, a, sk, D, eps1, dzscale, z, dz);
        for (int j = 0; j < D; ++j) {
            __stcg(z1 + k * D + j, z[j]);
            __stcg(dz1 + k * D + j, dz[j]);
        }
    }
    cluster_sync_acq_rel();
    // the vertex gather: vertices [rank nv / C, (rank + 1) nv / C)
    const long long q0 = (long long)rank * nv / fs.C, q1 = (long long)(rank + 1) * nv / fs.C;
    for (long long q = q0 + tid; q < q1; q += kFusedThreads)
        dt_gather_vertex<true>(q, ncorner, v, nv, D, cells, nc, vptr, vidx, z1, dz1, px);
}

template <class Real>
inline size_t dt_grad_fused_smem(int tile) {
    return sizeof(FusedRec<Real>) * (size_t)tile + sizeof(double) * kFusedThreads * (kDtGradOut + 6);
}

// source records per shared-memory tile for `total` source cells: all of them
// when they fit (a smaller footprint lets more CTAs share an SM), else DtTile::N
template <class Real>
inline int dt_fused_tile(long long total) {
    const long long t = (total + 31) / 32 * 32;
    return (int)(t < DtTile<Real>::N ? t : DtTile<Real>::N);
}

template <class Real>
inline size_t dt_fused_smem(long long total) {
    return sizeof(FusedRec<Real>) * (size_t)dt_fused_tile<Real>(total) + sizeof(double) * kFusedThreads * 7;
}

}  // namespace lddmm
