// Ragged (multi-request) launches for the serving engine: one launch sweeps
// the kernel sums of many independent problems of different sizes.
//
//   lddmm_ragged_shoot_f32c     shooting + regularisation energy of every request
//   lddmm_ragged_covector_f32c  Hamiltonian adjoint of every request
//   lddmm_ragged_applyk_f32c    independent applyK segments (K-metric dot products)
//   lddmm_ragged_dataterm_*     data-term values / gradients of every request
//
// Segment s owns its rows (offsets from the host), its own kernel width, its
// own source-chunk count and its own FP64 reduction tree, all functions of the
// segment's own shape only: a request's results are bit-identical whatever
// other requests share the launch.  Reference formulas: as the single-problem
// entry points (pointEvolution.py:666-817, kernelFunctions.f90:1-54,
// surfaces.py:1009-1276).
#include <type_traits>
#include <vector>

#include "dataterm_ops.cuh"
#include "host.h"
#include "ops2.cuh"
#include "pack.cuh"
#include "sweep_dispatch.cuh"

namespace lddmm {

constexpr int kRagThreads = 256;

// largest s with off[s] <= r (off has nseg+1 entries, off[0] = 0)
LDDMM_D int seg_lookup(const long long* off, int nseg, long long r) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per-segment device table of the ragged launches.
struct RagSeg {
    long long row0;      // first real row (points / cells) in the concatenated arrays
    long long n;         // real rows
    long long m0;        // first source row (ragged applyK / data terms) -- points or cells
    long long m;         // source rows
    long long tgt;       // first packed target row
    long long src;       // first packed source row
    long long tpad, spad;  // packed rows of this segment (targets, sources)
    long long part;      // first row of the partial-sum buffer
    int split;
    int nb;              // reduction blocks of this segment
    long long eoff;      // first energy partial of this segment
    double scale;        // coordinate prescale
    double dscale;       // derivative constant
    double center[3];
    double rw;
    double extra;        // dt, or sign of the target set, ...
    long long bkey[6];   // bounding-box keys (min x y z, max x y z), see bbox_key
    int bb0, nbb;        // first bounding-box block of this segment, block count
};

// Host-side plan of a ragged launch.
template <class Op>
struct RagPlan {
    std::vector<RagSeg> segs;
    std::vector<SegDesc> desc;
    long long tt = 0, ss = 0, parts = 0, eparts = 0;
    int items = 0;
};

template <class Op>
RagPlan<Op> rag_plan(const std::vector<long long>& n, const std::vector<long long>& m) {
    RagPlan<Op> p;
    const int nseg = (int)n.size();
    p.segs.resize(nseg);
    p.desc.resize(nseg);
    long long row = 0, mrow = 0;
    for (int s = 0; s < nseg; ++s) {
        const SinglePlan pl = plan_single<Op>(n[s], m[s]);
        RagSeg& g = p.segs[s];
        g.row0 = row;
        g.n = n[s];
        g.m0 = mrow;
        g.m = m[s];
        g.tgt = p.tt;
        g.src = p.ss;
        g.tpad = pl.n_tpad;
        g.spad = pl.m_pad;
        g.part = p.parts;
        g.split = pl.split;
        g.nb = (int)std::max<long long>(1, std::min<long long>(1024, (n[s] + kRagThreads - 1) / kRagThreads));
        g.eoff = p.eparts;
        SegDesc& d = p.desc[s];
        d.tgt = g.tgt;
        d.src = g.src;
        d.part = g.part;
        d.n_tgt = (int)n[s];
        d.n_src_tiles = pl.n_src_tiles;
        d.n_tb = pl.n_tb;
        d.split = pl.split;
        d.item0 = p.items;
        p.items += pl.n_tb * pl.split;
        p.tt += pl.n_tpad;
        p.ss += pl.m_pad;
        p.parts += (long long)pl.split * n[s];
        p.eparts += g.nb;
        row += n[s];
        mrow += m[s];
    }
    return p;
}

// ---- segment-local reductions ----------------------------------------------------
LDDMM_D double rag_block_sum(double v) {
    __shared__ double red[kRagThreads];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = kRagThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// Centre of the bounding box of each segment's rows: rows [row0, row0 + n) of x
// (x0 of a trajectory block when XT0: rows (T+1) row0 + i) and, if y, rows
// [m0, m0 + m) of y.  nbb blocks per segment reduce order-preserving keys with
// atomics into the segment's bkey (exact, order independent).
template <bool XT0>
static __global__ void rag_bbox_keys_kernel(RagSeg* segs, int nseg, const double* __restrict__ x,
                                            const double* __restrict__ y, int d, int T) {
    const int b = blockIdx.x;
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].bb0 <= b) lo = mid; else hi = mid - 1;
    }
    RagSeg& g = segs[lo];
    const int lb = b - g.bb0;
    const double* base = x + (XT0 ? (long long)(T + 1) * g.row0 : g.row0) * d;
    const long long tot = g.n + (y ? g.m : 0);
    long long l[3] = {kKeyMax, kKeyMax, kKeyMax}, h[3] = {kKeyMin, kKeyMin, kKeyMin};
    for (long long i = (long long)lb * blockDim.x + threadIdx.x; i < tot; i += (long long)g.nbb * blockDim.x) {
        const double* p = i < g.n ? base + i * d : y + (g.m0 + i - g.n) * d;
        for (int j = 0; j < d; ++j) {
            const long long k = bbox_key(p[j]);
            l[j] = min(l[j], k);
            h[j] = max(h[j], k);
        }
    }
    bbox_block_commit(l, h, g.bkey);
}

static __global__ void rag_bbox_finish_kernel(RagSeg* segs, int nseg, int d, int with_y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    RagSeg& g = segs[s];
    const bool nonempty = g.n + (with_y ? g.m : 0) > 0;
    for (int j = 0; j < 3; ++j)
        g.center[j] = (j < d && nonempty) ? 0.5 * (bbox_val(g.bkey[j]) + bbox_val(g.bkey[3 + j])) : 0.0;
}

// host: block layout of the bounding-box launch, initial keys; returns the block count
static int rag_bbox_prepare(std::vector<RagSeg>& segs, bool with_y) {
    int b = 0;
    for (RagSeg& g : segs) {
        const long long tot = g.n + (with_y ? g.m : 0);
        g.nbb = (int)std::max<long long>(1, std::min<long long>(256, (tot + 2047) / 2048));
        g.bb0 = b;
        b += g.nbb;
        for (int j = 0; j < 3; ++j) {
            g.bkey[j] = kKeyMax;
            g.bkey[3 + j] = kKeyMin;
        }
    }
    return b;
}

template <bool XT0>
static void rag_bbox_launch(RagSeg* dsegs, int nseg, int nbb, const double* x, const double* y, int d, int T,
                            cudaStream_t st) {
    rag_bbox_keys_kernel<XT0><<<nbb, kRagThreads, 0, st>>>(dsegs, nseg, x, y, d, T);
    rag_bbox_finish_kernel<<<(nseg + 127) / 128, 128, 0, st>>>(dsegs, nseg, d, y != nullptr ? 1 : 0);
}

LDDMM_D void put_dup(float4* planes, long long stride, long long i, const float* v, int NV) {
    for (int w = 0; w < (NV + 1) / 2; ++w) {
        const float a = v[2 * w], b = (2 * w + 1 < NV) ? v[2 * w + 1] : 0.f;
        planes[(long long)w * stride + i] = make_float4(a, a, b, b);
    }
}

LDDMM_D void put_plain(float4* planes, long long stride, long long i, const float* v, int nv, int nwords) {
    for (int w = 0; w < nwords; ++w) {
        float q[4];
        for (int k = 0; k < 4; ++k) q[k] = (w * 4 + k < nv) ? v[w * 4 + k] : 0.f;
        planes[(long long)w * stride + i] = make_float4(q[0], q[1], q[2], q[3]);
    }
}

// ---- ragged shooting ---------------------------------------------------------------
// xt / at of request s: blocks (T+1, n, d) / (T, n, d) at rows (T+1)*row0 / T*row0.
template <int D>
static __global__ void rag_shoot_pack_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ padoff,
                                             int nseg, const double* __restrict__ xt, const double* __restrict__ at,
                                             int T, int step, int d, float4* tgt, long long tstride, float4* src,
                                             long long sstride) {
    const long long total = padoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = seg_lookup(padoff, nseg, q);
        const RagSeg& g = segs[s];
        const long long i = q - padoff[s];
        float pos[3] = {0, 0, 0}, vals[2 * D];
        for (int k = 0; k < 2 * D; ++k) vals[k] = 0.f;
        if (i < g.n) {
            const double* x = xt + (((long long)(T + 1) * g.row0 + (long long)step * g.n + i) * d);
            const double* a = at + (((long long)T * g.row0 + (long long)step * g.n + i) * d);
            for (int j = 0; j < d; ++j) {
                pos[j] = (float)((x[j] - g.center[j]) * g.scale);
                vals[j] = pos[j];
                vals[D + j] = (float)a[j];
            }
        }
        if (i < g.tpad) put_plain(tgt, tstride, g.tgt + i, pos, 3, 1);
        if (i < g.spad) put_dup(src, sstride, g.src + i, vals, 2 * D);
    }
}

// v = sum of chunks, x_{t+1} = x_t + dt v, energy partial <a, v> per segment block
template <int D>
static __global__ void rag_shoot_combine_kernel(const RagSeg* __restrict__ segs, int nseg,
                                                const double* __restrict__ part, double* __restrict__ xt,
                                                const double* __restrict__ at, int T, int step, int d,
                                                double* __restrict__ epart) {
    // grid: blocks enumerate (segment, local block) pairs; eoff gives the first block of a segment
    const int b = blockIdx.x;
    int s = 0;
    {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].eoff <= b) lo = mid; else hi = mid - 1;
        }
        s = lo;
    }
    const RagSeg& g = segs[s];
    const int lb = b - (int)g.eoff;
    double e = 0.0;
    for (long long i = (long long)lb * blockDim.x + threadIdx.x; i < g.n; i += (long long)g.nb * blockDim.x) {
        const double* x0 = xt + (((long long)(T + 1) * g.row0 + (long long)step * g.n + i) * d);
        double* x1 = xt + (((long long)(T + 1) * g.row0 + (long long)(step + 1) * g.n + i) * d);
        const double* a0 = at + (((long long)T * g.row0 + (long long)step * g.n + i) * d);
        double v[D];
        for (int j = 0; j < D; ++j) v[j] = 0.0;
#pragma unroll 4
        for (int k = 0; k < g.split; ++k) {
            const double* pk = part + (g.part + (long long)k * g.n + i) * D;
            for (int j = 0; j < D; ++j) v[j] += pk[j];
        }
        for (int j = 0; j < d; ++j) {
            e += a0[j] * v[j];
            x1[j] = x0[j] + g.extra * v[j];
        }
    }
    const double r = rag_block_sum(e);
    if (threadIdx.x == 0) epart[(long long)step * 0 + b] += r;
}

// energy[s] = rw dt * sum of the segment's partials (fixed order)
static __global__ void rag_energy_kernel(const RagSeg* __restrict__ segs, int nseg, const double* __restrict__ epart,
                                         double scale_by_dt, double* __restrict__ energy, int use_rw) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const RagSeg& g = segs[s];
    double v = 0.0;
    for (int k = 0; k < g.nb; ++k) v += epart[g.eoff + k];
    energy[s] = (use_rw ? g.rw * g.extra : scale_by_dt) * v;
}

static int rag_copy_table(const void* host, size_t bytes, void* dev, cudaStream_t st) {
    return cuda_check(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st), "ragged table copy");
}

template <int KIND, int DEG, int D>
int rag_shoot_impl(int nseg, const int64_t* v_off, int d, const double* x0, const double* at, int T,
                   const double* sigma, int order, const double* rw, double* xt, double* energy, Workspace& ws,
                   cudaStream_t st) {
    using Op = OpApplyK2<KIND, DEG, D, D>;
    std::vector<long long> n(nseg);
    for (int s = 0; s < nseg; ++s) n[s] = v_off[s + 1] - v_off[s];
    RagPlan<Op> pl = rag_plan<Op>(n, n);
    std::vector<long long> padoff(nseg + 1, 0);
    for (int s = 0; s < nseg; ++s) padoff[s + 1] = padoff[s] + std::max(pl.segs[s].tpad, pl.segs[s].spad);
    RagSeg* dsegs = ws.take<RagSeg>(nseg);
    SegDesc* ddesc = ws.take<SegDesc>(nseg);
    long long* dpad = ws.take<long long>(nseg + 1);
    float4* tgt = ws.take<float4>((size_t)Op::PP * pl.tt);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.ss);
    double* part = ws.take<double>((size_t)pl.parts * D);
    double* epart = ws.take<double>((size_t)std::max<long long>(1, pl.eparts));
    if (ws.measuring()) return LDDMM_OK;
    for (int s = 0; s < nseg; ++s) {
        const KScale ks = kernel_scale<float>(KIND, order, sigma[s]);
        pl.segs[s].scale = ks.scale;
        pl.segs[s].dscale = ks.dscale;
        pl.segs[s].rw = rw[s];
        pl.segs[s].extra = 1.0 / T;
    }
    const int nbb = rag_bbox_prepare(pl.segs, false);
    LDDMM_TRY(rag_copy_table(pl.segs.data(), sizeof(RagSeg) * nseg, dsegs, st));
    LDDMM_TRY(rag_copy_table(pl.desc.data(), sizeof(SegDesc) * nseg, ddesc, st));
    LDDMM_TRY(rag_copy_table(padoff.data(), sizeof(long long) * (nseg + 1), dpad, st));
    LDDMM_TRY(cuda_check(cudaMemsetAsync(epart, 0, sizeof(double) * std::max<long long>(1, pl.eparts), st), "memset"));
    // xt[0] = x0 per request
    for (int s = 0; s < nseg; ++s)
        LDDMM_TRY(cuda_check(cudaMemcpyAsync(xt + (T + 1) * v_off[s] * d, x0 + v_off[s] * d, sizeof(double) * n[s] * d,
                                             cudaMemcpyDeviceToDevice, st), "ragged shoot copy"));
    rag_bbox_launch<false>(dsegs, nseg, nbb, x0, nullptr, d, 0, st);   // x0 rows [row0, row0 + n)
    KernelParams2 P{};
    P.src4 = src;
    P.src_stride = pl.ss;
    P.tgt4 = tgt;
    P.tgt_stride = pl.tt;
    const KScale ks0 = kernel_scale<float>(KIND, order, sigma[0]);
    for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks0.pk[j]);
    for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks0.pq[j]);
    SweepGrid grid{};
    grid.segs = ddesc;
    grid.nseg = nseg;
    grid.n_items = pl.items;
    for (int t = 0; t < T; ++t) {
        rag_shoot_pack_kernel<D><<<grid_for(padoff[nseg]), 256, 0, st>>>(dsegs, dpad, nseg, xt, at, T, t, d, tgt, pl.tt,
                                                                        src, pl.ss);
        sweep_kernel<Op><<<pl.items, Op::BLOCK, 0, st>>>(grid, P, part);
        rag_shoot_combine_kernel<D><<<(int)pl.eparts, kRagThreads, 0, st>>>(dsegs, nseg, part, xt, at, T, t, d, epart);
    }
    if (energy) rag_energy_kernel<<<(nseg + 127) / 128, 128, 0, st>>>(dsegs, nseg, epart, 0.0, energy, 1);
    return cuda_check(cudaGetLastError(), "ragged shoot");
}

// ---- ragged covector ---------------------------------------------------------------
// step t: targets (pos x_t, u = (p_{t+1} - 2 rw a_t, a_t)), sources (pos, v = (a_t, p_{t+1}))
template <int D>
static __global__ void rag_cov_pack_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ padoff,
                                           int nseg, const double* __restrict__ xt, const double* __restrict__ at,
                                           const double* __restrict__ pxt, int T, int step, int d, float4* tgt,
                                           long long tstride, float4* src, long long sstride) {
    const long long total = padoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = seg_lookup(padoff, nseg, q);
        const RagSeg& g = segs[s];
        const long long i = q - padoff[s];
        float pos[3] = {0, 0, 0}, u[2 * D], v[3 * D];
        for (int k = 0; k < 2 * D; ++k) u[k] = 0.f;
        for (int k = 0; k < 3 * D; ++k) v[k] = 0.f;
        if (i < g.n) {
            const double* x = xt + (((long long)(T + 1) * g.row0 + (long long)step * g.n + i) * d);
            const double* a = at + (((long long)T * g.row0 + (long long)step * g.n + i) * d);
            const double* p = pxt + (((long long)(T + 1) * g.row0 + (long long)(step + 1) * g.n + i) * d);
            for (int j = 0; j < d; ++j) {
                pos[j] = (float)((x[j] - g.center[j]) * g.scale);
                u[j] = (float)(p[j] - 2.0 * g.rw * a[j]);
                u[D + j] = (float)a[j];
                v[j] = pos[j];
                v[D + j] = (float)a[j];
                v[2 * D + j] = (float)p[j];
            }
        }
        if (i < g.tpad) {
            put_plain(tgt, tstride, g.tgt + i, pos, 3, 1);
            put_plain(tgt + tstride, tstride, g.tgt + i, u, 2 * D, (2 * D + 3) / 4);
        }
        if (i < g.spad) put_dup(src, sstride, g.src + i, v, 3 * D);
    }
}

template <int D>
static __global__ void rag_cov_combine_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ rowoff,
                                              int nseg, const double* __restrict__ part, const double* __restrict__ at,
                                              double* __restrict__ pxt, double* __restrict__ dat, int T, int step,
                                              int d) {
    const long long total = rowoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = seg_lookup(rowoff, nseg, q);
        const RagSeg& g = segs[s];
        const long long i = q - rowoff[s];
        const double* pn = pxt + (((long long)(T + 1) * g.row0 + (long long)(step + 1) * g.n + i) * d);
        double* pc = pxt + (((long long)(T + 1) * g.row0 + (long long)step * g.n + i) * d);
        const double* a = at + (((long long)T * g.row0 + (long long)step * g.n + i) * d);
        double* da = dat ? dat + (((long long)T * g.row0 + (long long)step * g.n + i) * d) : nullptr;
        double f[D];
        for (int j = 0; j < D; ++j) f[j] = 0.0;
#pragma unroll 4
        for (int k = 0; k < g.split; ++k) {
            const double* pk = part + (g.part + (long long)k * g.n + i) * D;
            for (int j = 0; j < D; ++j) f[j] += pk[j];
        }
        for (int j = 0; j < d; ++j) {
            pc[j] = pn[j] + g.extra * (g.dscale * f[j]);
            if (da) da[j] = 2.0 * g.rw * a[j] - pn[j];
        }
    }
}

template <int KIND, int QDEG, int D>
int rag_cov_impl(int nseg, const int64_t* v_off, int d, const double* xt, const double* at, int T,
                 const double* px1, const double* sigma, int order, const double* rw, double* pxt, double* dat,
                 Workspace& ws, cudaStream_t st) {
    constexpr int W = 2 * D;
    using Op = OpDiffKT2<KIND, QDEG, D, W>;
    constexpr int NT = 1 + (W + 3) / 4;
    std::vector<long long> n(nseg);
    for (int s = 0; s < nseg; ++s) n[s] = v_off[s + 1] - v_off[s];
    RagPlan<Op> pl = rag_plan<Op>(n, n);
    std::vector<long long> padoff(nseg + 1, 0), rowoff(nseg + 1, 0);
    for (int s = 0; s < nseg; ++s) {
        padoff[s + 1] = padoff[s] + std::max(pl.segs[s].tpad, pl.segs[s].spad);
        rowoff[s + 1] = rowoff[s] + n[s];
    }
    RagSeg* dsegs = ws.take<RagSeg>(nseg);
    SegDesc* ddesc = ws.take<SegDesc>(nseg);
    long long* dpad = ws.take<long long>(nseg + 1);
    long long* drow = ws.take<long long>(nseg + 1);
    float4* tgt = ws.take<float4>((size_t)NT * pl.tt);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.ss);
    double* part = ws.take<double>((size_t)pl.parts * D);
    if (ws.measuring()) return LDDMM_OK;
    for (int s = 0; s < nseg; ++s) {
        const KScale ks = kernel_scale<float>(KIND, order, sigma[s]);
        pl.segs[s].scale = ks.scale;
        pl.segs[s].dscale = ks.dscale;
        pl.segs[s].rw = rw[s];
        pl.segs[s].extra = 1.0 / T;
    }
    const int nbb = rag_bbox_prepare(pl.segs, false);
    LDDMM_TRY(rag_copy_table(pl.segs.data(), sizeof(RagSeg) * nseg, dsegs, st));
    LDDMM_TRY(rag_copy_table(pl.desc.data(), sizeof(SegDesc) * nseg, ddesc, st));
    LDDMM_TRY(rag_copy_table(padoff.data(), sizeof(long long) * (nseg + 1), dpad, st));
    LDDMM_TRY(rag_copy_table(rowoff.data(), sizeof(long long) * (nseg + 1), drow, st));
    for (int s = 0; s < nseg; ++s)
        LDDMM_TRY(cuda_check(cudaMemcpyAsync(pxt + ((T + 1) * v_off[s] + (long long)T * n[s]) * d, px1 + v_off[s] * d,
                                             sizeof(double) * n[s] * d, cudaMemcpyDeviceToDevice, st), "cov copy"));
    rag_bbox_launch<true>(dsegs, nseg, nbb, xt, nullptr, d, T, st);   // x_0 of each trajectory block
    KernelParams2 P{};
    P.src4 = src;
    P.src_stride = pl.ss;
    P.tgt4 = tgt;
    P.tgt_stride = pl.tt;
    const KScale ks0 = kernel_scale<float>(KIND, order, sigma[0]);
    for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks0.pk[j]);
    for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks0.pq[j]);
    SweepGrid grid{};
    grid.segs = ddesc;
    grid.nseg = nseg;
    grid.n_items = pl.items;
    for (int t = T - 1; t >= 0; --t) {
        rag_cov_pack_kernel<D><<<grid_for(padoff[nseg]), 256, 0, st>>>(dsegs, dpad, nseg, xt, at, pxt, T, t, d, tgt,
                                                                      pl.tt, src, pl.ss);
        sweep_kernel<Op><<<pl.items, Op::BLOCK, 0, st>>>(grid, P, part);
        rag_cov_combine_kernel<D><<<grid_for(rowoff[nseg]), 256, 0, st>>>(dsegs, drow, nseg, part, at, pxt, dat, T, t,
                                                                         d);
    }
    return cuda_check(cudaGetLastError(), "ragged covector");
}

// ---- ragged applyK (independent target / source segments) --------------------------
// segment s: targets x rows [row0, row0+n), sources y rows [m0, m0+m) with
// weights beta rows aligned with y; output f rows [foff_s, foff_s + n) (compact).
template <int D, int DIMB>
static __global__ void rag_applyk_pack_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ padoff,
                                              int nseg, const double* __restrict__ x, const double* __restrict__ y,
                                              const double* __restrict__ beta, int d, int dimb, float4* tgt,
                                              long long tstride, float4* src, long long sstride) {
    const long long total = padoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = seg_lookup(padoff, nseg, q);
        const RagSeg& g = segs[s];
        const long long i = q - padoff[s];
        if (i < g.tpad) {
            float pos[3] = {0, 0, 0};
            if (i < g.n)
                for (int j = 0; j < d; ++j) pos[j] = (float)((x[(g.row0 + i) * d + j] - g.center[j]) * g.scale);
            put_plain(tgt, tstride, g.tgt + i, pos, 3, 1);
        }
        if (i < g.spad) {
            float v[D + DIMB];
            for (int k = 0; k < D + DIMB; ++k) v[k] = 0.f;
            if (i < g.m) {
                for (int j = 0; j < d; ++j) v[j] = (float)((y[(g.m0 + i) * d + j] - g.center[j]) * g.scale);
                for (int c = 0; c < dimb && c < DIMB; ++c) v[D + c] = (float)beta[(g.m0 + i) * dimb + c];
            }
            put_dup(src, sstride, g.src + i, v, D + DIMB);
        }
    }
}

template <int DIMB>
static __global__ void rag_applyk_combine_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ rowoff,
                                                 int nseg, const double* __restrict__ part, int dimb,
                                                 double* __restrict__ f) {
    const long long total = rowoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = seg_lookup(rowoff, nseg, q);
        const RagSeg& g = segs[s];
        const long long i = q - rowoff[s];
        double v[DIMB];
        for (int c = 0; c < DIMB; ++c) v[c] = 0.0;
#pragma unroll 4
        for (int k = 0; k < g.split; ++k) {
            const double* pk = part + (g.part + (long long)k * g.n + i) * DIMB;
            for (int c = 0; c < DIMB; ++c) v[c] += pk[c];
        }
        for (int c = 0; c < dimb && c < DIMB; ++c) f[q * dimb + c] = v[c];
    }
}

template <int KIND, int DEG, int D, int DIMB>
int rag_applyk_impl(int nseg, const int64_t* t_start, const int64_t* t_count, const int64_t* s_start,
                    const int64_t* s_count, int d, const double* x, const double* y, const double* beta, int dimb,
                    const double* sigma, int order, double* f, Workspace& ws, cudaStream_t st) {
    using Op = OpApplyK2<KIND, DEG, D, DIMB>;
    std::vector<long long> n(nseg), m(nseg);
    for (int s = 0; s < nseg; ++s) {
        n[s] = t_count[s];
        m[s] = s_count[s];
    }
    RagPlan<Op> pl = rag_plan<Op>(n, m);
    std::vector<long long> padoff(nseg + 1, 0), rowoff(nseg + 1, 0);
    for (int s = 0; s < nseg; ++s) {
        pl.segs[s].row0 = t_start[s];
        pl.segs[s].m0 = s_start[s];
        padoff[s + 1] = padoff[s] + std::max(pl.segs[s].tpad, pl.segs[s].spad);
        rowoff[s + 1] = rowoff[s] + n[s];
    }
    RagSeg* dsegs = ws.take<RagSeg>(nseg);
    SegDesc* ddesc = ws.take<SegDesc>(nseg);
    long long* dpad = ws.take<long long>(nseg + 1);
    long long* drow = ws.take<long long>(nseg + 1);
    float4* tgt = ws.take<float4>((size_t)Op::PP * pl.tt);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.ss);
    double* part = ws.take<double>((size_t)pl.parts * DIMB);
    if (ws.measuring()) return LDDMM_OK;
    for (int s = 0; s < nseg; ++s) {
        const KScale ks = kernel_scale<float>(KIND, order, sigma[s]);
        pl.segs[s].scale = ks.scale;
        pl.segs[s].dscale = ks.dscale;
    }
    const int nbb = rag_bbox_prepare(pl.segs, true);
    LDDMM_TRY(rag_copy_table(pl.segs.data(), sizeof(RagSeg) * nseg, dsegs, st));
    LDDMM_TRY(rag_copy_table(pl.desc.data(), sizeof(SegDesc) * nseg, ddesc, st));
    LDDMM_TRY(rag_copy_table(padoff.data(), sizeof(long long) * (nseg + 1), dpad, st));
    LDDMM_TRY(rag_copy_table(rowoff.data(), sizeof(long long) * (nseg + 1), drow, st));
    rag_bbox_launch<false>(dsegs, nseg, nbb, x, y, d, 0, st);
    KernelParams2 P{};
    P.src4 = src;
    P.src_stride = pl.ss;
    P.tgt4 = tgt;
    P.tgt_stride = pl.tt;
    const KScale ks0 = kernel_scale<float>(KIND, order, sigma[0]);
    for (int j = 0; j < 5; ++j) P.pkd[j] = dup_coeff(ks0.pk[j]);
    for (int j = 0; j < 4; ++j) P.pqd[j] = dup_coeff(ks0.pq[j]);
    SweepGrid grid{};
    grid.segs = ddesc;
    grid.nseg = nseg;
    grid.n_items = pl.items;
    rag_applyk_pack_kernel<D, DIMB><<<grid_for(padoff[nseg]), 256, 0, st>>>(dsegs, dpad, nseg, x, y, beta, d, dimb,
                                                                             tgt, pl.tt, src, pl.ss);
    if (pl.items > 0) sweep_kernel<Op><<<pl.items, Op::BLOCK, 0, st>>>(grid, P, part);
    rag_applyk_combine_kernel<DIMB><<<grid_for(rowoff[nseg]), 256, 0, st>>>(dsegs, drow, nseg, part, dimb, f);
    return cuda_check(cudaGetLastError(), "ragged applyk");
}

// ---- ragged data terms ---------------------------------------------------------------
// request s: cells rows [row0, row0 + n) of c1/s1 (global vertex indices), target
// cells rows [m0, m0 + m) of c2/s2; sources of the sweep = its n cells then its m.
template <class Real>
static __global__ void rag_dt_pack_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ padoff,
                                          int nseg, int norm, int grad, const double* __restrict__ c1,
                                          const double* __restrict__ s1, const double* __restrict__ c2,
                                          const double* __restrict__ s2, int d, double eps1, double eps2,
                                          double sign2, float4* tgt, long long tstride, int tplanes, int tslots,
                                          float4* src, long long sstride, int splanes, int sslots, int dup,
                                          int sym_align) {
    const long long total = padoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int sg = seg_lookup(padoff, nseg, q);
        const RagSeg& g = segs[sg];
        const long long i = q - padoff[sg];
        if (i < g.tpad)
            dt_pack_record<Real>(norm, grad, true, i < g.n ? c1 + (g.row0 + i) * d : nullptr,
                                 i < g.n ? s1 + (g.row0 + i) * d : nullptr, d, eps1, 1.0, g.scale, g.center, tgt,
                                 tstride, g.tgt + i, tplanes, tslots);
        if (i < g.spad) {
            // target-shape cells start at n rounded up to sym_align (symmetric sweeps) or at n
            const long long n1s = sym_align > 0 ? (g.n + sym_align - 1) / sym_align * sym_align : g.n;
            const bool first = i < g.n, second = i >= n1s && i < n1s + g.m;
            const double* c = first ? c1 + (g.row0 + i) * d : (second ? c2 + (g.m0 + i - n1s) * d : nullptr);
            const double* sv = first ? s1 + (g.row0 + i) * d : (second ? s2 + (g.m0 + i - n1s) * d : nullptr);
            dt_pack_record<Real>(norm, grad, false, c, sv, d, first ? eps1 : eps2, first ? 1.0 : sign2, g.scale,
                                 g.center, src, sstride, g.src + i, splanes, sslots, dup != 0);
        }
    }
}

// energy partial of the segment's block: sum_k w1_k . z_k
static __global__ void rag_dt_value_kernel(const RagSeg* __restrict__ segs, int nseg, int norm,
                                           const double* __restrict__ part, int nout, const double* __restrict__ s1,
                                           int d, double eps1, double* __restrict__ epart) {
    const int b = blockIdx.x;
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].eoff <= b) lo = mid; else hi = mid - 1;
    }
    const RagSeg& g = segs[lo];
    const int lb = b - (int)g.eoff;
    double e = 0.0;
    for (long long i = (long long)lb * blockDim.x + threadIdx.x; i < g.n; i += (long long)g.nb * blockDim.x) {
        double z[4] = {0, 0, 0, 0};
#pragma unroll 4
        for (int k = 0; k < g.split; ++k) {
            const double* pk = part + (g.part + (long long)k * g.n + i) * nout;
            for (int c = 0; c < nout && c < 4; ++c) z[c] += pk[c];
        }
        const double* sv = s1 + (g.row0 + i) * d;
        if (norm == NCURRENT) {
            for (int j = 0; j < d; ++j) e += sv[j] * z[j];
        } else {
            e += vec_norm_eps(sv, d, eps1) * z[0];
        }
    }
    const double r = rag_block_sum(e);
    if (threadIdx.x == 0) epart[b] = r;
}

static __global__ void rag_dt_grad_kernel(const RagSeg* __restrict__ segs, const long long* __restrict__ rowoff,
                                          int nseg, int norm, const double* __restrict__ part, int nout,
                                          const double* __restrict__ s1, int d, double eps1, double fac,
                                          double* __restrict__ z1, double* __restrict__ dz1) {
    const long long total = rowoff[nseg];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int sg = seg_lookup(rowoff, nseg, q);
        const RagSeg& g = segs[sg];
        const long long i = q - rowoff[sg];
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 2
        for (int k = 0; k < g.split; ++k) {
            const double* pk = part + (g.part + (long long)k * g.n + i) * nout;
            for (int c = 0; c < nout && c < 8; ++c) acc[c] += pk[c];
        }
        const long long r = g.row0 + i;
        dt_grad_row(norm, acc, s1 + r * d, d, eps1, fac * g.dscale, z1 + r * d, dz1 + r * d);
    }
}

struct RagDataArgs {
    int nseg;
    int ncorner, norm;
    const int64_t* v_off;
    const int64_t* c_off;
    const int64_t* c2_off;
    const double* v;
    int d;
    const int64_t* cells;
    const double* c2;
    const double* s2;
    const double* sigma;
    int order;
    double eps1, eps2;
    const double* frame;   // host (nseg, 3) packing centres, or NULL: bounding-box centre per call
    double* energy;
    const int64_t* vptr;
    const int64_t* vidx;
    double* px;
};

// SYM (values): each segment's cell-cell self part is evaluated once per
// unordered pair (sweep_kernel<Op, true>); its target cells start at a tile.
template <class Real, class Op, int TSLOTS, int SSLOTS, int NT, bool SYM = false>
int rag_dt_sweep(const RagDataArgs& a, int kind, int grad, double sign2, const double* c1, const double* s1,
                 Workspace& ws, cudaStream_t st, RagPlan<Op>& pl, RagSeg*& dsegs, long long*& drow, double*& part) {
    const int nseg = a.nseg;
    std::vector<long long> n(nseg), m(nseg), n1s(nseg);
    for (int s = 0; s < nseg; ++s) {
        n[s] = a.c_off[s + 1] - a.c_off[s];
        n1s[s] = SYM ? (n[s] + Op::TILE - 1) / Op::TILE * Op::TILE : n[s];
        m[s] = n1s[s] + (a.c2_off[s + 1] - a.c2_off[s]);
    }
    pl = rag_plan<Op>(n, m);
    for (int s = 0; s < nseg; ++s) pl.desc[s].sym_tiles = SYM ? (int)(n1s[s] / Op::TILE) : 0;
    std::vector<long long> padoff(nseg + 1, 0), rowoff(nseg + 1, 0);
    for (int s = 0; s < nseg; ++s) {
        pl.segs[s].row0 = a.c_off[s];
        pl.segs[s].m0 = a.c2_off[s];
        pl.segs[s].m = a.c2_off[s + 1] - a.c2_off[s];
        padoff[s + 1] = padoff[s] + std::max(pl.segs[s].tpad, pl.segs[s].spad);
        rowoff[s + 1] = rowoff[s] + n[s];
    }
    dsegs = ws.take<RagSeg>(nseg);
    SegDesc* ddesc = ws.take<SegDesc>(nseg);
    long long* dpad = ws.take<long long>(nseg + 1);
    drow = ws.take<long long>(nseg + 1);
    float4* tgt = ws.take<float4>((size_t)NT * pl.tt);
    float4* src = ws.take<float4>((size_t)Op::NS * pl.ss);
    part = ws.take<double>((size_t)pl.parts * Op::NOUT);
    if (ws.measuring()) return LDDMM_OK;
    for (int s = 0; s < nseg; ++s) {
        const KScale ks = kernel_scale<Real>(kind, a.order, a.sigma[s]);
        pl.segs[s].scale = ks.scale;
        pl.segs[s].dscale = ks.dscale;
        if (a.frame)
            for (int j = 0; j < 3; ++j) pl.segs[s].center[j] = j < a.d ? a.frame[3 * s + j] : 0.0;
    }
    const int nbb = rag_bbox_prepare(pl.segs, a.c2 != nullptr);
    LDDMM_TRY(rag_copy_table(pl.segs.data(), sizeof(RagSeg) * nseg, dsegs, st));
    LDDMM_TRY(rag_copy_table(pl.desc.data(), sizeof(SegDesc) * nseg, ddesc, st));
    LDDMM_TRY(rag_copy_table(padoff.data(), sizeof(long long) * (nseg + 1), dpad, st));
    LDDMM_TRY(rag_copy_table(rowoff.data(), sizeof(long long) * (nseg + 1), drow, st));
    if (!a.frame) rag_bbox_launch<false>(dsegs, nseg, nbb, c1, a.c2, a.d, 0, st);
    typename Op::Params P{};
    P.src4 = src;
    P.src_stride = pl.ss;
    P.tgt4 = tgt;
    P.tgt_stride = pl.tt;
    const KScale ks0 = kernel_scale<Real>(kind, a.order, a.sigma[0]);
    set_data_poly<Op, Real>(P, ks0);
    rag_dt_pack_kernel<Real><<<grid_for(padoff[nseg]), 256, 0, st>>>(
        dsegs, dpad, nseg, a.norm, grad, c1, s1, a.c2, a.s2, a.d, a.eps1, a.eps2, sign2, tgt, pl.tt, NT, TSLOTS, src,
        pl.ss, Op::NS, SSLOTS, op_dup<Op>::value ? 1 : 0, SYM ? Op::TILE : 0);
    SweepGrid grid{};
    grid.segs = ddesc;
    grid.nseg = nseg;
    grid.n_items = pl.items;
    if (pl.items > 0) sweep_kernel<Op, SYM><<<pl.items, Op::BLOCK, 0, st>>>(grid, P, part);
    return cuda_check(cudaGetLastError(), "ragged data sweep");
}

template <class Real, int KIND, int PDEG, int QDEG, int D>
int rag_dt_impl(const RagDataArgs& a, Workspace& ws, cudaStream_t st) {
    constexpr int PW = Traits<Real>::PER_WORD;
    constexpr int PP = PointPlanes<Real>::N;
    const long long C = a.c_off[a.nseg];
    const long long NV = a.v_off[a.nseg];
    double* c1 = ws.take<double>((size_t)C * a.d);
    double* s1 = ws.take<double>((size_t)C * a.d);
    if (!ws.measuring())
        cell_geometry_kernel<<<grid_for(C), 256, 0, st>>>(a.ncorner, a.v, NV, a.d, a.cells, C, c1, s1);
    if (a.energy != nullptr) {
        RagSeg* dsegs = nullptr;
        long long* drow = nullptr;
        double* part = nullptr;
        int nout = 1, rc = LDDMM_OK;
        long long eparts = 0;
        if (a.norm == NVARIFOLD) {
            // FP32: packed-pair operator (two targets per slot, duplicated sources)
            using Op = std::conditional_t<(sizeof(Real) == 4 && D == 3), OpVariValue2<KIND, PDEG>,
                                          OpData<Real, KIND, PDEG, QDEG, D, M_VARI_VALUE>>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, 3, 4, PP + (3 + PW - 1) / PW, true>(a, KIND, 0, -2.0, c1, s1, ws, st, pl, dsegs,
                                                                       drow, part);
            nout = Op::NOUT;
            eparts = pl.eparts;
        } else if (a.norm == NCURRENT) {
            using Op = OpApplyK<Real, KIND, PDEG, D, D>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, 0, D, PP, true>(a, KIND, 0, -2.0, c1, s1, ws, st, pl, dsegs, drow, part);
            nout = Op::NOUT;
            eparts = pl.eparts;
        } else {
            using Op = OpApplyK<Real, KIND, PDEG, D, 1>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, 0, 1, PP, true>(a, KIND, 0, -2.0, c1, s1, ws, st, pl, dsegs, drow, part);
            nout = Op::NOUT;
            eparts = pl.eparts;
        }
        if (rc != LDDMM_OK) return rc;
        double* epart = ws.take<double>((size_t)std::max<long long>(1, eparts));
        if (!ws.measuring()) {
            rag_dt_value_kernel<<<(int)eparts, kRagThreads, 0, st>>>(dsegs, a.nseg, a.norm, part, nout, s1, a.d,
                                                                    a.eps1, epart);
            rag_energy_kernel<<<(a.nseg + 127) / 128, 128, 0, st>>>(dsegs, a.nseg, epart, 1.0, a.energy, 0);
        }
    }
    if (a.px != nullptr) {
        RagSeg* dsegs = nullptr;
        long long* drow = nullptr;
        double* part = nullptr;
        int nout = 1, rc = LDDMM_OK;
        constexpr bool PACK = sizeof(Real) == 4 && D == 3;   // FP32 surfaces: packed-pair operators
        if (a.norm == NVARIFOLD) {
            using Op = std::conditional_t<PACK, OpVariGrad2<KIND, PDEG, QDEG>,
                                          OpData<Real, KIND, PDEG, QDEG, D, M_VARI_GRAD>>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, 3, 4, PP + (3 + PW - 1) / PW>(a, KIND, 1, -1.0, c1, s1, ws, st, pl, dsegs,
                                                                       drow, part);
            nout = Op::NOUT;
        } else if (a.norm == NCURRENT) {
            using Op = std::conditional_t<PACK, OpCurGrad2<KIND, PDEG, QDEG>,
                                          OpData<Real, KIND, PDEG, QDEG, D, M_CUR_GRAD>>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, D, D, PP + (D + PW - 1) / PW>(a, KIND, 1, -1.0, c1, s1, ws, st, pl, dsegs,
                                                                       drow, part);
            nout = Op::NOUT;
        } else {
            using Op = OpData<Real, KIND, PDEG, QDEG, D, M_MEAS_GRAD>;
            RagPlan<Op> pl;
            rc = rag_dt_sweep<Real, Op, 0, 1, PP>(a, KIND, 1, -1.0, c1, s1, ws, st, pl, dsegs, drow, part);
            nout = Op::NOUT;
        }
        if (rc != LDDMM_OK) return rc;
        double* z1 = ws.take<double>((size_t)C * a.d);
        double* dz1 = ws.take<double>((size_t)C * a.d);
        if (!ws.measuring()) {
            const double fac = a.ncorner == 3 ? 1.0 / 3.0 : 0.5;
            rag_dt_grad_kernel<<<grid_for(C), 256, 0, st>>>(dsegs, drow, a.nseg, a.norm, part, nout, s1, a.d, a.eps1,
                                                           fac, z1, dz1);
            dt_gather_kernel<<<grid_for(NV), 256, 0, st>>>(a.ncorner, a.v, NV, a.d, a.cells, C, a.vptr, a.vidx, z1,
                                                           dz1, a.px);
        }
    }
    if (ws.measuring()) return LDDMM_OK;
    return cuda_check(cudaGetLastError(), "ragged dataterm");
}

// ---- dispatch, validation and workspace ---------------------------------------------------
template <class F>
int rag_dispatch_pq(int order, F&& f) {
    switch (order) {
        case 0: return f(IC<KLAP>{}, IC<0>{}, IC<0>{});
        case 1: return f(IC<KLAP>{}, IC<1>{}, IC<0>{});
        case 2: return f(IC<KLAP>{}, IC<2>{}, IC<1>{});
        case 3: return f(IC<KLAP>{}, IC<3>{}, IC<2>{});
        case 4: return f(IC<KLAP>{}, IC<4>{}, IC<3>{});
        default: return f(IC<KGAUSS>{}, IC<0>{}, IC<0>{});
    }
}

static int rag_check_offsets(int nseg, const int64_t* off, const char* name) {
    if (off == nullptr || off[0] != 0) {
        set_error("ragged: %s must start at 0", name);
        return LDDMM_ERR_ARG;
    }
    for (int s = 0; s < nseg; ++s)
        if (off[s + 1] < off[s] || off[s + 1] - off[s] > (1LL << 30)) {
            set_error("ragged: %s is not non-decreasing (segment %d)", name, s);
            return LDDMM_ERR_ARG;
        }
    return LDDMM_OK;
}

static int rag_check_sigma(int nseg, const double* sigma, int order) {
    if (sigma == nullptr || order < 0) {
        set_error("ragged: sigma array missing or order < 0");
        return LDDMM_ERR_ARG;
    }
    for (int s = 0; s < nseg; ++s)
        if (!(sigma[s] > 0)) {
            set_error("ragged: sigma[%d] must be > 0", s);
            return LDDMM_ERR_ARG;
        }
    return LDDMM_OK;
}

template <class Run>
int rag_run(Run run, void* wsp, size_t wsb, cudaStream_t st, const char* who) {
    Workspace meas;
    LDDMM_TRY(run(meas));
    if (wsp == nullptr || meas.off > wsb) {
        set_error("%s: workspace too small: need %zu bytes, got %zu", who, meas.off, wsb);
        return LDDMM_ERR_WORKSPACE;
    }
    // The segment tables are built on the host and copied to the device with
    // each call; a CUDA graph would keep the host address of that copy, so a
    // capturing stream is refused before anything is enqueued.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    LDDMM_TRY(cuda_check(cudaStreamIsCapturing(st, &cap), who));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("%s: ragged entry points cannot be captured into a CUDA graph (host-built segment tables)", who);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(wsp, "workspace"));
    Workspace ws;
    ws.base = static_cast<char*>(wsp);
    ws.cap = wsb;
    return run(ws);
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_ragged_shoot_f32c_workspace(int nreq, const int64_t* v_off, int d, int T, int order) {
    if (nreq < 1 || d < 1 || d > 3 || T < 1 || rag_check_offsets(nreq, v_off, "v_off") != LDDMM_OK) return 0;
    std::vector<double> sg(nreq, 1.0), rw(nreq, 1.0);
    Workspace ws;
    dispatch_kind_p(order, [&](auto kind, auto deg) {
        return dispatch_d(d, [&](auto D) {
            return rag_shoot_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value>(
                nreq, v_off, d, nullptr, nullptr, T, sg.data(), order, rw.data(), nullptr, nullptr, ws, 0);
        });
    });
    return ws.off + 256;
}

int lddmm_ragged_shoot_f32c(int nreq, const int64_t* v_off, int d, const double* x0, const double* at, int T,
                            const double* sigma, int order, const double* regweight, double* xt, double* energy,
                            void* workspace, size_t workspace_bytes, lddmm_stream_t stream) {
    if (nreq < 1 || d < 1 || d > 3 || T < 1) {
        set_error("ragged shoot: invalid arguments (nreq=%d d=%d T=%d)", nreq, d, T);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(rag_check_offsets(nreq, v_off, "v_off"));
    LDDMM_TRY(rag_check_sigma(nreq, sigma, order));
    if (regweight == nullptr) {
        set_error("ragged shoot: regweight array missing");
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(x0, "x0"));
    LDDMM_TRY(check_device_ptr(at, "at"));
    LDDMM_TRY(check_device_ptr(xt, "xt"));
    if (energy) LDDMM_TRY(check_device_ptr(energy, "energy"));
    cudaStream_t st = (cudaStream_t)stream;
    return rag_run([&](Workspace& ws) {
        return dispatch_kind_p(order, [&](auto kind, auto deg) {
            return dispatch_d(d, [&](auto D) {
                return rag_shoot_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value>(
                    nreq, v_off, d, x0, at, T, sigma, order, regweight, xt, energy, ws, st);
            });
        });
    }, workspace, workspace_bytes, st, "ragged shoot");
}

size_t lddmm_ragged_covector_f32c_workspace(int nreq, const int64_t* v_off, int d, int T, int order) {
    if (nreq < 1 || d < 1 || d > 3 || T < 1 || order == 0 ||
        rag_check_offsets(nreq, v_off, "v_off") != LDDMM_OK)
        return 0;
    std::vector<double> sg(nreq, 1.0), rw(nreq, 1.0);
    Workspace ws;
    dispatch_kind_q(order, [&](auto kind, auto deg) {
        return dispatch_d(d, [&](auto D) {
            return rag_cov_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value>(
                nreq, v_off, d, nullptr, nullptr, T, nullptr, sg.data(), order, rw.data(), nullptr, nullptr, ws, 0);
        });
    });
    return ws.off + 256;
}

int lddmm_ragged_covector_f32c(int nreq, const int64_t* v_off, int d, const double* xt, const double* at, int T,
                               const double* px1, const double* sigma, int order, const double* regweight,
                               double* pxt, double* dat, void* workspace, size_t workspace_bytes,
                               lddmm_stream_t stream) {
    if (nreq < 1 || d < 1 || d > 3 || T < 1 || order == 0) {
        set_error("ragged covector: invalid arguments (nreq=%d d=%d T=%d order=%d)", nreq, d, T, order);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(rag_check_offsets(nreq, v_off, "v_off"));
    LDDMM_TRY(rag_check_sigma(nreq, sigma, order));
    if (regweight == nullptr) {
        set_error("ragged covector: regweight array missing");
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(xt, "xt"));
    LDDMM_TRY(check_device_ptr(at, "at"));
    LDDMM_TRY(check_device_ptr(px1, "px1"));
    LDDMM_TRY(check_device_ptr(pxt, "pxt"));
    if (dat) LDDMM_TRY(check_device_ptr(dat, "dat"));
    cudaStream_t st = (cudaStream_t)stream;
    return rag_run([&](Workspace& ws) {
        return dispatch_kind_q(order, [&](auto kind, auto deg) {
            return dispatch_d(d, [&](auto D) {
                return rag_cov_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value>(
                    nreq, v_off, d, xt, at, T, px1, sigma, order, regweight, pxt, dat, ws, st);
            });
        });
    }, workspace, workspace_bytes, st, "ragged covector");
}

size_t lddmm_ragged_applyk_f32c_workspace(int nseg, const int64_t* t_count, const int64_t* s_count, int d, int dimb,
                                          int order) {
    if (nseg < 1 || d < 1 || d > 3 || dimb < 1 || dimb > 4 || t_count == nullptr || s_count == nullptr) return 0;
    std::vector<int64_t> zero(nseg, 0);
    std::vector<double> sg(nseg, 1.0);
    Workspace ws;
    dispatch_kind_p(order, [&](auto kind, auto deg) {
        return dispatch_d(d, [&](auto D) {
            return dispatch_dimb(dimb, [&](auto B) {
                return rag_applyk_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value,
                                       decltype(B)::value>(nseg, zero.data(), t_count, zero.data(), s_count, d,
                                                           nullptr, nullptr, nullptr, dimb, sg.data(), order,
                                                           nullptr, ws, 0);
            });
        });
    });
    return ws.off + 256;
}

int lddmm_ragged_applyk_f32c(int nseg, const int64_t* t_start, const int64_t* t_count, const int64_t* s_start,
                             const int64_t* s_count, int d, const double* x, const double* y, const double* beta,
                             int dimb, const double* sigma, int order, double* f, void* workspace,
                             size_t workspace_bytes, lddmm_stream_t stream) {
    if (nseg < 1 || d < 1 || d > 3 || dimb < 1 || dimb > 4 || !t_start || !t_count || !s_start || !s_count) {
        set_error("ragged applyk: invalid arguments (nseg=%d d=%d dimb=%d)", nseg, d, dimb);
        return LDDMM_ERR_ARG;
    }
    for (int s = 0; s < nseg; ++s)
        if (t_start[s] < 0 || s_start[s] < 0 || t_count[s] < 0 || s_count[s] < 0 || t_count[s] > (1LL << 30) ||
            s_count[s] > (1LL << 30)) {
            set_error("ragged applyk: negative or oversized segment %d", s);
            return LDDMM_ERR_ARG;
        }
    LDDMM_TRY(rag_check_sigma(nseg, sigma, order));
    LDDMM_TRY(check_device_ptr(x, "x"));
    LDDMM_TRY(check_device_ptr(y, "y"));
    LDDMM_TRY(check_device_ptr(beta, "beta"));
    LDDMM_TRY(check_device_ptr(f, "f"));
    cudaStream_t st = (cudaStream_t)stream;
    return rag_run([&](Workspace& ws) {
        return dispatch_kind_p(order, [&](auto kind, auto deg) {
            return dispatch_d(d, [&](auto D) {
                return dispatch_dimb(dimb, [&](auto B) {
                    return rag_applyk_impl<decltype(kind)::value, decltype(deg)::value, decltype(D)::value,
                                           decltype(B)::value>(nseg, t_start, t_count, s_start, s_count, d, x, y,
                                                               beta, dimb, sigma, order, f, ws, st);
                });
            });
        });
    }, workspace, workspace_bytes, st, "ragged applyk");
}

#define RAG_DT_BODY(REAL)                                                                                         \
    RagDataArgs a{nreq, cell_size, norm, v_off, c_off, c2_off, vertices, d, cells, tgt_centers, tgt_vectors,        \
                  sigma, order, eps1, eps2, frame, energy, vertex_ptr, vertex_idx, px};                            \
    auto run = [&](Workspace& ws) {                                                                                 \
        return rag_dispatch_pq(order, [&](auto kind, auto pdeg, auto qdeg) {                                        \
            return dispatch_d(d, [&](auto D) {                                                                      \
                return rag_dt_impl<REAL, decltype(kind)::value, decltype(pdeg)::value, decltype(qdeg)::value,     \
                                   decltype(D)::value>(a, ws, (cudaStream_t)stream);                                \
            });                                                                                                     \
        });                                                                                                         \
    };

static int rag_dt_validate(int nreq, int cell_size, int norm, const int64_t* v_off, const int64_t* c_off,
                           const int64_t* c2_off, int d, const double* sigma, int order, const double* vertices,
                           const int64_t* cells, const double* c2, const double* s2, double* energy,
                           const int64_t* vptr, const int64_t* vidx, double* px) {
    if (nreq < 1 || (cell_size != 2 && cell_size != 3) || norm < 0 || norm > 2 || d < 2 || d > 3 ||
        (cell_size == 3 && d != 3) || (norm == NVARIFOLD && cell_size != 3)) {
        set_error("ragged dataterm: invalid arguments (nreq=%d cell_size=%d norm=%d d=%d)", nreq, cell_size, norm, d);
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(rag_check_offsets(nreq, v_off, "v_off"));
    LDDMM_TRY(rag_check_offsets(nreq, c_off, "c_off"));
    LDDMM_TRY(rag_check_offsets(nreq, c2_off, "c2_off"));
    LDDMM_TRY(rag_check_sigma(nreq, sigma, order));
    if (energy == nullptr && px == nullptr) {
        set_error("ragged dataterm: nothing requested");
        return LDDMM_ERR_ARG;
    }
    if (px != nullptr && order == 0) {
        set_error("ragged dataterm: the order-0 Laplacian kernel is not differentiable");
        return LDDMM_ERR_ARG;
    }
    LDDMM_TRY(check_device_ptr(vertices, "vertices"));
    LDDMM_TRY(check_device_ptr(cells, "cells"));
    if (c2_off[nreq] > 0) {
        LDDMM_TRY(check_device_ptr(c2, "target centers"));
        LDDMM_TRY(check_device_ptr(s2, "target vectors"));
    }
    if (energy) LDDMM_TRY(check_device_ptr(energy, "energy"));
    if (px) {
        LDDMM_TRY(check_device_ptr(px, "px"));
        LDDMM_TRY(check_device_ptr(vptr, "vertex_ptr"));
        LDDMM_TRY(check_device_ptr(vidx, "vertex_idx"));
    }
    return LDDMM_OK;
}

#define RAG_DT_SIG                                                                                              \
    int nreq, int cell_size, int norm, const int64_t *v_off, const int64_t *c_off, const int64_t *c2_off,        \
        const double *vertices, int d, const int64_t *cells, const double *tgt_centers, const double *tgt_vectors, \
        const double *sigma, int order, double eps1, double eps2, const double *frame, double *energy,           \
        const int64_t *vertex_ptr, const int64_t *vertex_idx, double *px, void *workspace, size_t workspace_bytes,  \
        lddmm_stream_t stream

#define RAG_DT_ENTRY(REAL, WHO)                                                                                    \
    LDDMM_TRY(rag_dt_validate(nreq, cell_size, norm, v_off, c_off, c2_off, d, sigma, order, vertices, cells,       \
                              tgt_centers, tgt_vectors, energy, vertex_ptr, vertex_idx, px));                      \
    RAG_DT_BODY(REAL)                                                                                              \
    return rag_run(run, workspace, workspace_bytes, (cudaStream_t)stream, WHO);

int lddmm_ragged_dataterm_f32c(RAG_DT_SIG) { RAG_DT_ENTRY(float, "ragged dataterm") }
int lddmm_ragged_dataterm_f64(RAG_DT_SIG) { RAG_DT_ENTRY(double, "ragged dataterm") }

#define RAG_DT_WS(REAL)                                                                                            \
    if (nreq < 1 || (cell_size != 2 && cell_size != 3) || norm < 0 || norm > 2 || d < 2 || d > 3) return 0;       \
    if (rag_check_offsets(nreq, v_off, "v_off") || rag_check_offsets(nreq, c_off, "c_off") ||                     \
        rag_check_offsets(nreq, c2_off, "c2_off"))                                                                 \
        return 0;                                                                                                  \
    std::vector<double> sg(nreq, 1.0);                                                                             \
    const double* sigma = sg.data();                                                                               \
    const double *vertices = nullptr, *tgt_centers = nullptr, *tgt_vectors = nullptr;                              \
    const int64_t *cells = nullptr, *vertex_ptr = nullptr, *vertex_idx = nullptr;                                 \
    double* energy = want_energy ? reinterpret_cast<double*>(16) : nullptr;                                        \
    double* px = want_grad ? reinterpret_cast<double*>(16) : nullptr;                                              \
    double eps1 = 0, eps2 = 0;                                                                                     \
    const double* frame = nullptr;                                                                                 \
    void* stream = nullptr;                                                                                        \
    RAG_DT_BODY(REAL)                                                                                              \
    Workspace ws;                                                                                                  \
    if (run(ws) != LDDMM_OK) return 0;                                                                             \
    return ws.off + 256;

size_t lddmm_ragged_dataterm_f32c_workspace(int nreq, int cell_size, int norm, const int64_t* v_off,
                                            const int64_t* c_off, const int64_t* c2_off, int d, int order,
                                            int want_energy, int want_grad) {
    RAG_DT_WS(float)
}
size_t lddmm_ragged_dataterm_f64_workspace(int nreq, int cell_size, int norm, const int64_t* v_off,
                                           const int64_t* c_off, const int64_t* c2_off, int d, int order,
                                           int want_energy, int want_grad) {
    RAG_DT_WS(double)
}

}  // extern "C"
