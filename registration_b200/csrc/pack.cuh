// Packing kernels (FP64 user arrays -> prescaled FP32/FP64 planes) and the
// deterministic combine of per-chunk partial sums.
#pragma once
#include "common.cuh"
#include "ops.cuh"

namespace lddmm {

// Centre of the bounding box of x (n, d) and y (m, d): center[0..d).  The
// kernels are translation invariant, and packing coordinates relative to this
// centre halves the magnitude (and so the FP32 rounding error) of the packed
// coordinates.  One block; min/max do not depend on the reduction order.
static __global__ void bbox_center_kernel(const double* __restrict__ x, long long n, const double* __restrict__ y,
                                          long long m, int d, double* __restrict__ center) {
    __shared__ double lo[3][256], hi[3][256];
    double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    for (long long i = threadIdx.x; i < n + m; i += blockDim.x) {
        const double* p = i < n ? x + i * d : y + (i - n) * d;
        for (int j = 0; j < d; ++j) {
            l[j] = fmin(l[j], p[j]);
            h[j] = fmax(h[j], p[j]);
        }
    }
    for (int j = 0; j < 3; ++j) {
        lo[j][threadIdx.x] = l[j];
        hi[j][threadIdx.x] = h[j];
    }
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int j = 0; j < 3; ++j) {
                lo[j][threadIdx.x] = fmin(lo[j][threadIdx.x], lo[j][threadIdx.x + s]);
                hi[j][threadIdx.x] = fmax(hi[j][threadIdx.x], hi[j][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int j = 0; j < 3; ++j) center[j] = j < d && n + m > 0 ? 0.5 * (lo[j][0] + hi[j][0]) : 0.0;
}

// Points: value j of row i is (x[i*d + j] - center[j]) * scale (zero for j >= d or i >= n).
// FP32: one float4 word per row in plane 0.  FP64: two double2 words (planes 0, 1).
template <class Real>
static __global__ void pack_points_kernel(const double* __restrict__ x, long long n, int d, double scale,
                                          const double* __restrict__ center, float4* __restrict__ out,
                                          long long stride, long long n_pad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_pad;
         i += (long long)gridDim.x * blockDim.x) {
        double v[4] = {0, 0, 0, 0};
        if (i < n)
            for (int j = 0; j < d && j < 4; ++j) v[j] = (x[i * d + j] - (center ? center[j] : 0.0)) * scale;
        if constexpr (sizeof(Real) == 4) {
            out[i] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
        } else {
            double2* o = reinterpret_cast<double2*>(out);
            o[i] = make_double2(v[0], v[1]);
            o[stride + i] = make_double2(v[2], v[3]);
        }
    }
}

// Gather spec for value planes: value w of row i is src[i*row_stride + off[w]] * mult.
struct Gather {
    const double* src;
    long long row_stride;
    long long off[12];
    int nvals;
    double mult;
};

// Writes `g.nvals` values per row into consecutive planes starting at first_plane.
template <class Real>
static __global__ void pack_values_kernel(const Gather g, long long n, float4* __restrict__ out, long long stride,
                                   long long n_pad, int first_plane) {
    constexpr int PW = Traits<Real>::PER_WORD;
    const int nwords = (g.nvals + PW - 1) / PW;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_pad;
         i += (long long)gridDim.x * blockDim.x) {
        for (int w = 0; w < nwords; ++w) {
            Real v[PW];
            for (int q = 0; q < PW; ++q) {
                const int idx = w * PW + q;
                v[q] = (i < n && idx < g.nvals) ? (Real)(g.src[i * g.row_stride + g.off[idx]] * g.mult) : (Real)0;
            }
            float4* dst = out + (long long)(first_plane + w) * stride + i;
            if constexpr (sizeof(Real) == 4) {
                *dst = make_float4(v[0], v[1], v[2], v[3]);
            } else {
                *reinterpret_cast<double2*>(dst) = make_double2(v[0], v[1]);
            }
        }
    }
}

// out[i*out_ld + col0 + c] = scale * sum_{chunk < split} part[(chunk*n + i)*nout + c]
static __global__ void combine_kernel(const double* __restrict__ part, long long n, int nout, int split,
                                      double scale, double* __restrict__ out, long long out_ld, int col0) {
    const long long total = n * nout;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const long long i = q / nout;
        const int c = (int)(q - i * nout);
        double s = 0.0;
        for (int k = 0; k < split; ++k) s += part[((long long)k * n + i) * nout + c];
        out[i * out_ld + col0 + c] = scale * s;
    }
}

// Like combine_kernel but the partial rows hold `nout` values of which only
// the first `ncols` are written out.
static __global__ void combine_cols_kernel(const double* __restrict__ part, long long n, int nout, int ncols,
                                           int split, double scale, double* __restrict__ out, long long out_ld,
                                           int col0) {
    const long long total = n * ncols;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const long long i = q / ncols;
        const int c = (int)(q - i * ncols);
        double s = 0.0;
        for (int k = 0; k < split; ++k) s += part[((long long)k * n + i) * nout + c];
        out[i * out_ld + col0 + c] = scale * s;
    }
}

inline int grid_for(long long work, int block = 256, int max_blocks = 148 * 16) {
    long long b = (work + block - 1) / block;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

}  // namespace lddmm
