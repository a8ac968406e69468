// Packing kernels (FP64 user arrays -> prescaled FP32/FP64 planes) and the
// deterministic combine of per-chunk partial sums.
#pragma once
#include "common.cuh"
#include "ops.cuh"

namespace lddmm {

// Centre of the bounding box of x (n, d) and y (m, d): center[0..d).  The
// kernels are translation invariant, and packing coordinates relative to this
// centre halves the magnitude (and so the FP32 rounding error) of the packed
// coordinates.
//
// Many blocks reduce min / max of order-preserving 64-bit keys of the
// coordinates with atomicMin / atomicMax: min and max are exact, so the result
// does not depend on the order of the blocks.  The centre buffer holds
// kCenterWords doubles: the centre in [0, 4) and the six keys in [4, 10).
constexpr int kCenterWords = 16;
constexpr long long kKeyMax = 0x7FFFFFFFFFFFFFFFLL;
constexpr long long kKeyMin = -kKeyMax - 1;

// signed-integer order of the keys == numeric order of the doubles (no NaN)
LDDMM_D long long bbox_key(double v) {
    const long long b = __double_as_longlong(v);
    return b >= 0 ? b : (b ^ kKeyMax);
}

LDDMM_D double bbox_val(long long k) { return __longlong_as_double(k >= 0 ? k : (k ^ kKeyMax)); }

// warp + block reduction of per-thread key bounds, then one atomic per block
// and component into keys[0..3) (min) and keys[3..6) (max)
LDDMM_D void bbox_block_commit(long long (&l)[3], long long (&h)[3], long long* keys) {
    __shared__ long long sl[3][32], sh[3][32];
    for (int off = 16; off > 0; off >>= 1)
        for (int j = 0; j < 3; ++j) {
            l[j] = min(l[j], __shfl_down_sync(0xffffffffu, l[j], off));
            h[j] = max(h[j], __shfl_down_sync(0xffffffffu, h[j], off));
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
        for (int j = 0; j < 3; ++j) {
            sl[j][warp] = l[j];
            sh[j][warp] = h[j];
        }
    __syncthreads();
    if (warp == 0) {
        for (int j = 0; j < 3; ++j) {
            l[j] = lane < nw ? sl[j][lane] : kKeyMax;
            h[j] = lane < nw ? sh[j][lane] : kKeyMin;
        }
        for (int off = 16; off > 0; off >>= 1)
            for (int j = 0; j < 3; ++j) {
                l[j] = min(l[j], __shfl_down_sync(0xffffffffu, l[j], off));
                h[j] = max(h[j], __shfl_down_sync(0xffffffffu, h[j], off));
            }
        if (lane == 0)
            for (int j = 0; j < 3; ++j) {
                if (l[j] != kKeyMax) atomicMin(keys + j, l[j]);
                if (h[j] != kKeyMin) atomicMax(keys + 3 + j, h[j]);
            }
    }
}

static __global__ void bbox_init_kernel(long long* __restrict__ keys) {
    if (threadIdx.x < 6) keys[threadIdx.x] = threadIdx.x < 3 ? kKeyMax : kKeyMin;
}

static __global__ void bbox_keys_kernel(const double* __restrict__ x, long long n, const double* __restrict__ y,
                                        long long m, int d, long long* __restrict__ keys) {
    long long l[3] = {kKeyMax, kKeyMax, kKeyMax}, h[3] = {kKeyMin, kKeyMin, kKeyMin};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n + m;
         i += (long long)gridDim.x * blockDim.x) {
        const double* p = i < n ? x + i * d : y + (i - n) * d;
        for (int j = 0; j < d; ++j) {
            const long long k = bbox_key(p[j]);
            l[j] = min(l[j], k);
            h[j] = max(h[j], k);
        }
    }
    bbox_block_commit(l, h, keys);
}

static __global__ void bbox_finish_kernel(const long long* __restrict__ keys, int d, int nonempty,
                                          double* __restrict__ center) {
    if (threadIdx.x < 3) {
        const int j = threadIdx.x;
        center[j] = (j < d && nonempty) ? 0.5 * (bbox_val(keys[j]) + bbox_val(keys[3 + j])) : 0.0;
    }
}

// center: kCenterWords doubles of device memory (see above)
inline void launch_bbox_center(const double* x, long long n, const double* y, long long m, int d, double* center,
                               cudaStream_t st) {
    long long* keys = reinterpret_cast<long long*>(center + 4);
    const long long tot = n + m;
    const int blocks = (int)std::max<long long>(1, std::min<long long>(148 * 4, (tot + 2047) / 2048));
    bbox_init_kernel<<<1, 32, 0, st>>>(keys);
    bbox_keys_kernel<<<blocks, 256, 0, st>>>(x, n, y, m, d, keys);
    bbox_finish_kernel<<<1, 32, 0, st>>>(keys, d, tot > 0 ? 1 : 0, center);
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
