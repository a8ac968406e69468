// Common device helpers for the LDDMM kernel sums (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LDDMM_HD __host__ __device__ __forceinline__
#define LDDMM_D __device__ __forceinline__

namespace lddmm {

// Kernel families: Gaussian (Fortran `ord > 4`) and Laplacian/Matern of order 0..4.
enum KernelKind : int { KGAUSS = 0, KLAP = 1 };

// Fortran default-real literal 1e-8 of the zero-distance branch, promoted to real(8).
static constexpr double kZeroThresh = (double)1e-8f;

// ---------------------------------------------------------------------------
// Segments: one launch can sweep several independent problems (requests).
// Every block finds its segment by binary search over item0.
// ---------------------------------------------------------------------------
struct SegDesc {
    long long tgt;    // first target row in the packed target arrays
    long long src;    // first source row in the packed source arrays (TILE aligned)
    long long part;   // first row of this segment in the partial-sum buffer
    int n_tgt;        // targets
    int n_src_tiles;  // source tiles (sources zero-padded to a TILE multiple)
    int n_tb;         // target blocks
    int split;        // source chunks (one block per target block and chunk)
    int item0;        // first block index of this segment
    int sym_tiles;    // > 0: the first sym_tiles source tiles are the targets' own records and the
                      // sum is symmetric in (target, source): see sweep_kernel<Op, true>
};

struct SweepGrid {
    SegDesc seg0;        // used when nseg == 0 (single problem)
    const SegDesc* segs; // device table (ragged launches)
    int nseg;
    int n_items;
};

LDDMM_D SegDesc find_segment(const SweepGrid& g, int item) {
    if (g.nseg == 0) return g.seg0;
    int lo = 0, hi = g.nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (g.segs[mid].item0 <= item) lo = mid; else hi = mid - 1;
    }
    return g.segs[lo];
}

// ---------------------------------------------------------------------------
// FP32 arithmetic helpers
// ---------------------------------------------------------------------------
// 2^x on the multi-function unit (PTX ex2.approx.ftz.f32, relative error ~2^-22).
LDDMM_D float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

LDDMM_D float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Knuth TwoSum: s + e == a + b exactly.
LDDMM_D void two_sum_acc(float& s, float& c, float p) {
    float t = s + p;
    float bp = t - s;
    float e = (s - (t - bp)) + (p - bp);
    s = t;
    c += e;
}

// cp.async 16-byte global -> shared copy (L2 only), and group management.
LDDMM_D void cp_async16(void* smem, const void* gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
LDDMM_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
LDDMM_D void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

struct double4a {  // 32-byte record of four doubles
    double x, y, z, w;
};

}  // namespace lddmm
