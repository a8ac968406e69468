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

// Bulk copies on the copy engine (TMA), completing on a shared-memory
// mbarrier: one thread arms the barrier with the byte count and issues the
// copies; every thread waits for the barrier's phase.  No multicast.
LDDMM_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
LDDMM_D void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
LDDMM_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
LDDMM_D void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
LDDMM_D void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
LDDMM_D bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Polls of a bounded wait (about a second at most): a copy that has not
// completed by then never will, and the caller gives up instead of hanging.
constexpr int kWaitPolls = 1 << 24;
LDDMM_D bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    for (int i = 0; i < kWaitPolls; ++i) {
        if (mbar_test(bar, parity)) return true;
        if (i >= 32) __nanosleep(32);
    }
    return false;
}

struct double4a {  // 32-byte record of four doubles
    double x, y, z, w;
};

}  // namespace lddmm
