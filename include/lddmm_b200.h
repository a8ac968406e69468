/*
 * lddmm_b200.h -- C ABI of the B200 (sm_100a) point-LDDMM hot path.
 *
 * One shared library, liblddmm_b200.so, replaces the f2py Fortran module
 * `kernelFunctions_fort` of py-lddmm (source py-lddmm/kernelFunctions.f90) and
 * carries the fused shooting / adjoint / data-attachment operators that the
 * Python layer (py-lddmm pointEvolution.py, surfaces.py, curves.py) calls.
 *
 * Conventions (all entry points):
 *   - every array argument is a DEVICE pointer (cudaMalloc'd or managed),
 *     row-major and contiguous, FP64, exactly the shapes numpy hands to f2py;
 *     host pointers are rejected with LDDMM_ERR_ARG;
 *   - "x" arguments are targets and "y" arguments are sources, in the
 *     Fortran argument order (applyk(x, y, beta, ...));
 *   - `order > 4` selects the Gaussian kernel, 0..4 the Laplacian (Matern)
 *     order, as in the Fortran `ord` argument (KernelSpec forces 10 for
 *     'gauss');
 *   - nothing is allocated inside: scratch memory is the caller's
 *     `workspace` of `workspace_bytes` bytes, sized by the matching
 *     *_workspace() query on the same current device;
 *   - work is enqueued on `stream` (a cudaStream_t, 0 = legacy default) and
 *     the call returns without synchronising; results are deterministic
 *     (fixed reduction order) for a given device and shape;
 *   - return 0 on success or a negative LDDMM_ERR_* code; lddmm_last_error()
 *     gives a message for the calling thread.
 *
 * Precision variants:
 *   _f32c : FP32 pair arithmetic, FP32 partial sums over 32 sources folded
 *           into TwoSum-compensated accumulators, FP64 combine and outputs;
 *   _f64  : plain FP64 arithmetic with the Fortran's branches.
 */
#ifndef LDDMM_B200_H
#define LDDMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDDMM_OK 0
#define LDDMM_ERR_ARG (-1)         /* bad shape, order, sigma or pointer */
#define LDDMM_ERR_WORKSPACE (-2)   /* workspace missing or too small */
#define LDDMM_ERR_CUDA (-3)        /* CUDA runtime / launch error */
#define LDDMM_ERR_UNSUPPORTED (-4) /* valid in the reference, not built here */

#if defined(__GNUC__)
#define LDDMM_API __attribute__((visibility("default")))
#else
#define LDDMM_API
#endif

typedef void* lddmm_stream_t; /* cudaStream_t */

/* Message for the last failing call on this thread ("" if none). */
LDDMM_API const char* lddmm_last_error(void);
/* ABI version, bumped on any signature change. */
LDDMM_API int lddmm_abi_version(void);

/* ---- kernel sums: kernelFunctions_fort.applyk ------------------------------
 * Replaces applyk(x, y, beta, sig, ord, num_nodes, num_nodes_y, dim, dimb)
 * (py-lddmm/kernelFunctions.f90:1-54, called from kernelFunctions.py:320,327):
 *   f[k, :] = sum_l K(x_k, y_l) beta[l, :]
 * x (n, d) targets, y (m, d) sources, beta (m, dimb), f (n, dimb); d in 1..3. */
LDDMM_API size_t lddmm_applyk_f32c_workspace(int64_t n, int64_t m, int d, int dimb);
LDDMM_API int lddmm_applyk_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                      double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                      lddmm_stream_t stream);
LDDMM_API size_t lddmm_applyk_f64_workspace(int64_t n, int64_t m, int d, int dimb);
LDDMM_API int lddmm_applyk_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d, int dimb,
                     double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                     lddmm_stream_t stream);

/* ---- kernel sums: kernelFunctions_fort.applykdifft -------------------------
 * Replaces applykdifft(x, y, a1, a2, sig, ord, num_nodes, num_nodes_y, dim,
 * dimb, na) (py-lddmm/kernelFunctions.f90:56-114, kernelFunctions.py:421,423):
 *   f[k, :] = sum_l K'(x_k, y_l) 2 (x_k - y_l) sum_{i,c} a1[i,k,c] a2[i,l,c]
 * a1 (na, n, dimb), a2 (na, m, dimb), f (n, d); na*dimb <= 12; order != 0. */
LDDMM_API size_t lddmm_applykdifft_f32c_workspace(int64_t n, int64_t m, int na, int d, int dimb);
LDDMM_API int lddmm_applykdifft_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* a1,
                           const double* a2, int na, int d, int dimb, double sigma, int order, double* f,
                           void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_applykdifft_f64_workspace(int64_t n, int64_t m, int na, int d, int dimb);
LDDMM_API int lddmm_applykdifft_f64(const double* x, int64_t n, const double* y, int64_t m, const double* a1,
                          const double* a2, int na, int d, int dimb, double sigma, int order, double* f,
                          void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* ---- diagnostics ------------------------------------------------------------
 * No counterpart in the reference.  Launches `blocks` x `threads` threads that
 * each issue 8*iters FP32 FMAs (what = 0) or 8*iters MUFU ex2 (what = 1) and
 * write one float to out[blocks*threads].  Timed by the benchmark to measure
 * the issue-rate peaks that the kernel-sum roofline is quoted against. */
LDDMM_API int lddmm_probe_launch(int what, int blocks, int threads, int iters, float* out, lddmm_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* LDDMM_B200_H */
