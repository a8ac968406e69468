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
/* Allocation-free variant of lddmm_applyk_f32c -- no counterpart in the
 * reference.  For callers that cannot allocate GPU memory (a plug-in whose
 * host framework owns all device allocations, an FFI caller without a CUDA
 * allocator, a path where cudaMalloc / cudaFree would synchronise the device):
 * the caller passes the inputs and the output only, and the scratch memory is a
 * 32 MiB array in the library's static device memory (held by every GPU that
 * loads the library until exit).  Shapes whose scratch exceeds 32 MiB (about
 * n = m = 400,000 with dimb <= 4) return LDDMM_ERR_WORKSPACE before any launch.
 * All calls on a device share that array: calls that overlap on the GPU race,
 * so order them on one stream.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress); make it before any stream capture. */
LDDMM_API int lddmm_applyk_f32c_noalloc(const double* x, int64_t n, const double* y, int64_t m, const double* beta,
                                        int d, int dimb, double sigma, int order, double* f, lddmm_stream_t stream);
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

/* ---- divergence: Kernel.applyDivergence -------------------------------------
 * Replaces the dense numpy applyDivergence (py-lddmm/kernelFunctions.py:510-530,
 * used by landmarkDirectEvolutionEuler(withJacobian=True)), without the
 * kernel weight factor (the caller multiplies by KernelSpec.weight):
 *   f[k] = sum_l K'(x_k, y_l) 2 <x_k - y_l, a_l>
 * x (n, d) targets, y (m, d) sources, a (m, d), f (n). */
LDDMM_API size_t lddmm_applydiv_f32c_workspace(int64_t n, int64_t m, int d);
LDDMM_API int lddmm_applydiv_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* a, int d,
                                  double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                  lddmm_stream_t stream);
LDDMM_API size_t lddmm_applydiv_f64_workspace(int64_t n, int64_t m, int d);
LDDMM_API int lddmm_applydiv_f64(const double* x, int64_t n, const double* y, int64_t m, const double* a, int d,
                                 double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                 lddmm_stream_t stream);

/* ---- geodesic shooting: pointEvolution.landmarkDirectEvolutionEuler ----------
 * Replaces the T-step Euler loop of py-lddmm/pointEvolution.py:666-730 (no
 * affine part, no optional outputs):
 *   xt[0] = x0,  xt[t+1] = xt[t] + dt K(xt[t], xt[t]) at[t]
 * with dt = 1/T (the reference) when dt <= 0, or the given dt (a segment of a
 * longer shot), and, if energy != NULL, writes
 * energy[0] = sum_t rw dt <at[t], K(xt[t]) at[t]>,
 * the deformation cost of objectiveFunDef (py-lddmm/surfaceMatching.py:205-212,
 * curveMatching.py:168-173), from the same kernel sums.
 * x0 (n, d), at (T, n, d), xt (T+1, n, d); energy: one double on the device. */
LDDMM_API size_t lddmm_shoot_f32c_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_shoot_f32c(const double* x0, int64_t n, int d, const double* at, int T, double dt,
                               double sigma, int order, double regweight, double* xt, double* energy,
                               void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_shoot_f64_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_shoot_f64(const double* x0, int64_t n, int d, const double* at, int T, double dt,
                              double sigma, int order, double regweight, double* xt, double* energy,
                              void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* The same shot along a search direction: the momenta are
 *   at_try[t] = at[t] - (*eps) dir[t]   (eps: one double on the device)
 * written to at_try (T, n, d), then shot as above.  No single counterpart in
 * the reference: it is the trial step of SurfaceMatching / CurveMatching.updateTry
 * (py-lddmm/surfaceMatching.py:255-289, curveMatching.py:185-208), atTry =
 * at - eps dir followed by its objectiveFunDef shot, in one call whose eps
 * lives on the device (a CUDA graph can replay it for every trial step).
 * Same workspace as lddmm_shoot_*_workspace; the products and differences are
 * rounded as two FP64 operations, as numpy's at - eps * dir. */
LDDMM_API int lddmm_shoot_along_f32c(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                     const double* eps, int T, double dt, double sigma, int order, double regweight,
                                     double* at_try, double* xt, double* energy, void* workspace,
                                     size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_shoot_along_f64(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                    const double* eps, int T, double dt, double sigma, int order, double regweight,
                                    double* at_try, double* xt, double* energy, void* workspace,
                                    size_t workspace_bytes, lddmm_stream_t stream);

/* A batch of trial steps along one direction: step sizes eps[0..nbatch) on
 * the device, outputs stacked per step size: at_try (nbatch, T, n, d), xt
 * (nbatch, T+1, n, d), energy (nbatch) (may be NULL).  Slot b equals, bit for
 * bit, lddmm_shoot_along_* with eps[b].  No counterpart in the reference: the
 * step sizes cg's line search tries next (eps / 2^k while halving, eps 1.25^j
 * while growing; conjugateGradient.py:140-183) are shot side by side, one
 * thread-block cluster each, when the point set is small enough for a cluster
 * to leave most SMs idle (lddmm_trial_batch_size > 1); otherwise one after the
 * other.  1 <= nbatch <= 4096. */
LDDMM_API size_t lddmm_shoot_along_batch_f32c_workspace(int64_t n, int d, int T, int nbatch);
LDDMM_API int lddmm_shoot_along_batch_f32c(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                           const double* eps, int nbatch, int T, double dt, double sigma, int order,
                                           double regweight, double* at_try, double* xt, double* energy,
                                           void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_shoot_along_batch_f64_workspace(int64_t n, int d, int T, int nbatch);
LDDMM_API int lddmm_shoot_along_batch_f64(const double* x0, int64_t n, int d, const double* at, const double* dir,
                                          const double* eps, int nbatch, int T, double dt, double sigma, int order,
                                          double regweight, double* at_try, double* xt, double* energy,
                                          void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* How many trial steps of a problem (n points in d dimensions, a data term of
 * nc own and nc2 target cells; shot and value kernel sums in FP64 when
 * shot_fp64 / value_fp64, else FP32c) one batched launch runs side by side:
 * 1 when the batch would run one step size after the other (the general
 * path), else up to 24, bounded by the clusters of the shot and value kernels
 * that are resident on the device at once. */
LDDMM_API int lddmm_trial_batch_size(int64_t n, int d, int64_t nc, int64_t nc2, int shot_fp64, int value_fp64);

/* ---- Hamiltonian adjoint: landmarkHamiltonianCovector / Gradient --------------
 * Replaces the backward loop of py-lddmm/pointEvolution.py:735-765 and the
 * gradient of :793-817 (no affine part), given the trajectory xt:
 *   pxt[T] = px1,
 *   pxt[t] = pxt[t+1] + dt applyDiffKT(xt[t], [pxt[t+1], at[t], -2 rw at[t]],
 *                                             [at[t], pxt[t+1], at[t]]),
 *   dat[t] = 2 rw at[t] - pxt[t+1]          (dat may be NULL)
 * dt <= 0 means 1/T (the reference); a positive dt runs a segment of a longer
 * adjoint (checkpointed trajectories).
 * xt (T+1, n, d), at (T, n, d), px1 (n, d), pxt (T+1, n, d), dat (T, n, d). */
LDDMM_API size_t lddmm_covector_f32c_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_covector_f32c(const double* xt, int64_t n, int d, const double* at, int T, double dt,
                                  const double* px1, double sigma, int order, double regweight, double* pxt,
                                  double* dat, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_covector_f64_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_covector_f64(const double* xt, int64_t n, int d, const double* at, int T, double dt,
                                 const double* px1, double sigma, int order, double regweight, double* pxt,
                                 double* dat, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* ---- metric inner products of directions: Matching.dotProduct -----------------
 * Replaces the loops of py-lddmm/surfaceMatching.py:353-377 and
 * curveMatching.py:286-304 (no affine part):
 *   out[l] = sum_{t<T} sum_k <g2[l][t][k], sum_j K(xt[t][k], xt[t][j]) g1[t][j]>,  l < m <= 8
 * xt (>= T, n, d) the trajectory (rows 0..T-1), g1 (T, n, d), g2: a HOST array of
 * m device pointers to (T, n, d) arrays, out: m doubles on the device.  Kernel
 * sums in FP32 with compensated partials (f32c) or FP64, dot products and all
 * reductions in FP64 in a fixed order (two launches for all T steps). */
LDDMM_API size_t lddmm_metric_dots_f32c_workspace(int64_t n, int d, int T, int m);
LDDMM_API int lddmm_metric_dots_f32c(const double* xt, int64_t n, int d, int T, const double* g1,
                                     const double* const* g2, int m, double sigma, int order, double* out,
                                     void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_metric_dots_f64_workspace(int64_t n, int d, int T, int m);
LDDMM_API int lddmm_metric_dots_f64(const double* xt, int64_t n, int d, int T, const double* g1,
                                    const double* const* g2, int m, double sigma, int order, double* out,
                                    void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* ---- EPDiff shooting: pointEvolution.landmarkEPDiff ---------------------------
 * Replaces py-lddmm/pointEvolution.py:599-658 (no affine / optional outputs):
 *   xt[k+1] = xt[k] + dt K(xt[k]) at[k],
 *   at[k+1] = at[k] - dt applyDiffKT(xt[k], [at[k]], [at[k]])   (k < T-1)
 * x0, a0 (n, d), xt (T+1, n, d), at (T, n, d). */
LDDMM_API size_t lddmm_epdiff_f32c_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_epdiff_f32c(const double* x0, int64_t n, int d, const double* a0, int T, double sigma, int order,
                                double* xt, double* at, void* workspace, size_t workspace_bytes,
                                lddmm_stream_t stream);
LDDMM_API size_t lddmm_epdiff_f64_workspace(int64_t n, int d, int T);
LDDMM_API int lddmm_epdiff_f64(const double* x0, int64_t n, int d, const double* a0, int T, double sigma, int order,
                               double* xt, double* at, void* workspace, size_t workspace_bytes,
                               lddmm_stream_t stream);

/* ---- data attachment: surfaces / curves current, measure, varifold ------------
 * Replaces surfaces.{current,measure,varifold}Norm{0,Def,Gradient}
 * (py-lddmm/surfaces.py:1009-1276) and curves.{current,measure}Norm{0,Def,Gradient}
 * (py-lddmm/curves.py:539-703) -- the fun_obj0 / fun_obj / fun_objGrad plug-in
 * triple of SurfaceMatchingParam.errorType (surfaceMatching.py:29-40).
 *   cell_size   3: triangles (d = 3), 2: edges (d = 2 or 3)
 *   norm        0 current, 1 measure, 2 varifold (triangles only)
 *   vertices (nv, d) and cells (nc, cell_size) int64 of the deformed shape S1;
 *   tgt_centers / tgt_vectors (nc2, d): centres and surfels/tangents of the
 *   target shape S2 (nc2 = 0 for Norm0 of S1);
 *   eps1 / eps2: the constant under the square root of the cell weights of S1
 *   and S2 (1e-10 in the reference, 0 in curves.measureNorm0);
 *   energy (if not NULL): <S1,S1> - 2 <S1,S2>  (NormDef; Norm0 with nc2 = 0);
 *   px (if not NULL): the gradient of |S1 - S2|^2 w.r.t. the vertices (nv, d)
 *   (NormGradient); it needs the vertex -> (cell, corner) incidence in CSR form:
 *   vertex_ptr (nv+1), vertex_idx (nc*cell_size) with entries cell*cell_size+corner. */
LDDMM_API size_t lddmm_dataterm_f32c_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2,
                                               int order, int want_energy, int want_grad);
LDDMM_API int lddmm_dataterm_f32c(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                  const int64_t* cells, int64_t nc, const double* tgt_centers,
                                  const double* tgt_vectors, int64_t nc2, double sigma, int order, double eps1,
                                  double eps2, double* energy, const int64_t* vertex_ptr, const int64_t* vertex_idx,
                                  double* px, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_dataterm_f64_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc, int64_t nc2,
                                              int order, int want_energy, int want_grad);
LDDMM_API int lddmm_dataterm_f64(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                 const int64_t* cells, int64_t nc, const double* tgt_centers,
                                 const double* tgt_vectors, int64_t nc2, double sigma, int order, double eps1,
                                 double eps2, double* energy, const int64_t* vertex_ptr, const int64_t* vertex_idx,
                                 double* px, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* Values of a batch of vertex sets of the same shape (the final positions of
 * batched trial steps): vertex set b starts at vertices + b vertex_stride
 * (vertex_stride >= nv d), energy[b] as lddmm_dataterm_* with px NULL, bit for
 * bit.  One cluster per vertex set side by side for small shapes, else one
 * after the other.  1 <= nbatch <= 4096. */
LDDMM_API size_t lddmm_dataterm_value_batch_f32c_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc,
                                                           int64_t nc2, int order, int nbatch);
LDDMM_API int lddmm_dataterm_value_batch_f32c(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                              const int64_t* cells, int64_t nc, const double* tgt_centers,
                                              const double* tgt_vectors, int64_t nc2, double sigma, int order,
                                              double eps1, double eps2, int nbatch, int64_t vertex_stride,
                                              double* energy, void* workspace, size_t workspace_bytes,
                                              lddmm_stream_t stream);
LDDMM_API size_t lddmm_dataterm_value_batch_f64_workspace(int cell_size, int norm, int64_t nv, int d, int64_t nc,
                                                          int64_t nc2, int order, int nbatch);
LDDMM_API int lddmm_dataterm_value_batch_f64(int cell_size, int norm, const double* vertices, int64_t nv, int d,
                                             const int64_t* cells, int64_t nc, const double* tgt_centers,
                                             const double* tgt_vectors, int64_t nc2, double sigma, int order,
                                             double eps1, double eps2, int nbatch, int64_t vertex_stride,
                                             double* energy, void* workspace, size_t workspace_bytes,
                                             lddmm_stream_t stream);

/* ---- dense-weight kernel sums: kff.applykmat / kff.applykdiffmat ---------------
 * Replace py-lddmm/kernelFunctions.f90:499-552 and :554-610 (called by
 * Kernel.applyK(matrixWeights=True), kernelFunctions.py:310-329, and
 * Kernel.applyDiffKmat, kernelFunctions.py:405-410):
 *   applykmat:     f[k,:] = sum_l K(x_k, y_l) beta[k,l,:]       beta (n, m, dimb), dimb <= 8
 *   applykdiffmat: f[k,:] = sum_l K'(x_k, y_l) 2 (x_k - y_l) beta[k,l]   beta (n, m), f (n, d)
 * x: targets (n, d), y: sources (m, d).  HBM-bound on beta; no workspace. */
LDDMM_API int lddmm_applykmat_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                                   int dimb, double sigma, int order, double* f, lddmm_stream_t stream);
LDDMM_API int lddmm_applykmat_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                                  int dimb, double sigma, int order, double* f, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiffmat_f32c(const double* x, int64_t n, const double* y, int64_t m, const double* beta,
                                       int d, double sigma, int order, double* f, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiffmat_f64(const double* x, int64_t n, const double* y, int64_t m, const double* beta,
                                      int d, double sigma, int order, double* f, lddmm_stream_t stream);

/* ---- first / second derivative loops: kff.applykdiff1 ... applykdiff11and12 -----
 * Replace py-lddmm/kernelFunctions.f90:116-496 (Kernel.applyDiffK, applyDiffK2,
 * applyDiffK1and2, applyDDiffK11and12, kernelFunctions.py:391-455, and the
 * dense applyDDiffK11 / applyDDiffK12, :459-507), self-interaction over x (n, d):
 *   applykdiff1      f_k =  sum_l K' 2 <x_k-x_l, a1_k> a2_l
 *   applykdiff2      f_k = -sum_l K' 2 <x_k-x_l, a1_l> a2_l
 *   applykdiff1and2  f_k =  sum_l K' 2 <x_k-x_l, a1_k-a1_l> a2_l
 *   applykdiff11     f_k =  sum_l <a1_k,a2_l> (K'' 4 <x_k-x_l, p_k> (x_k-x_l) + K' 2 p_k)
 *   applykdiff12     f_k = -sum_l <a1_k,a2_l> (K'' 4 <x_k-x_l, p_l> (x_k-x_l) + K' 2 p_l)
 *   applykdiff11and12 f_k = sum_l <a1_k,a2_l> (K'' 4 <dx, p_k-p_l> dx + K' 2 (p_k-p_l))
 * a1, a2, p, f (n, d).  Order 0 is rejected; the 11 / 12 routines need a
 * Gaussian or a Laplacian of order >= 2 (K'' table c2_).  The reference's
 * 11 / 12 loops run over an undeclared y; these compute the intended y = x.
 * Workspace: lddmm_applykdiffx_*_workspace(routine, n, d, order) with routine
 * 1, 2, 3 (1and2), 11, 12, 13 (11and12). */
LDDMM_API size_t lddmm_applykdiffx_f32c_workspace(int routine, int64_t n, int d, int order);
LDDMM_API size_t lddmm_applykdiffx_f64_workspace(int routine, int64_t n, int d, int order);
LDDMM_API int lddmm_applykdiff1_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                     double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                     lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff1_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                    double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                    lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff2_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                     double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                     lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff2_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                    double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                                    lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff1and2_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                         double sigma, int order, double* f, void* workspace,
                                         size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff1and2_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                        double sigma, int order, double* f, void* workspace,
                                        size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff11_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                      const double* p, double sigma, int order, double* f, void* workspace,
                                      size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff11_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                     const double* p, double sigma, int order, double* f, void* workspace,
                                     size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff12_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                      const double* p, double sigma, int order, double* f, void* workspace,
                                      size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff12_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                     const double* p, double sigma, int order, double* f, void* workspace,
                                     size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff11and12_f32c(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                           const double* p, double sigma, int order, double* f, void* workspace,
                                           size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_applykdiff11and12_f64(const double* x, int64_t n, int d, const double* a1, const double* a2,
                                          const double* p, double sigma, int order, double* f, void* workspace,
                                          size_t workspace_bytes, lddmm_stream_t stream);

/* ---- affine kernel parts: KernelSpec(affine = 'affine' | 'euclidean') ----------
 * No f2py counterpart: py-lddmm/kernelFunctions.py:334-367 (applyK) and
 * :431-448 (applyDiffKT) add these terms in numpy after the kernel sums.
 * lddmm_moments_f64: out[i * dimb + j] = sum_l (x_l - c)_i a_l,j  (i < d, j < dimb)
 *   and out[d * dimb + j] = sum_l a_l,j; x (m, d), a (m, dimb), c (d) or NULL
 *   for 0; out: d * dimb + dimb doubles; dimb <= 4; FP64, fixed reduction order;
 *   workspace sized by lddmm_moments_f64_workspace.
 * lddmm_rows_affine_f64: f[k, j] += sum_q (u[k, q] - c[q]) W[q, j] + b[j]
 *   u (n, Q), c (Q) or NULL, W (Q, J), b (J) or NULL, f (n, J); Q <= 16, J <= 4. */
LDDMM_API size_t lddmm_moments_f64_workspace(int64_t m, int d, int dimb);
LDDMM_API int lddmm_moments_f64(const double* x, int64_t m, int d, const double* a, int dimb, const double* center,
                                double* out, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API int lddmm_rows_affine_f64(const double* u, int64_t n, int Q, const double* center, const double* W,
                                    const double* b, int J, double* f, lddmm_stream_t stream);

/* ---- ragged launches: many independent problems in one launch ----------------
 * No single counterpart in the reference (which solves one problem per process);
 * each segment computes exactly what the single-problem entry point above
 * computes for its own rows, with its own kernel width, and its results do not
 * depend on the other segments of the launch (per-segment chunking and FP64
 * reduction trees).  Offsets / sigma / regweight arrays are HOST arrays; the
 * segment tables built from them are copied to the device by each call, so a
 * call on a stream that is capturing a CUDA graph is refused (LDDMM_ERR_ARG)
 * before anything is enqueued.  The single-problem entry points above enqueue
 * only kernels, device-to-device copies and memsets and can be captured.
 *
 * Shooting / adjoint of nreq requests, request s owning points
 * [v_off[s], v_off[s+1]) (v_off has nreq+1 entries, v_off[0] = 0):
 *   x0 (v_off[nreq], d); at / dat: request s's (T, n_s, d) block at row T*v_off[s];
 *   xt / pxt: request s's (T+1, n_s, d) block at row (T+1)*v_off[s];
 *   px1: (v_off[nreq], d); energy[s] = rw_s dt sum_t <a_t, K(x_t) a_t>; dt = 1/T.
 * (pointEvolution.py:666-817, surfaceMatching.py:187-221) */
LDDMM_API size_t lddmm_ragged_shoot_f32c_workspace(int nreq, const int64_t* v_off, int d, int T, int order);
LDDMM_API int lddmm_ragged_shoot_f32c(int nreq, const int64_t* v_off, int d, const double* x0, const double* at,
                                      int T, const double* sigma, int order, const double* regweight, double* xt,
                                      double* energy, void* workspace, size_t workspace_bytes,
                                      lddmm_stream_t stream);
LDDMM_API size_t lddmm_ragged_covector_f32c_workspace(int nreq, const int64_t* v_off, int d, int T, int order);
LDDMM_API int lddmm_ragged_covector_f32c(int nreq, const int64_t* v_off, int d, const double* xt, const double* at,
                                         int T, const double* px1, const double* sigma, int order,
                                         const double* regweight, double* pxt, double* dat, void* workspace,
                                         size_t workspace_bytes, lddmm_stream_t stream);
/* applyK segments (kernelFunctions.py:161-179): segment s maps targets x rows
 * [t_start[s], +t_count[s]) and sources y rows [s_start[s], +s_count[s]) with
 * weights beta (rows aligned with y, dimb <= 4 columns) to f rows
 * [sum_{r<s} t_count[r], +t_count[s]) (compact, in segment order). */
LDDMM_API size_t lddmm_ragged_applyk_f32c_workspace(int nseg, const int64_t* t_count, const int64_t* s_count, int d,
                                                    int dimb, int order);
LDDMM_API int lddmm_ragged_applyk_f32c(int nseg, const int64_t* t_start, const int64_t* t_count,
                                       const int64_t* s_start, const int64_t* s_count, int d, const double* x,
                                       const double* y, const double* beta, int dimb, const double* sigma, int order,
                                       double* f, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
/* Data terms of nreq requests (surfaces.py:1009-1276, curves.py:539-703):
 * request s owns vertices [v_off[s], v_off[s+1]), cells [c_off[s], c_off[s+1])
 * (entries are GLOBAL vertex indices) and target cells [c2_off[s], c2_off[s+1]);
 * vertex_ptr (v_off[nreq]+1) / vertex_idx (c_off[nreq]*cell_size, entries
 * global cell*cell_size+corner) is the concatenated incidence; energy[nreq].
 * frame: NULL (each request is packed relative to the centre of the bounding box
 * of its cells, as the single-problem entry points do) or a HOST array
 * (nreq, 3) of fixed packing centres -- with a fixed centre the FP32 rounding
 * of the target cells is the same in every call, so differences of values
 * between calls (line searches) do not carry it. */
LDDMM_API size_t lddmm_ragged_dataterm_f32c_workspace(int nreq, int cell_size, int norm, const int64_t* v_off,
                                                      const int64_t* c_off, const int64_t* c2_off, int d, int order,
                                                      int want_energy, int want_grad);
LDDMM_API int lddmm_ragged_dataterm_f32c(int nreq, int cell_size, int norm, const int64_t* v_off,
                                         const int64_t* c_off, const int64_t* c2_off, const double* vertices, int d,
                                         const int64_t* cells, const double* tgt_centers, const double* tgt_vectors,
                                         const double* sigma, int order, double eps1, double eps2,
                                         const double* frame, double* energy,
                                         const int64_t* vertex_ptr, const int64_t* vertex_idx, double* px,
                                         void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
LDDMM_API size_t lddmm_ragged_dataterm_f64_workspace(int nreq, int cell_size, int norm, const int64_t* v_off,
                                                     const int64_t* c_off, const int64_t* c2_off, int d, int order,
                                                     int want_energy, int want_grad);
LDDMM_API int lddmm_ragged_dataterm_f64(int nreq, int cell_size, int norm, const int64_t* v_off,
                                        const int64_t* c_off, const int64_t* c2_off, const double* vertices, int d,
                                        const int64_t* cells, const double* tgt_centers, const double* tgt_vectors,
                                        const double* sigma, int order, double eps1, double eps2,
                                         const double* frame, double* energy,
                                        const int64_t* vertex_ptr, const int64_t* vertex_idx, double* px,
                                        void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* LDDMM_B200_H */
