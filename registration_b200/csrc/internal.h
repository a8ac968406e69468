// Internal (non-exported) entry points shared between translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace lddmm {

// lddmm_applyk_f32c on a given workspace, with at most `split_cap` source
// chunks (0 = no cap; a cap bounds the partial-sum buffer).
int applyk_f32c_in_workspace(const double* x, int64_t n, const double* y, int64_t m, const double* beta, int d,
                             int dimb, double sigma, int order, double* f, void* workspace, size_t workspace_bytes,
                             cudaStream_t stream, int split_cap);

// Workspace bytes of applyk_f32c_in_workspace for a shape and chunk cap
// (0 for an invalid shape).
size_t applyk_f32c_scratch_bytes(int64_t n, int64_t m, int d, int dimb, int split_cap);

}  // namespace lddmm
