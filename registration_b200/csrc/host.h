// Host-side helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/lddmm_b200.h"
#include "common.cuh"

namespace lddmm {

void set_error(const char* fmt, ...);

// Bump allocator over the caller's workspace.  With base == nullptr it only
// measures, so the *_workspace queries run exactly the same code as the calls.
struct Workspace {
    char* base = nullptr;
    size_t cap = 0;
    size_t off = 0;
    template <class T>
    T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
    bool measuring() const { return base == nullptr; }
    bool overflow() const { return base && off > cap; }
};

struct DeviceInfo {
    int device = 0;
    int sms = 148;
};
DeviceInfo device_info();

// Maximum resident blocks per SM of a kernel (cached by the caller per kernel).
int occupancy_blocks(const void* kernel, int block, size_t dyn_smem = 0);

// Number of source chunks for a sweep: enough items (target blocks x chunks)
// for about 8 waves of `slots` resident blocks, at least 2 source tiles per
// chunk.  `slots` is taken as 8 blocks per SM for every operator, so the split
// (and the workspace) depends only on the shape and the SM count.
inline int choose_split(int n_tb, int n_src_tiles, int slots) {
    if (n_tb <= 0 || n_src_tiles <= 0) return 1;
    long long want = (8LL * slots + n_tb - 1) / n_tb;
    int max_split = std::max(1, n_src_tiles / 2);
    return (int)std::max(1LL, std::min<long long>(want, max_split));
}

inline long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// Returns LDDMM_ERR_ARG unless ptr is device (or managed) memory.
int check_device_ptr(const void* ptr, const char* name);

inline int cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return LDDMM_ERR_CUDA;
    }
    return LDDMM_OK;
}

#define LDDMM_TRY(expr)                   \
    do {                                  \
        int _rc = (expr);                 \
        if (_rc != LDDMM_OK) return _rc;  \
    } while (0)

// Laplacian polynomial tables of py-lddmm/kernelFunctions.f90 (c_ :24-26,
// c1_ :85-86, c2_ :325) with their default-real (float32) literal values, or
// (exact = true) the exact rationals of the dense numpy path lapPol /
// lapPolDiff / lapPolDiff2 (kernelFunctions.py:58-103).
void laplacian_tables(int order, double P[5], double Q[4], double Rr[3], bool exact = false);

}  // namespace lddmm
