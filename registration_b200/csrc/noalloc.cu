// lddmm_applyk_f32c_noalloc: the FP32 compensated kernel sum applyK for
// callers that cannot allocate GPU memory.
//
// Some hosts of this code cannot call cudaMalloc: a plug-in whose host
// framework owns every device allocation (it hands over input and output
// buffers only), an FFI caller in a language runtime with no CUDA allocator,
// or a caller on a latency-critical path where cudaMalloc / cudaFree would
// synchronise the device.  This entry point takes only the inputs and the
// output; its scratch memory (packed points, per-chunk partial sums) is a
// file-scope array in the library's static device memory, which every GPU that
// loads the library holds until the process exits.
//
// Limits and sharing:
//   * the scratch holds kNoAllocScratchBytes (32 MiB): enough for about
//     n = m = 400,000 points with dimb <= 4; larger shapes are rejected with
//     LDDMM_ERR_WORKSPACE and a message, before any launch.  Within the limit
//     the number of source chunks is capped so the partial sums fit, which
//     can change the summation grouping (not the accuracy class) with respect
//     to lddmm_applyk_f32c.
//   * every call on a device uses the same array and leaves the last call's
//     contents in it.  Nothing in it has to start at zero: each call writes
//     every byte it later reads (packed points and partial sums).  Calls whose
//     work overlaps on the GPU (other streams, other host threads) race on
//     the array; order them on one stream.
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make that
//     first call before any stream capture.
#include <mutex>

#include "host.h"
#include "internal.h"

namespace lddmm {

static constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch on the current device (looked up once)
static int noalloc_scratch(void** out) {
    static std::mutex mu;
    static void* cached[64] = {nullptr};
    int dev = -1;
    LDDMM_TRY(cuda_check(cudaGetDevice(&dev), "noalloc: cudaGetDevice"));
    if (dev < 0 || dev >= 64) {
        set_error("noalloc: device index %d out of range", dev);
        return LDDMM_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (cached[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error("noalloc: cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
            return LDDMM_ERR_CUDA;
        }
        cached[dev] = p;
    }
    *out = cached[dev];
    return LDDMM_OK;
}

}  // namespace lddmm

extern "C" LDDMM_API int lddmm_applyk_f32c_noalloc(const double* x, int64_t n, const double* y, int64_t m,
                                                   const double* beta, int d, int dimb, double sigma, int order,
                                                   double* f, lddmm_stream_t stream) {
    using namespace lddmm;
    if (n < 0 || m < 0 || d < 1 || d > 3 || dimb < 1 || !(sigma > 0) || order < 0) {
        set_error("applyk_noalloc: invalid arguments (n=%lld m=%lld d=%d dimb=%d sigma=%g order=%d)",
                  (long long)n, (long long)m, d, dimb, sigma, order);
        return LDDMM_ERR_ARG;
    }
    if (n > (1LL << 30) || m > (1LL << 30)) {   // the same limit as lddmm_applyk_f32c
        set_error("applyk_noalloc: more than 2^30 points");
        return LDDMM_ERR_ARG;
    }
    int cap = 0;
    if (n > 0 && m > 0) {
        // largest chunk count whose workspace fits the static scratch
        const size_t one = applyk_f32c_scratch_bytes(n, m, d, dimb, 1);
        if (one == 0 || one > kNoAllocScratchBytes) {
            set_error("applyk_noalloc: n=%lld, m=%lld, dimb=%d needs %zu bytes of scratch; the static scratch holds "
                      "%zu (use lddmm_applyk_f32c with a workspace)",
                      (long long)n, (long long)m, dimb, one, kNoAllocScratchBytes);
            return LDDMM_ERR_WORKSPACE;
        }
        const size_t per_chunk = (size_t)n * (size_t)std::min(dimb, 4) * sizeof(double) + 256;
        cap = 1 + (int)std::min<size_t>((kNoAllocScratchBytes - one) / per_chunk, 1 << 20);
        while (cap > 1 && applyk_f32c_scratch_bytes(n, m, d, dimb, cap) > kNoAllocScratchBytes) --cap;
    }
    void* scratch = nullptr;
    LDDMM_TRY(noalloc_scratch(&scratch));
    return applyk_f32c_in_workspace(x, n, y, m, beta, d, dimb, sigma, order, f, scratch, kNoAllocScratchBytes,
                                    (cudaStream_t)stream, cap);
}
