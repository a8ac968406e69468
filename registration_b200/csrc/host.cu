// Host helpers: error strings, device info, pointer checks, coefficient tables.
#include <mutex>
#include <string>

#include "host.h"

namespace lddmm {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

DeviceInfo device_info() {
    static std::mutex mu;
    static int sms_cache[64] = {0};
    DeviceInfo di;
    cudaGetDevice(&di.device);
    if (di.device < 0 || di.device >= 64) return di;
    std::lock_guard<std::mutex> lk(mu);
    if (sms_cache[di.device] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, di.device) == cudaSuccess && v > 0)
            sms_cache[di.device] = v;
        else
            sms_cache[di.device] = 148;
    }
    di.sms = sms_cache[di.device];
    return di;
}

int occupancy_blocks(const void* kernel, int block, size_t dyn_smem) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, dyn_smem) != cudaSuccess || nb <= 0) {
        cudaGetLastError();
        return 1;
    }
    return nb;
}

int check_device_ptr(const void* ptr, const char* name) {
    if (ptr == nullptr) {
        set_error("%s is NULL", name);
        return LDDMM_ERR_ARG;
    }
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("%s: not a CUDA pointer (%s)", name, cudaGetErrorString(e));
        return LDDMM_ERR_ARG;
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) {
        set_error("%s must be device memory (got a host pointer)", name);
        return LDDMM_ERR_ARG;
    }
    return LDDMM_OK;
}

void laplacian_tables(int order, double P[5], double Q[4], double Rr[3], bool exact) {
    // rows of c_, c1_, c2_ (kernelFunctions.f90:24-26, 85-86, 325); the
    // literals are default-real, i.e. float32-rounded, unless `exact`.
    const double t3 = exact ? 1.0 / 3 : (double)(1.0f / 3.0f), t04 = exact ? 0.4 : (double)0.4f;
    const double t37 = exact ? 3.0 / 7 : (double)(3.0f / 7.0f);
    const double t15 = exact ? 1.0 / 15 : (double)(1.0f / 15.0f), t221 = exact ? 2.0 / 21 : (double)(2.0f / 21.0f);
    const double t105 = exact ? 1.0 / 105 : (double)(1.0f / 105.0f);
    const double t5 = exact ? 1.0 / 5 : (double)(1.0f / 5.0f), t7 = exact ? 1.0 / 7 : (double)(1.0f / 7.0f);
    const double t235 = exact ? 2.0 / 35 : (double)(2.0f / 35.0f), t35 = exact ? 1.0 / 35 : (double)(1.0f / 35.0f);
    const double p[5][5] = {{1, 0, 0, 0, 0}, {1, 1, 0, 0, 0}, {1, 1, t3, 0, 0}, {1, 1, t04, t15, 0},
                            {1, 1, t37, t221, t105}};
    const double q[5][4] = {{0, 0, 0, 0}, {1, 0, 0, 0}, {t3, t3, 0, 0}, {t5, t5, t15, 0}, {t7, t7, t235, t105}};
    const double r[5][3] = {{0, 0, 0}, {0, 0, 0}, {t3, 0, 0}, {t15, t15, 0}, {t35, t35, t105}};
    const int o = (order >= 0 && order <= 4) ? order : 0;
    for (int j = 0; j < 5; ++j) P[j] = p[o][j];
    for (int j = 0; j < 4; ++j) Q[j] = q[o][j];
    for (int j = 0; j < 3; ++j) Rr[j] = r[o][j];
}

}  // namespace lddmm

extern "C" const char* lddmm_last_error(void) { return lddmm::g_last_error.c_str(); }
extern "C" int lddmm_abi_version(void) { return 3; }
