// Error reporting and device queries of the C ABI.
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>

#include "snp_common.cuh"

namespace snp {

static thread_local char g_err[1024] = "";

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_err[0] = '\0'; }

int sm_count() {
    static std::mutex mu;
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
            cudaGetLastError();
            v = 148;
        }
        cached[dev] = v;
    }
    return cached[dev];
}

int resident_blocks(const void *kernel, int block, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, size_t, int>, int> cached;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = -1;
    }
    const auto key = std::make_tuple(kernel, block, smem, dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cached.find(key);
    if (it != cached.end()) return it->second;
    int v = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, block, smem) != cudaSuccess || v <= 0) {
        cudaGetLastError();
        v = 1;
    }
    if (v > 8) v = 8;
    cached[key] = v;
    return v;
}

}  // namespace snp

extern "C" {

const char *snp_last_error(void) { return snp::g_err; }

int snp_version(void) { return 1; }

}  // extern "C"
