// qssb_errors.cu - error reporting, version and device queries of the C ABI.
#include <stdio.h>
#include <string.h>

#include <atomic>

#include "qssb_internal.h"

namespace qssb {

static thread_local char g_last_error[512] = "";

int set_error(int code, const char* msg) {
    snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
    return code;
}

int set_cuda_error(cudaError_t err, const char* where) {
    snprintf(g_last_error, sizeof(g_last_error), "CUDA error %d (%s) at %s", (int)err,
             cudaGetErrorString(err), where);
    return QSSB_ERR_CUDA;
}

static std::atomic<long long> g_kernel_launches{0};

void note_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

int device_sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            sms <= 0)
            sms = 148;
        cached[dev] = sms;
    }
    return cached[dev];
}

}  // namespace qssb

extern "C" int qssb_version(void) { return QSSB_VERSION; }

extern "C" const char* qssb_last_error(void) { return qssb::g_last_error; }

extern "C" int64_t qssb_kernel_launches(void) {
    return (int64_t)qssb::g_kernel_launches.load(std::memory_order_relaxed);
}
