// capi.cu -- library-level C-ABI entry points (version, device check, error text).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>

#include "lcs_internal.h"

namespace {
thread_local char g_last_error[512] = "";
std::atomic<unsigned long long> g_launches{0};
}

void lcs_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" uint64_t lcs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int lcs_fail(int code, const char* msg)
{
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
    return code;
}

extern "C" const char* lcs_version(void) { return "lcs_b200 0.1.0 sm_100a"; }

extern "C" const char* lcs_last_error(void) { return g_last_error; }

extern "C" int lcs_device_check(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0)
        return lcs_fail(LCS_ERR_NO_DEVICE, "lcs_device_check: no such CUDA device");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return lcs_fail(LCS_ERR_CUDA, "lcs_device_check: cudaGetDeviceProperties failed");
    if (prop.major != 10)
        return lcs_fail(LCS_ERR_NO_DEVICE, "lcs_device_check: the library is built for sm_100a only");
    return LCS_OK;
}
