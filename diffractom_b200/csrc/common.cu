// Error reporting of the C ABI: a per-host-thread message and the launch check.
#include <stdarg.h>

#include "dfx_common.cuh"

namespace dfx {

static thread_local char g_msg[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
}

static unsigned long long g_launches = 0;   // kernels launched through this library (all host threads)

int launch_status(const char *what)
{
    __atomic_fetch_add(&g_launches, 1ULL, __ATOMIC_RELAXED);
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return DFX_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return DFX_ELAUNCH;
}

}  // namespace dfx

extern "C" int dfx_abi_version(void) { return DFX_ABI_VERSION; }

extern "C" const char *dfx_last_error(void) { return dfx::g_msg; }

extern "C" uint64_t dfx_launch_count(void) { return __atomic_load_n(&dfx::g_launches, __ATOMIC_RELAXED); }
