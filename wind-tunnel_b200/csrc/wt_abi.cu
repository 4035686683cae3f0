// Library-level entry points: error reporting, version, shape checks.
#include <cstdarg>
#include <cstdio>

#include "wt_common.cuh"

static thread_local char g_err[512] = "";

int wt_set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int wt_cuda_check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return wt_set_error(WT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return WT_OK;
}

extern "C" const char* wt_last_error(void) { return g_err; }

extern "C" int wt_abi_version(void) { return WT_ABI_VERSION; }

extern "C" int wt_check_dims(int32_t nx, int32_t ny, int32_t nz) {
    // nx even: the outlet cell x = nx-1 then never starts a warp, so its x = nx-2
    // neighbour is always the previous lane (k_step_bulk).
    if (nx < 4 || ny < 3 || nz < 3 || (nx & 1))
        return wt_set_error(WT_ERR_DIMS, "grid %dx%dx%d: need nx even and >= 4, ny >= 3, nz >= 3", nx, ny, nz);
    if ((int64_t)nx * ny * nz >= (1ll << 31))
        return wt_set_error(WT_ERR_DIMS, "grid %dx%dx%d: more than 2^31 - 1 cells", nx, ny, nz);
    return WT_OK;
}

extern "C" int64_t wt_population_bytes(int32_t precision, int64_t n) {
    switch (precision) {
        case WT_F32: return 19 * 4 * n;
        case WT_F16:
        case WT_BF16: return 19 * 2 * n;
        case WT_F64: return 19 * 8 * n;
        default: return -1;
    }
}
