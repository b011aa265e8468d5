// gkm_abi.cu -- status codes, the per-thread error message and device queries.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "gkm_common.cuh"

static thread_local char g_err[512] = "";

int gkm_fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

// Persistent index queries launched from a thread take at most this many
// blocks (0: one per SM).  A serving loop's side worker (ISM, GkmExplain) sets
// it so that its long queries leave SMs free for the scoring passes of other
// threads; nothing is shared between threads.
static thread_local int32_t g_grid_limit = 0;

extern "C" int gkm_set_thread_grid_limit(int32_t blocks)
{
    if (blocks < 0) return gkm_fail(GKM_ERR_INVALID, "grid limit %d < 0", blocks);
    g_grid_limit = blocks;
    return GKM_OK;
}

int gkm_query_blocks()
{
    const int n = gkm_sm_count();
    return g_grid_limit > 0 && g_grid_limit < n ? g_grid_limit : n;
}

int gkm_cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return GKM_OK;
    return gkm_fail(e == cudaErrorMemoryAllocation ? GKM_ERR_OOM : GKM_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
}

extern "C" int gkm_version(void) { return 1; }

extern "C" const char *gkm_last_error(void) { return g_err; }

extern "C" int gkm_device_info(int32_t *sm_count, int32_t *smem_per_block)
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return gkm_cuda_status(e == cudaSuccess ? cudaErrorNoDevice : e, "device");
    if (sm_count) *sm_count = gkm_sm_count();
    if (smem_per_block) *smem_per_block = gkm_smem_limit();
    return GKM_OK;
}
