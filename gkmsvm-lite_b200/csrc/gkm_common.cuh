// gkm_common.cuh -- device helpers and launch plumbing shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/gkm_b200.h"

#define GKM_FULL 0xFFFFFFFFu

// Status plumbing (gkm_abi.cu owns the thread-local message).
int gkm_fail(int code, const char *fmt, ...);
int gkm_cuda_status(cudaError_t e, const char *what);
#define GKM_CHECK_LAUNCH(what)                                   \
    do {                                                         \
        cudaError_t e_ = cudaGetLastError();                     \
        if (e_ != cudaSuccess) return gkm_cuda_status(e_, what); \
    } while (0)
#define GKM_TRY(expr)                  \
    do {                               \
        int s_ = (expr);               \
        if (s_ != GKM_OK) return s_;   \
    } while (0)

// Mismatching 2-bit positions of two packed windows (kernels/primitives.py:
// _packed_mismatches): XOR, fold each digit's two bits, popcount.
__device__ __forceinline__ int gkm_mism(uint32_t a, uint32_t b)
{
    uint32_t x = a ^ b;
    return __popc((x | (x >> 1)) & 0x55555555u);
}

// Packed reverse complement of one window: complement every base and reverse
// the digit order (bit-reverse the word, swap the two bits of each digit, shift
// the l digits down).
__device__ __forceinline__ uint32_t gkm_rc_word(uint32_t w, int l)
{
    uint32_t r = __brev(w);
    r = ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
    r >>= (32 - 2 * l);
    return r ^ ((1u << (2 * l)) - 1u);
}

// 64-bit shift with PTX clamping: shifts of 64 or more give 0, which drops
// mismatch counts past the packed fields.
__device__ __forceinline__ uint64_t gkm_shl64(uint64_t a, uint32_t s)
{
    uint64_t d;
    asm("shl.b64 %0, %1, %2;" : "=l"(d) : "l"(a), "r"(s));
    return d;
}

// Window weight of window i in a row of n windows (kernels/weighted.py:38-43
// depends only on |n/2 - i|; wd is that table, computed on the host exactly as
// the reference computes it).
__device__ __forceinline__ uint32_t gkm_wt(const uint8_t *wd, int n, int i)
{
    int d = n / 2 - i;
    return wd[d < 0 ? -d : d];
}

// Block-wide sum of doubles in a fixed order (deterministic): per-warp
// butterfly, then warp 0 over the warp sums.  scratch: >= 32 doubles.
__device__ __forceinline__ double gkm_block_sum(double v, double *scratch)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GKM_FULL, v, o);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = lane < nw ? scratch[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(GKM_FULL, t, o);
    }
    return t;  // valid in thread 0
}

__device__ __forceinline__ uint64_t gkm_block_sum_u64(uint64_t v, uint64_t *scratch)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GKM_FULL, v, o);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    uint64_t t = 0;
    if (warp == 0) {
        t = lane < nw ? scratch[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(GKM_FULL, t, o);
    }
    return t;  // valid in thread 0
}

// Internal launchers shared between translation units.
struct gkm_index {
    gkm_spec spec;
    int64_t S;           // columns (SVs)
    int64_t W;           // window slots per column row
    int32_t tiles;       // SV tiles
    int32_t tile_svs;    // SVs per tile (last may be short)
    int32_t nlev;        // dmax + 1 accumulator levels
    int64_t n_lmers;     // 4^l
    int64_t entries;     // indexed windows
    uint32_t *offsets;   // [tiles * n_lmers + 1] start of bucket (tile, v)
    uint32_t *bwords;    // [tiles * n_lmers] (start - tile start) << lb | length (saturated); unweighted only
    int32_t lb;          // length bits of a bucket word
    uint32_t *ent;       // [entries] local SV id (bits 0..23) | weight << 24 (weighted, or big tiles)
    uint16_t *ent16;     // [entries] local SV id (unweighted tiles of <= 65,536 SVs), else null
    uint32_t *masks;     // [n_masks] mask | level << 24
    int32_t n_masks;
    int64_t bytes;
    int32_t acc_bytes;   // shared memory left for counters in a query block
    int32_t wide;        // 1: 32-bit counters (weighted, or after a carry-log overflow)
    int32_t packed;      // narrow counters: 1 every level of an SV in one word, 0 two levels per word
    uint32_t pack_w[8];  // packed: bits of each level's field
    uint32_t wmax;       // largest window weight (1 unweighted)
    unsigned int *status; // [2] query event counts (see gkm_index_status)
    unsigned int *queues;            // [GKM_QUEUE_SLOTS] work-queue heads, one per call in flight
    mutable std::atomic<unsigned> next_queue{0};
};

// Concurrent query calls on one index (different streams) each take their own
// work-queue counter; more than this many in flight at once would share one.
#define GKM_QUEUE_SLOTS 64

// Kernels that run beside the index query (other streams of a serving loop)
// ask for the largest shared-memory carveout, the one the query needs: an SM
// whose blocks use another carveout must drain before the query's block can
// start on it.
#define GKM_PREFER_SHARED(fn) cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, \
                                                   (int)cudaSharedmemCarveoutMaxShared)

int gkm_smem_limit();
int gkm_sm_count();
// Blocks a persistent index query may take on the calling thread's launches:
// the SM count, or the thread's limit (gkm_set_thread_grid_limit) if lower.
int gkm_query_blocks();
