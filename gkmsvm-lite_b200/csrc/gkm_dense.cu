// gkm_dense.cu -- the dense form of the pairwise profile on the 5th-generation
// tensor cores (tcgen05).
//
// The number of positions at which two l-mers agree is the dot product of
// their one-hot encodings (4 bytes per position, 4l <= 64 bytes).  A CTA takes
// 128 query windows (operand A, [128, 64] uint8) and 256 SV windows (operand B,
// [256, 64] uint8, forward and RC windows of a chunk of SVs), and two
// tcgen05.mma.kind::i8 instructions (K = 32 bytes each) leave the 128 x 256
// match counts as int32 in tensor memory.  The epilogue reads them with
// tcgen05.ld, one query window per thread, and counts every pair with at
// least l - dmax matches into its (SV, mismatch level) -- integer and exact,
// the same profile as the ballot/popc join and the l-mer index.
//
// Operands sit in shared memory in the K-major no-swizzle core-matrix layout:
// byte k of row r at (k / 32) * rows * 32 + (r / 8) * 256 + ((k % 32) / 16) *
// 128 + (r % 8) * 16 + k % 16, so one MMA's operand is [rows, 32 bytes] with
// core matrices 8 rows x 16 bytes, 128 bytes apart along K and 256 bytes apart
// along rows.  One elected thread issues the MMAs and commits them to an
// mbarrier; every wait on it is bounded and sets an error flag on timeout.
#include <cuda_runtime.h>
#include <stdint.h>

#include "gkm_common.cuh"

namespace {

constexpr int DM = 128;          // query windows per tile (MMA M)
constexpr int DN = 256;          // SV windows per tile (MMA N)
constexpr int DKB = 64;          // one-hot bytes per window (4l <= 64)
constexpr int D_THREADS = 128;   // one warpgroup: a TMEM lane quadrant per warp
constexpr int D_SV_CHUNK = 8;    // SVs per CTA
constexpr int D_LEVELS = 16;
constexpr uint32_t D_TMEM_COLS = 256;
constexpr uint64_t D_WAIT_NS = 1000000000ull;  // give up on an MMA after 1 s

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (Blackwell version 1)
__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version
    return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
}

// instruction descriptor: kind::i8, unsigned A and B, int32 accumulate, K-major
// A and B, M = 128, N = 256
__host__ __device__ constexpr uint32_t make_idesc()
{
    return (2u << 4)                      // D format: S32
           | (0u << 7) | (0u << 10)       // A, B: unsigned 8-bit
           | ((uint32_t)(DN >> 3) << 17)  // N / 8
           | ((uint32_t)(DM >> 4) << 24); // M / 16
}

__device__ __forceinline__ uint32_t core_offset(int r, int chunk16, int rows)
{
    // byte offset of the 16-byte chunk chunk16 (0..3) of row r
    return (uint32_t)((chunk16 >> 1) * rows * 32 + (r >> 3) * 256 + (chunk16 & 1) * 128 + (r & 7) * 16);
}

// one-hot of a packed window, 16 bytes per chunk, with `bias` in byte 63
// (l <= 15 leaves bytes 60..63 free).  PAD or a missing window: all zero.
__device__ __forceinline__ void onehot_row(uint8_t *base, int r, int rows, uint32_t w, int l, uint32_t bias)
{
#pragma unroll
    for (int c = 0; c < 4; c++) {
        uint32_t word[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int pos = 4 * c + q;
            word[q] = (w != GKM_PAD && pos < l) ? (1u << (8 * ((w >> (2 * pos)) & 3u))) : 0u;
        }
        if (c == 3 && w != GKM_PAD) word[3] |= bias << 24;
        *(uint4 *)(base + core_offset(r, c, rows)) = make_uint4(word[0], word[1], word[2], word[3]);
    }
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// waits for the mbarrier phase with parity `phase` to complete; false after
// D_WAIT_NS of wall time
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase)
{
    const uint64_t t0 = global_ns();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
        if (global_ns() - t0 > D_WAIT_NS) return false;
    }
}

struct DenseArgs {
    gkm_spec spec;
    const uint32_t *bx;
    const int32_t *cx;
    int64_t Wx;
    const uint32_t *by;
    const uint32_t *ry;
    const int32_t *cy;
    int64_t S;
    int64_t Wy;
    double *raw;
    uint64_t *profile;
    int *error;
};

__global__ void __launch_bounds__(D_THREADS) dense_join_kernel(DenseArgs a)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *smA = sm;                                     // [DM, 64] core-matrix layout (8 KB)
    uint8_t *smB = sm + DM * DKB;                          // [DN, 64] (16 KB)
    uint16_t *col_sv = (uint16_t *)(smB + DN * DKB);       // [DN] SV of each B column (0xFFFF: none)
    uint8_t *col_w = (uint8_t *)(col_sv + DN);             // [DN] its window weight
    unsigned long long *cnt = (unsigned long long *)(((uintptr_t)(col_w + DN) + 15) & ~(uintptr_t)15);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;

    const gkm_spec &sp = a.spec;
    const int l = sp.l, dmax = sp.dmax;
    // a pair's accumulator is matches + bias_b (byte 63 of A is 1, of B is
    // bias_b): at least 32 -- bit 5 set -- exactly when it has at least l - dmax
    // matches, and below 48 since matches <= l <= 15.  Pairs with a PAD
    // window or a missing column accumulate 0.
    const uint32_t bias_b = 32u - (uint32_t)(l - dmax);
    const int64_t b = blockIdx.x;
    const int64_t s_lo = (int64_t)blockIdx.y * D_SV_CHUNK;
    const int nsv = (int)min((int64_t)D_SV_CHUNK, a.S - s_lo);
    const int tid = threadIdx.x, warp = tid >> 5;
    const bool has_rc = sp.include_rc && a.ry != nullptr;

    // an earlier CTA gave up on an MMA: skip the work (the outputs are
    // undefined and the host raises), so a failed launch ends quickly.  One
    // read, shared, so the whole block takes the same branch.
    if (tid == 0) failed = *(volatile int *)a.error != 0;
    __syncthreads();
    if (failed) return;
    for (int k = tid; k < D_SV_CHUNK * D_LEVELS; k += D_THREADS) cnt[k] = 0;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                     "r"(D_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    const int nx = a.cx[b];
    // SV windows of this chunk, listed SV by SV: forward windows then RC ones
    int ny_total = 0;
    for (int s = 0; s < nsv; s++) ny_total += (has_rc ? 2 : 1) * a.cy[s_lo + s];
    const uint32_t idesc = make_idesc();
    uint32_t phase = 0;

    for (int c0 = 0; c0 < ny_total && !failed; c0 += DN) {
        // B tile: column j = SV window c0 + j
        for (int j = tid; j < DN; j += D_THREADS) {
            int t = c0 + j, s = 0;
            uint32_t w = GKM_PAD;
            uint16_t sv = 0xFFFF;
            uint8_t wt = 0;
            if (t < ny_total) {
                for (; s < nsv; s++) {
                    const int n2 = (has_rc ? 2 : 1) * a.cy[s_lo + s];
                    if (t < n2) break;
                    t -= n2;
                }
                const int64_t sg = s_lo + s;
                const int ny = a.cy[sg];
                if (t < ny) {
                    w = a.by[sg * a.Wy + t];
                    wt = sp.weighted ? (uint8_t)gkm_wt(sp.wd, ny, t) : 1;
                } else {  // RC of forward window ny - 1 - (t - ny)
                    const int f = ny - 1 - (t - ny);
                    w = a.ry[sg * a.Wy + (a.Wy - 1 - f)];
                    wt = sp.weighted ? (uint8_t)gkm_wt(sp.wd, ny, f) : 1;
                }
                sv = (uint16_t)s;
            }
            onehot_row(smB, j, DN, w, l, bias_b);
            col_sv[j] = sv;
            col_w[j] = wt;
        }
        for (int r0 = 0; r0 < nx && !failed; r0 += DM) {
            // A tile: this thread's query window
            {
                const int i = r0 + tid;
                const uint32_t w = i < nx ? a.bx[b * a.Wx + i] : GKM_PAD;
                onehot_row(smA, tid, DM, w, l, 1u);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (tid == 0) {
#pragma unroll
                for (int kb = 0; kb < 2; kb++) {
                    const uint64_t da = make_sdesc(smem_addr(smA) + kb * DM * 32, 128, 256);
                    const uint64_t db = make_sdesc(smem_addr(smB) + kb * DN * 32, 128, 256);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(idesc), "r"(kb));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_addr(&mbar)));
            }
            if (!mbar_wait(smem_addr(&mbar), phase)) {
                failed = 1;
                atomicOr(a.error, 1);
            }
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");
            __syncthreads();
            if (failed) break;
            // epilogue: this thread's row (TMEM lane 32 * warp + lane)
            const int i = r0 + tid;
            const uint64_t wx = (i < nx && sp.weighted) ? gkm_wt(sp.wd, nx, i) : 1;
#pragma unroll 1
            for (int c = 0; c < DN / 32; c++) {
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                uint32_t any = 0;
#pragma unroll
                for (int j = 0; j < 32; j++) any |= v[j];
                if (any & 32u) {  // some pair of this row is within dmax here
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const int col = c * 32 + j;
                        if (v[j] & 32u)  // mismatches l - (v - bias_b)
                            atomicAdd(&cnt[col_sv[col] * D_LEVELS + (32 + dmax - (int)v[j])],
                                      (unsigned long long)(wx * col_w[col]));
                    }
                }
                __syncwarp();  // the next tcgen05.ld is warp-aligned
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;");
        }
        __syncthreads();  // B is rebuilt next
    }
    // a timed-out MMA may still be in flight: one more bounded wait before its
    // accumulator columns are released
    if (failed && tid == 0) mbar_wait(smem_addr(&mbar), phase ^ 1u);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(D_TMEM_COLS));
    if (failed) return;
    for (int s = tid; s < nsv; s += D_THREADS) {
        const int64_t sg = s_lo + s;
        double k = 0.0;
        for (int m = 0; m <= dmax; m++) k += sp.h[m] * (double)cnt[s * D_LEVELS + m];
        if (a.raw) a.raw[b * a.S + sg] = k;
        if (a.profile)
            for (int m = 0; m <= l; m++) a.profile[(b * a.S + sg) * (l + 1) + m] = m <= dmax ? cnt[s * D_LEVELS + m] : 0;
    }
}

}  // namespace

extern "C" int gkm_dense_pairwise(const gkm_spec *spec, const uint32_t *bx, const int32_t *cx, int64_t B,
                                  int64_t Wx, const uint32_t *by, const uint32_t *ry, const int32_t *cy, int64_t S,
                                  int64_t Wy, double *raw, uint64_t *profile, int32_t *error, gkm_stream_t stream)
{
    if (!spec) return gkm_fail(GKM_ERR_INVALID, "spec is null");
    if (spec->l < 1 || spec->l > 15) return gkm_fail(GKM_ERR_UNSUPPORTED, "the dense form needs l <= 15");
    if (spec->dmax < 0 || spec->dmax >= spec->l)
        return gkm_fail(GKM_ERR_UNSUPPORTED, "the dense form needs 0 <= dmax < l");
    if (spec->weighted && (!spec->wd || spec->wd_len < 1)) return gkm_fail(GKM_ERR_INVALID, "weighted spec without weights");
    if (B == 0 || S == 0) return GKM_OK;
    if (!bx || !cx || !by || !cy || !error) return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (B > 0x7FFFFFFFLL || (S + D_SV_CHUNK - 1) / D_SV_CHUNK > 65535)
        return gkm_fail(GKM_ERR_UNSUPPORTED, "too many rows or columns for one dense launch");
    DenseArgs a;
    a.spec = *spec;
    a.bx = bx;
    a.cx = cx;
    a.Wx = Wx;
    a.by = by;
    a.ry = ry;
    a.cy = cy;
    a.S = S;
    a.Wy = Wy;
    a.raw = raw;
    a.profile = profile;
    a.error = error;
    // operands + column tables + counters; 100 KB keeps at most two CTAs per
    // SM, so their 256 TMEM columns each always fit the SM's 512
    size_t smem = 100 * 1024;
    cudaFuncSetAttribute(dense_join_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)B, (unsigned)((S + D_SV_CHUNK - 1) / D_SV_CHUNK));
    dense_join_kernel<<<grid, D_THREADS, smem, (cudaStream_t)stream>>>(a);
    GKM_CHECK_LAUNCH("dense_join");
    return GKM_OK;
}
