// gkm_dense.cu -- the dense form of the pairwise profile on the 5th-generation
// tensor cores (tcgen05).
//
// The number of positions at which two l-mers agree is the dot product of
// their one-hot encodings (4 bytes per position, 4l <= 60 bytes).  A tile of
// 128 query windows (operand A, [128, 64] uint8) against 128 SV windows
// (operand B, [128, 64] uint8) is two tcgen05.mma.kind::i8 instructions
// (K = 32 bytes each) that leave the 128 x 128 match counts as int32 in tensor
// memory.  The epilogue counts every pair with at least l - dmax matches into
// its (SV, mismatch level) -- integer and exact, the same profile as the
// ballot/popc join and the l-mer index.
//
// Two kernels per launch:
//   dense_b_records  writes every B tile once to global memory as a record:
//                    the tile's one-hot bytes already in the shared-memory
//                    layout the MMA reads, then each column's chunk-local SV
//                    and window weight.  The SVs are taken D_CH at a time (a
//                    chunk); a chunk's windows -- forward then RC, SV after
//                    SV -- are packed into consecutive tiles across SV
//                    boundaries.
//   dense_pairs_kernel  one CTA per (query row, SV chunk), with warp roles:
//     - all warps first stage a segment of the row's one-hot (up to 1,024
//       windows: 8 A tiles; 512 for weighted kernels) in shared memory, where
//       it stays while every B tile of the chunk passes;
//     - one producer thread copies the chunk's B records, one per tile, into a
//       ring of 3 (4 weighted) buffers with cp.async.bulk (untiled, 16-byte aligned, a multiple
//       of 16 bytes, completing on the buffer's mbarrier);
//     - one thread issues the MMAs of every (B tile, A tile) pair, alternating
//       between two accumulators in tensor memory, and commits each to an
//       mbarrier;
//     - two epilogue warpgroups, one per accumulator, read a finished
//       accumulator into registers (tcgen05.ld, 16-bit packed), hand it
//       straight back to the MMA thread, and only then look for pairs within
//       dmax: an OR over each 32-column chunk and a warp ballot; the rare rows
//       with a hit leave their values in shared scratch and the warp walks
//       them one row at a time, a column per lane, into per-(SV, level)
//       counters (see the counting modes below).
// mbarriers hand buffers between the roles (full/empty pairs); every wait is
// bounded in time and raises the launch's error flag when it runs out, after
// which every role leaves its loop, the MMA thread waits (bounded) for its
// MMAs and the producer for its copies in flight, and the tensor memory is
// freed.
//
// Operands sit in shared memory in the K-major no-swizzle core-matrix layout:
// byte k of row r at (k / 32) * rows * 32 + (r / 8) * 256 + ((k % 32) / 16) *
// 128 + (r % 8) * 16 + k % 16, so one MMA's operand is [rows, 32 bytes] with
// core matrices 8 rows x 16 bytes, 128 bytes apart along K and 256 bytes apart
// along rows.
#include <cuda_runtime.h>
#include <stdint.h>

#include "gkm_common.cuh"

namespace {

constexpr int DM = 128;            // query windows per A tile (MMA M)
constexpr int DN = 128;            // SV windows per B tile (MMA N)
constexpr int DKB = 64;            // one-hot bytes per window
constexpr int D_CH = 16;           // SVs per chunk (per CTA)
constexpr int D_LEVELS = 16;
constexpr int D_EPI_WARPS = 8;     // warps 0..7: warpgroup w / 4 drains accumulator w / 4,
                                   // warp w reads TMEM lane quadrant w % 4
constexpr int D_PROD_WARP = D_EPI_WARPS;      // warp 8 (lane 0 copies)
constexpr int D_MMA_WARP = D_EPI_WARPS + 1;   // warp 9 (lane 0 issues)
constexpr int D_THREADS = (D_MMA_WARP + 1) * 32;
constexpr uint32_t D_TMEM_COLS = 2 * DN;  // two accumulators
constexpr int A_TILE = DM * DKB;   // 8 KB
constexpr int B_TILE = DN * DKB;   // 8 KB
constexpr int REC = B_TILE + 2 * DN;  // B record: one-hot, column SVs, column weights
constexpr uint64_t D_WAIT_NS = 1000000000ull;  // give up on a hand-off after 1 s
constexpr size_t D_REC_BUDGET = (size_t)1 << 30;  // B records per launch round
static_assert(REC % 16 == 0, "bulk copies move multiples of 16 bytes");

// Counting modes: unweighted launches count each pair 1 in the block's shared
// counters, 32-bit when no (row, SV) can reach 2^32 pairs, else 64-bit;
// weighted launches count pair weights (up to 255 x 255) in per-warp 32-bit
// counters flushed into the block's 64-bit counters before they could wrap.
enum { MODE_U32 = 0, MODE_U64 = 1, MODE_WEIGHTED = 2 };
constexpr int D_BBUF_MAX = 4;
constexpr int D_SCR_STRIDE = 20;   // scratch words per lane (16 used; 20 keeps 16-byte stores conflict-free)

// Shared-memory layout of a mode: staged query segment (A tiles), ring of B
// records, block counters, per-warp counters (weighted), hit scratch.  Each
// fits two CTAs per SM and requests more than a third of the SM's shared
// memory, so at most two CTAs share an SM and their 2 x 256 tensor-memory
// columns always fit its 512.
template <int MODE>
struct Cfg {
    static constexpr bool weighted = MODE == MODE_WEIGHTED;
    static constexpr int SEG = weighted ? 512 : 1024;  // query windows staged at a time
    static constexpr int BBUF = weighted ? 4 : 3;      // B records in flight
    static constexpr int OFF_A = 0;
    static constexpr int OFF_B = OFF_A + SEG * DKB;
    static constexpr int OFF_CNT = OFF_B + BBUF * REC;
    static constexpr int OFF_WCNT = OFF_CNT + D_CH * D_LEVELS * 8;
    static constexpr int OFF_SCR = OFF_WCNT + (weighted ? D_EPI_WARPS * D_CH * D_LEVELS * 4 : 0);
    static constexpr int USED = OFF_SCR + D_EPI_WARPS * 32 * D_SCR_STRIDE * 4;
    static constexpr int SMEM = ((USED + 1023) / 1024) * 1024;
    // a warp's counters gain at most its 32 rows x 128 columns of each of its
    // warpgroup's A tiles of one B tile, times the largest pair weight
    static constexpr uint64_t WARP_PAIRS_PER_B = 32ull * DN * (SEG / DM / 2);
    static_assert(OFF_B % 16 == 0 && OFF_CNT % 16 == 0 && OFF_WCNT % 16 == 0 && OFF_SCR % 16 == 0, "alignment");
    static_assert(BBUF <= D_BBUF_MAX, "barrier slots");
    static_assert(2 * (SMEM + 2048) <= 228 * 1024, "two CTAs per SM");
    static_assert(3 * (SMEM + 1024) > 228 * 1024, "at most two CTAs per SM");
    static_assert(WARP_PAIRS_PER_B * 255 * 255 < (1ull << 32), "per-warp counters cannot wrap");
};

// mbarriers (static shared memory)
enum {
    BAR_BFULL = 0,
    BAR_BEMPTY = BAR_BFULL + D_BBUF_MAX,
    BAR_TFULL = BAR_BEMPTY + D_BBUF_MAX,
    BAR_TEMPTY = BAR_TFULL + 2,
    BAR_DONE = BAR_TEMPTY + 2,
    N_BARS = BAR_DONE + 1
};

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
// A and B, M = DM, N = DN
__host__ __device__ constexpr uint32_t make_idesc()
{
    return (2u << 4)                      // D format: S32
           | (0u << 7) | (0u << 10)       // A, B: unsigned 8-bit
           | ((uint32_t)(DN >> 3) << 17)  // N / 8
           | ((uint32_t)(DM >> 4) << 24); // M / 16
}

__host__ __device__ __forceinline__ uint32_t core_offset(int r, int chunk16, int rows)
{
    // byte offset of the 16-byte chunk chunk16 (0..3) of row r
    return (uint32_t)((chunk16 >> 1) * rows * 32 + (r >> 3) * 256 + (chunk16 & 1) * 128 + (r & 7) * 16);
}

// one-hot of a packed window, 16 bytes per chunk, with `bias` in byte 63
// (l <= 15 leaves bytes 60..63 free).  PAD or a missing window: all zero.
__device__ __forceinline__ uint4 onehot_chunk(uint32_t w, int l, uint32_t bias, int c)
{
    uint32_t word[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int pos = 4 * c + q;
        word[q] = (w != GKM_PAD && pos < l) ? (1u << (8 * ((w >> (2 * pos)) & 3u))) : 0u;
    }
    if (c == 3 && w != GKM_PAD) word[3] |= bias << 24;
    return make_uint4(word[0], word[1], word[2], word[3]);
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool bar_test(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `bar` with parity `parity` to complete.  False when
// another role has aborted (*abort set) or after limit_ns, which sets *abort
// and the launch's error flag.  Hand-offs between roles wait up to the
// launch's role limit (D_WAIT_NS unless a test shortens it); the drain waits
// for copies and MMAs in flight always wait up to D_WAIT_NS.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, volatile int *abort, int *error,
                                         uint64_t limit_ns = D_WAIT_NS)
{
    const uint64_t t0 = global_ns();
    for (;;) {
        if (bar_test(bar, parity)) return true;
        if (*abort) return false;
        if (global_ns() - t0 > limit_ns) {
            *abort = 1;
            atomicOr(error, 1);
            return false;
        }
    }
}

__device__ __forceinline__ void bar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// 32 columns of this warp's 32 TMEM lanes, two 16-bit values per register
// (column 2i in the low half of v[i], column 2i + 1 in the high half)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.pack::16b.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
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
    int64_t chunk0;        // first SV chunk of this launch round
    int64_t max_tiles;     // record slots per chunk
    int flush_every;       // B tiles between flushes of the per-warp counters
    const uint8_t *rec;    // [chunks of the round][max_tiles] B records
    double *raw;
    uint64_t *profile;
    int *error;
    uint64_t role_wait_ns;  // limit of the hand-off waits between roles
};

// chunk-local windows of SV chunk `cg`: prefix counts pre[0..n] (n SVs)
__device__ __forceinline__ int chunk_prefix(const DenseArgs &a, int64_t cg, int *pre)
{
    const int64_t s_lo = cg * D_CH;
    const int n = (int)min((int64_t)D_CH, a.S - s_lo);
    const int mult = (a.spec.include_rc && a.ry) ? 2 : 1;
    pre[0] = 0;
    for (int s = 0; s < n; s++) pre[s + 1] = pre[s] + mult * a.cy[s_lo + s];
    return n;
}

// B records: block (tile i, chunk of the round), thread = column
__global__ void __launch_bounds__(DN) dense_b_records(DenseArgs a, uint8_t *rec)
{
    __shared__ int pre[D_CH + 1];
    __shared__ int nsv;
    const int64_t cl = blockIdx.y, cg = a.chunk0 + cl;
    if (threadIdx.x == 0) nsv = chunk_prefix(a, cg, pre);
    __syncthreads();
    const int ny_total = pre[nsv];
    const int i = blockIdx.x;
    if ((int64_t)i * DN >= ny_total) return;  // past this chunk's last tile
    const gkm_spec &sp = a.spec;
    const uint32_t bias_b = 32u - (uint32_t)(sp.l - sp.dmax);
    const int j = threadIdx.x, t = i * DN + j;
    uint32_t w = GKM_PAD;
    int s = 0;
    uint8_t wt = 0;
    if (t < ny_total) {
        while (t >= pre[s + 1]) s++;
        const int u = t - pre[s];
        const int64_t sg = cg * D_CH + s;
        const int ny = a.cy[sg];
        if (u < ny) {
            w = a.by[sg * a.Wy + u];
            wt = sp.weighted ? (uint8_t)gkm_wt(sp.wd, ny, u) : 1;
        } else {  // RC of forward window ny - 1 - (u - ny)
            const int f = ny - 1 - (u - ny);
            w = a.ry[sg * a.Wy + (a.Wy - 1 - f)];
            wt = sp.weighted ? (uint8_t)gkm_wt(sp.wd, ny, f) : 1;
        }
    }
    uint8_t *r = rec + (cl * a.max_tiles + i) * (int64_t)REC;
#pragma unroll
    for (int c = 0; c < 4; c++) *(uint4 *)(r + core_offset(j, c, DN)) = onehot_chunk(w, sp.l, bias_b, c);
    r[B_TILE + j] = (uint8_t)s;
    r[B_TILE + DN + j] = wt;
}

template <int MODE>
__global__ void __launch_bounds__(D_THREADS, 2) dense_pairs_kernel(DenseArgs a)
{
    using C = Cfg<MODE>;
    constexpr bool WEIGHTED = C::weighted;
    constexpr int D_SEG = C::SEG, D_BBUF = C::BBUF;
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *smA = sm + C::OFF_A;              // [D_SEG / DM] A tiles, core-matrix layout
    uint8_t *smB = sm + C::OFF_B;              // [D_BBUF] B records
    unsigned long long *cnt = (unsigned long long *)(sm + C::OFF_CNT);  // [D_CH][D_LEVELS]
    unsigned *cnt32 = (unsigned *)(sm + C::OFF_CNT);                     // the same, 32-bit (MODE_U32)
    unsigned *wcnt_all = (unsigned *)(sm + C::OFF_WCNT);  // [epilogue warp][D_CH][D_LEVELS] (weighted)
    uint32_t *scratch = (uint32_t *)(sm + C::OFF_SCR);    // [epilogue warp][lane][D_SCR_STRIDE]
    __shared__ __align__(8) uint64_t bars[N_BARS];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    __shared__ int pre[D_CH + 1];
    __shared__ int nsv_s;
    volatile int *abort = &abort_flag;

    const gkm_spec &sp = a.spec;
    const int l = sp.l, dmax = sp.dmax;
    // a pair's accumulator is matches + bias_b (byte 63 of A is 1, of B is
    // bias_b = 32 - (l - dmax)): at least 32 -- bit 5 set -- exactly when it
    // has at least l - dmax matches, and below 48 since matches <= l <= 15.
    // Pairs with a PAD window or a missing column accumulate 0.
    const int64_t b = blockIdx.x;
    const int64_t cl = blockIdx.y, cg = a.chunk0 + cl;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar0 = smem_addr(bars);
    auto bar = [&](int k) { return bar0 + 8u * (uint32_t)k; };

    // an earlier CTA gave up on a hand-off: skip the work (the outputs are
    // undefined and the host raises), so a failed launch ends quickly.  One
    // read, shared, so the whole block takes the same branch.
    if (tid == 0) abort_flag = *(volatile int *)a.error != 0;
    __syncthreads();
    if (abort_flag) return;

    for (int k = tid; k < D_CH * D_LEVELS; k += D_THREADS) cnt[k] = 0;
    if (WEIGHTED)
        for (int k = tid; k < D_EPI_WARPS * D_CH * D_LEVELS; k += D_THREADS) wcnt_all[k] = 0;
    if (tid == 0) {
        nsv_s = chunk_prefix(a, cg, pre);
        // B buffers: filled by the producer's copy, emptied by every epilogue
        // warp; accumulators: filled by the MMA commit, emptied by the four
        // warps of their warpgroup
        for (int k = 0; k < N_BARS; k++) {
            const uint32_t n = k < BAR_BEMPTY ? 1 : k < BAR_TFULL ? D_EPI_WARPS : k < BAR_TEMPTY ? 1
                             : k < BAR_DONE ? 4 : 1;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar(k)), "r"(n));
        }
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
    const int nsv = nsv_s;
    const int NB = (pre[nsv] + DN - 1) / DN;
    const int nx = a.cx[b];
    const uint32_t idesc = make_idesc();
    const uint8_t *rec = a.rec + cl * a.max_tiles * (int64_t)REC;
    uint32_t g_base = 0, t_base = 0;  // B tiles and tile pairs of earlier segments
    uint32_t copies = 0;              // B records the producer has requested

    for (int seg0 = 0; seg0 < nx && NB > 0; seg0 += D_SEG) {
        const int nseg = min(D_SEG, nx - seg0);
        const int NA = (nseg + DM - 1) / DM;
        // every warp: this segment's A tiles (rows past the row's end: zero)
        for (int r = tid; r < NA * DM; r += D_THREADS) {
            const uint32_t w = r < nseg ? a.bx[b * a.Wx + seg0 + r] : GKM_PAD;
            uint8_t *base = smA + (r / DM) * A_TILE;
#pragma unroll
            for (int c = 0; c < 4; c++) *(uint4 *)(base + core_offset(r % DM, c, DM)) = onehot_chunk(w, l, 1u, c);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();

        if (warp < D_EPI_WARPS) {
            // ---- epilogue: warpgroup eg drains the accumulator of the tiles t
            // with t % 2 == eg; TMEM lane quadrant `quad`, one query window per thread
            const uint32_t eg = (uint32_t)(warp >> 2);
            const int quad = warp & 3;
            uint32_t *scr = scratch + warp * 32 * D_SCR_STRIDE;
            unsigned *wcnt = wcnt_all + warp * D_CH * D_LEVELS;
            for (int bt = 0; bt < NB; bt++) {
                const uint32_t g = g_base + bt, buf = g % D_BBUF;
                const uint8_t *csv = smB + buf * REC + B_TILE, *cw = csv + DN;
                // wait for this B tile to land even when none of its tiles is
                // ours: the release below must not count toward an earlier
                // phase of the buffer while the other warpgroup still reads it
                bool ok = __all_sync(GKM_FULL, bar_wait(bar(BAR_BFULL + buf), (g / D_BBUF) & 1u, abort, a.error,
                                                                   a.role_wait_ns));
                if (!ok) break;
                for (int at = 0; at < NA; at++) {
                    const uint32_t t = t_base + (uint32_t)(bt * NA + at), slot = t & 1u;
                    if (slot != eg) continue;
                    ok = __all_sync(GKM_FULL, bar_wait(bar(BAR_TFULL + slot), (t >> 1) & 1u, abort, a.error,
                                                                  a.role_wait_ns));
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    // the whole accumulator row in 64 registers (values < 48), then
                    // the accumulator goes back to the MMA thread before any counting
                    uint32_t p[DN / 2];
                    const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + slot * DN;
#pragma unroll
                    for (int k = 0; k < DN / 32; k++) tmem_ld16(taddr + (uint32_t)(32 * k), p + 16 * k);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    asm volatile("tcgen05.fence::before_thread_sync;");
                    __syncwarp();
                    if (lane == 0) bar_arrive(bar(BAR_TEMPTY + slot));

                    const int r = at * DM + quad * 32 + lane;
                    const uint32_t wx = (sp.weighted && r < nseg) ? gkm_wt(sp.wd, nx, seg0 + r) : 1u;
#pragma unroll
                    for (int k = 0; k < DN / 32; k++) {
                        uint32_t o = 0;
#pragma unroll
                        for (int i = 0; i < 16; i++) o |= p[16 * k + i];
                        const bool mine = (o & 0x00200020u) != 0;  // a pair of this row within dmax
                        unsigned rows = __ballot_sync(GKM_FULL, mine);
                        if (rows == 0) continue;  // warp-uniform: the common case
                        // rows with a hit leave their 32 values in the warp's scratch;
                        // the warp then takes them one row at a time, a column per lane
                        if (mine) {
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                *(uint4 *)(scr + lane * D_SCR_STRIDE + 4 * i) =
                                    make_uint4(p[16 * k + 4 * i], p[16 * k + 4 * i + 1], p[16 * k + 4 * i + 2],
                                               p[16 * k + 4 * i + 3]);
                        }
                        __syncwarp();
                        const int col = 32 * k + lane;
                        const uint32_t base = (uint32_t)csv[col] * D_LEVELS + 32 + dmax, cw_l = cw[col];
                        while (rows) {
                            const int q = __ffs(rows) - 1;
                            rows &= rows - 1;
                            const uint32_t word = scr[q * D_SCR_STRIDE + (lane >> 1)];
                            const uint32_t v = (lane & 1) ? (word >> 16) : (word & 0xFFFFu);
                            // mismatches l - (v - bias_b)
                            if (MODE == MODE_WEIGHTED) {
                                const uint32_t wq = __shfl_sync(GKM_FULL, wx, q);
                                if (v & 32u) atomicAdd(wcnt + (base - v), wq * cw_l);
                            } else if (MODE == MODE_U32) {
                                if (v & 32u) atomicAdd(cnt32 + (base - v), 1u);
                            } else if (v & 32u) {
                                atomicAdd(cnt + (base - v), 1ull);
                            }
                        }
                        __syncwarp();  // scratch is rewritten by the next chunk
                    }
                }
                if (!ok) break;
                __syncwarp();  // B tile's column tables no longer read: hand the buffer back
                if (lane == 0) bar_arrive(bar(BAR_BEMPTY + buf));
                if (WEIGHTED && ((g + 1) % (uint32_t)a.flush_every == 0 || bt + 1 == NB)) {
                    // this warp's counts into the block's 64-bit counters
                    for (int k = lane; k < D_CH * D_LEVELS; k += 32) {
                        const unsigned c = wcnt[k];
                        if (c) {
                            atomicAdd(cnt + k, (unsigned long long)c);
                            wcnt[k] = 0;
                        }
                    }
                    __syncwarp();
                }
            }
        } else if (warp == D_PROD_WARP) {
            // ---- producer: one bulk copy per B record
            if (lane == 0) {
                for (int bt = 0; bt < NB; bt++) {
                    const uint32_t g = g_base + bt, buf = g % D_BBUF;
                    if (g >= D_BBUF &&
                        !bar_wait(bar(BAR_BEMPTY + buf), (g / D_BBUF - 1) & 1u, abort, a.error, a.role_wait_ns))
                        break;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar(BAR_BFULL + buf)),
                                 "r"((uint32_t)REC)
                                 : "memory");
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            smem_addr(smB + buf * REC)),
                        "l"(rec + (int64_t)bt * REC), "r"((uint32_t)REC), "r"(bar(BAR_BFULL + buf))
                        : "memory");
                    copies = g + 1;
                }
            }
        } else if (lane == 0) {
            // ---- MMA issue: every (B tile, A tile) pair, accumulators alternating
            bool ok = true;
            for (int bt = 0; bt < NB && ok; bt++) {
                const uint32_t g = g_base + bt, buf = g % D_BBUF;
                ok = bar_wait(bar(BAR_BFULL + buf), (g / D_BBUF) & 1u, abort, a.error, a.role_wait_ns);
                for (int at = 0; at < NA && ok; at++) {
                    const uint32_t t = t_base + (uint32_t)(bt * NA + at), slot = t & 1u;
                    if (t >= 2) ok = bar_wait(bar(BAR_TEMPTY + slot), ((t >> 1) - 1) & 1u, abort, a.error, a.role_wait_ns);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
                    for (int kb = 0; kb < 2; kb++) {
                        const uint64_t da = make_sdesc(smem_addr(smA + at * A_TILE) + kb * DM * 32, 128, 256);
                        const uint64_t db = make_sdesc(smem_addr(smB + buf * REC) + kb * DN * 32, 128, 256);
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + slot * DN),
                            "l"(da), "l"(db), "r"(idesc), "r"(kb));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        bar(BAR_TFULL + slot)));
                }
            }
        }
        g_base += (uint32_t)NB;
        t_base += (uint32_t)(NB * NA);
        __syncthreads();  // segment done (or abandoned): A is restaged next
        if (abort_flag) break;
    }
    if (abort_flag && warp == D_PROD_WARP && lane == 0) {
        // copies in flight land in the B buffers: wait for the last one of
        // each buffer (bounded) before the block's shared memory is released
        for (uint32_t g = copies > D_BBUF ? copies - D_BBUF : 0; g < copies; g++) {
            int ignore = 0;
            bar_wait(bar(BAR_BFULL + g % D_BBUF), (g / D_BBUF) & 1u, &ignore, a.error);
        }
    }
    // every MMA issued has completed before its accumulator columns are
    // released (bounded: on a stuck MMA the wait runs out and the error is set)
    if (warp == D_MMA_WARP && lane == 0) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            bar(BAR_DONE)));
        int ignore = 0;
        bar_wait(bar(BAR_DONE), 0u, &ignore, a.error);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(D_TMEM_COLS));
    if (abort_flag) return;
    for (int s = tid; s < nsv; s += D_THREADS) {
        const int64_t sg = cg * D_CH + s;
        auto count = [&](int m) -> uint64_t {
            return MODE == MODE_U32 ? (uint64_t)cnt32[s * D_LEVELS + m] : (uint64_t)cnt[s * D_LEVELS + m];
        };
        double k = 0.0;
        for (int m = 0; m <= dmax; m++) k += sp.h[m] * (double)count(m);
        if (a.raw) a.raw[b * a.S + sg] = k;
        if (a.profile)
            for (int m = 0; m <= l; m++) a.profile[(b * a.S + sg) * (l + 1) + m] = m <= dmax ? count(m) : 0;
    }
}

// Role hand-off wait limit of the dense launches made from this thread; 0:
// D_WAIT_NS.  Tests shorten it to make a hand-off wait run out.
static thread_local uint64_t g_role_wait_ns = 0;

}  // namespace

extern "C" int gkm_dense_set_role_wait(int64_t ns)
{
    if (ns < 0) return gkm_fail(GKM_ERR_INVALID, "wait limit %lld < 0", (long long)ns);
    g_role_wait_ns = (uint64_t)ns;
    return GKM_OK;
}

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
    if (B > 0x7FFFFFFFLL) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many rows for one dense launch");
    if ((int64_t)D_CH * 2 * Wy > 0x7FFFFFFFLL) return gkm_fail(GKM_ERR_UNSUPPORTED, "columns too long for one dense launch");
    cudaStream_t st = (cudaStream_t)stream;
    const int mult = (spec->include_rc && ry) ? 2 : 1;
    const int64_t chunks = (S + D_CH - 1) / D_CH;
    const int64_t max_tiles = (D_CH * mult * Wy + DN - 1) / DN;
    const size_t per_chunk = (size_t)max_tiles * REC;
    int64_t round = (int64_t)(D_REC_BUDGET / per_chunk);
    if (round < 1) round = 1;
    if (round > chunks) round = chunks;
    if (round > 65535) round = 65535;
    uint8_t *rec = nullptr;
    if (cudaMallocAsync(&rec, per_chunk * round, st) != cudaSuccess) return gkm_fail(GKM_ERR_OOM, "dense B records");
    // 32-bit block counters when no (row, SV) can reach 2^32 unweighted pairs
    const int mode = spec->weighted ? MODE_WEIGHTED
                     : (int64_t)Wx * mult * Wy < 0xFFFFFFFFLL ? MODE_U32 : MODE_U64;
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
    a.max_tiles = max_tiles;
    a.flush_every = (int)(0xFFFFFFFFull / (Cfg<MODE_WEIGHTED>::WARP_PAIRS_PER_B * 255ull * 255ull));
    a.rec = rec;
    a.raw = raw;
    a.profile = profile;
    a.error = error;
    a.role_wait_ns = g_role_wait_ns ? g_role_wait_ns : D_WAIT_NS;
    cudaFuncSetAttribute(dense_pairs_kernel<MODE_U32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         Cfg<MODE_U32>::SMEM);
    cudaFuncSetAttribute(dense_pairs_kernel<MODE_U64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         Cfg<MODE_U64>::SMEM);
    cudaFuncSetAttribute(dense_pairs_kernel<MODE_WEIGHTED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         Cfg<MODE_WEIGHTED>::SMEM);
    int s = GKM_OK;
    for (int64_t c0 = 0; c0 < chunks && s == GKM_OK; c0 += round) {
        const int64_t nc = chunks - c0 < round ? chunks - c0 : round;
        a.chunk0 = c0;
        dense_b_records<<<dim3((unsigned)max_tiles, (unsigned)nc), DN, 0, st>>>(a, rec);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            s = gkm_cuda_status(e, "dense_b_records");
            break;
        }
        const dim3 grid((unsigned)B, (unsigned)nc);
        if (mode == MODE_U32)
            dense_pairs_kernel<MODE_U32><<<grid, D_THREADS, Cfg<MODE_U32>::SMEM, st>>>(a);
        else if (mode == MODE_U64)
            dense_pairs_kernel<MODE_U64><<<grid, D_THREADS, Cfg<MODE_U64>::SMEM, st>>>(a);
        else
            dense_pairs_kernel<MODE_WEIGHTED><<<grid, D_THREADS, Cfg<MODE_WEIGHTED>::SMEM, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "dense_pairs");
    }
    cudaFreeAsync(rec, st);
    return s;
}
