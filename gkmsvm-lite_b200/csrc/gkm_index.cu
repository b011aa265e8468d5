// gkm_index.cu -- the SV l-mer index: built by an LSD radix sort of the packed
// l-mers of every SV window (forward and RC) into per-SV-tile CSR buckets, and
// queried by visiting each query window's d-mismatch neighbourhood.
//
// Query accumulators are integer pair counts per (SV, mismatch level) in
// shared memory, one SV tile per thread block; the FP64 epilogue weights them
// by h(m) and, for scoring, normalises, applies the RBF and reduces over the
// tile's SVs in a fixed order (deterministic), so no [rows, S] block is written.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <type_traits>

#include "gkm_common.cuh"

namespace {

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of uint32 (three phases, recursive on block sums)
// ---------------------------------------------------------------------------

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER_THREAD = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

__global__ void scan_tiles(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, int64_t n,
                           uint32_t *__restrict__ tile_sums)
{
    __shared__ uint32_t warp_tot[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_PER_THREAD;
    uint32_t v[SCAN_PER_THREAD];
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        uint32_t t = v[k];
        v[k] = run;
        run += t;
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(GKM_FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(GKM_FULL, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;
    }
    __syncthreads();
    uint32_t excl = x - run + (warp ? warp_tot[warp - 1] : 0);
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++)
        if (base + k < n) out[base + k] = v[k] + excl;
    if (threadIdx.x == SCAN_THREADS - 1 && tile_sums) tile_sums[blockIdx.x] = excl + run;
}

__global__ void scan_add(uint32_t *__restrict__ out, int64_t n, const uint32_t *__restrict__ tile_pref)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_pref[i / SCAN_TILE];
}

int scan_exclusive(const uint32_t *in, uint32_t *out, int64_t n, cudaStream_t st)
{
    if (n <= 0) return GKM_OK;
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 1) {
        scan_tiles<<<1, SCAN_THREADS, 0, st>>>(in, out, n, nullptr);
        GKM_CHECK_LAUNCH("scan");
        return GKM_OK;
    }
    uint32_t *sums = nullptr;
    if (cudaMallocAsync(&sums, sizeof(uint32_t) * tiles * 2, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "scan scratch");
    scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, sums);
    GKM_CHECK_LAUNCH("scan");
    int s = scan_exclusive(sums, sums + tiles, tiles, st);
    if (s == GKM_OK) {
        scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, sums + tiles);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "scan_add");
    }
    cudaFreeAsync(sums, st);
    return s;
}

// ---------------------------------------------------------------------------
// LSD radix sort of (key, value) pairs, 8-bit digits, stable
// ---------------------------------------------------------------------------

constexpr int RS_THREADS = 256;
constexpr int RS_SUB = 16;                       // sub-tiles of 256 keys per block
constexpr int RS_CHUNK = RS_THREADS * RS_SUB;    // keys per block

__global__ void radix_hist(const uint32_t *__restrict__ keys, int64_t n, int shift, uint32_t *__restrict__ hist,
                           int64_t nblocks)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * RS_CHUNK;
    for (int k = threadIdx.x; k < RS_CHUNK; k += RS_THREADS) {
        int64_t i = base + k;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: keys of a block go out in their input order within each digit.
__global__ void radix_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                              uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, int64_t n, int shift,
                              const uint32_t *__restrict__ pref, int64_t nblocks)
{
    constexpr int NWARP = RS_THREADS / 32;
    __shared__ uint32_t run[256];
    __shared__ uint32_t wcnt[NWARP][256];
    __shared__ uint32_t woff[NWARP][256];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    run[threadIdx.x] = pref[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    int64_t base = (int64_t)blockIdx.x * RS_CHUNK;
    for (int sub = 0; sub < RS_SUB; sub++) {
        for (int w = 0; w < NWARP; w++) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        int64_t i = base + (int64_t)sub * RS_THREADS + threadIdx.x;
        bool valid = i < n;
        uint32_t k = valid ? kin[i] : 0, v = valid ? vin[i] : 0;
        uint32_t d = (k >> shift) & 255u;
        uint32_t act = __ballot_sync(GKM_FULL, valid);
        uint32_t rank = 0;
        if (valid) {
            uint32_t peers = __match_any_sync(act, d);
            rank = __popc(peers & ((1u << lane) - 1u));
            if (rank == 0) wcnt[warp][d] = __popc(peers);
        }
        __syncthreads();
        {  // thread t owns digit t: prefix over warps
            uint32_t s = 0;
            for (int w = 0; w < NWARP; w++) {
                woff[w][threadIdx.x] = s;
                s += wcnt[w][threadIdx.x];
            }
            wcnt[0][threadIdx.x] = s;  // sub-tile total for the digit (read after sync)
        }
        __syncthreads();
        if (valid) {
            uint32_t pos = run[d] + woff[warp][d] + rank;
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncthreads();
        run[threadIdx.x] += wcnt[0][threadIdx.x];
        __syncthreads();
    }
}

int radix_sort(uint32_t *&keys, uint32_t *&vals, uint32_t *&ktmp, uint32_t *&vtmp, int64_t n, int bits,
               cudaStream_t st)
{
    if (n <= 1) return GKM_OK;
    int64_t nb = (n + RS_CHUNK - 1) / RS_CHUNK;
    uint32_t *hist = nullptr;
    if (cudaMallocAsync(&hist, sizeof(uint32_t) * 256 * nb * 2, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "radix sort scratch");
    int s = GKM_OK;
    for (int shift = 0; shift < bits && s == GKM_OK; shift += 8) {
        radix_hist<<<(unsigned)nb, RS_THREADS, 0, st>>>(keys, n, shift, hist, nb);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            s = gkm_cuda_status(e, "radix_hist");
            break;
        }
        s = scan_exclusive(hist, hist + 256 * nb, 256 * nb, st);
        if (s != GKM_OK) break;
        radix_scatter<<<(unsigned)nb, RS_THREADS, 0, st>>>(keys, vals, ktmp, vtmp, n, shift, hist + 256 * nb, nb);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            s = gkm_cuda_status(e, "radix_scatter");
            break;
        }
        uint32_t *t = keys;
        keys = ktmp;
        ktmp = t;
        t = vals;
        vals = vtmp;
        vtmp = t;
    }
    cudaFreeAsync(hist, st);
    return s;
}

// ---------------------------------------------------------------------------
// Index build
// ---------------------------------------------------------------------------

__global__ void entry_counts(const int32_t *__restrict__ counts, int64_t S, int nb, uint32_t *__restrict__ out)
{
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) out[s] = (uint32_t)counts[s] * nb;
}

// Entries in column order: each SV's forward windows, then its RC windows in
// RC-row order (kernels/lmer_index.py:171-176), so a stable sort keeps every
// bucket ascending by SV.  key = tile << 2l | l-mer; value = local SV id |
// window weight << 24.
__global__ void entry_gen(gkm_spec spec, const uint32_t *__restrict__ fwd, const uint32_t *__restrict__ rc,
                          const int32_t *__restrict__ counts, const uint32_t *__restrict__ base, int64_t S,
                          int64_t W, int tile_svs, uint32_t *__restrict__ keys, uint32_t *__restrict__ vals)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= S * W) return;
    int64_t s = idx / W;
    int j = (int)(idx - s * W);
    int n = counts[s];
    if (j >= n) return;
    uint32_t tile = (uint32_t)(s / tile_svs);
    uint32_t local = (uint32_t)(s - (int64_t)tile * tile_svs);
    uint32_t hi = tile << (2 * spec.l);
    uint32_t e0 = base[s];
    uint32_t wf = spec.weighted ? gkm_wt(spec.wd, n, j) : 1u;
    keys[e0 + j] = hi | fwd[s * W + j];
    vals[e0 + j] = local | (wf << 24);
    if (spec.include_rc && rc) {
        // RC-row position W - n + j holds rc(forward window n - 1 - j)
        uint32_t wr = spec.weighted ? gkm_wt(spec.wd, n, n - 1 - j) : 1u;
        keys[e0 + n + j] = hi | rc[s * W + (W - n + j)];
        vals[e0 + n + j] = local | (wr << 24);
    }
}

__global__ void narrow_entries(const uint32_t *__restrict__ vals, int64_t n, uint16_t *__restrict__ out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint16_t)(vals[i] & 0xFFFFu);
}

__global__ void bucket_offsets(const uint32_t *__restrict__ keys, int64_t E, int64_t nbuckets,
                               uint32_t *__restrict__ off)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > E) return;
    int64_t lo = i == 0 ? 0 : (int64_t)keys[i - 1] + 1;
    int64_t hi = i == E ? nbuckets : (int64_t)keys[i];
    for (int64_t k = lo; k <= hi; k++) off[k] = (uint32_t)i;
}

// One 32-bit word per bucket for the query's lookups, so that a lookup is one
// load: (bucket begin - its tile's first entry) << lb | bucket length, the
// length saturated at 2^lb - 1 (a bucket that long is read from the offsets).
__global__ void bucket_words(const uint32_t *__restrict__ off, int64_t nbuckets, int64_t n_lmers, int lb,
                             uint32_t *__restrict__ bw)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbuckets) return;
    const uint32_t base = off[(i / n_lmers) * n_lmers], b = off[i], n = off[i + 1] - b;
    const uint32_t lmask = (1u << lb) - 1u;
    bw[i] = ((b - base) << lb) | (n < lmask ? n : lmask);
}

// ---------------------------------------------------------------------------
// Index query
// ---------------------------------------------------------------------------

constexpr int Q_THREADS = 1024;
constexpr int Q_WARPS = Q_THREADS / 32;
constexpr int LOG_CAP = 64;            // carry events a block can log (narrow counters)
constexpr int MASKS_SMEM_MAX = 6144;   // neighbour masks staged in shared memory up to this
// MODE_COUNT: an item covers a range of a row's windows (a row split) and adds
// its exact per-(SV, level) counts into gcount; a finish kernel turns the
// summed counts into K_raw, profiles or scores.
enum { MODE_SCORE = 0, MODE_RAW = 1, MODE_COUNT = 2 };

// Narrow (C16) counters: 32-bit words split into fields, one level of one SV
// per field.  Paired layout: two 16-bit fields per word, levels 2j and 2j+1 of
// an SV in word j * tile_svs + s.  Packed layout (unweighted, <= 4 levels):
// every level of SV s in word s, field m at bit shift(m) and width(m), so a
// tile holds twice the SVs.  Field g of a layout: shift (fsh >> 5g) & 31,
// width (fw >> 5g) & 31; nf fields per word.
struct Narrow {
    int packed, nf;
    uint32_t fsh, fw;
    __device__ __forceinline__ uint32_t shift(int g) const { return (fsh >> (5 * g)) & 31u; }
    __device__ __forceinline__ uint32_t mask(int g) const
    {
        const uint32_t w = (fw >> (5 * g)) & 31u;
        return w ? (1u << w) - 1u : 0xFFFFFFFFu;  // width 0 stands for 32
    }
    __device__ __forceinline__ uint32_t width(int g) const
    {
        const uint32_t w = (fw >> (5 * g)) & 31u;
        return w ? w : 32u;
    }
    // counter word and field of level m of local SV s
    __device__ __forceinline__ uint32_t word(int m, int St, int s) const
    {
        return packed ? (uint32_t)s : (uint32_t)((m >> 1) * St + s);
    }
    __device__ __forceinline__ int field(int m) const { return packed ? m : (m & 1); }
};

struct QueryArgs {
    const uint32_t *bx;
    const int32_t *cx;
    int64_t W;
    const int32_t *order;
    int64_t diag_offset;  // >= 0: row r is column diag_offset + r
    // index
    const uint32_t *off;
    const uint32_t *bw;   // bucket words (bucket_words)
    int lb;               // length bits of a bucket word
    const void *ent;      // uint16 local ids, or uint32 id | weight << 24
    const uint32_t *masks;
    int n_masks;
    int64_t n_lmers;
    int64_t S;
    int tile_svs;
    int sub_svs;          // SVs per accumulation pass (wide counters)
    int nlev;
    int dmax;
    double h[16];
    Narrow nw;            // narrow counters' layout
    const uint8_t *wd;
    const uint8_t *wq;    // [rows, W] query window weights (null: from the row's count)
    unsigned int *status; // [2] event counts: a block's carry log overflowed, a wide counter wrapped
    unsigned int *queue;  // work-queue head: items (tile, row) handed out tile-major
    int64_t B;            // rows
    int tiles;
    // 32-bit counters: the most one query window can add to one counter (its
    // SV's windows x the largest weight product); an item whose windows times
    // this stays below 2^32 cannot wrap a counter, and adds without checking
    uint64_t wide_bound;
    int skip_empty;       // rows without windows write nothing (their outputs are never read)
    int nsplit;           // items per (row, tile): window ranges of split_w windows
    int split_w;
    unsigned long long *gcount;  // MODE_COUNT: [B, S, nlev] summed counts (gpack: [B, S, (nlev + 1) / 2])
    int gpack;            // MODE_COUNT: two levels per 64-bit count, 32 bits each (no count reaches 2^32)
    // score
    const double *inv_dx;
    const double *inv_ds;
    const double *coef;
    double gamma;
    int rbf;
    double *partial;  // [B, tiles]
    // raw
    double *raw;
    uint64_t *profile;
    int l;
};

// Shared memory of a query block: staged masks and the carry log, then the
// counters.
__host__ __device__ inline size_t query_fixed_smem(int n_masks)
{
    size_t m = n_masks <= MASKS_SMEM_MAX ? (size_t)n_masks * 4 : 0;
    m = (m + 15) & ~(size_t)15;
    return m + LOG_CAP * 4 + 64;
}

// C16: unweighted pair counts in narrow fields (Narrow).  A field that passes
// its largest value carries into the next field (or out of the word); the
// carry-logged adder sees that in the value atomicAdd returns and logs it, and
// the epilogue adds the carries back, so the counts stay exact.
template <bool C16, bool C64>
__device__ __forceinline__ int64_t read_count(const uint32_t *acc, const uint32_t *log, int nlog, int m, int St,
                                              int s, const Narrow &nw)
{
    if (C64) return (int64_t)((const unsigned long long *)acc)[m * St + s];
    if (!C16) return acc[m * St + s];
    const uint32_t word = nw.word(m, St, s);
    const int g = nw.field(m);
    int64_t f = (acc[word] >> nw.shift(g)) & nw.mask(g);
    // a logged carry out of field g took 2^width from it; one out of field
    // g - 1 added 1 to it
    for (int e = 0; e < nlog; e++) {
        const uint32_t ev = log[e];
        if ((ev >> 3) != word) continue;
        const int eg = (int)(ev & 7u);
        if (eg == g)
            f += (int64_t)1 << nw.width(g);
        else if (eg + 1 == g)
            f -= 1;
    }
    return f;
}

// Carry-logged narrow counter update: add 1 to field g of word.  A field that
// was all ones carries into the next (which may carry on in turn; the top
// field's carry leaves the word): each carry is logged as (word, field), and
// read_count adds it back.
__device__ __forceinline__ void count_narrow(uint32_t *acc, uint32_t word, int g, const Narrow &nw, int *nlog,
                                             uint32_t *log, unsigned int *status)
{
    const uint32_t old = atomicAdd(acc + word, 1u << nw.shift(g));
    for (; g < nw.nf; g++) {
        const uint32_t mk = nw.mask(g);
        if (((old >> nw.shift(g)) & mk) != mk) break;
        const int p0 = atomicAdd(nlog, 1);
        if (p0 < LOG_CAP)
            log[p0] = (word << 3) | (uint32_t)g;
        else
            atomicAdd(status, 1u);
    }
}

// Index entry k: 16-bit local SV id (unweighted tiles of <= 65,536 SVs), or
// local id | window weight << 24.
template <bool E16>
__device__ __forceinline__ uint32_t load_entry(const void *ent, uint32_t k)
{
    if (E16) return (uint32_t)__ldg((const uint16_t *)ent + k);
    return __ldg((const uint32_t *)ent + k);
}

// Persistent blocks take (SV tile, row) items: each warp takes whole query
// windows (rows shorter than the warp count: (window, mask chunk) units split
// evenly); each lane one neighbour mask per chunk of 32, scanning its bucket
// four entries at a time (one vector load); the next chunk's bucket bounds
// are loaded while this chunk's entries are counted.  Counts go to narrow
// shared fields by plain adds, checked exactly at the end of the item (a
// carry makes the decoded fields sum to less than the adds made), and the
// rare item that carried is redone with the carry-logged adds.  Wide counters
// are 32-bit, or 64-bit (C64) for the rerun of a weighted call whose 32-bit
// count wrapped.
template <bool WEIGHTED, int MODE, bool C16, bool E16, bool RANGE, bool C64 = false>
__global__ void __launch_bounds__(Q_THREADS, 1) index_query(QueryArgs a)
{
    extern __shared__ __align__(16) uint8_t smraw[];
    __shared__ double red[32];
    __shared__ int nlog;
    __shared__ unsigned long long chk[2];  // decoded field sum, plain adds made
    const int n_masks = a.n_masks;
    uint32_t *sm_masks = n_masks <= MASKS_SMEM_MAX ? (uint32_t *)smraw : nullptr;
    uint32_t *sm_log = (uint32_t *)(smraw + ((sm_masks ? (size_t)n_masks * 4 : 0) + 15 & ~(size_t)15));
    uint32_t *sm_acc = (uint32_t *)(smraw + query_fixed_smem(n_masks));
    __shared__ unsigned int item_s;
    if (sm_masks)
        for (int k = threadIdx.x; k < n_masks; k += Q_THREADS) sm_masks[k] = a.masks[k];
    const uint32_t *masks = sm_masks ? sm_masks : a.masks;
    const int St = a.tile_svs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // persistent: each block takes (tile, row) items off the work queue,
    // tile-major so that one SV tile's index is what L2 holds, rows in the order
    // given (longest first)
    for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_s = atomicAdd(a.queue, 1u);
    __syncthreads();
    const unsigned int item = item_s;
    const int64_t per_tile = a.B * a.nsplit;
    if ((int64_t)item >= per_tile * a.tiles) break;
    const int t = (int)(item / per_tile);
    const int64_t rem = item - (int64_t)t * per_tile;
    const int64_t r = rem / a.nsplit;
    const int ks = (int)(rem - r * a.nsplit);
    const int64_t row = a.order ? a.order[r] : r;
    const int64_t s0 = (int64_t)t * St;
    const int ns = (int)min((int64_t)St, a.S - s0);
    const int64_t lo_g = a.diag_offset >= 0 ? a.diag_offset + row : 0;
    if (MODE == MODE_RAW && s0 + ns <= lo_g) continue;  // tile wholly below the diagonal
    const uint32_t lo = (uint32_t)(lo_g > s0 ? lo_g - s0 : 0);
    const int n = a.cx[row];
    // this item's windows [i0, i1) of the row (the whole row unless split)
    const int i0 = min(n, ks * a.split_w), i1 = min(n, i0 + a.split_w);
    if ((MODE == MODE_COUNT || a.skip_empty) && i0 >= i1) continue;
    const uint32_t *x = a.bx + row * a.W;
    const uint32_t *off = a.off + (int64_t)t * a.n_lmers;
    const uint32_t *bw = WEIGHTED ? nullptr : a.bw + (int64_t)t * a.n_lmers;
    const uint32_t tbase = __ldg(off), lmask = (1u << a.lb) - 1u;
    const double inv_dx = MODE == MODE_SCORE ? a.inv_dx[row] : 0.0;
    double part = 0.0;
    const int sub = C16 ? ns : a.sub_svs;
    if (MODE == MODE_SCORE && i0 >= i1) {
        // a row without windows (rows of length 0 pad a batch to its graph
        // bucket): every K(row, s) is 0, so each SV's term is coef f(0), with
        // the arithmetic and order of a one-pass flush below -- no counters to
        // clear, no walk
        for (int s = threadIdx.x; s < ns; s += Q_THREADS) {
            const int64_t sg = s0 + s;
            const double kn = 0.0 * inv_dx * a.inv_ds[sg];
            part += a.coef[sg] * (a.rbf ? exp(a.gamma * (kn - 1.0)) : kn);
        }
    } else
    for (int sub_lo = 0; sub_lo < ns; sub_lo += sub) {
        const int sub_n = min(sub, ns - sub_lo);
        const int stride = C16 ? St : sub_n;
        const int nacc = C16 ? (a.nw.packed ? St : ((a.nlev + 1) / 2) * St) : a.nlev * sub_n;
        const uint32_t id_lo = max((uint32_t)sub_lo, lo), id_hi = (uint32_t)(sub_lo + sub_n);
        // narrow counters: a first attempt with plain shared adds (no return
        // value, no per-hit carry test), checked exactly at the end -- the
        // decoded fields sum to the hits counted unless some field carried;
        // only then the item is redone with the carry-logged adds
        bool logged = false;
        for (;;) {
        for (int k = threadIdx.x; k < (C64 ? 2 * nacc : nacc); k += Q_THREADS) sm_acc[k] = 0;
        if (threadIdx.x == 0) {
            nlog = 0;
            chk[0] = chk[1] = 0;
        }
        __syncthreads();
        unsigned long long lane_hits = 0;  // plain adds this lane made
        const int nwin = i1 - i0;
        const bool wide_safe = !C16 && (unsigned long long)nwin * a.wide_bound < (1ull << 32);
        const int nchunk = (n_masks + 31) >> 5;
        // per lane: its mask's bucket (begin, length) and counter slot (C16:
        // word base of the level (0 packed, the level pair's row paired) | the
        // level's field in bits 29..31; wide: row base of the level)
        auto lane_mask = [&](uint32_t u, int c, uint32_t &b0, uint32_t &n0, uint32_t &sl) {
            b0 = n0 = sl = 0;
            if (c >= n_masks) return;
            const uint32_t mk = masks[c];
            const uint32_t v = u ^ (mk & 0x00FFFFFFu);
            const uint32_t lev = mk >> 24;
            sl = C16 ? (a.nw.packed ? lev << 29 : ((lev >> 1) * (uint32_t)St) | ((lev & 1u) << 29))
                     : lev * (uint32_t)stride - (uint32_t)sub_lo;
            if (WEIGHTED) {
                b0 = __ldg(off + v);
                n0 = __ldg(off + v + 1) - b0;
            } else {
                // one load (measured on 5,000 config-3 t=3 queries: 400.6 ->
                // 383.9 ms; the weighted walk, 4-byte entries, was 2 % slower)
                const uint32_t w = __ldg(bw + v);
                b0 = tbase + (w >> a.lb);
                n0 = w & lmask;
                if (n0 == lmask) n0 = __ldg(off + v + 1) - b0;  // a long bucket
            }
        };
        auto window_weight = [&](int i) -> uint32_t {
            return WEIGHTED ? (a.wq ? (uint32_t)a.wq[row * a.W + i] : gkm_wt(a.wd, n, i)) : 1u;
        };
        // the chunk being counted: this lane's bucket (beg, len), its counter
        // slot, and the query window's weight
        uint32_t wq = 1, beg = 0, len = 0, slot = 0;
        // one index entry en of this lane's bucket: counter word base + id
        // (C16: add `add` to it, the level's field g; wide: row base).
        // PLAIN (a compile-time flag of the counting loops): C16 plain adds
        // (not the carry-logged retry), wide adds that cannot wrap
        auto count_hit = [&](auto PLAIN, uint32_t en, uint32_t base, uint32_t add, int g) {
            constexpr bool plain = decltype(PLAIN)::value;
            const uint32_t id = E16 ? en : (en & 0x00FFFFFFu);
            if (RANGE && (id < id_lo || id >= id_hi)) return;
            if (C16) {
                if (!plain) {
                    count_narrow(sm_acc, base + id, g, a.nw, &nlog, sm_log, a.status);
                } else {
                    atomicAdd(sm_acc + base + id, add);
                    if (RANGE) lane_hits++;  // else the chunk's bucket length is counted whole
                }
            } else if (C64) {
                atomicAdd((unsigned long long *)sm_acc + base + id,
                          (unsigned long long)(WEIGHTED ? wq * (en >> 24) : 1u));
            } else {
                const uint32_t inc = WEIGHTED ? wq * (en >> 24) : 1u;
                if (plain) {
                    atomicAdd(sm_acc + base + id, inc);
                } else {
                    const uint32_t old = atomicAdd(sm_acc + base + id, inc);
                    if (old + inc < old) atomicAdd(a.status + 1, 1u);
                }
            }
        };
        // this lane's bucket [beg, beg + len) in aligned blocks of four
        // entries, several blocks per iteration with all their loads in flight
        // before any is counted; the warp runs as many iterations as its
        // longest bucket needs.  Measured: 2-byte entries (8-byte blocks) 2
        // blocks 417 ms, 3: 405, 4: 401 on 5,000 config-3 queries, one block
        // 500; with packed counters (larger buckets) 4: 341.6 ms, 5: 340.5, 6:
        // 338.1, six spilling registers where the SV range is tested (RANGE);
        // 4-byte entries (16-byte blocks) 1 block 1,841 ms, 2: 1,591, 4: 1,753
        // on 10,000 config-3 queries of the weighted t=5 kernel (3: 2 % faster
        // there, 5 % slower on the config-2 Gram)
        auto walk = [&](auto PLAIN) {
            constexpr int NB = E16 ? (RANGE ? 4 : 6) : 2;
            const uint32_t end = beg + len;
            const int g = C16 ? (int)(slot >> 29) : 0;  // the level's field
            const uint32_t base = C16 ? slot & 0x1FFFFFFFu : slot, add = C16 ? 1u << a.nw.shift(g) : 0u;
            if (!RANGE) lane_hits += len;
            for (uint32_t e = beg & ~3u; __any_sync(GKM_FULL, e < end); e += 4 * NB) {
                uint32_t en[4 * NB];
                if (E16) {
                    uint2 w[NB];
#pragma unroll
                    for (int k = 0; k < NB; k++)
                        w[k] = e + 4 * k < end ? __ldg((const uint2 *)((const uint16_t *)a.ent + e + 4 * k))
                                               : make_uint2(0, 0);
#pragma unroll
                    for (int k = 0; k < NB; k++) {
                        en[4 * k] = w[k].x & 0xFFFFu;
                        en[4 * k + 1] = w[k].x >> 16;
                        en[4 * k + 2] = w[k].y & 0xFFFFu;
                        en[4 * k + 3] = w[k].y >> 16;
                    }
                } else {
                    uint4 w[NB];
#pragma unroll
                    for (int k = 0; k < NB; k++)
                        w[k] = e + 4 * k < end ? __ldg((const uint4 *)((const uint32_t *)a.ent + e + 4 * k))
                                               : make_uint4(0, 0, 0, 0);
#pragma unroll
                    for (int k = 0; k < NB; k++) {
                        en[4 * k] = w[k].x;
                        en[4 * k + 1] = w[k].y;
                        en[4 * k + 2] = w[k].z;
                        en[4 * k + 3] = w[k].w;
                    }
                }
                // the iteration's slots inside [beg, end) as one bit mask
                const uint32_t lo = beg > e ? min(beg - e, 4u * NB) : 0u;
                const uint32_t hi = end > e ? min(end - e, 4u * NB) : 0u;
                const uint32_t valid = hi > lo ? ((1u << hi) - 1u) ^ ((1u << lo) - 1u) : 0u;
#pragma unroll
                for (int q = 0; q < 4 * NB; q++)
                    if (valid & (1u << q)) count_hit(PLAIN, en[q], base, add, g);
            }
        };
        // the item's windows to the warps, counted in one of two compiled forms
        auto count_item = [&](auto PLAIN) {
            if (nwin >= Q_WARPS) {
                // the row's windows to the warps in turn, all masks of a window in
                // one warp
                for (int i = i0 + warp; i < i1; i += Q_WARPS) {
                    const uint32_t u = x[i];
                    wq = window_weight(i);
                    lane_mask(u, lane, beg, len, slot);
                    for (int c0 = 0; c0 < n_masks; c0 += 32) {
                        // the next chunk's buckets, loaded while this one is counted
                        uint32_t nbeg, nlen, nslot;
                        lane_mask(u, c0 + 32 + lane, nbeg, nlen, nslot);
                        walk(PLAIN);
                        beg = nbeg;
                        len = nlen;
                        slot = nslot;
                    }
                }
            } else {
                // rows of fewer windows than warps (ISM window sets, the ends of
                // row splits): (window, chunk of 32 masks) units, window-major, in
                // one contiguous range per warp, so every warp has work
                const int64_t nunit = (int64_t)nwin * nchunk;
                const int64_t ub = nunit * warp / Q_WARPS, ue = nunit * (warp + 1) / Q_WARPS;
                if (ub < ue) {
                    int win = (int)(ub / nchunk), ch = (int)(ub - (int64_t)win * nchunk);
                    uint32_t u = x[i0 + win];
                    wq = window_weight(i0 + win);
                    lane_mask(u, ch * 32 + lane, beg, len, slot);
                    for (int64_t un = ub; un < ue; un++) {
                        // the next unit's window and buckets, loaded while this one is counted
                        int nw = win, nc = ch + 1;
                        if (nc == nchunk) {
                            nw = win + 1;
                            nc = 0;
                        }
                        uint32_t nu = u, nwq = wq, nbeg = 0, nlen = 0, nslot = 0;
                        if (un + 1 < ue) {
                            if (nw != win) {
                                nu = x[i0 + nw];
                                nwq = window_weight(i0 + nw);
                            }
                            lane_mask(nu, nc * 32 + lane, nbeg, nlen, nslot);
                        }
                        walk(PLAIN);
                        beg = nbeg;
                        len = nlen;
                        slot = nslot;
                        win = nw;
                        ch = nc;
                        u = nu;
                        wq = nwq;
                    }
                }
            }
        };
        if (C16 ? !logged : wide_safe)
            count_item(std::true_type{});
        else
            count_item(std::false_type{});
        __syncthreads();
        if (!C16 || logged) break;
        {
            unsigned long long fs = 0, hs = lane_hits;
            for (int k = threadIdx.x; k < nacc; k += Q_THREADS) {
                const uint32_t v = sm_acc[k];
                for (int g = 0; g < a.nw.nf; g++) fs += (v >> a.nw.shift(g)) & a.nw.mask(g);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                fs += __shfl_xor_sync(GKM_FULL, fs, o);
                hs += __shfl_xor_sync(GKM_FULL, hs, o);
            }
            if (lane == 0) {
                atomicAdd(&chk[0], fs);
                atomicAdd(&chk[1], hs);
            }
        }
        __syncthreads();
        const bool exact = chk[0] == chk[1];
        __syncthreads();  // every thread has read chk before the retry resets it
        if (exact) break;
        logged = true;
        }
        const int nl = min(nlog, LOG_CAP);
        if (MODE == MODE_COUNT) {
            for (int s = sub_lo + threadIdx.x; s < sub_lo + sub_n; s += Q_THREADS) {
                if (a.gpack) {
                    // levels 2j and 2j + 1 in one add: half the global atomics
                    const int gw = (a.nlev + 1) >> 1;
                    unsigned long long *g = a.gcount + (row * a.S + s0 + s) * gw;
                    for (int j = 0; j < gw; j++) {
                        const uint64_t c0 = (uint64_t)read_count<C16, C64>(sm_acc, sm_log, nl, 2 * j, stride,
                                                                           s - sub_lo, a.nw);
                        const uint64_t c1 = 2 * j + 1 < a.nlev
                                                ? (uint64_t)read_count<C16, C64>(sm_acc, sm_log, nl, 2 * j + 1,
                                                                                 stride, s - sub_lo, a.nw)
                                                : 0;
                        const uint64_t v = c0 | (c1 << 32);
                        if (v) atomicAdd(g + j, (unsigned long long)v);
                    }
                } else {
                    unsigned long long *g = a.gcount + (row * a.S + s0 + s) * a.nlev;
                    for (int m = 0; m < a.nlev; m++) {
                        const int64_t c = read_count<C16, C64>(sm_acc, sm_log, nl, m, stride, s - sub_lo, a.nw);
                        if (c) atomicAdd(g + m, (unsigned long long)c);
                    }
                }
            }
        } else
        for (int s = sub_lo + threadIdx.x; s < sub_lo + sub_n; s += Q_THREADS) {
            double k = 0.0;
            for (int m = 0; m < a.nlev; m++)
                k += a.h[m] * (double)read_count<C16, C64>(sm_acc, sm_log, nl, m, stride, s - sub_lo, a.nw);
            const int64_t sg = s0 + s;
            if (MODE == MODE_SCORE) {
                const double kn = k * inv_dx * a.inv_ds[sg];
                part += a.coef[sg] * (a.rbf ? exp(a.gamma * (kn - 1.0)) : kn);
            } else if (s >= (int)lo) {
                if (a.raw) a.raw[row * a.S + sg] = k;
                if (a.profile) {
                    uint64_t *pp = a.profile + (row * a.S + sg) * (a.l + 1);
                    for (int m = 0; m <= a.l; m++)
                        pp[m] = m < a.nlev ? (uint64_t)read_count<C16, C64>(sm_acc, sm_log, nl, m, stride, s - sub_lo, a.nw) : 0;
                }
            }
        }
        __syncthreads();
    }
    if (MODE == MODE_SCORE) {
        part = gkm_block_sum(part, red);
        if (threadIdx.x == 0) a.partial[row * a.tiles + t] = part;
    }
    }
}

__global__ void finish_scores(const double *__restrict__ partial, int64_t B, int tiles, double bias,
                              double *__restrict__ out)
{
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double s = 0.0;
    for (int t = 0; t < tiles; t++) s += partial[b * tiles + t];
    out[b] = s + bias;
}

// V[v] over every tile's bucket of v (lmer_table.py:35-55)
__global__ void lmer_weights_kernel(const uint32_t *__restrict__ off, const uint32_t *__restrict__ ent,
                                    const uint16_t *__restrict__ ent16, int64_t n_lmers, int tiles, int tile_svs,
                                    int weighted, const double *__restrict__ c_sv, double *__restrict__ V)
{
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_lmers) return;
    double acc = 0.0;
    for (int t = 0; t < tiles; t++) {
        uint32_t b = off[t * n_lmers + v], e = off[t * n_lmers + v + 1];
        for (uint32_t k = b; k < e; k++) {
            uint32_t en = ent16 ? (uint32_t)ent16[k] | (1u << 24) : ent[k];
            double c = c_sv[(int64_t)t * tile_svs + (en & 0x00FFFFFFu)];
            acc += weighted ? c * (double)(en >> 24) : c;
        }
    }
    V[v] = acc;
}

}  // namespace

int gkm_smem_limit()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

int gkm_sm_count()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

extern "C" int gkm_index_create(const gkm_spec *spec, const uint32_t *fwd, const uint32_t *rc,
                                const int32_t *counts, int64_t S, int64_t W, const uint32_t *masks,
                                int32_t n_masks, int32_t tile_svs, gkm_index_t **out, gkm_stream_t stream)
{
    if (!spec || !out) return gkm_fail(GKM_ERR_INVALID, "null spec or out");
    *out = nullptr;
    if (spec->l < 1 || spec->l > 12) return gkm_fail(GKM_ERR_UNSUPPORTED, "the l-mer index needs l <= 12");
    if (S < 1 || W < 1) return gkm_fail(GKM_ERR_INVALID, "empty columns");
    if (S > (1 << 24) * 64LL) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many columns");
    if (!masks || n_masks < 1) return gkm_fail(GKM_ERR_INVALID, "no neighbour masks");
    if (spec->weighted && !spec->wd) return gkm_fail(GKM_ERR_INVALID, "weighted spec without weights");
    cudaStream_t st = (cudaStream_t)stream;
    int nlev = spec->dmax + 1;
    // counter bytes per SV: narrow fields (unweighted) or 32-bit (weighted)
    int acc_bytes = gkm_smem_limit() - 1024 - (int)query_fixed_smem(n_masks);
    // narrow counters: every level of an SV in one 32-bit word where the
    // counts fit fields of these widths (measured per-(row, 36,000-SV tile)
    // maxima on 256 config-3 queries of 50..2,000 bp, l = 11, d = 3: 14, 59,
    // 451 and 3,196 per level; random matches grow 4x for each l below, so
    // d = 3 packs at l = 11..12 and d = 2 (8 / 10 / 14 bits) at l >= 8; a field
    // that overflows is carried exactly by the per-item check and the carry
    // log), else two 16-bit levels per word
    static const uint32_t pack4[4] = {4, 7, 9, 12}, pack3[3] = {8, 10, 14};
    const int packed = !spec->weighted && ((nlev == 4 && spec->l >= 11 && spec->l <= 12) ||
                                           (nlev == 3 && spec->l >= 8));
    int per_sv = spec->weighted ? 4 * nlev : packed ? 4 : 4 * ((nlev + 1) / 2);
    int max_tile = (acc_bytes / per_sv) & ~1;
    if (max_tile < 2) return gkm_fail(GKM_ERR_UNSUPPORTED, "%d mismatch levels do not fit shared memory", nlev);
    if (tile_svs <= 0) {
        int64_t T = (S + max_tile - 1) / max_tile;
        tile_svs = (int32_t)((S + T - 1) / T);
        tile_svs += tile_svs & 1;
    }
    if (tile_svs > max_tile || tile_svs > (1 << 24)) return gkm_fail(GKM_ERR_INVALID, "tile_svs %d too large", tile_svs);
    if (tile_svs & 1) tile_svs++;
    int64_t T = (S + tile_svs - 1) / tile_svs;
    int tile_bits = 0;
    while ((1LL << tile_bits) < T) tile_bits++;
    if (2 * spec->l + tile_bits > 32) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many SV tiles for l = %d", spec->l);
    int nb = (spec->include_rc && rc) ? 2 : 1;

    gkm_index *ix = new gkm_index();
    ix->spec = *spec;
    ix->S = S;
    ix->W = W;
    ix->tiles = (int32_t)T;
    ix->tile_svs = tile_svs;
    ix->nlev = nlev;
    ix->n_lmers = (int64_t)1 << (2 * spec->l);
    ix->n_masks = n_masks;
    ix->acc_bytes = acc_bytes;
    ix->wide = spec->weighted ? 1 : 0;
    ix->packed = packed;
    for (int m = 0; m < nlev && packed; m++) ix->pack_w[m] = nlev == 4 ? pack4[m] : pack3[m];
    ix->wmax = 1;
    if (spec->weighted) {
        // the largest window weight, from the device table (once per index)
        uint8_t *h = (uint8_t *)malloc(spec->wd_len > 0 ? spec->wd_len : 1);
        if (!h || cudaMemcpyAsync(h, spec->wd, spec->wd_len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            free(h);
            gkm_index_free(ix);
            return gkm_fail(GKM_ERR_CUDA, "window weight table");
        }
        ix->wmax = 0;
        for (int32_t k = 0; k < spec->wd_len; k++) ix->wmax = h[k] > ix->wmax ? h[k] : ix->wmax;
        free(h);
        if (ix->wmax == 0) ix->wmax = 1;
    }
    int status = GKM_OK;
    uint32_t *ecount = nullptr, *base = nullptr, *keys = nullptr, *vals = nullptr, *kt = nullptr, *vt = nullptr;
    uint32_t total = 0;
    int64_t nbuckets = T * ix->n_lmers;
    do {
        if (cudaMallocAsync(&ecount, sizeof(uint32_t) * (S + 1) * 2, st) != cudaSuccess) {
            status = gkm_fail(GKM_ERR_OOM, "index build scratch");
            break;
        }
        base = ecount + S + 1;
        entry_counts<<<(unsigned)((S + 255) / 256), 256, 0, st>>>(counts, S, nb, ecount);
        cudaMemsetAsync(ecount + S, 0, sizeof(uint32_t), st);
        if ((status = scan_exclusive(ecount, base, S + 1, st)) != GKM_OK) break;
        if (cudaMemcpyAsync(&total, base + S, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            status = gkm_cuda_status(cudaGetLastError(), "index size");
            break;
        }
        ix->entries = total;
        size_t eb = sizeof(uint32_t) * (total ? total : 1);
        if (cudaMallocAsync(&keys, eb, st) != cudaSuccess || cudaMallocAsync(&vals, eb, st) != cudaSuccess ||
            cudaMallocAsync(&kt, eb, st) != cudaSuccess || cudaMallocAsync(&vt, eb, st) != cudaSuccess) {
            status = gkm_fail(GKM_ERR_OOM, "index entries (%u)", total);
            break;
        }
        int64_t n = S * W;
        entry_gen<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*spec, fwd, rc, counts, base, S, W, tile_svs, keys, vals);
        GKM_CHECK_LAUNCH("entry_gen");
        if ((status = radix_sort(keys, vals, kt, vt, total, 2 * spec->l + tile_bits, st)) != GKM_OK) break;
        if (cudaMalloc(&ix->offsets, sizeof(uint32_t) * (nbuckets + 1)) != cudaSuccess) {
            status = gkm_fail(GKM_ERR_OOM, "index offsets");
            break;
        }
        bucket_offsets<<<(unsigned)((total + 1 + 255) / 256), 256, 0, st>>>(keys, total, nbuckets, ix->offsets);
        GKM_CHECK_LAUNCH("bucket_offsets");
        if (!spec->weighted) {
            // bucket words (unweighted queries): begins relative to their tile
            // take the bits the largest tile needs, the length the rest (<= 8)
            uint32_t *bounds = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(T + 1));
            if (!bounds || cudaMemcpy2DAsync(bounds, sizeof(uint32_t), ix->offsets, sizeof(uint32_t) * ix->n_lmers,
                                             sizeof(uint32_t), (size_t)(T + 1), cudaMemcpyDeviceToHost,
                                             st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                free(bounds);
                status = gkm_cuda_status(cudaGetLastError(), "index tile bounds");
                break;
            }
            uint32_t max_e = 0;
            for (int64_t t = 0; t < T; t++) max_e = bounds[t + 1] - bounds[t] > max_e ? bounds[t + 1] - bounds[t] : max_e;
            free(bounds);
            int bits = 0;
            while (bits < 32 && (max_e >> bits) != 0) bits++;
            ix->lb = 32 - bits < 8 ? 32 - bits : 8;
            if (ix->lb < 1) {
                status = gkm_fail(GKM_ERR_UNSUPPORTED, "an SV tile of %u index entries", max_e);
                break;
            }
            if (cudaMalloc(&ix->bwords, sizeof(uint32_t) * nbuckets) != cudaSuccess) {
                status = gkm_fail(GKM_ERR_OOM, "index bucket words");
                break;
            }
            bucket_words<<<(unsigned)((nbuckets + 255) / 256), 256, 0, st>>>(ix->offsets, nbuckets, ix->n_lmers,
                                                                             ix->lb, ix->bwords);
            GKM_CHECK_LAUNCH("bucket_words");
        }
        bool compact = !spec->weighted && tile_svs <= 65536;
        // queries read entries in aligned blocks of four: pad the arrays by a block
        size_t eb16 = sizeof(uint16_t) * ((size_t)total + 8);
        eb = sizeof(uint32_t) * ((size_t)total + 8);
        if ((compact ? cudaMalloc(&ix->ent16, eb16) : cudaMalloc(&ix->ent, eb)) != cudaSuccess ||
            cudaMalloc(&ix->masks, sizeof(uint32_t) * n_masks) != cudaSuccess ||
            cudaMalloc(&ix->status, 2 * sizeof(unsigned int)) != cudaSuccess ||
            cudaMalloc(&ix->queues, sizeof(unsigned int) * GKM_QUEUE_SLOTS) != cudaSuccess) {
            status = gkm_fail(GKM_ERR_OOM, "index entries");
            break;
        }
        if (compact) {
            cudaMemsetAsync(ix->ent16, 0, eb16, st);
            narrow_entries<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(vals, total, ix->ent16);
            GKM_CHECK_LAUNCH("narrow_entries");
            eb = eb16;
        } else {
            cudaMemsetAsync(ix->ent, 0, eb, st);
            cudaMemcpyAsync(ix->ent, vals, sizeof(uint32_t) * (size_t)total, cudaMemcpyDeviceToDevice, st);
        }
        cudaMemcpyAsync(ix->masks, masks, sizeof(uint32_t) * n_masks, cudaMemcpyDeviceToDevice, st);
        cudaMemsetAsync(ix->status, 0, 2 * sizeof(unsigned int), st);
        ix->bytes = (int64_t)sizeof(uint32_t) * ((ix->bwords ? 2 : 1) * nbuckets + 1) + (int64_t)eb +
                    sizeof(uint32_t) * n_masks;
    } while (0);
    cudaFreeAsync(ecount, st);
    cudaFreeAsync(keys, st);
    cudaFreeAsync(vals, st);
    cudaFreeAsync(kt, st);
    cudaFreeAsync(vt, st);
    if (status == GKM_OK) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) status = gkm_cuda_status(e, "index build");
    }
    if (status != GKM_OK) {
        gkm_index_free(ix);
        return status;
    }
    *out = ix;
    return GKM_OK;
}

extern "C" int gkm_index_free(gkm_index_t *ix)
{
    if (!ix) return GKM_OK;
    cudaFree(ix->offsets);
    cudaFree(ix->bwords);
    cudaFree(ix->ent);
    cudaFree(ix->ent16);
    cudaFree(ix->masks);
    cudaFree(ix->status);
    cudaFree(ix->queues);
    delete ix;
    return GKM_OK;
}

extern "C" int gkm_index_status(gkm_index_t *ix, uint32_t *counts, int32_t wide, gkm_stream_t stream)
{
    if (!ix) return gkm_fail(GKM_ERR_INVALID, "null index");
    if (counts) {
        cudaError_t e = cudaMemcpyAsync(counts, ix->status, 2 * sizeof(unsigned int), cudaMemcpyDefault,
                                        (cudaStream_t)stream);
        if (e != cudaSuccess) return gkm_cuda_status(e, "index status");
    }
    // weighted: 32-bit counters, or 64-bit (2); unweighted: narrow (0) or 32-bit
    if (wide >= 0) ix->wide = ix->spec.weighted ? (wide == 2 ? 2 : 1) : (wide ? 1 : 0);
    return GKM_OK;
}

extern "C" int gkm_index_info(const gkm_index_t *ix, int64_t *entries, int32_t *tiles, int32_t *tile_svs,
                              int64_t *device_bytes)
{
    if (!ix) return gkm_fail(GKM_ERR_INVALID, "null index");
    if (entries) *entries = ix->entries;
    if (tiles) *tiles = ix->tiles;
    if (tile_svs) *tile_svs = ix->tile_svs;
    if (device_bytes) *device_bytes = ix->bytes;
    return GKM_OK;
}

static QueryArgs query_args(const gkm_index_t *ix, const uint32_t *bx, const int32_t *cx, int64_t W)
{
    QueryArgs a = {};
    a.bx = bx;
    a.cx = cx;
    a.W = W;
    a.diag_offset = -1;
    a.nsplit = 1;
    a.split_w = (int)(W > 0x7FFFFFFF ? 0x7FFFFFFF : W);
    a.gcount = nullptr;
    a.off = ix->offsets;
    a.bw = ix->bwords;
    a.lb = ix->lb;
    a.ent = ix->ent16 ? (const void *)ix->ent16 : (const void *)ix->ent;
    a.masks = ix->masks;
    a.n_masks = ix->n_masks;
    a.n_lmers = ix->n_lmers;
    a.S = ix->S;
    a.tile_svs = ix->tile_svs;
    a.sub_svs = ix->acc_bytes / ((ix->wide == 2 ? 8 : 4) * ix->nlev);
    a.status = ix->status;
    a.nlev = ix->nlev;
    a.dmax = ix->spec.dmax;
    for (int m = 0; m < 16; m++) a.h[m] = ix->spec.h[m];
    a.wd = ix->spec.wd;
    a.l = ix->spec.l;
    a.wide_bound = (uint64_t)(ix->spec.include_rc ? 2 : 1) * (uint64_t)ix->W * ix->wmax * ix->wmax;
    a.nw.packed = ix->packed;
    if (ix->packed) {
        a.nw.nf = ix->nlev;
        uint32_t sh = 0;
        for (int g = 0; g < ix->nlev; g++) {
            a.nw.fsh |= sh << (5 * g);
            a.nw.fw |= (ix->pack_w[g] & 31u) << (5 * g);
            sh += ix->pack_w[g];
        }
    } else {
        a.nw.nf = 2;
        a.nw.fsh = 16u << 5;
        a.nw.fw = 16u | (16u << 5);
    }
    return a;
}

template <bool WEIGHTED, int MODE, bool C16, bool E16, bool C64 = false>
static void launch_query(unsigned grid, size_t smem, cudaStream_t st, const QueryArgs &a)
{
    // ids need a range test only for a self-Gram's diagonal or wide sub-ranges
    if (C16 && a.diag_offset < 0) {
        cudaFuncSetAttribute(index_query<WEIGHTED, MODE, C16, E16, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        index_query<WEIGHTED, MODE, C16, E16, false><<<grid, Q_THREADS, smem, st>>>(a);
    } else {
        cudaFuncSetAttribute(index_query<WEIGHTED, MODE, C16, E16, true, C64>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        index_query<WEIGHTED, MODE, C16, E16, true, C64><<<grid, Q_THREADS, smem, st>>>(a);
    }
}

template <int MODE>
static int query_launch(const gkm_index_t *ix, const QueryArgs &a, int64_t B, cudaStream_t st)
{
    if (B * ix->tiles * a.nsplit > 0xFFFFFFFFLL - 2LL * gkm_sm_count())
        return gkm_fail(GKM_ERR_UNSUPPORTED, "too many (row, tile) items for one launch");
    size_t smem = query_fixed_smem(ix->n_masks) + 16 + (size_t)ix->acc_bytes;
    // one resident block per SM, fed by the work queue (a counter of the
    // index's pool, one per call in flight)
    QueryArgs q = a;
    q.B = B;
    q.tiles = ix->tiles;
    unsigned slot = ix->next_queue.fetch_add(1) % GKM_QUEUE_SLOTS;
    q.queue = ix->queues + slot;
    cudaError_t e0 = cudaMemsetAsync(q.queue, 0, sizeof(unsigned int), st);
    if (e0 != cudaSuccess) return gkm_cuda_status(e0, "index queue");
    int64_t items = B * ix->tiles * a.nsplit;
    const int blocks = gkm_query_blocks();
    unsigned grid = (unsigned)(items < blocks ? items : blocks);
    if (ix->spec.weighted && ix->wide == 2)
        launch_query<true, MODE, false, false, true>(grid, smem, st, q);
    else if (ix->spec.weighted)
        launch_query<true, MODE, false, false>(grid, smem, st, q);
    else if (ix->ent16 && ix->wide)
        launch_query<false, MODE, false, true>(grid, smem, st, q);
    else if (ix->ent16)
        launch_query<false, MODE, true, true>(grid, smem, st, q);
    else if (ix->wide)
        launch_query<false, MODE, false, false>(grid, smem, st, q);
    else
        launch_query<false, MODE, true, false>(grid, smem, st, q);
    GKM_CHECK_LAUNCH("index_query");
    return GKM_OK;
}

// Row splits for small batches: when (rows x tiles) items cannot fill the GPU,
// each row's windows are cut into nsplit ranges of at least 32 windows, so
// items = rows x tiles x nsplit; the summed counts (B x S x levels x 8 B) are
// kept within 256 MB.  1: no split.
static int split_plan(const gkm_index_t *ix, int64_t B, int64_t W)
{
    // (measured on 1..64 rows of 300..2,000 bp, t=3 and t=5 on 72,000 SVs:
    // ranges of at least 64, 96 or 160 windows, or one item per block, were
    // as fast or slower)
    const int64_t items = B * ix->tiles, target = 2LL * gkm_query_blocks();
    if (items >= target || W < 64) return 1;
    if (B * ix->S * ix->nlev * 8 > (256LL << 20)) return 1;
    int64_t ns = (target + items - 1) / items;
    if (ns > W / 32) ns = W / 32;
    return ns < 2 ? 1 : (int)ns;
}

// K_raw / profiles / per-(row, tile) score partials from summed counts, each
// SV's levels in a fixed order (deterministic)
struct CountFinish {
    const unsigned long long *g;
    int64_t B, S;
    int nlev, l, tiles, tile_svs;
    int gpack;  // two levels per count (see QueryArgs::gpack)
    __device__ __forceinline__ uint64_t count(int64_t i, int m) const
    {
        if (!gpack) return g[i * nlev + m];
        return (g[i * ((nlev + 1) >> 1) + (m >> 1)] >> (32 * (m & 1))) & 0xFFFFFFFFull;
    }
    double h[16];
    double *raw;
    uint64_t *profile;
    const double *inv_dx, *inv_ds, *coef;
    double gamma;
    int rbf;
    double *partial;
};

__global__ void count_finish_raw(CountFinish f)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= f.B * f.S) return;
    double k = 0.0;
    for (int m = 0; m < f.nlev; m++) k += f.h[m] * (double)f.count(i, m);
    if (f.raw) f.raw[i] = k;
    if (f.profile)
        for (int m = 0; m <= f.l; m++) f.profile[i * (f.l + 1) + m] = m < f.nlev ? f.count(i, m) : 0;
}

__global__ void count_finish_score(CountFinish f)
{
    __shared__ double red[32];
    const int t = blockIdx.x;
    const int64_t row = blockIdx.y;
    const int64_t s0 = (int64_t)t * f.tile_svs, s1 = min(f.S, s0 + f.tile_svs);
    const double inv_dx = f.inv_dx[row];
    double part = 0.0;
    for (int64_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        double k = 0.0;
        for (int m = 0; m < f.nlev; m++) k += f.h[m] * (double)f.count(row * f.S + s, m);
        const double kn = k * inv_dx * f.inv_ds[s];
        part += f.coef[s] * (f.rbf ? exp(f.gamma * (kn - 1.0)) : kn);
    }
    part = gkm_block_sum(part, red);
    if (threadIdx.x == 0) f.partial[row * f.tiles + t] = part;
}

// split counts hold two levels per 64-bit word when no (row, SV, level) count
// can reach 2^32: rows of W windows x the SV rows' window slots (both strands)
// x the largest weight product
static int split_gpack(const gkm_index_t *ix, int64_t W)
{
    const uint64_t bound = (uint64_t)(ix->spec.include_rc ? 2 : 1) * (uint64_t)ix->W * ix->wmax * ix->wmax;
    return W > 0 && (uint64_t)W < (1ull << 32) / bound;
}

// the split query into freshly zeroed counts (caller frees *g)
static int query_split(const gkm_index_t *ix, QueryArgs a, int64_t B, int64_t W, int nsplit,
                       unsigned long long **g, cudaStream_t st)
{
    a.gpack = split_gpack(ix, W);
    const int gw = a.gpack ? (ix->nlev + 1) / 2 : ix->nlev;
    const size_t bytes = sizeof(unsigned long long) * (size_t)(B * ix->S * gw);
    if (cudaMallocAsync((void **)g, bytes, st) != cudaSuccess) return gkm_fail(GKM_ERR_OOM, "split counts");
    cudaError_t e = cudaMemsetAsync(*g, 0, bytes, st);
    if (e != cudaSuccess) return gkm_cuda_status(e, "split counts");
    a.nsplit = nsplit;
    a.split_w = (int)((W + nsplit - 1) / nsplit);
    a.gcount = *g;
    a.order = nullptr;
    return query_launch<MODE_COUNT>(ix, a, B, st);
}

static CountFinish count_finish_args(const gkm_index_t *ix, const unsigned long long *g, int64_t B, int64_t W)
{
    CountFinish f = {};
    f.g = g;
    f.B = B;
    f.gpack = split_gpack(ix, W);
    f.S = ix->S;
    f.nlev = ix->nlev;
    f.l = ix->spec.l;
    f.tiles = ix->tiles;
    f.tile_svs = ix->tile_svs;
    for (int m = 0; m < 16; m++) f.h[m] = ix->spec.h[m];
    return f;
}

extern "C" int gkm_index_pairwise(const gkm_index_t *ix, const uint32_t *bx, const int32_t *cx, int64_t B,
                                  int64_t W, int64_t diag_offset, double *raw, uint64_t *profile,
                                  gkm_stream_t stream)
{
    if (!ix || !bx || !cx) return gkm_fail(GKM_ERR_INVALID, "null index or rows");
    if (B == 0) return GKM_OK;
    QueryArgs a = query_args(ix, bx, cx, W);
    a.diag_offset = diag_offset;
    a.raw = raw;
    a.profile = profile;
    cudaStream_t st = (cudaStream_t)stream;
    const int nsplit = diag_offset < 0 ? split_plan(ix, B, W) : 1;
    if (nsplit == 1) return query_launch<MODE_RAW>(ix, a, B, st);
    unsigned long long *g = nullptr;
    int s = query_split(ix, a, B, W, nsplit, &g, st);
    if (s == GKM_OK) {
        CountFinish f = count_finish_args(ix, g, B, W);
        f.raw = raw;
        f.profile = profile;
        GKM_PREFER_SHARED(count_finish_raw);
        count_finish_raw<<<(unsigned)((B * ix->S + 255) / 256), 256, 0, st>>>(f);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "count_finish_raw");
    }
    if (g) cudaFreeAsync(g, st);
    return s;
}

extern "C" int gkm_index_score(const gkm_index_t *ix, const uint32_t *bx, const int32_t *cx, int64_t B,
                               int64_t W, const double *inv_dx, const double *inv_ds, const double *coef,
                               double gamma, int32_t rbf, double bias, const int32_t *order, double *scores,
                               gkm_stream_t stream)
{
    if (!ix || !bx || !cx || !inv_dx || !inv_ds || !coef || !scores)
        return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (B < 0 || W < 1) return gkm_fail(GKM_ERR_INVALID, "rows %lld, windows per row %lld", (long long)B, (long long)W);
    if (B == 0) return GKM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    double *partial = nullptr;
    if (cudaMallocAsync(&partial, sizeof(double) * B * ix->tiles, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "score partials");
    QueryArgs a = query_args(ix, bx, cx, W);
    a.order = order;
    a.inv_dx = inv_dx;
    a.inv_ds = inv_ds;
    a.coef = coef;
    a.gamma = gamma;
    a.rbf = rbf;
    a.partial = partial;
    const int nsplit = split_plan(ix, B, W);
    int s = GKM_OK;
    if (nsplit == 1) {
        s = query_launch<MODE_SCORE>(ix, a, B, st);
    } else {
        unsigned long long *g = nullptr;
        s = query_split(ix, a, B, W, nsplit, &g, st);
        if (s == GKM_OK) {
            CountFinish f = count_finish_args(ix, g, B, W);
            f.inv_dx = inv_dx;
            f.inv_ds = inv_ds;
            f.coef = coef;
            f.gamma = gamma;
            f.rbf = rbf;
            f.partial = partial;
            GKM_PREFER_SHARED(count_finish_score);
            count_finish_score<<<dim3((unsigned)ix->tiles, (unsigned)B), 256, 0, st>>>(f);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) s = gkm_cuda_status(e, "count_finish_score");
        }
        if (g) cudaFreeAsync(g, st);
    }
    if (s == GKM_OK) {
        GKM_PREFER_SHARED(finish_scores);
        finish_scores<<<(unsigned)((B + 255) / 256), 256, 0, st>>>(partial, B, ix->tiles, bias, scores);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "finish_scores");
    }
    cudaFreeAsync(partial, st);
    return s;
}

extern "C" int gkm_index_lmer_weights(const gkm_index_t *ix, const double *c_sv, double *V, gkm_stream_t stream)
{
    if (!ix || !c_sv || !V) return gkm_fail(GKM_ERR_INVALID, "null argument");
    int64_t n = ix->n_lmers;
    lmer_weights_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        ix->offsets, ix->ent, ix->ent16, n, ix->tiles, ix->tile_svs, ix->spec.weighted, c_sv, V);
    GKM_CHECK_LAUNCH("lmer_weights");
    return GKM_OK;
}

__global__ void index_count_kernel(const uint32_t *__restrict__ bx, const int32_t *__restrict__ cx, int64_t B,
                                   int64_t W, const uint32_t *__restrict__ off, const uint32_t *__restrict__ masks,
                                   int n_masks, int64_t n_lmers, int tiles, unsigned long long *__restrict__ out)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long hits = 0, looks = 0;
    if (idx < B * W) {
        int64_t b = idx / W;
        int i = (int)(idx - b * W);
        if (i < cx[b]) {
            uint32_t u = bx[idx];
            looks = n_masks;
            for (int c = 0; c < n_masks; c++) {
                uint32_t v = u ^ (__ldg(masks + c) & 0x00FFFFFFu);
                for (int t = 0; t < tiles; t++) hits += off[t * n_lmers + v + 1] - off[t * n_lmers + v];
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        hits += __shfl_xor_sync(GKM_FULL, hits, o);
        looks += __shfl_xor_sync(GKM_FULL, looks, o);
    }
    if ((threadIdx.x & 31) == 0 && (hits || looks)) {
        atomicAdd(out, looks);
        atomicAdd(out + 1, hits);
    }
}

extern "C" int gkm_index_count(const gkm_index_t *ix, const uint32_t *bx, const int32_t *cx, int64_t B, int64_t W,
                               uint64_t *out, gkm_stream_t stream)
{
    if (!ix || !bx || !cx || !out) return gkm_fail(GKM_ERR_INVALID, "null argument");
    int64_t n = B * W;
    if (n == 0) return GKM_OK;
    index_count_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        bx, cx, B, W, ix->offsets, ix->masks, ix->n_masks, ix->n_lmers, ix->tiles, (unsigned long long *)out);
    GKM_CHECK_LAUNCH("index_count");
    return GKM_OK;
}

// ---------------------------------------------------------------------------
// ISM through the index (kernels/lmer_index_cpu.py:203-285): K(mutant, s) =
// ref[b, s] + K(mutated windows, s) - K(reference windows, s), over the <= l
// windows covering the mutated base p (they keep their slot weights,
// ism.py:276-295).  Per chunk of positions, one query covers
//   * the three mutant window sets of each (p, b), one query row each (the
//     reference base's own set is the reference and its delta exactly 0), and
//   * every reference window the chunk's positions touch, once, as a row of
//     its own: a position's reference-window term is the sum of the rows of
//     the windows covering it (each window covers l positions, so querying it
//     once instead of once per covered position drops (l - 1) / l of that part).
// ---------------------------------------------------------------------------

// the base at p as packed in the first window covering it (-1: none covers p)
__device__ __forceinline__ int ism_ref_base(const uint32_t *fwd, int64_t b, int64_t W, int64_t p, int a_s, int a_e)
{
    return a_e > a_s ? (int)((fwd[b * W + a_s] >> (2 * (p - a_s))) & 3u) : -1;
}

// rows of one chunk: 3 mutant sets per (position, row), then per row the
// reference windows p0 - l + 1 .. p0 + np - 1; every query row has l slots
struct IsmChunk {
    int64_t np, B, nw0;  // positions, rows, reference windows per row (np + l - 1)
    __host__ __device__ int64_t mut_rows() const { return 3 * np * B; }
    __host__ __device__ int64_t rows() const { return mut_rows() + B * nw0; }
};

__global__ void ism_rows_kernel(gkm_spec spec, const uint32_t *__restrict__ fwd, const int32_t *__restrict__ cnt,
                                int64_t W, int64_t p0, IsmChunk ck, uint32_t *__restrict__ rows,
                                int32_t *__restrict__ rcount, uint8_t *__restrict__ rwt)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= ck.rows()) return;
    const int l = spec.l;
    uint32_t *row = rows + r * l;
    uint8_t *wt = rwt ? rwt + r * l : nullptr;
    for (int j = 0; j < l; j++) {
        row[j] = GKM_PAD;
        if (wt) wt[j] = 0;
    }
    if (r < ck.mut_rows()) {
        const int64_t item = r / 3, p = p0 + item / ck.B, b = item % ck.B;
        const int n = cnt[b];
        const int a_s = (int)(p - l + 1 > 0 ? p - l + 1 : 0), a_e = (int)(p + 1 < n ? p + 1 : n);
        const int na = a_e > a_s ? a_e - a_s : 0;
        const int xp = ism_ref_base(fwd, b, W, p, a_s, a_e);
        const int k = (int)(r - item * 3);       // the k-th base other than xp
        const int v = k + (k >= xp ? 1 : 0);
        rcount[r] = na;
        for (int j = 0; j < na; j++) {
            const int i = a_s + j;
            const uint32_t sh = 2u * (uint32_t)(p - i);
            row[j] = (fwd[b * W + i] & ~(3u << sh)) | ((uint32_t)v << sh);
            if (wt) wt[j] = (uint8_t)gkm_wt(spec.wd, n, i);
        }
    } else {
        const int64_t k = r - ck.mut_rows(), b = k / ck.nw0;
        const int64_t i = p0 - l + 1 + (k - b * ck.nw0);
        const bool in = i >= 0 && i < cnt[b];
        rcount[r] = in ? 1 : 0;
        if (in) {
            row[0] = fwd[b * W + i];
            if (wt) wt[0] = (uint8_t)gkm_wt(spec.wd, cnt[b], (int)i);
        }
    }
}

// one block per (position, row) of the chunk: the three mutants' scores minus
// the reference score; the reference base's own delta is exactly 0
__global__ void ism_index_finish(const double *__restrict__ kbuf, int64_t S, const uint32_t *__restrict__ fwd,
                                 const int32_t *__restrict__ cnt, int64_t W, int64_t L, int l, int64_t p0,
                                 IsmChunk ck, const double *__restrict__ ref, const double *__restrict__ ref_score,
                                 const double *__restrict__ inv_dmut, const double *__restrict__ inv_ds,
                                 const double *__restrict__ coef, double gamma, int rbf, double *__restrict__ out)
{
    __shared__ double red[32];
    const int64_t item = blockIdx.x, p = p0 + item / ck.B, b = item % ck.B;
    const int n = cnt[b];
    const int a_s = (int)(p - l + 1 > 0 ? p - l + 1 : 0), a_e = (int)(p + 1 < n ? p + 1 : n);
    const int xp = ism_ref_base(fwd, b, W, p, a_s, a_e);
    if (a_e <= a_s) {  // no window covers p
        if (threadIdx.x < 4) out[(b * 4 + threadIdx.x) * L + p] = 0.0;
        return;
    }
    // rows of the reference windows a_s .. a_e - 1 of row b
    const double *kw = kbuf + (ck.mut_rows() + b * ck.nw0 + (a_s - (p0 - l + 1))) * S;
    const double *km = kbuf + item * 3 * S;
    const double *rr = ref + b * S;
    double z[3];
    for (int k = 0; k < 3; k++) {
        const int v = k + (k >= xp ? 1 : 0);
        z[k] = inv_dmut[((int64_t)v * L + p) * ck.B + b];
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
        double k0 = 0.0;
        for (int j = 0; j < a_e - a_s; j++) k0 += kw[j * S + s];
        const double base = rr[s] - k0, ds = inv_ds[s], c = coef[s];
        for (int k = 0; k < 3; k++) {
            const double kn = (base + km[k * S + s]) * z[k] * ds;
            acc[k] += c * (rbf ? exp(gamma * (kn - 1.0)) : kn);
        }
    }
    for (int k = 0; k < 3; k++) {
        const double t = gkm_block_sum(acc[k], red);
        const int v = k + (k >= xp ? 1 : 0);
        if (threadIdx.x == 0) out[(b * 4 + v) * L + p] = t - ref_score[b];
    }
    if (threadIdx.x == 0) out[(b * 4 + xp) * L + p] = 0.0;
}

// Reference scores of the rows, sum_s coef_s f(ref[b, s] inv_dx[b] inv_ds[s]),
// with ism_index_finish's arithmetic and reduction order (256 threads, s
// strided), so that a mutant's delta is the difference of two sums taken alike
__global__ void ism_ref_score(const double *__restrict__ ref, int64_t S, const double *__restrict__ inv_dx,
                              const double *__restrict__ inv_ds, const double *__restrict__ coef, double gamma,
                              int rbf, double *__restrict__ out)
{
    __shared__ double red[32];
    const int64_t b = blockIdx.x;
    const double z = inv_dx[b];
    double acc = 0.0;
    for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
        const double kn = ref[b * S + s] * z * inv_ds[s];
        acc += coef[s] * (rbf ? exp(gamma * (kn - 1.0)) : kn);
    }
    acc = gkm_block_sum(acc, red);
    if (threadIdx.x == 0) out[b] = acc;
}

static size_t ism_align(size_t n) { return (n + 255) & ~(size_t)255; }

// workspace bytes of a chunk: the rows' reference scores, query rows (l
// slots), their counts and slot weights, and their K_raw rows
static size_t ism_chunk_bytes(const gkm_index_t *ix, const IsmChunk &ck)
{
    const size_t rows = (size_t)ck.rows(), l = (size_t)ix->spec.l;
    return ism_align((size_t)ck.B * 8) + ism_align(rows * l * 4) + ism_align(rows * 4) + ism_align(rows * l) +
           rows * (size_t)ix->S * 8;
}

extern "C" int gkm_index_mutants_workspace(const gkm_index_t *ix, int64_t B, int64_t L, int64_t *min_bytes,
                                           int64_t *all_bytes)
{
    if (!ix || B < 0 || L < 0) return gkm_fail(GKM_ERR_INVALID, "null index or negative size");
    const int64_t l = ix->spec.l;
    if (min_bytes) *min_bytes = (int64_t)ism_chunk_bytes(ix, IsmChunk{1, B, l});
    if (all_bytes) *all_bytes = (int64_t)ism_chunk_bytes(ix, IsmChunk{L, B, L + l - 1});
    return GKM_OK;
}

extern "C" int gkm_index_mutants(const gkm_index_t *ix, const uint32_t *fwd, const int32_t *counts, int64_t B,
                                 int64_t W, int64_t L, const double *ref_raw, const double *ref_score,
                                 const double *inv_dx, const double *inv_dmut, const double *inv_ds,
                                 const double *coef, double gamma, int32_t rbf, double *out, void *workspace,
                                 int64_t workspace_bytes, gkm_stream_t stream)
{
    if (!ix || !fwd || !counts || !ref_raw || !inv_dmut || !inv_ds || !coef || !out)
        return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (!ref_score && !inv_dx) return gkm_fail(GKM_ERR_INVALID, "reference scores need inv_dx");
    if (B < 0 || L < 0 || W < 0) return gkm_fail(GKM_ERR_INVALID, "negative size");
    if (B == 0 || L == 0) return GKM_OK;
    if (!workspace || ((uintptr_t)workspace & 255))
        return gkm_fail(GKM_ERR_INVALID, "ISM workspace must be non-null and 256-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    const int l = ix->spec.l;
    const int64_t S = ix->S;
    // the most positions per chunk the workspace holds
    int64_t np = 0;
    for (int64_t lo = 1, hi = L; lo <= hi;) {
        const int64_t mid = lo + (hi - lo) / 2;
        if ((int64_t)ism_chunk_bytes(ix, IsmChunk{mid, B, mid + l - 1}) <= workspace_bytes) {
            np = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (np == 0)
        return gkm_fail(GKM_ERR_CAPACITY, "ISM workspace of %lld bytes holds no position (needs %lld)",
                        (long long)workspace_bytes, (long long)ism_chunk_bytes(ix, IsmChunk{1, B, l}));
    double *rscore = (double *)workspace;  // the first bytes of the workspace
    if (ref_score) {
        cudaError_t e = cudaMemcpyAsync(rscore, ref_score, sizeof(double) * B, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return gkm_cuda_status(e, "ISM reference scores");
    } else {
        GKM_PREFER_SHARED(ism_ref_score);
        ism_ref_score<<<(unsigned)B, 256, 0, st>>>(ref_raw, S, inv_dx, inv_ds, coef, gamma, rbf, rscore);
        GKM_CHECK_LAUNCH("ism_ref_score");
    }
    for (int64_t p0 = 0; p0 < L; p0 += np) {
        const int64_t n_p = min(np, L - p0);
        const IsmChunk ck{n_p, B, n_p + l - 1};
        const int64_t rows = ck.rows();
        if (rows > 0x7FFFFFFFLL) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many ISM rows in one chunk");
        uint8_t *w = (uint8_t *)workspace + ism_align((size_t)B * 8);
        uint32_t *qrows = (uint32_t *)w;
        w += ism_align((size_t)rows * l * 4);
        int32_t *qcnt = (int32_t *)w;
        w += ism_align((size_t)rows * 4);
        uint8_t *qwt = w;
        w += ism_align((size_t)rows * l);
        double *kbuf = (double *)w;
        GKM_PREFER_SHARED(ism_rows_kernel);
        ism_rows_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(ix->spec, fwd, counts, W, p0, ck, qrows, qcnt,
                                                                        ix->spec.weighted ? qwt : nullptr);
        GKM_CHECK_LAUNCH("ism_rows");
        QueryArgs a = query_args(ix, qrows, qcnt, l);
        a.wq = ix->spec.weighted ? qwt : nullptr;
        a.raw = kbuf;
        // query rows with no window (positions past a row's end, rows of
        // length 0 padding a batch) are never read by ism_index_finish
        a.skip_empty = 1;
        GKM_TRY(query_launch<MODE_RAW>(ix, a, rows, st));
        GKM_PREFER_SHARED(ism_index_finish);
        ism_index_finish<<<(unsigned)(n_p * B), 256, 0, st>>>(kbuf, S, fwd, counts, W, L, l, p0, ck, ref_raw,
                                                             rscore, inv_dmut, inv_ds, coef, gamma, rbf, out);
        GKM_CHECK_LAUNCH("ism_index_finish");
    }
    return GKM_OK;
}


// ---------------------------------------------------------------------------
// gkm_index_score_noalloc: the same scores as gkm_index_score for callers that
// must not allocate device memory while they run -- an application that owns
// the whole device heap through its own pool, a real-time serving loop that
// may not block in the allocator, or code that calls in from a context where
// cudaMalloc is forbidden.  The per-(row, SV tile) partial sums that
// gkm_index_score allocates per call live instead in the fixed array below,
// which every device that loads this library holds until the process exits.
// ---------------------------------------------------------------------------

#include <mutex>

#define GKM_NOALLOC_MAX_PARTIALS (1 << 19)  // rows x SV tiles per call: 4 MiB of doubles
#define GKM_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_noalloc_partials[GKM_NOALLOC_MAX_PARTIALS];

// Device address of g_noalloc_partials on the current device.  In host code
// the array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device (with that device current), cached.
// The cache lives as long as the device's context: a process that calls
// cudaDeviceReset must not call gkm_index_score_noalloc on that device again
// (the cached address would belong to the destroyed context).
static int noalloc_partials(double **out)
{
    static std::mutex mu;
    static double *addr[GKM_NOALLOC_MAX_DEVICES] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gkm_cuda_status(e, "gkm_index_score_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= GKM_NOALLOC_MAX_DEVICES)
        return gkm_fail(GKM_ERR_UNSUPPORTED, "gkm_index_score_noalloc: device %d beyond %d", dev,
                        GKM_NOALLOC_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return gkm_cuda_status(e, "gkm_index_score_noalloc: cudaGetSymbolAddress");
        addr[dev] = (double *)p;
    }
    *out = addr[dev];
    return GKM_OK;
}

extern "C" int gkm_index_score_noalloc(const gkm_index_t *ix, const uint32_t *bx, const int32_t *cx, int64_t B,
                                       int64_t W, const double *inv_dx, const double *inv_ds, const double *coef,
                                       double gamma, int32_t rbf, double bias, const int32_t *order,
                                       double *scores, gkm_stream_t stream)
{
    if (!ix || !bx || !cx || !inv_dx || !inv_ds || !coef || !scores)
        return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (B < 0 || W < 1)
        return gkm_fail(GKM_ERR_INVALID, "gkm_index_score_noalloc: rows %lld, windows per row %lld", (long long)B,
                        (long long)W);
    if (B == 0) return GKM_OK;
    if (B * (int64_t)ix->tiles > GKM_NOALLOC_MAX_PARTIALS)
        return gkm_fail(GKM_ERR_CAPACITY,
                        "gkm_index_score_noalloc: %lld rows x %d SV tiles exceed its fixed scratch of %d "
                        "partial sums; score at most %lld rows per call",
                        (long long)B, ix->tiles, GKM_NOALLOC_MAX_PARTIALS,
                        (long long)(GKM_NOALLOC_MAX_PARTIALS / ix->tiles));
    double *partial = nullptr;
    GKM_TRY(noalloc_partials(&partial));
    cudaStream_t st = (cudaStream_t)stream;
    // Every (row, tile) partial is written before finish_scores reads it, so
    // nothing in the scratch has to start at zero.
    QueryArgs a = query_args(ix, bx, cx, W);
    a.order = order;
    a.inv_dx = inv_dx;
    a.inv_ds = inv_ds;
    a.coef = coef;
    a.gamma = gamma;
    a.rbf = rbf;
    a.partial = partial;
    GKM_TRY(query_launch<MODE_SCORE>(ix, a, B, st));
    finish_scores<<<(unsigned)((B + 255) / 256), 256, 0, st>>>(partial, B, ix->tiles, bias, scores);
    GKM_CHECK_LAUNCH("finish_scores");
    return GKM_OK;
}
