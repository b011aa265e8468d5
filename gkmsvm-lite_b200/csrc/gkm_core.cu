// gkm_core.cu -- packing, self-kernels, the ballot/popc pair join, the l-mer
// table, ISM's mutant self-kernels and the dense FP64 epilogues.
//
// Mismatch counts are accumulated as integers: per-lane 16-bit fields of a
// uint64 (four mismatch levels per word, gkm_shl64 drops levels past the
// word), flushed into uint64 totals before a field can overflow.  The FP64
// weighting sum_m h(m) n_m happens once per (row, column).
#include <cuda_runtime.h>
#include <stdint.h>

#include "gkm_common.cuh"

namespace {

constexpr int SELF_THREADS = 256;
constexpr int SMEM_WINDOWS = 12288;  // rows staged in shared memory up to this

// staged-window capacity of a launch over rows of W window slots: the
// shared memory is sized to the rows, not to the limit, so short rows leave
// room for more blocks per SM
static int staged_windows(int64_t W) { return (int)(W < 1 ? 1 : W < SMEM_WINDOWS ? W : SMEM_WINDOWS); }

// ---------------------------------------------------------------------------
// Packing (kernels/packed.py:130-187)
// ---------------------------------------------------------------------------

__global__ void pack_kernel(const uint8_t *__restrict__ codes, const int64_t *__restrict__ lengths,
                            int64_t B, int64_t L, int l, uint32_t *__restrict__ fwd,
                            uint32_t *__restrict__ rc, int32_t *__restrict__ counts)
{
    int64_t W = L - l + 1;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * W) return;
    int64_t b = idx / W, i = idx - b * W;
    int64_t n = W;
    if (lengths) {
        n = lengths[b] - l + 1;
        n = n < 0 ? 0 : (n > W ? W : n);
    }
    if (i == 0 && counts) counts[b] = (int32_t)n;
    uint32_t w = GKM_PAD;
    if (i < n) {
        const uint8_t *c = codes + b * L + i;
        w = 0;
        for (int k = 0; k < l; k++) w |= ((uint32_t)(c[k] & 3u)) << (2 * k);
    }
    fwd[idx] = w;
    if (rc) rc[b * W + (W - 1 - i)] = w == GKM_PAD ? GKM_PAD : gkm_rc_word(w, l);
}

// ---------------------------------------------------------------------------
// Pair counting
// ---------------------------------------------------------------------------

template <int NW>
struct Packed {
    uint64_t w[NW];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < NW; k++) w[k] = 0;
    }
    // add a (<= 16 bits) to level m's field; levels past 4*NW drop out
    __device__ __forceinline__ void add(uint32_t m, uint64_t a)
    {
#pragma unroll
        for (int k = 0; k < NW; k++) w[k] += gkm_shl64(a, 16u * (m - 4u * k));
    }
    // tot[m] += scale * field m
    __device__ __forceinline__ void flush(uint64_t *tot, uint64_t scale)
    {
#pragma unroll
        for (int k = 0; k < NW; k++) {
#pragma unroll
            for (int f = 0; f < 4; f++) tot[4 * k + f] += scale * ((w[k] >> (16 * f)) & 0xFFFFu);
            w[k] = 0;
        }
    }
};

// Row staged for the self-kernel: f[k] its forward windows, r[k] = rc(f[k]).
struct RowView {
    const uint32_t *f;   // forward windows (smem or global)
    const uint32_t *r;   // rc(f[k]) at k (smem), or the RC row read reversed
    int64_t W;           // row stride of the global RC row (reverse read)
    bool reversed;       // r is the global RC row: rc(f[k]) = r[W - 1 - k]
    __device__ __forceinline__ uint32_t rcf(int k) const { return reversed ? r[W - 1 - k] : r[k]; }
};

// Per-thread partial pair counts of one row against itself: forward x forward
// and forward x RC, each unordered pair once (j > i doubled, j == i once),
// kernels/direct.py:109-137.
template <int NW>
__device__ void self_pairs(const RowView rv, int n, bool has_rc, const uint8_t *wd, bool weighted,
                           uint64_t *tot)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    Packed<NW> acc;
    acc.zero();
    for (int i = warp; i < n; i += nw) {
        uint32_t fi = rv.f[i];
        uint64_t wi = weighted ? gkm_wt(wd, n, i) : 1;
        int it = 0;
        for (int j = i + 1 + lane; j < n; j += 32) {
            uint64_t wj = weighted ? gkm_wt(wd, n, j) : 1;
            acc.add((uint32_t)gkm_mism(fi, rv.f[j]), wj);
            if (has_rc) acc.add((uint32_t)gkm_mism(fi, rv.rcf(j)), wj);
            if (++it == 128) {  // 2 * 255 * 128 < 2^16
                acc.flush(tot, 2 * wi);
                it = 0;
            }
        }
        acc.flush(tot, 2 * wi);
        if (lane == 0) {
            tot[0] += wi * wi;  // m(f_i, f_i) = 0
            if (has_rc) {
                int m = gkm_mism(fi, rv.rcf(i));
                if (m < 4 * NW) tot[m] += wi * wi;
            }
        }
    }
}

// Block reduction of per-thread level totals; result in sums[] (smem, all threads).
template <int NL>
__device__ void block_reduce_levels(uint64_t *tot, uint64_t *red, uint64_t *sums)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int m = 0; m < NL; m++) {
        uint64_t v = tot[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GKM_FULL, v, o);
        if (lane == 0) red[warp * NL + m] = v;
    }
    __syncthreads();
    if (threadIdx.x < NL) {
        uint64_t s = 0;
        for (int w = 0; w < nw; w++) s += red[w * NL + threadIdx.x];
        sums[threadIdx.x] = s;
    }
    __syncthreads();
}

// sw: windows the shared memory holds per strand (2 * sw words)
__device__ __forceinline__ RowView stage_row(const uint32_t *fwd, const uint32_t *rc, int64_t W,
                                             int n, bool has_rc, uint32_t *sm, int sw)
{
    RowView rv;
    rv.W = W;
    if (n <= sw) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            sm[k] = fwd[k];
            if (has_rc) sm[sw + k] = rc[W - 1 - k];
        }
        rv.f = sm;
        rv.r = sm + sw;
        rv.reversed = false;
    } else {
        rv.f = fwd;
        rv.r = rc;
        rv.reversed = true;
    }
    __syncthreads();
    return rv;
}

// Self-kernel of one row per block, optionally fused with the l-mer table sum
// (svm.py:559-582: score = sum_i wt_i table[x_i] / sqrt(K(x, x)) + b).
template <int NW>
__global__ void __launch_bounds__(SELF_THREADS) self_kernel(
    gkm_spec spec, const uint32_t *__restrict__ fwd, const uint32_t *__restrict__ rc,
    const int32_t *__restrict__ counts, int64_t W, double *__restrict__ diag,
    uint64_t *__restrict__ profile, const double *__restrict__ table, double bias, int normalize,
    double *__restrict__ scores, double *__restrict__ raw_out, int sw)
{
    constexpr int NL = 4 * NW;
    extern __shared__ uint32_t sm[];
    __shared__ uint64_t red[(SELF_THREADS / 32) * NL];
    __shared__ uint64_t sums[NL];
    __shared__ double dred[32];
    int64_t b = blockIdx.x;
    int n = counts[b];
    bool has_rc = spec.include_rc && rc != nullptr;
    const uint32_t *frow = fwd + b * W;
    RowView rv = stage_row(frow, has_rc ? rc + b * W : nullptr, W, n, has_rc, sm, sw);
    uint64_t tot[NL];
#pragma unroll
    for (int m = 0; m < NL; m++) tot[m] = 0;
    self_pairs<NW>(rv, n, has_rc, spec.wd, spec.weighted, tot);
    block_reduce_levels<NL>(tot, red, sums);
    double k = 0.0;
#pragma unroll
    for (int m = 0; m < NL; m++)
        if (m <= spec.dmax) k += spec.h[m] * (double)sums[m];
    if (threadIdx.x == 0) {
        if (diag) diag[b] = k;
        if (profile)
            for (int m = 0; m <= spec.l; m++)
                profile[b * (spec.l + 1) + m] = (m < NL && m <= spec.dmax) ? sums[m] : 0;
    }
    if (table) {
        double t = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double a = spec.weighted ? (double)gkm_wt(spec.wd, n, i) : 1.0;
            t += a * table[rv.f[i]];
        }
        t = gkm_block_sum(t, dred);
        if (threadIdx.x == 0) {
            if (raw_out) raw_out[b] = t;
            double s = normalize ? t / sqrt(fmax(k, 1e-10)) : t;
            scores[b] = s + bias;
        }
    }
}

// ---------------------------------------------------------------------------
// Pair join by warp ballot/popc: K_raw[b, s] over every window pair
// ---------------------------------------------------------------------------

constexpr int JOIN_WARPS = 8;

template <int NW>
__global__ void __launch_bounds__(JOIN_WARPS * 32) join_kernel(
    gkm_spec spec, const uint32_t *__restrict__ bx, const int32_t *__restrict__ cx, int64_t Wx,
    const uint32_t *__restrict__ by, const uint32_t *__restrict__ ry, const int32_t *__restrict__ cy,
    int64_t S, int64_t Wy, double *__restrict__ raw, uint64_t *__restrict__ profile)
{
    constexpr int NL = 4 * NW;
    extern __shared__ uint32_t xs[];  // query row windows
    int64_t b = blockIdx.x;
    int nx = cx[b];
    for (int i = threadIdx.x; i < nx; i += blockDim.x) xs[i] = bx[b * Wx + i];
    __syncthreads();
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t s = (int64_t)blockIdx.y * JOIN_WARPS + warp;
    if (s >= S) return;
    int ny = cy[s];
    bool has_rc = spec.include_rc && ry != nullptr;
    int nt = has_rc ? 2 * ny : ny;
    const int dmax = spec.dmax;
    uint64_t tot[NL];
#pragma unroll
    for (int m = 0; m < NL; m++) tot[m] = 0;
    for (int c0 = 0; c0 < nt; c0 += 32) {
        int t = c0 + lane;
        uint32_t y = GKM_PAD;
        uint64_t wy = 1;
        if (t < nt) {
            if (t < ny) {
                y = by[s * Wy + t];
                if (spec.weighted) wy = gkm_wt(spec.wd, ny, t);
            } else {  // RC window of forward window ny - 1 - (t - ny)
                int f = ny - 1 - (t - ny);
                y = ry[s * Wy + (Wy - 1 - f)];
                if (spec.weighted) wy = gkm_wt(spec.wd, ny, f);
            }
        }
        Packed<NW> acc;
        acc.zero();
        int hits = 0;
        for (int i = 0; i < nx; i++) {
            int m = y == GKM_PAD ? 99 : gkm_mism(xs[i], y);
            if (__ballot_sync(GKM_FULL, m <= dmax)) {
                if (spec.weighted) {
                    if (m <= dmax) acc.add((uint32_t)m, gkm_wt(spec.wd, nx, i));
                    if (++hits == 256) {  // 255 * 256 < 2^16
                        acc.flush(tot, wy);
                        hits = 0;
                    }
                } else {
#pragma unroll
                    for (int lev = 0; lev < NL; lev++)
                        if (lev <= dmax) tot[lev] += __popc(__ballot_sync(GKM_FULL, m == lev));
                }
            }
        }
        if (spec.weighted) acc.flush(tot, wy);
    }
    if (spec.weighted) {
#pragma unroll
        for (int m = 0; m < NL; m++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tot[m] += __shfl_xor_sync(GKM_FULL, tot[m], o);
    }
    if (lane == 0) {
        double k = 0.0;
#pragma unroll
        for (int m = 0; m < NL; m++)
            if (m <= dmax) k += spec.h[m] * (double)tot[m];
        if (raw) raw[b * S + s] = k;
        if (profile)
            for (int m = 0; m <= spec.l; m++)
                profile[(b * S + s) * (spec.l + 1) + m] = (m < NL && m <= dmax) ? tot[m] : 0;
    }
}

// ---------------------------------------------------------------------------
// l-mer table (lmer_table.py:58-98): table[u] = sum_t h(level_t) V[u ^ mask_t]
// ---------------------------------------------------------------------------

__global__ void lmer_table_kernel(gkm_spec spec, const double *__restrict__ V,
                                  const uint32_t *__restrict__ masks, int n_masks,
                                  double *__restrict__ table, int64_t n_lmers)
{
    __shared__ double hs[16];
    if (threadIdx.x < 16) hs[threadIdx.x] = threadIdx.x <= spec.l ? spec.h[threadIdx.x] : 0.0;
    __syncthreads();
    int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_lmers) return;
    double acc = 0.0;
    for (int t = 0; t < n_masks; t++) {
        uint32_t mk = __ldg(masks + t);
        double v = __ldg(V + ((uint32_t)u ^ (mk & 0x00FFFFFFu)));
        acc += hs[mk >> 24] * v;
    }
    table[u] = acc;
}

// ---------------------------------------------------------------------------
// ISM: mutant self-kernels and table deltas (ism.py:118-144, 254-320;
// kernels/direct.py:160-201)
// ---------------------------------------------------------------------------

constexpr int MUT_THREADS = 128;

// Per (position p, row b): for each substituted base v the change in pair
// counts of the row's self-kernel, from the pairs touching the windows A that
// cover p.  Pairs (i in A, j not in A) stand for both orders (x2); pairs inside
// A are counted once per order.  The reference base gives new == old, so its
// change is exactly 0.
template <int NW>
__global__ void __launch_bounds__(MUT_THREADS) mutant_kernel(
    gkm_spec spec, const uint32_t *__restrict__ fwd, const int32_t *__restrict__ counts, int64_t B,
    int64_t W, int64_t L, const double *__restrict__ diag, double *__restrict__ mut_diag,
    const double *__restrict__ table, const double *__restrict__ ref_raw, int normalize,
    double *__restrict__ ism_out, int sw)
{
    constexpr int NL = 4 * NW;
    // the pair counts with base v at p, v = 0..3; the reference base's are
    // the row's own (its substitution changes nothing), so they serve as "old"
    constexpr int NA = 4;
    extern __shared__ uint32_t sm[];
    __shared__ uint64_t red[(MUT_THREADS / 32) * NA * NL];
    __shared__ uint64_t sums[NA * NL];
    int64_t p = blockIdx.x, b = blockIdx.y;
    int n = counts[b];
    int l = spec.l;
    int a_s = (int)(p - l + 1 > 0 ? p - l + 1 : 0);
    int a_e = (int)(p + 1 < n ? p + 1 : n);
    double d0 = diag ? diag[b] : 0.0;
    if (a_s >= a_e) {  // p past the row's windows: nothing changes
        if (threadIdx.x < 4) {
            if (mut_diag) mut_diag[(threadIdx.x * L + p) * B + b] = d0;
            if (ism_out) ism_out[(b * 4 + threadIdx.x) * L + p] = 0.0;
        }
        return;
    }
    bool has_rc = spec.include_rc != 0;
    const uint32_t *frow = fwd + b * W;
    uint32_t *f = sm;  // [n] forward, [n] rc(f)
    bool in_smem = n <= sw;
    if (in_smem) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            uint32_t w = frow[k];
            f[k] = w;
            f[sw + k] = gkm_rc_word(w, l);
        }
        __syncthreads();
    }
    const uint32_t *F = in_smem ? f : frow;
    const int na = a_e - a_s;
    const int xp = (int)((F[a_s] >> (2 * (p - a_s))) & 3u);  // the row's base at p
    const uint8_t *wd = spec.wd;
    const bool wt = spec.weighted != 0;
    uint64_t tot[NA][NL];
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
        for (int m = 0; m < NL; m++) tot[a][m] = 0;
    if (diag || mut_diag) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            uint32_t fj = F[j];
            uint32_t rj = in_smem ? f[sw + j] : gkm_rc_word(fj, l);
            bool jin = j >= a_s && j < a_e;
            uint64_t wj = wt ? gkm_wt(wd, n, j) : 1;
            Packed<NW> acc[NA];
#pragma unroll
            for (int a = 0; a < NA; a++) acc[a].zero();
            for (int ii = 0; ii < na; ii++) {
                int i = a_s + ii;
                uint32_t fi = F[i];
                uint64_t wi = wt ? gkm_wt(wd, n, i) : 1;
                uint32_t sh = 2u * (uint32_t)(p - i);
                if (!jin) {
                    // only window i changes: its mismatches with j away from
                    // offset k = p - i, plus one where j's base at k is not v
                    const uint32_t keep = ~(1u << sh);
                    uint32_t x = fi ^ fj;
                    const uint32_t mf = (uint32_t)__popc((x | (x >> 1)) & 0x55555555u & keep);
                    const uint32_t bf = (fj >> sh) & 3u;
                    x = fi ^ rj;
                    const uint32_t mr = (uint32_t)__popc((x | (x >> 1)) & 0x55555555u & keep);
                    const uint32_t br = (rj >> sh) & 3u;
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        acc[v].add(mf + (bf != (uint32_t)v), wi);
                        if (has_rc) acc[v].add(mr + (br != (uint32_t)v), wi);
                    }
                    continue;
                }
                uint32_t cleared = fi & ~(3u << sh);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    uint32_t fn = cleared | ((uint32_t)v << sh);
                    // both windows change
                    const uint32_t shj = 2u * (uint32_t)(p - j);
                    const uint32_t gj = (fj & ~(3u << shj)) | ((uint32_t)v << shj);
                    const uint32_t grj = gkm_rc_word(gj, l);
                    acc[v].add((uint32_t)gkm_mism(fn, gj), wi);
                    if (has_rc) acc[v].add((uint32_t)gkm_mism(fn, grj), wi);
                }
            }
            uint64_t scale = (jin ? 1 : 2) * wj;  // 2 * 11 * 255 < 2^16
#pragma unroll
            for (int a = 0; a < NA; a++) acc[a].flush(tot[a], scale);
        }
        // block reduction of the NA * NL totals
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int a = 0; a < NA; a++)
#pragma unroll
            for (int m = 0; m < NL; m++) {
                uint64_t v = tot[a][m];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GKM_FULL, v, o);
                if (lane == 0) red[(warp * NA + a) * NL + m] = v;
            }
        __syncthreads();
        for (int k = threadIdx.x; k < NA * NL; k += blockDim.x) {
            uint64_t s = 0;
            for (int w = 0; w < nw; w++) s += red[w * NA * NL + k];
            sums[k] = s;
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) {
        int v = threadIdx.x;
        double md = d0;
        if (diag || mut_diag) {
            double delta = 0.0;
            for (int m = 0; m < NL && m <= spec.dmax; m++) {
                int64_t dn = (int64_t)(sums[v * NL + m] - sums[xp * NL + m]);
                delta += spec.h[m] * (double)dn;
            }
            md = d0 + delta;
            if (mut_diag) mut_diag[((int64_t)v * L + p) * B + b] = md;
        }
        if (ism_out) {
            double r = ref_raw[b];
            double dt = 0.0;
            for (int i = a_s; i < a_e; i++) {
                uint32_t fi = F[i];
                uint32_t sh = 2u * (uint32_t)(p - i);
                uint32_t fn = (fi & ~(3u << sh)) | ((uint32_t)v << sh);
                double a = wt ? (double)gkm_wt(wd, n, i) : 1.0;
                dt += a * (table[fn] - table[fi]);
            }
            double kn = r + dt;
            double out;
            if (normalize)
                out = kn / sqrt(fmax(md, 1e-10)) - r / sqrt(fmax(d0, 1e-10));
            else
                out = kn - r;
            ism_out[(b * 4 + v) * L + p] = out;
        }
    }
}

// ---------------------------------------------------------------------------
// Dense FP64 epilogues over materialised [rows, S] blocks
// ---------------------------------------------------------------------------

__global__ void raw_score_kernel(const double *__restrict__ raw, int64_t S, const double *__restrict__ dx,
                                 const double *__restrict__ ds, const double *__restrict__ coef,
                                 double gamma, int rbf, double bias, double *__restrict__ out)
{
    __shared__ double red[32];
    int64_t b = blockIdx.x;
    double acc = 0.0;
    for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
        double k = raw[b * S + s];
        if (dx) k /= fmax(sqrt(dx[b] * ds[s]), 1e-10);
        if (rbf) k = exp(gamma * (k - 1.0));
        acc += coef[s] * k;
    }
    acc = gkm_block_sum(acc, red);
    if (threadIdx.x == 0) out[b] = acc + bias;
}

__global__ void impact_kernel(const double *__restrict__ raw, int64_t n, int64_t S,
                              const double *__restrict__ dr, const double *__restrict__ ds,
                              const double *__restrict__ coef, double gamma, int rbf,
                              double *__restrict__ out)
{
    __shared__ double red[32];
    int64_t b = blockIdx.x;
    double fl = rbf ? exp(-gamma) : 0.0;
    double acc = 0.0;
    for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
        double k = raw[b * S + s];
        double dk = raw[(n + b) * S + s] - k;
        if (dr) {
            double z = fmax(sqrt(dr[b] * ds[s]), 1e-10);
            k /= z;
            dk /= z;
        }
        if (rbf) {
            if (k <= 0) continue;
            dk *= (exp(gamma * (k - 1.0)) - fl) / k;
        }
        acc += coef[s] * dk;
    }
    acc = gkm_block_sum(acc, red);
    if (threadIdx.x == 0) out[b] = acc;
}

__global__ void gram_finish_kernel(const double *__restrict__ raw, int64_t N, int64_t M,
                                   const double *__restrict__ dx, const double *__restrict__ dy,
                                   double gamma, int rbf, int symmetric, double *__restrict__ out)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * M) return;
    int64_t r = idx / M, c = idx - r * M;
    int64_t rr = r, cc = c;
    if (symmetric && c < r) {  // mirror the upper triangle exactly
        rr = c;
        cc = r;
    }
    double k = raw[rr * M + cc];
    if (dx) k /= fmax(sqrt(dx[rr] * dy[cc]), 1e-10);
    if (rbf) k = exp(gamma * (k - 1.0));
    out[idx] = k;
}

int nw_for(int dmax)
{
    return dmax < 4 ? 1 : (dmax < 8 ? 2 : 4);
}

int check_spec(const gkm_spec *spec)
{
    if (!spec) return gkm_fail(GKM_ERR_INVALID, "spec is null");
    if (spec->l < 1 || spec->l > GKM_MAX_L) return gkm_fail(GKM_ERR_INVALID, "l must be in 1..15, got %d", spec->l);
    if (spec->dmax < 0 || spec->dmax > spec->l) return gkm_fail(GKM_ERR_INVALID, "dmax %d out of range", spec->dmax);
    if (spec->weighted && (!spec->wd || spec->wd_len < 1)) return gkm_fail(GKM_ERR_INVALID, "weighted spec without weights");
    return GKM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Entry points (C ABI)
// ---------------------------------------------------------------------------

extern "C" int gkm_pack(const gkm_spec *spec, const uint8_t *codes, const int64_t *lengths, int64_t B,
                        int64_t L, uint32_t *fwd, uint32_t *rc, int32_t *counts, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (L < spec->l) return gkm_fail(GKM_ERR_INVALID, "Sequence length %lld is shorter than window length %d", (long long)L, spec->l);
    if (!codes || !fwd) return gkm_fail(GKM_ERR_INVALID, "null codes or output");
    int64_t W = L - spec->l + 1;
    int64_t n = B * W;
    if (n == 0) return GKM_OK;
    GKM_PREFER_SHARED(pack_kernel);
    pack_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(codes, lengths, B, L, spec->l, fwd, rc, counts);
    GKM_CHECK_LAUNCH("pack");
    return GKM_OK;
}

static int self_launch(const gkm_spec *spec, const uint32_t *fwd, const uint32_t *rc, const int32_t *counts,
                       int64_t B, int64_t W, double *diag, uint64_t *profile, const double *table, double bias,
                       int normalize, double *scores, double *raw, cudaStream_t st)
{
    if (B == 0) return GKM_OK;
    const int sw = staged_windows(W);
    size_t smem = (size_t)2 * sw * sizeof(uint32_t);
    int nw = nw_for(spec->dmax);
#define GKM_SELF(NW)                                                                                  \
    do {                                                                                              \
        cudaFuncSetAttribute(self_kernel<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        GKM_PREFER_SHARED(self_kernel<NW>);                                                            \
        self_kernel<NW><<<(unsigned)B, SELF_THREADS, smem, st>>>(*spec, fwd, rc, counts, W, diag,      \
                                                                 profile, table, bias, normalize,     \
                                                                 scores, raw, sw);                    \
    } while (0)
    if (nw == 1) GKM_SELF(1);
    else if (nw == 2) GKM_SELF(2);
    else GKM_SELF(4);
#undef GKM_SELF
    GKM_CHECK_LAUNCH("self_kernel");
    return GKM_OK;
}

extern "C" int gkm_self_kernel(const gkm_spec *spec, const uint32_t *fwd, const uint32_t *rc,
                               const int32_t *counts, int64_t B, int64_t W, double *diag,
                               uint64_t *profile, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (!fwd || !counts) return gkm_fail(GKM_ERR_INVALID, "null windows or counts");
    return self_launch(spec, fwd, rc, counts, B, W, diag, profile, nullptr, 0.0, 0, nullptr, nullptr,
                       (cudaStream_t)stream);
}

extern "C" int gkm_table_score(const gkm_spec *spec, const double *table, const uint32_t *fwd,
                               const uint32_t *rc, const int32_t *counts, int64_t B, int64_t W, double bias,
                               int32_t normalize, double *scores, double *raw, double *diag,
                               gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (!table || !scores) return gkm_fail(GKM_ERR_INVALID, "null table or scores");
    return self_launch(spec, fwd, rc, counts, B, W, diag, nullptr, table, bias, normalize, scores, raw,
                       (cudaStream_t)stream);
}

extern "C" int gkm_join_pairwise(const gkm_spec *spec, const uint32_t *bx, const int32_t *cx, int64_t B,
                                 int64_t Wx, const uint32_t *by, const uint32_t *ry, const int32_t *cy,
                                 int64_t S, int64_t Wy, double *raw, uint64_t *profile, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (B == 0 || S == 0) return GKM_OK;
    if (Wx > 56000) return gkm_fail(GKM_ERR_UNSUPPORTED, "query rows longer than 56,000 windows");
    size_t smem = (size_t)Wx * sizeof(uint32_t);
    dim3 grid((unsigned)B, (unsigned)((S + JOIN_WARPS - 1) / JOIN_WARPS));
    if (grid.y > 65535) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many columns for one join launch");
    cudaStream_t st = (cudaStream_t)stream;
    int nw = nw_for(spec->dmax);
#define GKM_JOIN(NW)                                                                                   \
    do {                                                                                               \
        cudaFuncSetAttribute(join_kernel<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
        join_kernel<NW><<<grid, JOIN_WARPS * 32, smem, st>>>(*spec, bx, cx, Wx, by, ry, cy, S, Wy, raw, \
                                                             profile);                                 \
    } while (0)
    if (nw == 1) GKM_JOIN(1);
    else if (nw == 2) GKM_JOIN(2);
    else GKM_JOIN(4);
#undef GKM_JOIN
    GKM_CHECK_LAUNCH("join");
    return GKM_OK;
}

extern "C" int gkm_lmer_table(const gkm_spec *spec, const double *V, const uint32_t *masks, int32_t n_masks,
                              double *table, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (spec->l > 12) return gkm_fail(GKM_ERR_UNSUPPORTED, "l-mer tables need l <= 12");
    int64_t n = (int64_t)1 << (2 * spec->l);
    lmer_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*spec, V, masks, n_masks,
                                                                                   table, n);
    GKM_CHECK_LAUNCH("lmer_table");
    return GKM_OK;
}

// DeltaSVM weights read off the l-mer table (svm.py:667-704): out[idx], idx in
// DeltaSVM order (first base most significant), = table[idx with its digits
// reversed] times the lone window's weight, divided by sqrt(K(u, u)) of the
// l-mer alone when qnorm (h(0), plus h(m(u, rc u)) with RC, times the weight
// squared).
__global__ void deltasvm_table_kernel(gkm_spec sp, const double *__restrict__ table, double wt, int qnorm,
                                      double *__restrict__ out, int64_t n)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int l = sp.l;
    const uint32_t u = (uint32_t)idx;
    uint32_t packed = 0;
    for (int p = 0; p < l; p++) packed |= ((u >> (2 * (l - 1 - p))) & 3u) << (2 * p);
    double w = table[packed] * wt;
    if (qnorm) {
        double self_k = sp.h[0];
        if (sp.include_rc) self_k = self_k + sp.h[gkm_mism(packed, gkm_rc_word(packed, l))];
        self_k = self_k * (wt * wt);
        w = w / sqrt(fmax(self_k, 1e-10));
    }
    out[idx] = w;
}

extern "C" int gkm_deltasvm_table(const gkm_spec *spec, const double *table, double window_weight,
                                  int32_t query_norm, double *out, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (!table || !out) return gkm_fail(GKM_ERR_INVALID, "null table or out");
    if (spec->l > 12) return gkm_fail(GKM_ERR_UNSUPPORTED, "l-mer tables need l <= 12");
    int64_t n = (int64_t)1 << (2 * spec->l);
    deltasvm_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*spec, table, window_weight,
                                                                                        query_norm, out, n);
    GKM_CHECK_LAUNCH("deltasvm_table");
    return GKM_OK;
}

static int mutant_launch(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts, int64_t B,
                         int64_t W, int64_t L, const double *diag, double *mut_diag, const double *table,
                         const double *ref_raw, int normalize, double *out, cudaStream_t st)
{
    if (B == 0 || L == 0) return GKM_OK;
    if (B > 65535) return gkm_fail(GKM_ERR_UNSUPPORTED, "more than 65,535 rows per ISM launch");
    const int sw = staged_windows(W);
    size_t smem = (size_t)2 * sw * sizeof(uint32_t);
    dim3 grid((unsigned)L, (unsigned)B);
    int nw = nw_for(spec->dmax);
#define GKM_MUT(NW)                                                                                      \
    do {                                                                                                 \
        cudaFuncSetAttribute(mutant_kernel<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
        GKM_PREFER_SHARED(mutant_kernel<NW>);                                                            \
        mutant_kernel<NW><<<grid, MUT_THREADS, smem, st>>>(*spec, fwd, counts, B, W, L, diag, mut_diag,  \
                                                           table, ref_raw, normalize, out, sw);          \
    } while (0)
    if (nw == 1) GKM_MUT(1);
    else if (nw == 2) GKM_MUT(2);
    else GKM_MUT(4);
#undef GKM_MUT
    GKM_CHECK_LAUNCH("mutant");
    return GKM_OK;
}

extern "C" int gkm_mutant_diag(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts, int64_t B,
                               int64_t W, int64_t L, const double *diag, double *mut_diag, gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (!diag || !mut_diag) return gkm_fail(GKM_ERR_INVALID, "null diag or mut_diag");
    return mutant_launch(spec, fwd, counts, B, W, L, diag, mut_diag, nullptr, nullptr, 0, nullptr,
                         (cudaStream_t)stream);
}

extern "C" int gkm_ism_table(const gkm_spec *spec, const double *table, const uint32_t *fwd,
                             const int32_t *counts, int64_t B, int64_t W, int64_t L, const double *ref_raw,
                             const double *diag, double *mut_diag, int32_t normalize, double *out,
                             gkm_stream_t stream)
{
    GKM_TRY(check_spec(spec));
    if (!table || !ref_raw || !out) return gkm_fail(GKM_ERR_INVALID, "null table, ref_raw or out");
    if (normalize && !diag) return gkm_fail(GKM_ERR_INVALID, "normalize needs diag");
    return mutant_launch(spec, fwd, counts, B, W, L, normalize ? diag : nullptr, mut_diag, table, ref_raw,
                         normalize, out, (cudaStream_t)stream);
}

extern "C" int gkm_raw_score(const double *raw, int64_t B, int64_t S, const double *dx, const double *ds,
                             const double *coef, double gamma, int32_t rbf, double bias, double *scores,
                             gkm_stream_t stream)
{
    if (B == 0) return GKM_OK;
    GKM_PREFER_SHARED(raw_score_kernel);
    raw_score_kernel<<<(unsigned)B, 256, 0, (cudaStream_t)stream>>>(raw, S, dx, ds, coef, gamma, rbf, bias, scores);
    GKM_CHECK_LAUNCH("raw_score");
    return GKM_OK;
}

extern "C" int gkm_impact(const double *raw, int64_t n, int64_t S, const double *dr, const double *ds,
                          const double *coef, double gamma, int32_t rbf, double *out, gkm_stream_t stream)
{
    if (n == 0) return GKM_OK;
    GKM_PREFER_SHARED(impact_kernel);
    impact_kernel<<<(unsigned)n, 256, 0, (cudaStream_t)stream>>>(raw, n, S, dr, ds, coef, gamma, rbf, out);
    GKM_CHECK_LAUNCH("impact");
    return GKM_OK;
}

extern "C" int gkm_gram_finish(const double *raw, int64_t N, int64_t M, const double *dx, const double *dy,
                               double gamma, int32_t rbf, int32_t symmetric, double *out, gkm_stream_t stream)
{
    int64_t n = N * M;
    if (n == 0) return GKM_OK;
    if (symmetric && N != M) return gkm_fail(GKM_ERR_INVALID, "symmetric Gram must be square");
    gram_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(raw, N, M, dx, dy, gamma, rbf,
                                                                                     symmetric, out);
    GKM_CHECK_LAUNCH("gram_finish");
    return GKM_OK;
}
