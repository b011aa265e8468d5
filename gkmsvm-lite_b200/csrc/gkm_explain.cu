// gkm_explain.cu -- GkmExplain through l-mer weights (explain/cpu.py:69-207,
// explain/lmer.py:31-188 of gkmsvm-lite).
//
// A warp owns one query window u; its lanes walk the neighbour masks.  For a
// neighbour v = u ^ mask with weight V(v) (the SVs' l-mer weights, or for RBF
// models the per-query SV weights summed over the index entries of v), each
// position k of the window gets table_a(m) V(v) when the mask leaves k alone
// (the SV base there is u_k) and table_b(m) V(v) on base u_k ^ d otherwise
// (d the mask's digit at k).  Lanes keep, per position, the "same" sum and the
// three "different" sums in registers; the warp reduces them and writes the
// window's [4, l] attribution, and a second pass adds the <= l windows that
// cover each position in a fixed order (deterministic, no atomics).
#include <cuda_runtime.h>
#include <stdint.h>

#include "gkm_common.cuh"

namespace {

constexpr int LMAX = 12;
constexpr int EX_WARPS = 4;

struct ExplainArgs {
    const uint32_t *fwd;
    const int32_t *cnt;
    int64_t W;
    int l;
    const double *V;      // [4^l] or null
    // index path
    const uint32_t *off;
    const uint32_t *ent;
    const uint16_t *ent16;
    int tiles;
    int tile_svs;
    int64_t n_lmers;
    int64_t S;
    const double *w;      // [B, S]
    int weighted;
    const uint8_t *wd;
    const uint32_t *masks;
    int n_masks;
    const double *ta;
    const double *tb;
    int perturbation;
    double *part;         // [B, W, 4, l]
};

__global__ void __launch_bounds__(EX_WARPS * 32) explain_windows(ExplainArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t win = (int64_t)blockIdx.x * EX_WARPS + (threadIdx.x >> 5);
    const int64_t b = blockIdx.y;
    if (win >= a.W) return;
    const int n = a.cnt[b];
    double *out = a.part + ((b * a.W + win) * 4) * a.l;
    if (win >= n) {  // PAD window: nothing
        if (lane < 4 * a.l) out[lane] = 0.0;
        if (lane + 32 < 4 * a.l) out[lane + 32] = 0.0;
        return;
    }
    const uint32_t u = a.fwd[b * a.W + win];
    const int l = a.l;
    double same[LMAX], d1[LMAX], d2[LMAX], d3[LMAX];
#pragma unroll
    for (int k = 0; k < LMAX; k++) same[k] = d1[k] = d2[k] = d3[k] = 0.0;
    const double *wrow = a.w ? a.w + b * a.S : nullptr;
    for (int c = lane; c < a.n_masks; c += 32) {
        const uint32_t mk = __ldg(a.masks + c);
        const uint32_t mask = mk & 0x00FFFFFFu;
        const uint32_t v = u ^ mask;
        double val;
        if (a.V) {
            val = __ldg(a.V + v);
        } else {
            val = 0.0;
            for (int t = 0; t < a.tiles; t++) {
                const uint32_t *o = a.off + (int64_t)t * a.n_lmers;
                const uint32_t e0 = __ldg(o + v), e1 = __ldg(o + v + 1);
                const double *wt = wrow + (int64_t)t * a.tile_svs;
                for (uint32_t e = e0; e < e1; e++) {
                    const uint32_t en = a.ent16 ? (uint32_t)__ldg(a.ent16 + e) | (1u << 24) : __ldg(a.ent + e);
                    double x = __ldg(wt + (en & 0x00FFFFFFu));
                    val += a.weighted ? x * (double)(en >> 24) : x;
                }
            }
        }
        if (val == 0.0) continue;
        const int lev = (int)(mk >> 24);
        const double av = val * __ldg(a.ta + lev), bv = val * __ldg(a.tb + lev);
#pragma unroll
        for (int k = 0; k < LMAX; k++) {
            const uint32_t d = (mask >> (2 * k)) & 3u;
            same[k] += d == 0 ? av : 0.0;
            d1[k] += d == 1 ? bv : 0.0;
            d2[k] += d == 2 ? bv : 0.0;
            d3[k] += d == 3 ? bv : 0.0;
        }
    }
#pragma unroll
    for (int k = 0; k < LMAX; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            same[k] += __shfl_xor_sync(GKM_FULL, same[k], o);
            d1[k] += __shfl_xor_sync(GKM_FULL, d1[k], o);
            d2[k] += __shfl_xor_sync(GKM_FULL, d2[k], o);
            d3[k] += __shfl_xor_sync(GKM_FULL, d3[k], o);
        }
    }
    const double wx = a.weighted ? (double)gkm_wt(a.wd, n, (int)win) : 1.0;
    // lane k < l writes position k: bases u_k ^ d
#pragma unroll
    for (int k = 0; k < LMAX; k++) {
        if (lane == k && k < l) {
            const uint32_t uk = (u >> (2 * k)) & 3u;
            double by[4];
            by[0] = a.perturbation ? 0.0 : same[k];
            by[1] = d1[k] + (a.perturbation ? same[k] : 0.0);
            by[2] = d2[k] + (a.perturbation ? same[k] : 0.0);
            by[3] = d3[k] + (a.perturbation ? same[k] : 0.0);
#pragma unroll
            for (int d = 0; d < 4; d++) out[(uk ^ d) * l + k] = wx * by[d];
        }
    }
}

// out[b, base, p] = inv_dx[b] * sum over windows i covering p of part[b, i, base, p - i]
__global__ void explain_gather(const double *__restrict__ part, const int32_t *__restrict__ cnt, int64_t B,
                               int64_t W, int64_t L, int l, const double *__restrict__ inv_dx,
                               double *__restrict__ out)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * 4 * L) return;
    int64_t b = idx / (4 * L);
    int64_t r = idx - b * 4 * L;
    int base = (int)(r / L);
    int64_t p = r - (int64_t)base * L;
    int n = cnt[b];
    int64_t i0 = p - l + 1 > 0 ? p - l + 1 : 0;
    int64_t i1 = p < n - 1 ? p : n - 1;
    double s = 0.0;
    for (int64_t i = i0; i <= i1; i++) s += part[((b * W + i) * 4 + base) * l + (p - i)];
    out[idx] = s * inv_dx[b];
}


// Per-SV GkmExplain (explain/cpu.py:14-66) for models the l-mer path does not
// take (l > 12): a block per query window i of row b; its warps sweep every
// SV window (forward, then RC, SV after SV), a lane per window, and take the
// pairs within the cutoff (ballot) one at a time in lane order; lane k adds
// the pair's contribution at position k to its four per-base registers.  The
// warps' [4, l] sums are added in warp order: deterministic.
constexpr int PX_WARPS = 8;

struct PairsArgs {
    const uint32_t *fwd;
    const int32_t *cnt;
    int64_t W;
    const uint32_t *by;
    const uint32_t *ry;
    const int32_t *cy;
    int64_t S;
    int64_t Wy;
    const double *w;  // [B, S] per-(row, SV) weight
    int l;
    int min_matches;
    int weighted;
    int include_rc;
    const uint8_t *wd;
    const double *ta;
    const double *tb;
    int perturbation;
    double *part;  // [B, W, 4, l]
};

__global__ void __launch_bounds__(PX_WARPS * 32) explain_pairs(PairsArgs a)
{
    __shared__ double red[PX_WARPS][4][16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t i = blockIdx.x, b = blockIdx.y;
    const int n = a.cnt[b];
    const int l = a.l;
    double *out = a.part + ((b * a.W + i) * 4) * l;
    if (i >= n) {  // past the row's windows: nothing
        for (int t = threadIdx.x; t < 4 * l; t += blockDim.x) out[t] = 0.0;
        return;
    }
    const uint32_t u = a.fwd[b * a.W + i];
    const double wx = a.weighted ? (double)gkm_wt(a.wd, n, (int)i) : 1.0;
    const int xk = lane < l ? (int)((u >> (2 * lane)) & 3u) : 0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const bool rc = a.include_rc && a.ry != nullptr;
    for (int64_t s = warp; s < a.S; s += PX_WARPS) {
        const double ws = a.w[b * a.S + s];
        const int ny = a.cy[s];
        const int nt = rc ? 2 * ny : ny;
        if (ws == 0.0) continue;
        for (int c0 = 0; c0 < nt; c0 += 32) {
            const int t = c0 + lane;
            uint32_t v = GKM_PAD;
            double wy = 1.0;
            if (t < nt) {
                if (t < ny) {
                    v = a.by[s * a.Wy + t];
                    if (a.weighted) wy = (double)gkm_wt(a.wd, ny, t);
                } else {  // RC of forward window ny - 1 - (t - ny)
                    const int f = ny - 1 - (t - ny);
                    v = a.ry[s * a.Wy + (a.Wy - 1 - f)];
                    if (a.weighted) wy = (double)gkm_wt(a.wd, ny, f);
                }
            }
            const int mm = v == GKM_PAD ? 99 : gkm_mism(u, v);
            unsigned hits = __ballot_sync(GKM_FULL, l - mm >= a.min_matches);
            while (hits) {
                const int h = __ffs(hits) - 1;
                hits &= hits - 1;
                const uint32_t vh = __shfl_sync(GKM_FULL, v, h);
                const int mh = __shfl_sync(GKM_FULL, mm, h);
                const double ew = ws * wx * __shfl_sync(GKM_FULL, wy, h);
                if (lane < l) {
                    const int yk = (int)((vh >> (2 * lane)) & 3u);
                    const double av = ew * a.ta[mh], bv = ew * a.tb[mh];
                    if (!a.perturbation) {
                        const double val = xk == yk ? av : bv;
#pragma unroll
                        for (int d = 0; d < 4; d++) acc[d] += d == yk ? val : 0.0;
                    } else if (xk == yk) {
#pragma unroll
                        for (int d = 0; d < 4; d++) acc[d] += d != yk ? av : 0.0;
                    } else {
#pragma unroll
                        for (int d = 0; d < 4; d++) acc[d] += d == yk ? bv : 0.0;
                    }
                }
            }
        }
    }
    if (lane < l)
        for (int d = 0; d < 4; d++) red[warp][d][lane] = acc[d];
    __syncthreads();
    for (int t = threadIdx.x; t < 4 * l; t += blockDim.x) {
        const int d = t / l, k = t - d * l;
        double sum = 0.0;
        for (int q = 0; q < PX_WARPS; q++) sum += red[q][d][k];
        out[d * l + k] = sum;  // base d at position i + k
    }
}

}  // namespace

extern "C" int gkm_explain_lmer(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts, int64_t B,
                                int64_t W, int64_t L, const double *inv_dx, const double *V,
                                const gkm_index_t *index, const double *w, const uint32_t *masks, int32_t n_masks,
                                const double *table_a, const double *table_b, int32_t perturbation, double *out,
                                gkm_stream_t stream)
{
    if (!spec || !fwd || !counts || !inv_dx || !masks || !table_a || !table_b || !out)
        return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (spec->l > LMAX) return gkm_fail(GKM_ERR_UNSUPPORTED, "GkmExplain l-mer path needs l <= %d", LMAX);
    if (!V && !(index && w)) return gkm_fail(GKM_ERR_INVALID, "need V, or an index and per-query weights");
    if (B == 0 || W == 0) return GKM_OK;
    if (B > 65535) return gkm_fail(GKM_ERR_UNSUPPORTED, "more than 65,535 rows per explain launch");
    cudaStream_t st = (cudaStream_t)stream;
    double *part = nullptr;
    if (cudaMallocAsync(&part, sizeof(double) * B * W * 4 * spec->l, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "explain scratch");
    ExplainArgs a = {};
    a.fwd = fwd;
    a.cnt = counts;
    a.W = W;
    a.l = spec->l;
    a.V = V;
    if (!V) {
        a.off = index->offsets;
        a.ent = index->ent;
        a.ent16 = index->ent16;
        a.tiles = index->tiles;
        a.tile_svs = index->tile_svs;
        a.n_lmers = index->n_lmers;
        a.S = index->S;
        a.w = w;
    }
    a.weighted = spec->weighted;
    a.wd = spec->wd;
    a.masks = masks;
    a.n_masks = n_masks;
    a.ta = table_a;
    a.tb = table_b;
    a.perturbation = perturbation;
    a.part = part;
    dim3 grid((unsigned)((W + EX_WARPS - 1) / EX_WARPS), (unsigned)B);
    explain_windows<<<grid, EX_WARPS * 32, 0, st>>>(a);
    int s = GKM_OK;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_windows");
    if (s == GKM_OK) {
        int64_t n = B * 4 * L;
        explain_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, counts, B, W, L, spec->l, inv_dx, out);
        e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_gather");
    }
    cudaFreeAsync(part, st);
    return s;
}

extern "C" int gkm_explain_pairs(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts, int64_t B,
                                 int64_t W, int64_t L, const double *inv_dx, const uint32_t *by, const uint32_t *ry,
                                 const int32_t *cy, int64_t S, int64_t Wy, const double *w, const double *table_a,
                                 const double *table_b, int32_t min_matches, int32_t perturbation, double *out,
                                 gkm_stream_t stream)
{
    if (!spec || !fwd || !counts || !inv_dx || !by || !cy || !w || !table_a || !table_b || !out)
        return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (spec->l < 1 || spec->l > 15) return gkm_fail(GKM_ERR_INVALID, "l must be in 1..15");
    if (spec->weighted && (!spec->wd || spec->wd_len < 1)) return gkm_fail(GKM_ERR_INVALID, "weighted spec without weights");
    if (B == 0 || W == 0 || L == 0) return GKM_OK;
    if (B > 65535 || W > 0x7FFFFFFFLL) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many rows or windows per launch");
    cudaStream_t st = (cudaStream_t)stream;
    double *part = nullptr;
    if (cudaMallocAsync(&part, sizeof(double) * B * W * 4 * spec->l, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "explain scratch");
    PairsArgs a = {};
    a.fwd = fwd;
    a.cnt = counts;
    a.W = W;
    a.by = by;
    a.ry = ry;
    a.cy = cy;
    a.S = S;
    a.Wy = Wy;
    a.w = w;
    a.l = spec->l;
    a.min_matches = min_matches;
    a.weighted = spec->weighted;
    a.include_rc = spec->include_rc;
    a.wd = spec->wd;
    a.ta = table_a;
    a.tb = table_b;
    a.perturbation = perturbation;
    a.part = part;
    explain_pairs<<<dim3((unsigned)W, (unsigned)B), PX_WARPS * 32, 0, st>>>(a);
    int s = GKM_OK;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_pairs");
    if (s == GKM_OK) {
        int64_t n = B * 4 * L;
        explain_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, counts, B, W, L, spec->l, inv_dx, out);
        e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_gather");
    }
    cudaFreeAsync(part, st);
    return s;
}
