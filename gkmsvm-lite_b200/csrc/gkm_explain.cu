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
// (nsplit > 1: part is [nsplit, B, W, 4, l], the splits added in order)
__global__ void explain_gather(const double *__restrict__ part, const int32_t *__restrict__ cnt, int64_t B,
                               int64_t W, int64_t L, int l, const double *__restrict__ inv_dx,
                               double *__restrict__ out, int nsplit = 1)
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
    const int64_t zs = B * W * 4 * l;
    for (int64_t i = i0; i <= i1; i++)
        for (int z = 0; z < nsplit; z++) s += part[z * zs + ((b * W + i) * 4 + base) * l + (p - i)];
    out[idx] = s * inv_dx[b];
}


// Per-SV GkmExplain (explain/cpu.py:14-66) for models the l-mer path does not
// take (l > 12, ...).  A block owns a tile of PX_QT query windows of row b and
// a range of SVs (split z of PX splits); its warps form PX_G groups that take
// the range's SVs in turn, and within a group each warp owns PX_QPW of the
// tile's windows.  A warp loads 32 SV windows (forward, then RC), one a lane,
// and tests each against its PX_QPW query windows (XOR + popcount + ballot):
// one load serves PX_QPW tests.  Pairs within the cutoff are rare and taken one
// at a time in lane order; lane k adds the pair's contribution at position k
// to the query's [4, l] sums in shared memory (each address has one writer in
// a group).  The groups' sums are added in group order and the splits in split
// order by the gather: deterministic for a given SV count.
constexpr int PX_QT = 32;
constexpr int PX_G = 2;
constexpr int PX_WARPS = 8;
constexpr int PX_QPW = PX_QT * PX_G / PX_WARPS;
constexpr int PX_LMAX = 16;
static_assert(PX_WARPS % PX_G == 0 && (PX_WARPS / PX_G) * PX_QPW == PX_QT, "tile split");

struct PairsArgs {
    const uint32_t *fwd;
    const int32_t *cnt;
    int64_t B;
    int64_t W;
    const uint32_t *by;
    const uint32_t *ry;
    const int32_t *cy;
    int64_t S;
    int64_t Wy;
    int nsplit;
    const double *w;  // [B, S] per-(row, SV) weight
    int l;
    int min_matches;
    int weighted;
    const uint8_t *wd;
    const double *ta;
    const double *tb;
    int perturbation;
    double *part;  // [nsplit, B, W, 4, l]
};

__global__ void __launch_bounds__(PX_WARPS * 32, 5) explain_pairs(PairsArgs a)
{
    __shared__ double acc[PX_G][PX_QT][4][PX_LMAX];
    __shared__ double wxs[PX_QT];
    __shared__ uint32_t us[PX_QT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t b = blockIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * PX_QT;
    const int n = a.cnt[b];
    if (i0 >= n) return;  // the gather reads windows < n only
    const int l = a.l;
    const int nq = (int)(n - i0 < PX_QT ? n - i0 : PX_QT);
    for (int t = threadIdx.x; t < PX_G * PX_QT * 4 * PX_LMAX; t += blockDim.x) (&acc[0][0][0][0])[t] = 0.0;
    for (int q = threadIdx.x; q < PX_QT; q += blockDim.x) {
        us[q] = q < nq ? a.fwd[b * a.W + i0 + q] : 0u;
        wxs[q] = q < nq && a.weighted ? (double)gkm_wt(a.wd, n, (int)(i0 + q)) : 1.0;
    }
    __syncthreads();
    const int g = warp / (PX_WARPS / PX_G);
    const int q0 = (warp % (PX_WARPS / PX_G)) * PX_QPW;
    const int mq = nq - q0 < PX_QPW ? (nq - q0 > 0 ? nq - q0 : 0) : PX_QPW;  // this warp's live windows
    uint32_t u[PX_QPW];
#pragma unroll
    for (int j = 0; j < PX_QPW; j++) u[j] = us[q0 + j];
    const int64_t z = blockIdx.z;
    const int64_t s0 = z * a.S / a.nsplit, s1 = (z + 1) * a.S / a.nsplit;
    const bool rc = a.ry != nullptr;
    const int dmax = l - a.min_matches;  // largest mismatch count of a contributing pair
    for (int64_t s = s0 + g; s < s1 && mq > 0; s += PX_G) {
        const double ws = a.w[b * a.S + s];
        if (ws == 0.0) continue;
        const int ny = a.cy[s];
        const int nt = rc ? 2 * ny : ny;
        const uint32_t *fy = a.by + s * a.Wy;
        const uint32_t *ry = rc ? a.ry + s * a.Wy + (a.Wy - ny) : nullptr;  // RC of forward ny-1-r at r
        for (int c0 = 0; c0 < nt; c0 += 32) {
            const int t = c0 + lane;
            const bool live = t < nt;
            const uint32_t v = !live ? 0u : (t < ny ? __ldg(fy + t) : __ldg(ry + (t - ny)));
            // the lane's hits over its warp's query windows, one bit each
            unsigned hm = 0;
#pragma unroll
            for (int j = 0; j < PX_QPW; j++) hm |= (unsigned)(j < mq && live && gkm_mism(u[j], v) <= dmax) << j;
            if (!__any_sync(GKM_FULL, hm)) continue;  // the common case
#pragma unroll
            for (int j = 0; j < PX_QPW; j++) {
                unsigned hits = __ballot_sync(GKM_FULL, (hm >> j) & 1u);
                while (hits) {
                    const int h = __ffs(hits) - 1;
                    hits &= hits - 1;
                    const uint32_t vh = __shfl_sync(GKM_FULL, v, h);
                    const int th = c0 + h;
                    const int mh = gkm_mism(u[j], vh);
                    // an RC window carries its forward window's weight
                    const double wy = a.weighted ? (double)gkm_wt(a.wd, ny, th < ny ? th : 2 * ny - 1 - th) : 1.0;
                    const double ew = ws * wxs[q0 + j] * wy;
                    if (lane < l) {
                        const int xk = (int)((u[j] >> (2 * lane)) & 3u);
                        const int yk = (int)((vh >> (2 * lane)) & 3u);
                        double *r = &acc[g][q0 + j][0][lane];
                        if (!a.perturbation) {
                            r[yk * PX_LMAX] += ew * (xk == yk ? a.ta[mh] : a.tb[mh]);
                        } else if (xk == yk) {
                            const double av = ew * a.ta[mh];
#pragma unroll
                            for (int d = 0; d < 4; d++)
                                if (d != yk) r[d * PX_LMAX] += av;
                        } else {
                            r[yk * PX_LMAX] += ew * a.tb[mh];
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    double *out = a.part + ((z * a.B + b) * a.W + i0) * 4 * l;
    for (int t = threadIdx.x; t < nq * 4 * l; t += blockDim.x) {
        const int q = t / (4 * l), r = t - q * 4 * l, d = r / l, k = r - d * l;
        double sum = 0.0;
#pragma unroll
        for (int gg = 0; gg < PX_G; gg++) sum += acc[gg][q][d][k];
        out[t] = sum;  // base d at position i0 + q + k
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
    GKM_PREFER_SHARED(explain_windows);
    explain_windows<<<grid, EX_WARPS * 32, 0, st>>>(a);
    int s = GKM_OK;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_windows");
    if (s == GKM_OK) {
        int64_t n = B * 4 * L;
        GKM_PREFER_SHARED(explain_gather);
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
    if (spec->include_rc && !ry) return gkm_fail(GKM_ERR_INVALID, "RC windows missing");
    if (B == 0 || W == 0 || L == 0) return GKM_OK;
    const int64_t tiles = (W + PX_QT - 1) / PX_QT;
    if (B > 65535 || tiles > 0x7FFFFFFFLL) return gkm_fail(GKM_ERR_UNSUPPORTED, "too many rows or windows per launch");
    // SV splits: a fixed function of S (the summation order then does not
    // depend on the batch), enough blocks for the GPU at small batches
    const int nsplit = (int)(S < 1 ? 1 : (S + 31) / 32 < 16 ? (S + 31) / 32 : 16);
    cudaStream_t st = (cudaStream_t)stream;
    double *part = nullptr;
    if (cudaMallocAsync(&part, sizeof(double) * nsplit * B * W * 4 * spec->l, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "explain scratch");
    PairsArgs a = {};
    a.fwd = fwd;
    a.cnt = counts;
    a.B = B;
    a.W = W;
    a.by = by;
    a.ry = spec->include_rc ? ry : nullptr;
    a.cy = cy;
    a.S = S;
    a.Wy = Wy;
    a.nsplit = nsplit;
    a.w = w;
    a.l = spec->l;
    a.min_matches = min_matches;
    a.weighted = spec->weighted;
    a.wd = spec->wd;
    a.ta = table_a;
    a.tb = table_b;
    a.perturbation = perturbation;
    a.part = part;
    int s = GKM_OK;
    if (S > 0) {
        explain_pairs<<<dim3((unsigned)tiles, (unsigned)B, (unsigned)nsplit), PX_WARPS * 32, 0, st>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_pairs");
    } else {
        cudaError_t e = cudaMemsetAsync(part, 0, sizeof(double) * B * W * 4 * spec->l, st);
        if (e != cudaSuccess) s = gkm_cuda_status(e, "explain scratch");
    }
    if (s == GKM_OK) {
        int64_t n = B * 4 * L;
        GKM_PREFER_SHARED(explain_gather);
        explain_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, counts, B, W, L, spec->l, inv_dx, out,
                                                                    nsplit);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_gather");
    }
    cudaFreeAsync(part, st);
    return s;
}
