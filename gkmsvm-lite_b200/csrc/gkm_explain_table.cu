// gkm_explain_table.cu -- the GkmExplain table of a linear model on the GPU
// (explain/table.py:14-169 of gkmsvm-lite).
//
// A query window u gets, at each position k and base u_k ^ d, the sum over
// l-mers v of V[v] t_d(m(u ^ v)) [(u ^ v)_k == d], where m counts the nonzero
// 2-bit digits and t_0 = table_a, t_1..3 = table_b.  Over all 4^l windows that
// is an XOR convolution, A[:, d, k] = H(H(V) H(G_kd)) / 4^l with the radix-4
// Walsh-Hadamard transform H (H H = 4^l I) and G_kd(z) = [z_k == d] t_d(m(z)).
// H(G_kd) is H(G_0d) with digits 0 and k swapped, so the table takes 5
// transforms of [4^l] vectors and one of the [4^l, 4l] table's rows.  Every
// transform pass is one kernel over the 4^l / 4 butterflies (x columns): HBM
// bandwidth bound, about 35 GB of traffic at l = 11 (the [4^11, 44] float64
// table is 1.5 GB).
//
// Lookups: each window's row A[u] ([4, l], times the window's weight, the
// perturbation deltas folded in) becomes its [4, l] part, and the parts of the
// windows covering each position are added in window order (explain_gather in
// gkm_explain.cu does the same for the per-window neighbour sums).
#include <cuda_runtime.h>
#include <stdint.h>

#include "gkm_common.cuh"

namespace {

constexpr int ET_LMAX = 12;

// one radix-4 pass with digit stride h over a [n, C] row-major array: each
// butterfly takes rows i, i + h, i + 2h, i + 3h of one column
__global__ void wht4_pass(double *__restrict__ a, int64_t n, int C, int64_t h)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (n / 4) * C) return;
    const int64_t j = t / C;
    const int c = (int)(t - j * C);
    const int64_t i = (j / h) * 4 * h + j % h;
    double *p0 = a + i * C + c, *p1 = p0 + h * C, *p2 = p1 + h * C, *p3 = p2 + h * C;
    const double a0 = *p0, a1 = *p1, a2 = *p2, a3 = *p3;
    const double s01 = a0 + a1, d01 = a0 - a1, s23 = a2 + a3, d23 = a2 - a3;
    *p0 = s01 + s23;
    *p1 = d01 + d23;
    *p2 = s01 - s23;
    *p3 = d01 - d23;
}

int wht4(double *a, int64_t n, int C, int l, cudaStream_t st)
{
    const int64_t work = (n / 4) * C;
    int64_t h = 1;
    for (int pass = 0; pass < l; pass++, h *= 4) {
        wht4_pass<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(a, n, C, h);
        GKM_CHECK_LAUNCH("wht4_pass");
    }
    return GKM_OK;
}

// G_d(z) = [z_0 == d] t_d(m(z)) for d = 0..3 ([4, n])
__global__ void explain_g_init(double *__restrict__ g, int64_t n, int l, const double *__restrict__ ta,
                               const double *__restrict__ tb)
{
    const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= n) return;
    int m = 0;
    for (int k = 0; k < l; k++) m += ((z >> (2 * k)) & 3) != 0;
    const int z0 = (int)(z & 3);
    for (int d = 0; d < 4; d++) g[d * n + z] = z0 == d ? (d == 0 ? ta[m] : tb[m]) : 0.0;
}

// A[z, d, k] = fv[z] / n * fg[d, z with digits 0 and k swapped]
__global__ void explain_fill_products(const double *__restrict__ fv, const double *__restrict__ fg, int64_t n, int l,
                                      double *__restrict__ A)
{
    const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= n) return;
    const int64_t z0 = z & 3;
    const double f = fv[z] / (double)n;
    double *row = A + z * 4 * l;
    for (int k = 0; k < l; k++) {
        const int64_t sk = 2 * k, zk = (z >> sk) & 3;
        const int64_t w = (z & ~((int64_t)3 << sk) & ~(int64_t)3) | (z0 << sk) | zk;
        for (int d = 0; d < 4; d++) row[d * l + k] = f * fg[d * n + w];
    }
}

// one window's part [4, l] from its table row: base u_k ^ d at position k gets
// A[u, d, k] (perturbation: the other three bases also get A[u, 0, k], the
// window's own base nothing), times the window weight
__global__ void explain_table_parts(const double *__restrict__ A, const uint32_t *__restrict__ fwd,
                                    const int32_t *__restrict__ cnt, int64_t B, int64_t W, int l, int weighted,
                                    const uint8_t *__restrict__ wd, int perturbation, double *__restrict__ part)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * W * 4 * l) return;
    const int k = (int)(t % l);
    const int base = (int)((t / l) % 4);
    const int64_t bw = t / (4 * l);
    const int64_t b = bw / W, i = bw - b * W;
    const int n = cnt[b];
    double v = 0.0;
    if (i < n) {
        const uint32_t u = fwd[b * W + i];
        const int uk = (int)((u >> (2 * k)) & 3u);
        const int d = base ^ uk;
        const double *row = A + (int64_t)u * 4 * l;
        if (perturbation)
            v = d == 0 ? 0.0 : row[d * l + k] + row[k];
        else
            v = row[d * l + k];
        if (weighted) v *= (double)gkm_wt(wd, n, (int)i);
    }
    part[t] = v;
}

// out[b, base, p] = inv_dx[b] * sum over windows i covering p of part[b, i, base, p - i]
__global__ void explain_table_gather(const double *__restrict__ part, const int32_t *__restrict__ cnt, int64_t B,
                                     int64_t W, int64_t L, int l, const double *__restrict__ inv_dx,
                                     double *__restrict__ out)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * 4 * L) return;
    const int64_t b = idx / (4 * L);
    const int64_t r = idx - b * 4 * L;
    const int base = (int)(r / L);
    const int64_t p = r - (int64_t)base * L;
    const int n = cnt[b];
    const int64_t i0 = p - l + 1 > 0 ? p - l + 1 : 0;
    const int64_t i1 = p < n - 1 ? p : n - 1;
    double s = 0.0;
    for (int64_t i = i0; i <= i1; i++) s += part[((b * W + i) * 4 + base) * l + (p - i)];
    out[idx] = s * inv_dx[b];
}

}  // namespace

extern "C" int gkm_explain_table_build(const gkm_spec *spec, const double *V, const double *table_a,
                                       const double *table_b, double *A, gkm_stream_t stream)
{
    if (!spec || !V || !table_a || !table_b || !A) return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (spec->l < 1 || spec->l > ET_LMAX)
        return gkm_fail(GKM_ERR_UNSUPPORTED, "explain tables need l <= %d", ET_LMAX);
    cudaStream_t st = (cudaStream_t)stream;
    const int l = spec->l;
    const int64_t n = (int64_t)1 << (2 * l);
    double *fv = nullptr, *fg = nullptr;
    if (cudaMallocAsync(&fv, sizeof(double) * n, st) != cudaSuccess ||
        cudaMallocAsync(&fg, sizeof(double) * 4 * n, st) != cudaSuccess) {
        if (fv) cudaFreeAsync(fv, st);
        return gkm_fail(GKM_ERR_OOM, "explain table transforms");
    }
    int s = GKM_OK;
    do {
        cudaError_t e = cudaMemcpyAsync(fv, V, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            s = gkm_cuda_status(e, "explain table V");
            break;
        }
        explain_g_init<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(fg, n, l, table_a, table_b);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            s = gkm_cuda_status(e, "explain_g_init");
            break;
        }
        if ((s = wht4(fv, n, 1, l, st)) != GKM_OK) break;
        for (int d = 0; d < 4 && s == GKM_OK; d++) s = wht4(fg + d * n, n, 1, l, st);
        if (s != GKM_OK) break;
        explain_fill_products<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(fv, fg, n, l, A);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            s = gkm_cuda_status(e, "explain_fill_products");
            break;
        }
        s = wht4(A, n, 4 * l, l, st);  // the 4l inverse transforms together, down A's rows
    } while (0);
    cudaFreeAsync(fv, st);
    cudaFreeAsync(fg, st);
    return s;
}

extern "C" int gkm_explain_table(const gkm_spec *spec, const double *A, const uint32_t *fwd, const int32_t *counts,
                                 int64_t B, int64_t W, int64_t L, const double *inv_dx, int32_t perturbation,
                                 double *out, gkm_stream_t stream)
{
    if (!spec || !A || !fwd || !counts || !inv_dx || !out) return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (spec->l < 1 || spec->l > ET_LMAX)
        return gkm_fail(GKM_ERR_UNSUPPORTED, "explain tables need l <= %d", ET_LMAX);
    if (spec->weighted && (!spec->wd || spec->wd_len < 1))
        return gkm_fail(GKM_ERR_INVALID, "weighted spec without weights");
    if (B == 0 || W == 0 || L == 0) return GKM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int l = spec->l;
    double *part = nullptr;
    if (cudaMallocAsync(&part, sizeof(double) * B * W * 4 * l, st) != cudaSuccess)
        return gkm_fail(GKM_ERR_OOM, "explain table parts");
    int s = GKM_OK;
    const int64_t np = B * W * 4 * l;
    explain_table_parts<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(A, fwd, counts, B, W, l, spec->weighted,
                                                                       spec->wd, perturbation, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = gkm_cuda_status(e, "explain_table_parts");
    if (s == GKM_OK) {
        const int64_t no = B * 4 * L;
        explain_table_gather<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(part, counts, B, W, L, l, inv_dx, out);
        if ((e = cudaGetLastError()) != cudaSuccess) s = gkm_cuda_status(e, "explain_table_gather");
    }
    cudaFreeAsync(part, st);
    return s;
}
