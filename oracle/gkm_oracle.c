/*
 * gkm_oracle.c -- CPU restatement of gkmsvm-lite's pairwise gapped-k-mer kernel
 * path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the
 * bench's CPU-baseline leg call it as the checker; no product code links it.
 *
 * Every function states the reference code it restates (paths are relative to
 * the gkmsvm-lite source tree, src/gkmsvm/...).
 *
 * Conventions (kernels/packed.py:27-53, 130-187):
 *   - a window is l bases packed 2 bits each into a uint32, position k in bits
 *     2k..2k+1 (A=0 C=1 G=2 T=3);
 *   - PAD = 0xFFFFFFFF marks "no window" past a shorter row's last window (and
 *     sits first in a reverse-complement row);
 *   - the RC row is the forward row reversed, each window complemented and
 *     digit-reversed, PAD staying PAD.
 *
 * Profiles: n_m(x, y) = number of window pairs (weighted: sum of w_i w_j) with m
 * mismatches, m = 0..l.  The reference's raw kernel is sum_m h(m) n_m
 * (kernels/direct.py:23-42, kernels/weighted.py:47-69).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <pthread.h>

#define PAD 0xFFFFFFFFu

static inline int mism(uint32_t a, uint32_t b)
{
    /* kernels/primitives.py:_packed_mismatches */
    uint32_t x = a ^ b;
    return __builtin_popcount(((x >> 1) | x) & 0x55555555u);
}

static inline uint32_t rc_word(uint32_t w, int l)
{
    /* kernels/primitives.py:_rc_window */
    uint32_t out = 0;
    for (int k = 0; k < l; k++)
        out |= (3u - ((w >> (2 * k)) & 3u)) << (2 * (l - 1 - k));
    return out;
}

/* kernels/packed.py:130-187 (pack, pack_both, _rc_windows).  lengths may be
 * NULL (every row L long).  rc may be NULL. */
void orc_pack(const uint8_t *codes, const int64_t *lengths, int64_t B, int64_t L,
              int l, uint32_t *fwd, uint32_t *rc)
{
    int64_t W = L - l + 1;
    for (int64_t b = 0; b < B; b++) {
        int64_t n = W;
        if (lengths) {
            n = lengths[b] - l + 1;
            if (n < 0) n = 0;
            if (n > W) n = W;
        }
        const uint8_t *c = codes + b * L;
        for (int64_t i = 0; i < W; i++) {
            uint32_t w = 0;
            for (int k = 0; k < l; k++) w |= ((uint32_t)(c[i + k] & 3u)) << (2 * k);
            fwd[b * W + i] = i < n ? w : PAD;
        }
        if (rc) {
            for (int64_t j = 0; j < W; j++) {
                uint32_t w = fwd[b * W + (W - 1 - j)];
                rc[b * W + j] = w == PAD ? PAD : rc_word(w, l);
            }
        }
    }
}

/* Per-pair mismatch profiles between rows bx [B, Wx] and rows by [S, Wy]
 * (kernels/direct.py:23-42 counted per level instead of summed through h;
 * weighted form kernels/weighted.py:47-69).  wx [B, Wx] / wy [S, Wy] uint8
 * window weights or NULL (all 1).  out [B, S, l+1] uint64.  PAD skipped. */
void orc_profiles(const uint32_t *bx, const uint8_t *wx, int64_t B, int64_t Wx,
                  const uint32_t *by, const uint8_t *wy, int64_t S, int64_t Wy,
                  int l, uint64_t *out)
{
    int nl = l + 1;
    for (int64_t b = 0; b < B; b++) {
        for (int64_t s = 0; s < S; s++) {
            uint64_t *o = out + (b * S + s) * nl;
            memset(o, 0, sizeof(uint64_t) * nl);
            for (int64_t i = 0; i < Wx; i++) {
                uint32_t u = bx[b * Wx + i];
                if (u == PAD) continue;
                uint64_t a = wx ? wx[b * Wx + i] : 1;
                for (int64_t j = 0; j < Wy; j++) {
                    uint32_t v = by[s * Wy + j];
                    if (v == PAD) continue;
                    uint64_t c = wy ? wy[s * Wy + j] : 1;
                    o[mism(u, v)] += a * c;
                }
            }
        }
    }
}

/* Self-kernel profiles K(x, x): each row's forward windows against its forward
 * windows and (rc != NULL) its RC windows, every pair visited
 * (kernels/direct.py:109-137 and kernels/weighted.py:91-118 visit each
 * unordered pair once; the counts are the same).  w [B, W] forward weights or
 * NULL; an RC window carries the weight of the forward window it came from
 * (kernels/packed.py:105-122, rc=True reverses the row).  out [B, l+1]. */
void orc_self_profiles(const uint32_t *fwd, const uint32_t *rc, const uint8_t *w,
                       int64_t B, int64_t W, int l, uint64_t *out)
{
    int nl = l + 1;
    for (int64_t b = 0; b < B; b++) {
        uint64_t *o = out + b * nl;
        memset(o, 0, sizeof(uint64_t) * nl);
        const uint32_t *f = fwd + b * W;
        for (int64_t i = 0; i < W; i++) {
            if (f[i] == PAD) continue;
            uint64_t a = w ? w[b * W + i] : 1;
            for (int64_t j = 0; j < W; j++) {
                if (f[j] != PAD) o[mism(f[i], f[j])] += a * (w ? w[b * W + j] : 1);
                if (rc) {
                    uint32_t r = rc[b * W + j];
                    if (r == PAD) continue;
                    /* rc position j holds rc(f[W-1-j]) with that window's weight */
                    uint64_t c = w ? w[b * W + (W - 1 - j)] : 1;
                    o[mism(f[i], r)] += a * c;
                }
            }
        }
    }
}

typedef struct {
    const uint32_t *fwd, *rc;
    const uint8_t *w;
    int64_t B, W;
    int l;
    uint64_t *out;
    int64_t *next_row;
} self_job;

static void *self_worker(void *arg)
{
    self_job *j = (self_job *)arg;
    for (;;) {
        int64_t b = __atomic_fetch_add(j->next_row, 1, __ATOMIC_RELAXED);
        if (b >= j->B) break;
        orc_self_profiles(j->fwd + b * j->W, j->rc ? j->rc + b * j->W : NULL, j->w ? j->w + b * j->W : NULL, 1,
                          j->W, j->l, j->out + b * (j->l + 1));
    }
    return NULL;
}

/* orc_self_profiles over nthreads threads, rows handed out one at a time. */
void orc_self_profiles_mt(const uint32_t *fwd, const uint32_t *rc, const uint8_t *w,
                          int64_t B, int64_t W, int l, uint64_t *out, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    int64_t next_row = 0;
    self_job j = {fwd, rc, w, B, W, l, out, &next_row};
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, self_worker, &j);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
}

/* ------------------------------------------------------------------------ */
/* l-mer index and fused query + reduce: the reference CPU path that the bench
 * times as its baseline (kernels/lmer_index.py:161-200 build;
 * kernels/lmer_index_cpu.py:11-19 _counting_sort, :23-37 _add_window,
 * :71-120 _query_reduce_cpu).  Threads: pthreads taking rows one at a time
 * from a shared counter (as a parallel loop with dynamic scheduling would),
 * one length-S accumulator per thread, zeroed as it is reduced. */

typedef struct {
    int l;
    int64_t n_lmers;
    int64_t *offsets; /* [n_lmers + 1] */
    int32_t *ids;     /* SV id per entry, ascending within a bucket */
    uint8_t *vals;    /* entry window weight, or NULL */
    int64_t S;
} orc_index;

/* Build the CSR over the SVs' forward then RC windows (columns in order, so the
 * counting sort leaves every bucket ascending by SV).  wf/wr: [S, W] weights
 * of the forward / RC rows, or NULL. */
void *orc_index_build(const uint32_t *fwd, const uint32_t *rc, const uint8_t *wf,
                      const uint8_t *wr, int64_t S, int64_t W, int l)
{
    orc_index *ix = (orc_index *)calloc(1, sizeof(orc_index));
    ix->l = l;
    ix->S = S;
    ix->n_lmers = (int64_t)1 << (2 * l);
    int64_t n = ix->n_lmers;
    ix->offsets = (int64_t *)calloc(n + 1, sizeof(int64_t));
    int nblk = rc ? 2 : 1;
    for (int64_t s = 0; s < S; s++)
        for (int k = 0; k < nblk; k++) {
            const uint32_t *row = (k ? rc : fwd) + s * W;
            for (int64_t j = 0; j < W; j++)
                if ((int64_t)row[j] < n) ix->offsets[row[j] + 1]++;
        }
    for (int64_t v = 0; v < n; v++) ix->offsets[v + 1] += ix->offsets[v];
    int64_t total = ix->offsets[n];
    ix->ids = (int32_t *)malloc(sizeof(int32_t) * (total ? total : 1));
    ix->vals = (wf ? (uint8_t *)malloc(total ? total : 1) : NULL);
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * n);
    memcpy(fill, ix->offsets, sizeof(int64_t) * n);
    for (int64_t s = 0; s < S; s++)
        for (int k = 0; k < nblk; k++) {
            const uint32_t *row = (k ? rc : fwd) + s * W;
            const uint8_t *wrow = wf ? ((k ? wr : wf) + s * W) : NULL;
            for (int64_t j = 0; j < W; j++) {
                uint32_t v = row[j];
                if ((int64_t)v >= n) continue;
                int64_t e = fill[v]++;
                ix->ids[e] = (int32_t)s;
                if (ix->vals) ix->vals[e] = wrow[j];
            }
        }
    free(fill);
    return ix;
}

void orc_index_free(void *p)
{
    orc_index *ix = (orc_index *)p;
    if (!ix) return;
    free(ix->offsets);
    free(ix->ids);
    free(ix->vals);
    free(ix);
}

int64_t orc_index_entries(void *p) { return ((orc_index *)p)->offsets[((orc_index *)p)->n_lmers]; }

static inline void add_window(const orc_index *ix, double *acc, uint32_t w, double scale,
                              const uint32_t *masks, const double *weights, int nm,
                              int64_t lo)
{
    if ((int64_t)w >= ix->n_lmers) return; /* PAD */
    for (int t = 0; t < nm; t++) {
        int64_t v = (int64_t)(w ^ masks[t]);
        double wt = scale * weights[t];
        for (int64_t e = ix->offsets[v + 1] - 1; e >= ix->offsets[v]; e--) {
            int64_t s = ix->ids[e];
            if (s < lo) break;
            acc[s] += ix->vals ? wt * ix->vals[e] : wt;
        }
    }
}

typedef struct {
    const orc_index *ix;
    const uint32_t *bx;
    int64_t B, W;
    const uint8_t *wx; /* [B, W] query weights or NULL */
    const uint32_t *masks;
    const double *weights;
    int nm;
    const double *inv_dx, *inv_ds, *coef;
    double gamma;
    int rbf;
    double *out;
    int64_t *next_row; /* shared: rows are handed out one at a time */
} reduce_job;

static void *reduce_worker(void *arg)
{
    reduce_job *j = (reduce_job *)arg;
    int64_t S = j->ix->S;
    double *acc = (double *)calloc(S ? S : 1, sizeof(double));
    double floor_ = j->rbf ? exp(-j->gamma) : 1.0;
    for (;;) {
        int64_t b = __atomic_fetch_add(j->next_row, 1, __ATOMIC_RELAXED);
        if (b >= j->B) break;
        for (int64_t i = 0; i < j->W; i++) {
            double a = j->wx ? (double)j->wx[b * j->W + i] : 1.0;
            add_window(j->ix, acc, j->bx[b * j->W + i], a, j->masks, j->weights, j->nm, 0);
        }
        double scale = j->inv_dx[b], total = 0.0;
        if (j->rbf) {
            double g = j->gamma * scale;
            for (int64_t s = 0; s < S; s++) {
                total += j->coef[s] * exp(g * acc[s] * j->inv_ds[s]);
                acc[s] = 0.0;
            }
            total *= floor_;
        } else {
            for (int64_t s = 0; s < S; s++) {
                total += j->coef[s] * acc[s] * j->inv_ds[s];
                acc[s] = 0.0;
            }
            total *= scale;
        }
        j->out[b] = total;
    }
    free(acc);
    return NULL;
}

/* sum_s coef_s f(K_raw[b, s] inv_dx[b] inv_ds[s]) [B] (f = exp(gamma (k - 1))
 * when rbf, else identity), as kernels/lmer_index_cpu.py:71-120. */
void orc_index_reduce(void *p, const uint32_t *bx, const uint8_t *wx, int64_t B,
                      int64_t W, const uint32_t *masks, const double *weights, int nm,
                      const double *inv_dx, const double *inv_ds, const double *coef,
                      double gamma, int rbf, double *out, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    int64_t next_row = 0;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    reduce_job j = {(orc_index *)p, bx, B, W, wx, masks, weights, nm,
                    inv_dx, inv_ds, coef, gamma, rbf, out, &next_row};
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, reduce_worker, &j);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
}

/* K_raw [B, S] through the index (kernels/lmer_index_cpu.py:41-67), one row at
 * a time; diag_offset >= 0 leaves columns below diag_offset + b at 0. */
void orc_index_pairwise(void *p, const uint32_t *bx, const uint8_t *wx, int64_t B,
                        int64_t W, const uint32_t *masks, const double *weights, int nm,
                        int64_t diag_offset, double *raw)
{
    orc_index *ix = (orc_index *)p;
    for (int64_t b = 0; b < B; b++) {
        double *acc = raw + b * ix->S;
        memset(acc, 0, sizeof(double) * ix->S);
        int64_t lo = diag_offset >= 0 ? diag_offset + b : 0;
        for (int64_t i = 0; i < W; i++) {
            double a = wx ? (double)wx[b * W + i] : 1.0;
            add_window(ix, acc, bx[b * W + i], a, masks, weights, nm, lo);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* GkmExplain per-SV pair loop (explain/cpu.py:14-66): [B, 4, seqlen]
 * attributions of packed_x [B, W] against packed_y [S, Wy] (forward then RC
 * windows), eff_coef [B, S], tables a/b indexed by mismatch count, weights
 * wx [B, W] / wy [S, Wy] (NULL: all 1). */
void orc_explain_pairs(const uint32_t *px, int64_t B, int64_t W, const uint32_t *py,
                       int64_t S, int64_t Wy, const double *ta, const double *tb,
                       const double *eff, int l, int min_matches, int64_t seqlen,
                       int perturbation, const uint8_t *wx, const uint8_t *wy,
                       double *out)
{
    memset(out, 0, sizeof(double) * B * 4 * seqlen);
    for (int64_t b = 0; b < B; b++) {
        double *res = out + b * 4 * seqlen;
        for (int64_t s = 0; s < S; s++) {
            double ec = eff[b * S + s];
            for (int64_t i = 0; i < W; i++) {
                uint32_t u = px[b * W + i];
                if (u == PAD) continue;
                for (int64_t j = 0; j < Wy; j++) {
                    uint32_t v = py[s * Wy + j];
                    if (v == PAD) continue;
                    int mm = mism(u, v);
                    if (l - mm < min_matches) continue;
                    double ew = ec;
                    if (wx) ew *= (double)wx[b * W + i] * (double)wy[s * Wy + j];
                    double av = ew * ta[mm], bv = ew * tb[mm];
                    for (int k = 0; k < l; k++) {
                        int xk = (u >> (2 * k)) & 3, yk = (v >> (2 * k)) & 3;
                        int64_t pos = k + i;
                        if (!perturbation) {
                            res[yk * seqlen + pos] += xk == yk ? av : bv;
                        } else if (xk == yk) {
                            for (int h = 0; h < 4; h++)
                                if (h != yk) res[h * seqlen + pos] += av;
                        } else {
                            res[yk * seqlen + pos] += bv;
                        }
                    }
                }
            }
        }
    }
}
