/*
 * gkm_b200.h -- C ABI of the B200 (sm_100a) gapped-k-mer kernel library.
 *
 * Plain pointers and sizes; every array argument is DEVICE memory unless its
 * comment says host; every call is asynchronous on the given CUDA stream and
 * returns a status (GKM_OK = 0).  gkm_last_error() describes the last failure
 * of the calling thread.
 *
 * Each entry point replaces one operation of gkmsvm-lite's kernel operator
 * API (paths relative to its source tree, src/gkmsvm/); that operator is cited
 * beside it.  Packed windows: a window of l bases is a uint32 with position k
 * in bits 2k..2k+1 (A=0 C=1 G=2 T=3); GKM_PAD marks no window (past a shorter
 * row's last window; first in a reverse-complement row).
 */
#ifndef GKM_B200_H
#define GKM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *gkm_stream_t; /* cudaStream_t */

#define GKM_PAD 0xFFFFFFFFu
#define GKM_MAX_L 15

enum {
    GKM_OK = 0,
    GKM_ERR_INVALID = 1,     /* bad argument: shape, l, null pointer ...      */
    GKM_ERR_CUDA = 2,        /* a CUDA call failed                            */
    GKM_ERR_OOM = 3,         /* device memory exhausted                        */
    GKM_ERR_CAPACITY = 4,    /* a counter or table limit was exceeded          */
    GKM_ERR_UNSUPPORTED = 5  /* the shape needs a path this build lacks        */
};

/* A kernel type after KERNEL_BUILDERS (svm.py:95-106): the pair weight h(m)
 * by mismatch count and the window weights of -t 4/-t 5. */
typedef struct gkm_spec {
    int32_t l;          /* window length, 1..15 */
    int32_t include_rc; /* 1: the reverse complement adds a column block */
    int32_t weighted;   /* 1: centre-weighted windows (kernels/weighted.py) */
    int32_t dmax;       /* largest m with h[m] != 0 */
    double h[16];       /* h[m], m = 0..l; 0 past dmax */
    const uint8_t *wd;  /* device [wd_len]: window weight by |n/2 - i| */
    int32_t wd_len;     /* > the longest row's window count when weighted */
} gkm_spec;

typedef struct gkm_index gkm_index_t; /* SV l-mer index (opaque) */

int gkm_version(void);
const char *gkm_last_error(void);
/* Number of SMs of the current device and its opt-in shared memory per block. */
int gkm_device_info(int32_t *sm_count, int32_t *smem_per_block);
/* Persistent index queries launched from the calling thread take at most
 * `blocks` blocks (0: one per SM, the default).  Thread-local.  A serving loop
 * gives its ISM / GkmExplain worker thread a limit so those long queries leave
 * SMs to the scoring passes other threads launch.  No counterpart in
 * gkmsvm-lite, which has no serving loop. */
int gkm_set_thread_grid_limit(int32_t blocks);

/* Packed forward and RC windows of [B, L] base codes; counts[b] = windows of
 * row b, lengths (nullable) = each row's length.
 * Replaces PackedGkmKernel.pack / pack_both (kernels/packed.py:130-187). */
int gkm_pack(const gkm_spec *spec, const uint8_t *codes, const int64_t *lengths,
             int64_t B, int64_t L, uint32_t *fwd, uint32_t *rc, int32_t *counts,
             gkm_stream_t stream);

/* K_raw(x, x) [B] (and, nullable, its profile [B, l+1] of pair counts by
 * mismatch count, forward and RC blocks summed).
 * Replaces raw_diag_packed (kernels/direct.py:109-137, 294-306;
 * kernels/weighted.py:91-118, 440-471). */
int gkm_self_kernel(const gkm_spec *spec, const uint32_t *fwd, const uint32_t *rc,
                    const int32_t *counts, int64_t B, int64_t W, double *diag,
                    uint64_t *profile, gkm_stream_t stream);

/* Pairwise K_raw [B, S] (nullable) and profiles [B, S, l+1] (nullable) of rows
 * bx against columns by (+ their RC ry when include_rc) by warp ballot/popc
 * over every window pair.
 * Replaces PackedGkmKernel.raw_packed's pair loop (kernels/packed.py:191-228,
 * kernels/direct.py:23-42, kernels/weighted.py:47-69). */
int gkm_join_pairwise(const gkm_spec *spec, const uint32_t *bx, const int32_t *cx,
                      int64_t B, int64_t Wx, const uint32_t *by, const uint32_t *ry,
                      const int32_t *cy, int64_t S, int64_t Wy, double *raw,
                      uint64_t *profile, gkm_stream_t stream);

/* The same pairwise K_raw and profiles as gkm_join_pairwise, computed on the
 * tensor cores: match counts of 128 query windows x 128 column windows as one
 * int8 one-hot product (tcgen05.mma kind::i8, int32 accumulators in tensor
 * memory), pairs within dmax counted exactly in the epilogue.  Allocates up to
 * 1 GiB of transient device memory per launch round for its pre-built column
 * tiles.  Needs
 * 0 <= dmax < l <= 15.  error (device int32, caller-zeroed): set non-zero if
 * an MMA did not complete within its wait limit (outputs then undefined).
 * Replaces the same pair loop as gkm_join_pairwise (kernels/packed.py:191-228,
 * kernels/direct.py:23-42, kernels/weighted.py:47-69). */
int gkm_dense_pairwise(const gkm_spec *spec, const uint32_t *bx, const int32_t *cx,
                       int64_t B, int64_t Wx, const uint32_t *by, const uint32_t *ry,
                       const int32_t *cy, int64_t S, int64_t Wy, double *raw,
                       uint64_t *profile, int32_t *error, gkm_stream_t stream);
/* Test hook: the limit (ns) of the dense kernel's waits on hand-offs between
 * its roles (B record landed, accumulator ready or handed back), for the
 * dense launches made from the calling thread; 0 restores the default 1 s.
 * A wait that runs out sets the call's error flag; the kernel still waits
 * (up to 1 s) for its copies and MMAs in flight and frees its tensor memory.
 * No counterpart in gkmsvm-lite. */
int gkm_dense_set_role_wait(int64_t ns);

/* Builds the l-mer index over S columns (radix sort of the packed l-mers of
 * their forward and RC windows into per-SV-tile CSR buckets).  masks [n_masks]
 * (device): the XOR neighbour masks within dmax, each with its mismatch count
 * in bits 24..31.  tile_svs 0: chosen for shared memory.
 * Replaces LmerIndex.__init__ (kernels/lmer_index.py:161-200). */
int gkm_index_create(const gkm_spec *spec, const uint32_t *fwd, const uint32_t *rc,
                     const int32_t *counts, int64_t S, int64_t W, const uint32_t *masks,
                     int32_t n_masks, int32_t tile_svs, gkm_index_t **out,
                     gkm_stream_t stream);
int gkm_index_free(gkm_index_t *index);
int gkm_index_info(const gkm_index_t *index, int64_t *entries, int32_t *tiles,
                   int32_t *tile_svs, int64_t *device_bytes);
/* Copies, in stream order (cudaMemcpyAsync), the index's two event counts
 * into counts[2] (nullable; host or device memory): [0] query blocks whose
 * narrow-counter carries outgrew their log, [1] 32-bit counters that wrapped.
 * The counts only grow: a call whose window (copy before, copy after, on its
 * stream) sees [0] change reruns with 32-bit counters; one that sees [1]
 * change reruns with 64-bit counters (weighted kernels).  wide >= 0 selects,
 * for unweighted kernels, 32-bit counters (1) or narrow counters with the
 * carry log (0); for weighted kernels, 64-bit counters (2) or 32-bit (0, 1).
 * Unweighted 32-bit counters wrap only past 2^32 matching window pairs of one
 * (row, SV) pair; [1] moving there is an error. */
int gkm_index_status(gkm_index_t *index, uint32_t *counts, int32_t wide, gkm_stream_t stream);

/* K_raw [B, S] (nullable) and profiles [B, S, l+1] (nullable) through the
 * index; diag_offset >= 0: row b is column diag_offset + b of a self-Gram and
 * only its columns from there on are written.
 * Replaces LmerIndex.pairwise (kernels/lmer_index.py:239-268, 400-441). */
int gkm_index_pairwise(const gkm_index_t *index, const uint32_t *bx, const int32_t *cx,
                       int64_t B, int64_t W, int64_t diag_offset, double *raw,
                       uint64_t *profile, gkm_stream_t stream);

/* scores[b] = sum_s coef[s] f(K_raw(b, s) inv_dx[b] inv_ds[s]) + bias, f the
 * identity or exp(gamma (k - 1)) (rbf), with no [B, S] block.  order
 * (nullable, [B]): the order rows are handed out in.
 * Replaces LmerIndex.reduce (kernels/lmer_index.py:275-298,
 * kernels/lmer_index_cpu.py:71-120) and GkmSVM._sv_scores (svm.py:368-405). */
int gkm_index_score(const gkm_index_t *index, const uint32_t *bx, const int32_t *cx,
                    int64_t B, int64_t W, const double *inv_dx, const double *inv_ds,
                    const double *coef, double gamma, int32_t rbf, double bias,
                    const int32_t *order, double *scores, gkm_stream_t stream);

/* gkm_index_score without any device allocation, for callers that cannot
 * allocate while scoring (a process whose device heap is owned by its own
 * pool, a serving loop that must not block in the allocator).  No counterpart
 * in gkmsvm-lite.  Its per-(row, SV tile) partial sums live in one fixed
 * 4 MiB device array that the library holds on every device it is loaded on
 * until exit, so B x tiles must be <= 524,288 (GKM_ERR_CAPACITY otherwise).
 * The first call on a device looks that array's address up
 * (cudaGetSymbolAddress): make it before any stream capture.  The address is
 * kept for the life of the device's context: do not call this again on a
 * device after cudaDeviceReset.  All calls share the array, so calls that
 * overlap on the GPU (other streams, other threads) race; serialise them.
 * Exactness, as for gkm_index_score: unweighted indexes count in narrow fields
 * with a per-block carry log; a block whose log overflows only raises event
 * count [0] of gkm_index_status, so a caller that needs exact scores reads
 * those counts before and after the call and, if [0] moved, rescores with
 * 32-bit counters (gkm_index_status wide = 1). */
int gkm_index_score_noalloc(const gkm_index_t *index, const uint32_t *bx, const int32_t *cx,
                            int64_t B, int64_t W, const double *inv_dx, const double *inv_ds,
                            const double *coef, double gamma, int32_t rbf, double bias,
                            const int32_t *order, double *scores, gkm_stream_t stream);

/* Work counts of an index query over rows bx: lookups (query windows x
 * neighbour masks) and hits (index entries those lookups visit, all tiles);
 * out [2] uint64, accumulated.  Used to state the algorithmic bytes of a
 * query (kernels/lmer_index_cpu.py:23-37 visits the same). */
int gkm_index_count(const gkm_index_t *index, const uint32_t *bx, const int32_t *cx,
                    int64_t B, int64_t W, uint64_t *out, gkm_stream_t stream);

/* V[v] = sum over index entries of l-mer v of c_sv[sv] times the entry's
 * window weight, [4^l].
 * Replaces sv_lmer_weights (lmer_table.py:35-55). */
int gkm_index_lmer_weights(const gkm_index_t *index, const double *c_sv, double *V,
                           gkm_stream_t stream);

/* table[u] = sum_{v within dmax of u} h(m(u, v)) V[v] over all 4^l l-mers.
 * Replaces build_lmer_table (lmer_table.py:58-98). */
int gkm_lmer_table(const gkm_spec *spec, const double *V, const uint32_t *masks,
                   int32_t n_masks, double *table, gkm_stream_t stream);

/* DeltaSVM weights [4^l] in DeltaSVM order (first base most significant) read
 * off the l-mer table: table[digit-reversed index] * window_weight, divided by
 * sqrt(max(K(u, u), 1e-10)) of the l-mer alone when query_norm.
 * Replaces _deltasvm_weights_from_table / _lmer_self_kernels (svm.py:667-704). */
int gkm_deltasvm_table(const gkm_spec *spec, const double *table, double window_weight,
                       int32_t query_norm, double *out, gkm_stream_t stream);

/* scores[b] = sum_i wt_i table[x_i] / sqrt(max(K(x, x), 1e-10)) + bias (plain
 * sum without normalize); raw and diag (nullable) get the two parts.
 * Replaces GkmSVM._table_raw / _score_lmer_table (svm.py:559-582). */
int gkm_table_score(const gkm_spec *spec, const double *table, const uint32_t *fwd,
                    const uint32_t *rc, const int32_t *counts, int64_t B, int64_t W,
                    double bias, int32_t normalize, double *scores, double *raw,
                    double *diag, gkm_stream_t stream);

/* K_raw(mutant, mutant) [4, L, B] for every single-base substitution, from the
 * pairs touching the windows that cover the substituted base.
 * Replaces raw_diag_mutants (kernels/direct.py:160-201, 265-292;
 * kernels/weighted.py:153-197). */
int gkm_mutant_diag(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts,
                    int64_t B, int64_t W, int64_t L, const double *diag,
                    double *mut_diag, gkm_stream_t stream);

/* ISM deltas [B, 4, L] from the l-mer table; with normalize the mutant
 * self-kernels are computed in the same pass (written to mut_diag [4, L, B]
 * when it is not null) and diag = K(x, x) is required; 0 past each row's
 * windows.  ref_raw [B] = sum_i wt_i table[x_i].
 * Replaces _ism_table (ism.py:118-144) with _mutants (ism.py:254-273). */
int gkm_ism_table(const gkm_spec *spec, const double *table, const uint32_t *fwd,
                  const int32_t *counts, int64_t B, int64_t W, int64_t L,
                  const double *ref_raw, const double *diag, double *mut_diag,
                  int32_t normalize, double *out, gkm_stream_t stream);

/* ISM deltas [B, 4, L] through the index for any kernel (RBF included):
 * K(mutant, s) = ref_raw[b, s] + K(new windows, s) - K(old windows, s), the
 * old windows' term summed from one query row per reference window.
 * inv_dmut [4, L, B]: 1 / sqrt(K(mutant, mutant)) (all 1 unnormalised).
 * Allocates nothing: workspace (256-byte aligned, workspace_bytes) holds the
 * query rows and K_raw rows of as many positions per pass as fit; it must
 * hold at least gkm_index_mutants_workspace's min_bytes (GKM_ERR_CAPACITY
 * otherwise); all_bytes does every position in one pass.  ref_score [B]
 * (nullable): the rows' scores without bias; null computes them from ref_raw
 * and inv_dx with the arithmetic of the mutants' sums (one pass over ref_raw
 * instead of another index query).
 * Replaces LmerIndex.mutants (kernels/lmer_index.py:326-374,
 * kernels/lmer_index_cpu.py:203-285). */
int gkm_index_mutants_workspace(const gkm_index_t *index, int64_t B, int64_t L, int64_t *min_bytes,
                                int64_t *all_bytes);
int gkm_index_mutants(const gkm_index_t *index, const uint32_t *fwd, const int32_t *counts,
                      int64_t B, int64_t W, int64_t L, const double *ref_raw,
                      const double *ref_score, const double *inv_dx,
                      const double *inv_dmut, const double *inv_ds, const double *coef,
                      double gamma, int32_t rbf, double *out, void *workspace,
                      int64_t workspace_bytes, gkm_stream_t stream);

/* scores[b] = sum_s coef[s] f(raw[b, s] / max(sqrt(dx[b] ds[s]), 1e-10)) + bias
 * over a materialised [B, S] block (dx, ds nullable: no normalisation).
 * Replaces _normalized_dot (svm.py:42-61). */
int gkm_raw_score(const double *raw, int64_t B, int64_t S, const double *dx,
                  const double *ds, const double *coef, double gamma, int32_t rbf,
                  double bias, double *scores, gkm_stream_t stream);

/* Mutation impact [n] from raw [2n, S] = [ref rows; alt rows].
 * Replaces _impact_cpu (explain/impact.py:22-48). */
int gkm_impact(const double *raw, int64_t n, int64_t S, const double *dr,
               const double *ds, const double *coef, double gamma, int32_t rbf,
               double *out, gkm_stream_t stream);

/* GkmExplain through l-mer weights: each query window visits the l-mers within
 * the explain cutoff (masks with their mismatch count in bits 24..31) and adds
 * a(m) or b(m) times the neighbour's weight to each position.  Weights come
 * from V [4^l] (non-RBF) or, with index and w [B, S], from the sum of w[b, sv]
 * over the index entries of the neighbour (RBF).  out [B, 4, L].
 * Replaces _explain_lmer_cpu / _explain_index_cpu (explain/cpu.py:69-207). */
int gkm_explain_lmer(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts,
                     int64_t B, int64_t W, int64_t L, const double *inv_dx,
                     const double *V, const gkm_index_t *index, const double *w,
                     const uint32_t *masks, int32_t n_masks, const double *table_a,
                     const double *table_b, int32_t perturbation, double *out,
                     gkm_stream_t stream);

/* GkmExplain by the per-SV pair loop, for models the l-mer path does not take
 * (l > 12, a neighbourhood larger than the SVs, no l-mer index): every query
 * window against every SV window by (SV s) forward and, with include_rc, RC
 * (by / ry [S, Wy] from gkm_pack, cy [S] their counts); a pair with at least
 * min_matches matching positions adds a(m) or b(m) times w[b, s] (and the two
 * window weights when weighted) to each position.  w [B, S]: coef_s /
 * sqrt(K(sv_s, sv_s)), times the RBF scale of K(x_b, sv_s) for RBF models;
 * inv_dx [B] scales each row.  out [B, 4, L]; deterministic.
 * Replaces _explain_cpu / _explain_gpu (explain/cpu.py:14-66,
 * explain/core.py:170-247). */
int gkm_explain_pairs(const gkm_spec *spec, const uint32_t *fwd, const int32_t *counts,
                      int64_t B, int64_t W, int64_t L, const double *inv_dx,
                      const uint32_t *by, const uint32_t *ry, const int32_t *cy,
                      int64_t S, int64_t Wy, const double *w, const double *table_a,
                      const double *table_b, int32_t min_matches, int32_t perturbation,
                      double *out, gkm_stream_t stream);

/* The GkmExplain table of a linear model: A [4^l, 4, l] float64 (caller
 * allocates, 1.5 GB at l = 11), every l-mer's attribution, from V [4^l] and
 * the level tables table_a / table_b [l + 2] (device), by radix-4
 * Walsh-Hadamard transforms.  l <= 12.
 * Replaces _build_explain_table (explain/table.py:58-113). */
int gkm_explain_table_build(const gkm_spec *spec, const double *V, const double *table_a,
                            const double *table_b, double *A, gkm_stream_t stream);

/* GkmExplain attributions out [B, 4, L] read from the table A: one row per
 * query window (times its window weight), added over the windows covering each
 * position, times inv_dx.  perturbation: the perturbation-mode table.
 * Replaces _explain_table_cpu (explain/table.py:117-147). */
int gkm_explain_table(const gkm_spec *spec, const double *A, const uint32_t *fwd,
                      const int32_t *counts, int64_t B, int64_t W, int64_t L,
                      const double *inv_dx, int32_t perturbation, double *out,
                      gkm_stream_t stream);

/* Normalised, finished Gram [N, M] from raw (upper triangle when symmetric,
 * mirrored exactly).  Replaces compute_gram's tile finish (gram.py:82-106). */
int gkm_gram_finish(const double *raw, int64_t N, int64_t M, const double *dx,
                    const double *dy, double gamma, int32_t rbf, int32_t symmetric,
                    double *out, gkm_stream_t stream);

/* Host: the support-vector section of an LS-GKM model file (the text after
 * its "SV" line), lines "<coefficient> <sequence>", blank lines skipped.  With
 * codes NULL, counts: *n_sv lines and *max_len, the longest sequence.  Else
 * fills coef [n], lengths [n] and codes [capacity, width] (A C G T = 0..3,
 * lower case too; N and other letters stored as 0, zero padded) and sets
 * *n_other, the SVs holding letters other than ACGTN.  A line with fewer than
 * two fields, a coefficient strtod does not read whole, or a non-ASCII byte
 * fails with GKM_ERR_INVALID and its line number within the section in
 * *bad_line (nullable).
 * Replaces the SV loop of load_lsgkm_model and build_model's encoding
 * (importers/lsgkm.py:68-85, importers/__init__.py:53-113). */
int gkm_lsgkm_parse_svs(const char *text, int64_t len, int64_t capacity, int64_t width,
                        double *coef, int64_t *lengths, uint8_t *codes, int64_t *n_sv,
                        int64_t *max_len, int64_t *n_other, int64_t *bad_line);

/* Kernel-column provider of gkm_smo_solve: writes, for k < count, column
 * idx[k] of the normalized kernel (K(:, idx[k]), N doubles, HOST memory) to
 * out[k * N ...]; returns 0, or non-zero to stop the solver. */
typedef int (*gkm_columns_cb)(int32_t count, const int32_t *idx, double *out, void *ctx);

/* SMO training over n dual variables of N sequences (HOST arrays): signs y
 * [n] (+1/-1), linear term p [n], variable t using column t mod N; C-SVC is
 * n = N, p = -1; epsilon-SVR is n = 2N, y = (+1, -1), p = (eps - z, eps + z).
 * diag [N] (nullable: 1) the kernel's diagonal.  Second-order working-set
 * selection, an LRU cache of cache_columns columns, columns fetched through
 * `columns` (with up to prefetch - 1 likely next ones while the cache has
 * room).  coef [n] = y_t alpha_t, bias = -rho (score = K coef + bias).
 * Replaces csmo_solve (_csmo.c:186) and _smo_csolver (solver.py:260-392). */
int gkm_smo_solve(int32_t n, int32_t N, const double *y, const double *p, const double *diag,
                  double C_pos, double C_neg, double tol, int64_t max_iter, int32_t cache_columns,
                  int32_t prefetch, gkm_columns_cb columns, void *ctx, double *coef, double *bias,
                  int64_t *iterations, int32_t verbose);

#ifdef __cplusplus
}
#endif
#endif /* GKM_B200_H */
