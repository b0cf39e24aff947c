/*
 * libumap_b200 — C ABI of the B200 (sm_100a) UMAP hot path.
 *
 * The reference (hanxiao/mlx-vis 0.7.0) has no FFI: its hot path is Python
 * calling MLX built-ins.  Each entry point below replaces one reference call
 * site, cited as file:line relative to the reference checkout.
 *
 * Conventions
 *  - Every function returns an int status (UMAPB_OK == 0).  On failure
 *    umapb_last_error() returns a message for the calling thread.
 *  - Array arguments are DEVICE pointers, row-major, caller-owned.  The library
 *    allocates no device memory: functions that need scratch take a caller-owned
 *    workspace whose size the matching *_workspace query returns.
 *  - All work is enqueued on `stream` (a cudaStream_t; NULL = legacy default).
 *    Calls are asynchronous; results are valid once the stream is synchronised.
 *  - Kernels with device-side waits bound every wait in time.  If one expires
 *    the kernel abandons its work and writes a non-zero code into the int32
 *    device status word at the start of the workspace; umapb_read_status()
 *    copies it back (synchronising the stream) and turns it into a status.
 */
#ifndef UMAP_B200_H_
#define UMAP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UMAPB_OK 0
#define UMAPB_ERR_ARG 1          /* invalid argument (shape, k, null pointer, ...) */
#define UMAPB_ERR_UNSUPPORTED 2  /* valid request outside the implemented envelope */
#define UMAPB_ERR_CUDA 3         /* CUDA runtime/driver error (launch, encode, ...) */
#define UMAPB_ERR_WORKSPACE 4    /* workspace null or smaller than the query said */
#define UMAPB_ERR_DEVICE 5       /* a kernel reported a device-side failure (bounded wait expired) */

typedef struct CUstream_st* umapb_stream_t;

/* Message for the last failed call on this thread ("" if none). */
const char* umapb_last_error(void);
/* ABI version of this library. */
int umapb_abi_version(void);
/* Number of CUDA kernels this library has enqueued in this process so far
 * (kernels recorded into a CUDA graph count once, at capture). */
unsigned long long umapb_kernel_launches(void);
/* Synchronises `stream`, reads the device status word at `workspace` and
 * returns UMAPB_OK or UMAPB_ERR_DEVICE (with a message). */
int umapb_read_status(const void* workspace, umapb_stream_t stream);
/* Time limit in nanoseconds of the spectral power iteration's grid barrier, for
 * launches made after the call (process-wide; 0 restores the default of 2 s).
 * No counterpart in the reference, which has no device-side waits. */
int umapb_set_wait_limit_ns(unsigned long long ns);

/* ---------------------------------------------------------------------------
 * Exact brute-force kNN — replaces mlx_vis/_knn.py:47-88 (chunked
 * |x|^2+|y|^2-2x.y GEMM, self += 1e30, full-row argsort, first k, sqrt).
 * BF16 tcgen05 distance tiles with a fused per-row top-(k+extra) selection,
 * then an exact FP32 rerank of those candidates.
 *   X        (n, d) float32
 *   out_idx  (n, k) int32   ascending distance, self excluded
 *   out_dist (n, k) float32 Euclidean (squared != 0: squared distances)
 * Requires 1 <= k <= n-1.  Lists of k + extra <= 128 candidates come from the
 * fused tiles and the rerank; longer ones (k <= 4096) from exact FP32-level
 * distance tiles (the split-precision GEMM) and a per-row radix select, which
 * uses no candidates (extra is ignored there; umapb_knn_brute_timed refuses them).
 * ------------------------------------------------------------------------- */
int umapb_knn_brute_workspace(int64_t n, int64_t d, int32_t k, int32_t extra, size_t* bytes);
int umapb_knn_brute(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                    int32_t* out_idx, float* out_dist, void* workspace, size_t workspace_bytes,
                    umapb_stream_t stream);
/* The same call with CUDA events between its three launches (operand prep, the
 * tensor-core distance tiles with the fused top-(k+extra), the FP32 rerank);
 * synchronises and writes the three stage times in milliseconds to stage_ms[3].
 * For profiling; the results equal umapb_knn_brute's. */
int umapb_knn_brute_timed(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                          int32_t* out_idx, float* out_dist, void* workspace, size_t workspace_bytes,
                          float* stage_ms, umapb_stream_t stream);
/* The kNN of the query rows [row_begin, row_begin + row_count) of X against all
 * n rows (self excluded): out_idx / out_dist (row_count, k), the same values as
 * those rows of umapb_knn_brute.  The row split of the reference's chunked loop
 * (mlx_vis/_knn.py:58-79) spread over GPUs: each rank takes one block of rows
 * and the (n, k) result is gathered (mlx_vis_b200/_distributed.py). */
int umapb_knn_brute_rows_workspace(int64_t n, int64_t d, int32_t k, int32_t extra, int64_t row_begin,
                                   int64_t row_count, size_t* bytes);
int umapb_knn_brute_rows(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                         int64_t row_begin, int64_t row_count, int32_t* out_idx, float* out_dist,
                         void* workspace, size_t workspace_bytes, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Allocation-free brute-force kNN.  No counterpart in the reference: an extra
 * entry point for callers that cannot allocate device memory (cudaMalloc and
 * cudaFree synchronise the device, fail when another framework's pooled
 * allocator owns the memory, and thin FFI bindings may be unable to keep a
 * workspace alive).  Same arguments and results as umapb_knn_brute without the
 * workspace: the scratch is a static device array of
 * UMAPB_NOALLOC_SCRATCH_BYTES per GPU, held from library load until exit.
 *   - requests needing more scratch (about 3.8 KB per row at d = 784, k = 15)
 *     fail with UMAPB_ERR_UNSUPPORTED;
 *   - the first call on a device looks up the array's address on that device;
 *     make it before any stream capture;
 *   - every call reuses the same array: calls that overlap on the GPU race, so
 *     serialise them (one stream, or wait between calls);
 *   - device_status (device int32, may be NULL) receives the kernels'
 *     bounded-wait status (0 = ok) once the stream reaches the end of the call.
 * ------------------------------------------------------------------------- */
#define UMAPB_NOALLOC_SCRATCH_BYTES (32u << 20)
int umapb_knn_brute_noalloc(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                            int32_t* out_idx, float* out_dist, int32_t* device_status, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * NNDescent — replaces NNDescent.build (mlx_vis/_nndescent/nndescent.py:34-403);
 * the host keeps the reference's iteration control and random draws.  k <= 32.
 * umapb_nnd_sqnorms:  sq[i] = |X_i|^2 (X float32, or FP16 when half != 0).
 * umapb_nnd_to_half:  FP16 copy of (n, dd) FP32 rows into rows of pitch ldh >= dd
 *                     (zero padded; the FP16 iterations 1-4 use ldh = dd rounded
 *                     up to a multiple of 8).
 * umapb_nnd_gather:   dist[i][p] = max(sq_i + sq_j - 2 X_i.X_j, 0) for j = idx[i][p]
 *                     in FP32 (_gather_dists, nndescent.py:573-612); with
 *                     sort_rows != 0 each row is then sorted by (distance, id)
 *                     (the initial sort, nndescent.py:63-65).
 * umapb_nnd_gather_pairs: the same distances for the pairs (i, j = idx[i][p]) with
 *                     i < r1 whose later row max(i, j) lies in [r0, r1); called once
 *                     per row block [r0, r1) of an upload in row order, it computes
 *                     every pair once, as soon as both rows are on the device, with
 *                     the same values umapb_nnd_gather gives.  idx is not changed.
 *                     k <= 32.
 * umapb_nnd_sort_rows: each row of (dist, idx) sorted by (distance, id), k <= 32; after
 *                     the last block, the pair gathers and this equal
 *                     umapb_nnd_gather with sort_rows != 0.
 * umapb_nnd_reverse:  reverse candidates (_compute_reverse_candidates,
 *                     nndescent.py:406-436): slot p of row j = p-th smallest source
 *                     i with j in idx[i], 0 when j has fewer in-edges.
 * umapb_nnd_iteration: one iteration for all rows (nndescent.py:221-280 full path,
 *                     103-217 converging path): candidates [idx row | first j_nn
 *                     of the rows of its first mc_new neighbours (NEW first when
 *                     converging) | rev row], first occurrence of a duplicate kept,
 *                     distances in the space Xd (rows of dd values at a pitch of
 *                     ldx; FP16 rows need ldx % 8 == 0 and zero padding; FP16
 *                     dot products are rounded to FP16 when half != 0), stored distances reused for current
 *                     neighbours unless recompute_cur, self and duplicates 1e30,
 *                     the k smallest (distance, id) kept; flags_new = positional
 *                     change flags, *changed (device uint64) += their count,
 *                     *evals (device uint64, nullable) += distances evaluated.
 *                     Rows without a NEW flag are copied on the converging path.
 *                     Full path only: with nnbuf (from umapb_nnd_join with the same
 *                     idx_old, mc_new, j_nn) the nn-of-nn distances are read from
 *                     it; with curd (from the same join) the current-neighbour
 *                     distances of positions < mc_new when recompute_cur, and the
 *                     distance of a reverse candidate j of row i as curd[j][p] where
 *                     idx_old[j][p] == i, p < mc_new (the join's d(j, i)); both
 *                     nullable.  order (nullable, a permutation of the rows) sets
 *                     which rows run side by side, for cache locality only.
 * umapb_nnd_join:     the nn-of-nn candidate distances of one full-path iteration
 *                     as blocks per source: for every row i and source position
 *                     p < mc, s = idx_old[i][p], nnbuf[i][p*j_nn + j] =
 *                     d(i, idx_old[s][j]) for j < j_nn and (curd nullable)
 *                     curd[i][p] = d(i, s), with the distance rule of
 *                     umapb_nnd_iteration (FP16 dot rounded when half != 0; FP32
 *                     rows need dd % 4 == 0).  *evals (nullable) += dots computed.
 *                     Sources are taken in the order of `order` (nullable, a
 *                     permutation; for cache locality only).  With mc == k its
 *                     buckets are the reverse-candidate buckets: rev_out
 *                     (nullable) then receives what umapb_nnd_reverse would write.
 * umapb_nnd_sqrt:     Euclidean distances sqrt(max(d2, 0)) (nndescent.py:400).
 * umapb_nnd_random_start: the reference's random start drawn on the device
 *                     (nndescent.py:47-57, 72-82): from the NumPy legacy state in
 *                     `state` (device uint32[628]: MT19937 key[624], pos,
 *                     has_gauss, gauss as a double, low word first — the layout of
 *                     np.random.get_state()), idx (n, k) = randint(0, n - 1)
 *                     shifted past the row index, then P (d, pd1) and P2 (d, pd2) =
 *                     float32(float32(randn) / sqrt(pd)) for pd > 0 (0 skips the
 *                     draw); `state` is overwritten with the state after the draws.
 *                     With a workspace (size from the _workspace query) the draws
 *                     run grid-wide on words generated ahead with a 10-sigma
 *                     margin (a shortfall is redone on the device by one CTA);
 *                     without one, one CTA walks the stream.  Streams longer than
 *                     86,720 words are generated in segments of 65,536 words on
 *                     separate CTAs, each started by jumping ahead; the first such
 *                     call per device copies the jump polynomials to the device
 *                     and synchronises the stream once (under stream capture the
 *                     call generates on one CTA instead).
 * umapb_mt_jump_poly: host only (no GPU needed), for tests and other hosts: the
 *                     jump polynomial x^D mod phi for D = b * 65536 words (*words_ahead
 *                     receives D), 1 <= b <= 1024, as 312 words (bit i of word i/64
 *                     = coefficient of x^i); phi is MT19937's characteristic
 *                     polynomial (degree 19937).  Raw words then satisfy
 *                     x[n + D] = XOR over set bits i of x[n + i] for n >= 1.
 * ------------------------------------------------------------------------- */
int umapb_nnd_sqnorms(const void* X, int64_t n, int32_t dd, int32_t half, float* sq, umapb_stream_t stream);
int umapb_nnd_to_half(const float* X, int64_t n, int32_t dd, int32_t ldh, void* H, umapb_stream_t stream);
int umapb_nnd_gather(const float* X, const float* sq, int64_t n, int32_t dd, int32_t* idx, float* dist, int32_t k,
                     int32_t sort_rows, umapb_stream_t stream);
int umapb_nnd_gather_pairs(const float* X, const float* sq, int64_t n, int32_t dd, const int32_t* idx, float* dist,
                           int32_t k, int64_t r0, int64_t r1, umapb_stream_t stream);
int umapb_nnd_sort_rows(int32_t* idx, float* dist, int64_t n, int32_t k, umapb_stream_t stream);
int umapb_nnd_reverse_workspace(int64_t n, int32_t k, size_t* bytes);
int umapb_nnd_reverse(const int32_t* idx, int64_t n, int32_t k, int32_t* rev, void* workspace,
                      size_t workspace_bytes, umapb_stream_t stream);
int umapb_nnd_join_workspace(int64_t n, int32_t k, int32_t mc, size_t* bytes);
int umapb_nnd_join(const void* Xd, const float* sqd, int32_t dd, int32_t ldx, int32_t half, const int32_t* idx_old,
                   const int32_t* order, int64_t n, int32_t k, int32_t mc, int32_t j_nn, float* nnbuf, float* curd,
                   int32_t* rev_out, unsigned long long* evals, void* workspace, size_t workspace_bytes,
                   umapb_stream_t stream);
/* umapb_nnd_join_new: the blocked join of the converging path (nndescent.py:103-126):
 * the sources of row i are the first mc of its neighbours in NEW-first stable order
 * (none for a row without a NEW flag, whose list the iteration keeps); FP32 rows of
 * dd floats (pitch dd, dd % 4 == 0); nnbuf[i][p*j_nn + j] = d(i, idx_old[s_p][j])
 * for the p-th source s_p; pass nnbuf (and no curd) to the converging
 * umapb_nnd_iteration.  Workspace: umapb_nnd_join_workspace(n, k, mc). */
int umapb_nnd_join_new(const float* X, const float* sq, int32_t dd, const int32_t* idx_old, const uint8_t* flags_old,
                       const int32_t* order, int64_t n, int32_t k, int32_t mc, int32_t j_nn, float* nnbuf,
                       unsigned long long* evals, void* workspace, size_t workspace_bytes, umapb_stream_t stream);
int umapb_nnd_iteration(const void* Xd, const float* sqd, int32_t dd, int32_t ldx, int32_t half, const int32_t* idx_old,
                        const float* dist_old, const uint8_t* flags_old, const int32_t* rev, const int32_t* order,
                        const float* nnbuf, const float* curd, int64_t n, int32_t k,
                        int32_t mc_new, int32_t j_nn, int32_t converging, int32_t recompute_cur, int32_t* idx_new,
                        float* dist_new, uint8_t* flags_new, unsigned long long* changed,
                        unsigned long long* evals, umapb_stream_t stream);
int umapb_nnd_sqrt(const float* d2, int64_t count, float* out, umapb_stream_t stream);
int umapb_nnd_random_start_workspace(int64_t n, int32_t k, int32_t d, int32_t pd1, int32_t pd2, size_t* bytes);
int umapb_nnd_random_start(uint32_t* state, int64_t n, int32_t k, int32_t d, int32_t* idx, float* P, int32_t pd1,
                           float* P2, int32_t pd2, void* workspace, size_t workspace_bytes,
                           umapb_stream_t stream);
int umapb_mt_jump_poly(int32_t b, uint64_t* out, int64_t* words_ahead);
/* umapb_legacy_normal: count values float32(loc + scale * g) with g NumPy's legacy
 * standard normals drawn from `state` (same buffer layout as above; overwritten
 * with the state after the draws) — RandomState(seed).normal(loc, scale, count)
 * cast to float32, as the spectral init's noise (umap.py:344-346).  Workspace as
 * for umapb_nnd_random_start. */
int umapb_legacy_normal_workspace(int64_t count, size_t* bytes);
int umapb_legacy_normal(uint32_t* state, int64_t count, double loc, double scale, float* out, void* workspace,
                        size_t workspace_bytes, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fuzzy simplicial set — replaces UMAP._fuzzy_simplicial_set
 * (mlx_vis/_umap/umap.py:199-270, with _searchsorted 8-22).
 * Per-row rho and sigma bisection (64 steps, target log2 k, tolerance 1e-5) in
 * FP64 (fp64_bisection != 0) or FP32 (the reference's precision); weights
 * exp(-max(d-rho,0)/max(sigma,1e-10)); symmetrisation w + w' - w*w' over the
 * n*k directed edges; prune w < max(w)/n_epochs keeping row-major order.
 *   knn_idx (n, k) int32, knn_dist (n, k) float32 (Euclidean, ascending)
 *   rows/cols/vals: capacity n*k; *n_edges (device int64) receives the count.
 *   rho_out, sigma_out: optional (n,) float32 (may be NULL).
 * ------------------------------------------------------------------------- */
int umapb_fuzzy_workspace(int64_t n, int32_t k, size_t* bytes);
int umapb_fuzzy(const int32_t* knn_idx, const float* knn_dist, int64_t n, int32_t k, int32_t n_epochs,
                int32_t fp64_bisection, int32_t* rows, int32_t* cols, float* vals, int64_t* n_edges,
                float* rho_out, float* sigma_out, void* workspace, size_t workspace_bytes, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Spectral initialisation — replaces UMAP._spectral_init power iteration
 * (mlx_vis/_umap/umap.py:298-348).  Graph in row-major edge order (as
 * umapb_fuzzy writes it), `n_edges` a device int64, `e_cap` its capacity.
 *   V0    (n, dim+1) float32 start block (the reference draws it from mx.random)
 *   noise (n, dim)   float32 N(0, 1e-4) draw added after the 10/max|e| scaling
 *   Y     (n, dim)   float32 output, min-max scaled to [0, 10] per column
 * 1 <= dim <= 32.  Each power iteration is one CSR SpMV that also accumulates
 * the FP64 Gram matrix; orthonormalisation uses its Cholesky factor (the same Q
 * as the reference's modified Gram-Schmidt).  For dim <= 4 all iterations run
 * in one cooperative launch whose grid barrier is a bounded wait: when it gives
 * up, the status word at the start of the workspace is non-zero and Y is not a
 * valid embedding.
 * umapb_spectral_fallback: the reference's fallback to a random start
 * (umap.py:354-357) without a host round trip: if the status word of the
 * spectral workspace is non-zero, Y (n, dim) is overwritten on the device with
 * 0.01 * the N(0, 1) stream of umapb_normal_fill(seed); otherwise Y is kept.
 * Enqueue it on the same stream right after umapb_spectral.
 * ------------------------------------------------------------------------- */
/* Standard normal draws for the spectral start block V0 — stands in for
 * mx.random.normal((n, c+1)) after mx.random.seed (umap.py:134-135, 325),
 * whose bit stream MLX does not specify: Philox4x32-10 + Box-Muller. */
int umapb_normal_fill(float* out, int64_t count, uint64_t seed, umapb_stream_t stream);
int umapb_spectral_workspace(int64_t n, int32_t dim, int64_t e_cap, int32_t n_iter, size_t* bytes);
int umapb_spectral(const int32_t* rows, const int32_t* cols, const float* vals, const int64_t* n_edges,
                   int64_t e_cap, int64_t n, int32_t dim, const float* V0, int32_t n_iter, const float* noise,
                   float* Y, void* workspace, size_t workspace_bytes, umapb_stream_t stream);
int umapb_spectral_fallback(const void* workspace, float* Y, int64_t n, int32_t dim, uint64_t seed,
                            umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Layout optimisation — replaces UMAP._optimize / _sgd_step
 * (mlx_vis/_umap/umap.py:359-449).
 * umapb_layout_prepare: epochs_per_sample = n_epochs / (n_epochs * w/max w)
 *   in float32 (umap.py:398-403) into eps[e_cap]; next[e] = eps[e].
 * umapb_layout_epochs: runs epochs [epoch_begin, epoch_end).  An edge is active
 *   in an epoch when next <= epoch (then next += eps, float32), exactly the
 *   reference's host schedule.  Each epoch reads the epoch-start Y and
 *   accumulates all moves before applying them (the reference's synchronous
 *   scatter-add semantics).  Negative tails come from a counter-based Philox
 *   stream keyed by (seed, epoch, edge, sample).
 * umapb_layout_epoch_injected: one epoch whose negative tails are given in the
 *   reference's order (sample j pairs head ef[j % A] with neg_to[j], A = number
 *   of active edges, umap.py:433-436); neg_count must equal neg_rate * A.
 * Y (n, dim) float32 is updated in place; dim in {1, 2, 3, 4}.
 * ------------------------------------------------------------------------- */
int umapb_layout_workspace(int64_t n, int32_t dim, int64_t e_cap, size_t* bytes);
int umapb_layout_prepare(const float* vals, const int64_t* n_edges, int64_t e_cap, int32_t n_epochs, float* eps,
                         float* next, void* workspace, size_t workspace_bytes, umapb_stream_t stream);
int umapb_layout_epochs(float* Y, int64_t n, int32_t dim, const int32_t* rows, const int32_t* cols,
                        const float* eps, float* next, const int64_t* n_edges, int64_t e_cap, int32_t epoch_begin,
                        int32_t epoch_end, int32_t n_epochs, float a, float b, float learning_rate,
                        int32_t neg_rate, uint64_t seed, void* workspace, size_t workspace_bytes,
                        umapb_stream_t stream);
/* umapb_layout_epochs_graph: the same epochs, recorded into a CUDA graph and
 * launched as one unit; the executable graph is cached per device and updated
 * in place on later calls (same epoch count -> same topology), so the per-call
 * host cost is the recording, not an instantiation.  The stream must not be under
 * capture already. */
int umapb_layout_epochs_graph(float* Y, int64_t n, int32_t dim, const int32_t* rows, const int32_t* cols,
                        const float* eps, float* next, const int64_t* n_edges, int64_t e_cap, int32_t epoch_begin,
                        int32_t epoch_end, int32_t n_epochs, float a, float b, float learning_rate,
                        int32_t neg_rate, uint64_t seed, void* workspace, size_t workspace_bytes,
                        umapb_stream_t stream);
/* Number of edges active in `epoch` given the current `next` values (written to
 * the device int64 *count) — the emptiness test of umap.py:409-414/424 that
 * decides whether the reference runs an epoch and calls epoch_callback.  Uses
 * the layout workspace. */
int umapb_layout_count_active(const float* next, const int64_t* n_edges, int64_t n, int32_t dim, int64_t e_cap,
                              int32_t epoch, int64_t* count, void* workspace, size_t workspace_bytes,
                              umapb_stream_t stream);
int umapb_layout_epoch_injected(float* Y, int64_t n, int32_t dim, const int32_t* rows, const int32_t* cols,
                                const float* eps, float* next, const int64_t* n_edges, int64_t e_cap,
                                int32_t epoch, int32_t n_epochs, float a, float b, float learning_rate,
                                int32_t neg_rate, const int32_t* neg_to, int64_t neg_count, void* workspace,
                                size_t workspace_bytes, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Learned warm-start encoder d -> 512 -> 512 -> c (GELU).  New: the reference
 * has no learned initialisation (its closest idiom is the MMAE MLP + AdamW step,
 * mlx_vis/_mmae/mmae.py:22-38, 258-281).
 * umapb_gemm_bf16: C[M,N] = sum_k A[m,k] B[n,k] on tcgen05 tensor cores, A and B
 *   BF16 row-major with pitches lda, ldb (multiples of 8, >= K), FP32 accumulation,
 *   fused epilogue: UMAPB_GEMM_F32 (C, ldc; with ksplit > 1 the K blocks are split
 *   over ksplit CTAs per tile and C holds ksplit slices of M x ldc, slice s at
 *   C + s M ldc, whose sum is the product); UMAPB_GEMM_BIAS_GELU (Z = C + bias,
 *   H = bf16(gelu(Z)), optional H^T);
 *   UMAPB_GEMM_GELU_BACK (H = bf16(C * gelu'(Z)), optional H^T, optional column
 *   sums of H in colsum, zeroed by the call).  *status (device int32) reports an
 *   expired bounded wait.
 * umapb_mlp_convert: X f32 (rows x d; row r taken from row row_idx[r] when row_idx,
 *   a device int64 array, is given) -> BF16 (rows x ldx, zero padded) and an
 *   optional transposed BF16 copy (d x rows, pitch ldt).
 * umapb_mlp_head_forward: Y = H W^T + b for the last layer (c <= 4, FP32 W).
 * umapb_mlp_head_backward: MSE loss mean_b |Y - T|^2 (device f32; T row t_idx[b] when
 *   the device int64 array t_idx is given), dY, dW = dY^T H2,
 *   db = sum dY, dZ2 = bf16((dY W) * gelu'(Z2)) row-major and transposed, and
 *   dbias2 = column sums of dZ2 (loss, dW, db, dbias2 zeroed by the call).
 * umapb_adamw: decoupled-weight-decay Adam on n_groups (<= 8) FP32 master
 *   tensors in one launch (host arrays of device pointers and shapes), bias-
 *   corrected at the step number *step (device memory, so a captured step can
 *   replay), writing optional BF16 copies (p_bf16 / ldb) and transposed BF16
 *   copies (p_bf16_t / ldbt); p_bf16 / p_bf16_t may be null or hold null entries.
 *   With g_slices (host array, may be null) group k's gradient is the sum of
 *   g_slices[k] slices g[k] + s g_stride[k] (the K-sliced GEMM output); the sum
 *   is written back to the first slice.
 * ------------------------------------------------------------------------- */
#define UMAPB_GEMM_F32 0
#define UMAPB_GEMM_BIAS_GELU 1
#define UMAPB_GEMM_GELU_BACK 2
int umapb_gemm_bf16(const void* A, const void* B, int32_t M, int32_t N, int32_t K, int32_t lda, int32_t ldb,
                    int32_t epilogue, int32_t ksplit, float* C, int32_t ldc, const float* bias, float* Z, int32_t ldz,
                    void* H, int32_t ldh, void* HT, int32_t ldt, float* colsum, int32_t* status,
                    umapb_stream_t stream);
int umapb_mlp_convert(const float* X, const int64_t* row_idx, int32_t rows, int32_t d, int32_t ldx, void* Xb,
                      void* XT, int32_t ldt, umapb_stream_t stream);
int umapb_mlp_head_forward(const void* H, int32_t ldh, int32_t B, int32_t Hd, const float* W, const float* bias,
                           int32_t c, float* Y, umapb_stream_t stream);
int umapb_mlp_head_backward(const float* Y, const float* T, const int64_t* t_idx, int32_t B, int32_t c,
                            const float* W, int32_t Hd,
                            const float* Z2, int32_t ldz, const void* H2, int32_t ldh2, float* dY, float* dW,
                            float* db, void* dZ2, int32_t lddz, void* dZ2T, int32_t ldt, float* dbias2, float* loss,
                            umapb_stream_t stream);
int umapb_adamw(int32_t n_groups, float* const* p, float* const* g, const int32_t* g_slices,
                const int64_t* g_stride, float* const* m, float* const* v, const int32_t* rows, const int32_t* cols,
                void* const* p_bf16, const int32_t* ldb,
                void* const* p_bf16_t, const int32_t* ldbt, float lr, float beta1, float beta2, float eps,
                float weight_decay, const int32_t* step, umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Dense FP32 products on the BF16 tensor cores, column means and a key sort.
 * Replace the reference's FP32 GEMMs of the NNDescent projections X @ P, X @ P2
 * (mlx_vis/_nndescent/nndescent.py:72-82, 229-233) and of PCA (covariance and
 * projection, mlx_vis/_umap/umap.py:92-111), and the row order NNDescent runs in.
 * umapb_split3: operand rows for umapb_gemm_split3 from a row-major FP32 matrix S
 *   (rows x cols, pitch lds), with the optional per-column mu subtracted: each
 *   value x as three BF16 parts x0 + x1 + x2 (24 significant bits) at column
 *   offsets 0, kp, 2 kp of an operand row of 3 kp BF16 (zero padded past K).
 *   transpose == 0: operand row r = S row r (K = cols); != 0: operand row c =
 *   S column c (K = rows).  kp: a multiple of 64, >= K.
 * umapb_gemm_split3: C[m][n] = sum_k A[m][k] B[n][k] from split operands A3
 *   (M x 3kp) and B3 (N x 3kp): six tcgen05 products per K block (x0y0, x0y1,
 *   x1y0, x0y2, x2y0, x1y1) in one FP32 accumulator, error at FP32 level.  With
 *   ksplit > 1 the K range is cut into slices, slice z written at C + z M ldc
 *   (sum them with umapb_sum_slices).  *status (device int32) receives the
 *   bounded-wait status.
 * umapb_colmean: mean[c] over the rows (FP64 partial sums in a fixed order).
 * umapb_sum_slices: out[t] = scale * sum_z C[z count + t].
 * umapb_sort_keys: order = the stable ascending order of the n float keys
 *   keys[0], keys[stride], ... (no NaN).
 * ------------------------------------------------------------------------- */
int umapb_split3(const float* S, int64_t rows, int64_t cols, int64_t lds, const float* mu, int32_t transpose,
                 int32_t kp, void* out, umapb_stream_t stream);
int umapb_gemm_split3(const void* A3, const void* B3, int32_t M, int32_t N, int32_t kp, int32_t ksplit, float* C,
                      int32_t ldc, int32_t* status, umapb_stream_t stream);
int umapb_colmean_workspace(int64_t rows, int64_t cols, size_t* bytes);
int umapb_colmean(const float* S, int64_t rows, int64_t cols, int64_t lds, float* mean, void* workspace,
                  size_t workspace_bytes, umapb_stream_t stream);
int umapb_sum_slices(const float* C, int32_t slices, int64_t count, float scale, float* out, umapb_stream_t stream);
int umapb_sort_keys_workspace(int64_t n, size_t* bytes);
int umapb_sort_keys(const float* keys, int64_t n, int64_t stride, int32_t* order, void* workspace,
                    size_t workspace_bytes,
                    umapb_stream_t stream);

/* ---------------------------------------------------------------------------
 * Access-rate probes (measurement; no reference counterpart).  The caller times one
 * launch; they give the measured ceilings the two gather-bound steps are reported
 * against.
 * umapb_probe_random_access: threads (a multiple of 256) x per_thread rounds of one
 *   random row read of dim floats (dim 1, 2 or 4) from table (n rows) and, every
 *   red_every rounds (0: never), one random vector atomic add of dim floats into
 *   dtable -- the access mix of a layout epoch.  sink: 4 device floats.
 * umapb_probe_row_gather: one warp per entry of ids reads the row of row_bytes (a
 *   multiple of 16, 16-byte aligned table) -- the candidate-row reads of the
 *   NNDescent join.  Ids outside [0, rows) are skipped.  sink: 16 device bytes.
 * ------------------------------------------------------------------------- */
int umapb_probe_random_access(const float* table, float* dtable, int64_t n, int32_t dim, int64_t threads,
                              int32_t per_thread, int32_t red_every, float* sink, umapb_stream_t stream);
int umapb_probe_row_gather(const void* table, int64_t rows, int32_t row_bytes, const int32_t* ids, int64_t count,
                           void* sink, umapb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* UMAP_B200_H_ */
