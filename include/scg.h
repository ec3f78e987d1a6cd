/*
 * scg.h -- C ABI of the B200 search library (libscgpu.so).
 *
 * The drop-in boundary for the search path of marker68/second-candidate:
 * plain pointers and sizes, int status returns, no C++ or CUDA types.  The
 * reference's own C++ classes (PQQuery, MultiQuery, SCQuery, Encoder,
 * SCEncoder) are header-only and non-virtual; the drop-in headers under
 * second-candidate_b200/cpp/ keep their names and signatures and forward to
 * these entry points.  Each declaration names the reference interface it
 * replaces (file:line in the reference tree).
 *
 * Status codes: SCG_OK (0) or a negative SCG_ERR_*; scg_last_error() returns
 * the message of the last failure on the calling thread.  Device-side caps
 * (cell budgets, iteration limits) end a query with a status, never a trap.
 */
#ifndef SCG_H_
#define SCG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCG_OK 0
#define SCG_ERR_ARG (-1)    /* invalid argument or shape                        */
#define SCG_ERR_OOM (-2)    /* device or host allocation failed                 */
#define SCG_ERR_IO (-3)     /* file missing, short or malformed                 */
#define SCG_ERR_CUDA (-4)   /* CUDA runtime error                               */
#define SCG_ERR_CAP (-5)    /* a per-query device budget was exceeded           */
#define SCG_ERR_STATE (-6)  /* call order (e.g. search before codebooks/index)  */
#define SCG_PENDING 1       /* scg_server_wait: the request has not finished     */

/* Search modes: the three reference entry points. */
#define SCG_IVFADC 0  /* PQQuery::search_ivfadc      query.h:202-325        */
#define SCG_IMI 1     /* MultiQuery::search_multi2   multi_query.h:62-273   */
#define SCG_SC2 2     /* SCQuery::search_mr_ivf      sc_query.h:60-256      */
#define SCG_SC3 3     /* SCQuery::search_mr_ivf3     sc_query.h:265-475     */

/* Arithmetic of the per-query tables and of the ADC sum.  The three
 * tensor-core forms build the tables as tcgen05 GEMMs with FP32 accumulation
 * and use the fused per-vector ADC term in the scan. */
#define SCG_FP32_EXACT 0 /* the reference's float operations in its order      */
#define SCG_FAST 1       /* BF16 hi/lo split operands, 3 products: ~2^-15 relative */
#define SCG_BF16 2       /* one BF16 product per term                          */
#define SCG_FP16 3       /* one FP16 product per term (operands must fit FP16)  */

typedef struct scg_index scg_index;

typedef struct {
    int mode;       /* SCG_IVFADC / SCG_IMI / SCG_SC2 / SCG_SC3                    */
    int R;          /* results per query (1..1024)                                 */
    int w;          /* cell cap: popped cells (IVFADC, IMI) or non-empty cells (SC) */
    int T;          /* candidate target: stop after the cell that reaches T         */
    int precision;  /* SCG_FP32_EXACT, SCG_FAST, SCG_BF16 or SCG_FP16                */
    int rerank;     /* 0: ADC distances.  -1: the reference's real_dist branch
                       (query.h:307-312, multi_query.h:255-259,
                       sc_query.h:232-236) -- every visited candidate scored
                       by its exact distance, the R smallest returned.
                       L > 0 (R <= L <= 1024): only the ADC top-L shortlist
                       re-ranked by that exact distance.  Both need the raw
                       vectors (scg_load_raw / scg_load_raw_u8).             */
} scg_search_params;

/* Message of the last failing call on this thread (always NUL-terminated). */
int scg_last_error(char *buf, int len);

/* Creates an empty index on CUDA device `device`.  Replaces the PQQuery /
 * MultiQuery / SCQuery constructors (query.cpp:19-32, multi_query.cpp:15-17,
 * sc_query.cpp:17-25). */
int scg_index_create(scg_index **out, int device);

/* Frees all device memory of the index.  Replaces ~PQQuery (query.cpp:37-61). */
int scg_index_destroy(scg_index *h);

/* Codebooks from memory: cq is [mc][kc][dim/mc], pq is [mp][kp][dim/mp]
 * (the arrays load_codebook fills, sc_utilities.h:897-980). */
int scg_load_codebooks(scg_index *h, const float *cq, int kc, int mc,
                       const float *pq, int kp, int mp, int dim);

/* Codebooks from two .ctr_ files.  Replaces PQQuery::load_codebooks
 * (query.cpp:66-75). */
int scg_load_codebooks_file(scg_index *h, const char *cq_path, const char *pq_path);

/* The CSR index: L[ncells] inclusive prefix counts, pid[N], codes[N][mp] in
 * cell order (the arrays PQQuery::load_encoded_data builds, query.cpp:82-165).
 * ncells must be kc^mc (IVFADC/IMI), kc^2 (second candidate, mc = 1) or kc^3
 * (second candidate with three nearest centroids, mc = 1, kc <= 1024). */
int scg_load_csr(scg_index *h, const int *L, const int *pid, const uint8_t *codes,
                 int64_t N, int64_t ncells);

/* Reads an .edat_ file with kc^nc cells (nc = mc for IVFADC/IMI indexes, 2 or
 * 3 for second-candidate indexes).  Replaces PQQuery::load_encoded_data
 * (query.cpp:82-165) and SCQuery::load_encoded_data (sc_query.cpp:36-123). */
int scg_load_encoded_file(scg_index *h, const char *path, int nc);

/* Raw vectors [N][dim] (float, row = the vector's id), for the shortlist
 * re-rank.  Replaces PQQuery::load_data (query.h:82-86). */
int scg_load_raw(scg_index *h, const float *X, int64_t N);

/* The same for uint8 vectors (e.g. .bvecs data): the exact distances are
 * those of their float copies, with a quarter of the device memory. */
int scg_load_raw_u8(scg_index *h, const uint8_t *X, int64_t N);

/* Query-independent tables: ||c||^2, ||r||^2, 2<c,r> and the per-vector ADC
 * term of the fast form.  Replaces PQQuery::pre_compute1 (query.h:91-149). */
int scg_precompute(scg_index *h);

/* Batched search with HOST buffers (batches of 1024 or more queries run in
 * 2 or 4 chunks over two streams, so that copies overlap the search):
 * Q[nq][dim] in, ids[nq][R], dists[nq][R],
 * sums[nq] out (sums may be NULL).  Each query returns its top min(R, sum)
 * candidates in ascending distance (equal distances by id); unused slots hold
 * id -1 and distance +inf.  `sum` is the candidate count the reference
 * returns by reference.  Replaces one call per query of search_ivfadc
 * (query.h:202), search_multi2 (multi_query.h:62) or search_mr_ivf
 * (sc_query.h:60); per-query tables (pre_compute2, query.h:154-184) are built
 * inside. */
int scg_search(scg_index *h, const scg_search_params *p, const float *Q, int nq,
               int *ids, float *dists, int *sums);

/* The same with DEVICE buffers, enqueued on `stream` (a cudaStream_t, or NULL
 * for the index's own stream); returns once the work is enqueued and
 * synchronises only to read the status word. */
int scg_search_device(scg_index *h, const scg_search_params *p, const float *dQ, int nq,
                      int *d_ids, float *d_dists, int *d_sums, void *stream);

/* scg_search_device replayed from a CUDA graph: the first call with a given
 * set of arguments (parameters, buffers, batch size, stream, per-query
 * targets) runs the search once, captures its launch sequence (tables,
 * coarse prefixes, selection, scan, re-rank, status copy) on `stream` (which
 * must be the caller's, not NULL) and instantiates it; later calls with the
 * same arguments launch the graph (one launch instead of about eight).  The
 * buffers' contents may change between calls, their addresses may not.
 * Synchronises to read the status word, like scg_search_device.  No
 * counterpart in the reference. */
int scg_search_graph(scg_index *h, const scg_search_params *p, const float *dQ, int nq,
                     int *d_ids, float *d_dists, int *d_sums, void *stream);

/* scg_search_device without any device allocation, for callers that cannot
 * allocate at search time (a memory pool that forbids cudaMalloc, or an
 * allocator owned by someone else).  No counterpart in the reference.  All
 * scratch -- per-query tables, cell records, scan survivors -- comes from one
 * 48 MiB file-scope device array that every GPU loading the library holds
 * until exit.  Limits: the per-query tables of nq queries must fit beside the
 * search slots (SCG_ERR_CAP names the largest nq for the index), and each
 * query may enumerate at most 8192 cells and keep 8192 scan survivors
 * (SCG_ERR_CAP otherwise).  The first call on a device looks up the array's
 * device address; make that first call before any stream capture.  Like
 * scg_search_device, every call synchronises `stream` to read the kernels'
 * status word before it returns.  Every call shares the one array: calls that
 * overlap on the GPU (other streams, other threads, the same device) race and
 * must be serialised by the caller.  The tensor-core forms (SCG_FAST,
 * SCG_BF16, SCG_FP16) need the per-vector term, built by an earlier call of
 * scg_search or scg_search_device in one of them (SCG_ERR_STATE otherwise). */
int scg_search_device_noalloc(scg_index *h, const scg_search_params *p, const float *dQ, int nq,
                              int *d_ids, float *d_dists, int *d_sums, void *stream);

/* Batched pre_compute2 (query.h:154-184, with the sequencing of lines 167
 * and 179 as intended): d_diff_qc[nq][mc*kc] = ||c||^2 - 2<q_part, c> and
 * d_diff_qr[nq][mp*kp] = ||r||^2 - 2<q_sub, r>, device buffers, in the
 * arithmetic of `precision` (SCG_FP32_EXACT: bit-identical to the
 * reference). */
int scg_query_tables_device(scg_index *h, int precision, const float *dQ, int nq,
                            float *d_diff_qc, float *d_diff_qr, void *stream);

/* Autotuner of the scan's chunking: times the fused search kernel on the
 * given device batch with 2, 4 and 8 candidates per lane per claimed chunk
 * (64, 128, 256 candidates per warp claim), keeps the fastest for this
 * index and the scan form of p->precision, and reports it (*choice; ms[3]
 * the best time of each, may be NULL).  Outputs are written as by
 * scg_search_device.  No counterpart in the reference. */
int scg_autotune(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids,
                 float *d_dists, int *d_sums, int *choice, float *ms);

/* Record of scg_autotune_ex: each knob's candidates with their best device
 * time (ms, tables + selection + scan + re-rank of the batch) and the pick. */
typedef struct {
    int upl;                   /* scan candidates per lane: 2, 4 or 8          */
    float upl_ms[3];
    int prefix;                /* sorted coarse-prefix length: 0 (the density
                                  rule), 128, 256 or 512                       */
    float prefix_ms[4];
    int split;                 /* 1: selection and scan as two kernels,
                                  0: one fused kernel                          */
    float split_ms[2];         /* [0] split, [1] fused                         */
    int shortlist;             /* rerank > 0: the shortlist length to use (the
                                  fastest tried whose top-R ids equal those of
                                  p->rerank on >= min_agree of the queries)    */
    int shortlist_L[5];        /* lengths tried: R, 2R, 4R, ... <= 1024        */
    float shortlist_ms[5];
    float shortlist_agree[5];  /* share of queries with the same top-R ids     */
} scg_tune_record;

/* Wider autotuner: on the given device batch, times the scan's candidates
 * per lane, the sorted coarse-prefix length and the kernel organisation in
 * turn and keeps the fastest of each for this index (the results of a
 * search do not depend on any of them); with p->rerank > 0 it also times
 * shortlists of R, 2R, 4R, ... <= 1024 candidates and reports the fastest one
 * that keeps the top-R ids of p->rerank on >= min_agree of the queries
 * (advice: the caller sets rerank).  Outputs are written as by
 * scg_search_device.  No counterpart in the reference. */
int scg_autotune_ex(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids,
                    float *d_dists, int *d_sums, float min_agree, scg_tune_record *rec);

/* Sets the scan's candidates per lane (2, 4 or 8) for the scan form of
 * `precision` without timing. */
int scg_set_scan_tuning(scg_index *h, int precision, int upl);

/* Kernel organisation of the search: on (the default), cell selection and
 * the ADC scan run as two persistent kernels (the scan kernel holds more
 * resident warps per SM); off, as one fused kernel.  Both give identical
 * results; SCG_SC3 searches always use the fused kernel. */
int scg_set_kernel_split(scg_index *h, int on);

/* Per-query candidate targets (device pointer to nq ints) for the next
 * scg_search_device call; NULL restores the single T of the parameters. */
int scg_set_query_targets(scg_index *h, const int *d_T);

/* Rank limit M of the coarse lists (the M argument of search_multi2,
 * multi_query.h:62-128; search_mr_ivf, sc_query.h:60-106; search_mr_ivf3):
 * the IMI and second-candidate walks of later searches use only ranks
 * 0..M-1 of each sorted coarse list, and stop when that grid is exhausted.
 * 0 (the default) or M >= kc: all ranks.  The reference sorts only the top
 * M ranks but lets its walk continue into the unsorted rest; where its walk
 * stays inside ranks 0..M-1 the two agree.  IVFADC has no rank limit. */
int scg_set_rank_limit(scg_index *h, int M);

/* Budgets of the traversal: the most cells one query may enumerate
 * (default 131072).  Larger budgets cost device memory per resident CTA. */
int scg_set_cell_budget(scg_index *h, int max_cells);

/* Encoder: X[n][dim] float rows -> cid[n][mc] (uint16) and codes[n][mp]
 * (uint8), first-minimum argmin with double accumulation exactly as
 * Encoder::encode<T> (encoder.h:69-192).  Host buffers. */
int scg_encode(scg_index *h, const float *X, int64_t n, uint16_t *cid, uint8_t *codes);

/* Second-candidate encoder (mc = 1): cid[n][nc] nearest coarse centroids in
 * ascending distance, codes of the residual to the nearest, as
 * SCEncoder::encode<T> (sc_encoder.h:205-332).  Host buffers. */
int scg_sc_encode(scg_index *h, const float *X, int64_t n, int nc, uint16_t *cid,
                  uint8_t *codes);

/* Index build on the device: encodes dX[n][dim] (device rows, ids 0..n-1;
 * nc = 0 IVF/IMI codes with kc^mc cells, nc = 2 or 3 second-candidate codes
 * with kc^nc cells), orders the rows by cell and by id inside a cell, and
 * loads the resulting CSR into the index -- the arrays Encoder::distribution /
 * SCEncoder::distribution write and load_encoded_data reads back
 * (encoder.cpp:170-305, sc_encoder.cpp:17-182, query.cpp:82-165).  With
 * nc = 3 a row's cell is its own (nn1, nn2, nn3); the reference's
 * distribution reads a misaligned window of the centroid ids there
 * (sc_encoder.cpp:41-59 advances by 2 per row). */
int scg_build_index(scg_index *h, const float *dX, int64_t n, int nc, void *stream);

/* Writes the index's CSR as an .edat_ file (int32 non-empty cells, int32 N,
 * then per cell in id order: int32 L, int32 pid[L], uint8 codes[L][mp]), the
 * format of Encoder::output (encoder.cpp:230-305), with 64-bit file offsets. */
int scg_write_edat(scg_index *h, const char *path);

/* Codebook training on device `device` (stream may be NULL): from n training
 * rows dX[n][dim] on the device, the coarse codebook d_cq[mc][kc][dim/mc]
 * (kc = 1: the zero centroid of plain PQ) and the residual PQ codebook
 * d_pq[mp][kp][dim/mp], each by k-means++ seeding (seeded, deterministic)
 * and `iters` Lloyd steps with FP64 centroid means; assignments use
 * tensor-core distance tables.  Replaces PQQuantizer::create_sub_quantizers
 * / calc_residual_vector (quantizer.h:235-272, 456-510) with greg_kmeans
 * (k-means.h:671-912), whose Lloyd loop stops after one pass. */
int scg_train_codebooks(const float *dX, int64_t n, int dim, int mc, int kc, int mp, int kp, int iters,
                        uint64_t seed, float *d_cq, float *d_pq, int device, void *stream);

/* k-means of nseg segments at once, HOST buffers: X[n][dim] (segment j =
 * dims [j dim/nseg, (j+1) dim/nseg)), centers[nseg][k][dim/nseg] and labels
 * [nseg][n] (may be NULL) out; k-means++ seeding (deterministic per seed) and
 * `iters` Lloyd steps with FP64 means, on device `device`.  The clustering of
 * PQQuantizer::create_sub_quantizers (quantizer.h:235-272) with greg_kmeans
 * (k-means.h:671-912) replaced by the published algorithm. */
int scg_kmeans(const float *X, int64_t n, int dim, int nseg, int k, int iters, uint64_t seed,
               float *centers, int *labels, int device);

/* Exact nearest neighbour of each query among base rows, all buffers on the
 * device: dX[n][dim] and dQ[nq][dim] float32 in, d_ids[nq] (row index) and
 * d_dists[nq] (may be NULL; the squared distance of distance_l2_square --
 * float differences squared and summed in double, stored as float) out.
 * Equal distances keep the lowest row index.  The ground truth that
 * Evaluation::load_groundtruth / calc_recall (evaluation.h:34-92) read from
 * a file made outside the reference; candidates are ranked by tcgen05
 * split-BF16 distance tiles over chunks of rows and every row within their
 * error margin of the chunk minimum is re-scored exactly, so the result is
 * the brute-force argmin.  Synchronises `stream` before it returns. */
int scg_exact_nn(const float *dX, int64_t n, const float *dQ, int nq, int dim, int *d_ids, float *d_dists,
                 int device, void *stream);

/* Encoder arithmetic (scg_encode, scg_sc_encode, scg_encode_device, and the
 * index build).  SCG_ENC_TENSOR (the default): distances ranked by tcgen05
 * split-BF16 GEMM tiles, every centroid within the tiles' error margin of the
 * minimum (of the nc-th smallest, for the second candidate's nc nearest
 * coarse centroids) re-scored with the reference's double arithmetic and its
 * float-rounded comparisons where it has them -- the codes are the
 * reference's.  SCG_ENC_EXACT: every distance in double (one thread per
 * row). */
#define SCG_ENC_EXACT 0
#define SCG_ENC_TENSOR 1
int scg_set_encoder(scg_index *h, int method);

/* Device-buffer form of the two encoders (X, cid, codes on the device). */
int scg_encode_device(scg_index *h, const float *dX, int64_t n, int nc, uint16_t *d_cid,
                      uint8_t *d_codes, void *stream);

/* Per-query facts of the last search call on this index: visited non-empty
 * cells and visited empty cells (the `e` output of search_multi2,
 * multi_query.h:170), host buffers of nq ints (either may be NULL). */
int scg_last_query_stats(scg_index *h, int *nvis, int *empty, int nq);

/* Device time in milliseconds of the kernels of the last search call,
 * measured with CUDA events on its stream: ms[0] the per-query tables and
 * coarse-list prefixes, ms[1] cell selection + scan, ms[2] the shortlist
 * re-rank (0 without one), ms[3] and ms[4] the selection kernel and the scan
 * kernel alone when they ran as two kernels (0 otherwise).  After scg_search (host buffers), which
 * runs large batches in chunks over two streams, the figures are those of
 * the last chunk on the index's own stream.  n is the capacity of ms. */
int scg_last_timings(scg_index *h, float *ms, int n);

/* Kernels the index's last search launched on its own stream: the tables,
 * query norms, coarse prefixes, selection, scan, top-R merge and re-rank
 * kernels that ran (and the per-vector term when that call built it; a
 * search the pool sent to the fused kernel counts both runs).  After
 * scg_search (host buffers) the figure is that of the last chunk on the
 * index's own stream.  No counterpart in the reference (no GPU code). */
int scg_last_launches(scg_index *h, int *count);

/* Copies the cell lengths back as the reference's inclusive prefix L[ncells]
 * (the array PQQuery::entropy reads, query.cpp:168-182). */
int scg_cell_counts(scg_index *h, int *L, int64_t ncells);

/* Diagnostics: with counters on, each search accumulates per-phase cycle
 * counts of the search kernels (thread 0 of every CTA, summed over queries):
 * [0] coarse-list sort, [1] staircase rounds' enumeration, [2] cut,
 * [3] compaction, [4] scan rounds, [5] final merge inside the scan kernel
 * (for a query handed to the warp-wide merge kernel: the hand-off only),
 * [6] scan survivors,
 * [7] queries the warp-wide selection deferred, [8] rounds, [9] bisection steps, [10] enumerated cells,
 * [11] complete sorts, [14] the rounds' bisections, in the scan-only
 * kernel [12] the LUT (or query) staging and [13] the warm-up scores and
 * threshold, and [15] the warp-wide selection (per query, every phase; the
 * block-wide counters then cover the queries it deferred).  n is the
 * capacity of out (<= 16). */
int scg_set_phase_counters(scg_index *h, int on);
int scg_last_phase_counters(scg_index *h, long long *out, int n);

/* ------------------------------------------------------------------------
 * Request loop with continuous batching.  No counterpart in the reference
 * (its query objects serve one query per call on the calling thread).
 *
 * A server holds `slots` CUDA streams, each with its own search workspace,
 * and a device arena of `arena_bytes` for per-request buffers (queries,
 * tables, outputs).  Requests -- a batch of 1..max_batch queries with its own
 * parameters (R <= max_R, T, w, precision, rerank) -- are submitted from any
 * thread with HOST buffers that must stay valid until the request is waited
 * for.  A worker thread admits requests in arrival order whenever a slot is
 * free and the arena has room, runs them concurrently on the device, and
 * completes them as their streams finish.  A request larger than the arena is
 * refused at submit (SCG_ERR_CAP).  Results are identical to the same request
 * alone.  The index must not be reloaded while a server runs on it. */
typedef struct scg_server scg_server;

int scg_server_create(scg_index *h, int slots, int max_batch, int max_R, size_t arena_bytes,
                      scg_server **out);

/* Queues a request; *ticket identifies it to scg_server_wait. */
int scg_server_submit(scg_server *s, const scg_search_params *p, const float *Q, int nq,
                      int *ids, float *dists, int *sums, uint64_t *ticket);

/* Waits for a request (timeout_s < 0: without limit).  Returns its status,
 * or SCG_PENDING if the timeout expired first (the ticket stays valid).  On
 * completion *latency_ms (may be NULL) is the time from submit to the end of
 * its copy-out, and the ticket is released. */
int scg_server_wait(scg_server *s, uint64_t ticket, double timeout_s, double *latency_ms);

/* The same with times_ms[3] (may be NULL): submit to completion, submit to
 * admission (time queued for a slot or memory), admission to completion. */
int scg_server_wait_times(scg_server *s, uint64_t ticket, double timeout_s, double *times_ms);

/* Completed requests, the most requests ever in flight at once, and the
 * requests waiting for a slot or memory now. */
int scg_server_stats(scg_server *s, long long *completed, int *max_inflight, int *queued);

/* Finishes every queued and running request, then frees the server.
 * Tickets not yet waited for are released. */
int scg_server_destroy(scg_server *s);

/* cudaMalloc calls the library has made for its own device buffers in this
 * process so far (index arrays, search workspaces, arenas; never the
 * caller's buffers).  A server reserves every per-slot buffer at
 * scg_server_create, so serving requests of up to max_batch queries adds
 * none: a cudaFree inside the request loop would wait for every slot.  No
 * counterpart in the reference (it allocates no device memory). */
int scg_device_allocations(long long *count);

/* Index facts: dim, mc, kc, mp, kp, N (any pointer may be NULL). */
int scg_index_info(scg_index *h, int *dim, int *mc, int *kc, int *mp, int *kp, int64_t *N);

#ifdef __cplusplus
}
#endif
#endif
