/*
 * fap_b200.h -- C ABI of the B200 (sm_100a) per-subgraph APSP solve path.
 *
 * Every function returns an int status (FAP_OK = 0, negative on error; the
 * message is in fap_last_error(), per host thread).  Nothing calls exit().
 * Handles are not thread-safe: use one fap_ctx per host thread.
 *
 * The path replaces the reference's kernel ABI
 *   fap/kernel/cuda/cuda_kernel.h:21-24  handle_boundry_Nvidia_GPU  (stage 1, SSSP)
 *   fap/kernel/cuda/cuda_kernel.h:29     floyd_GPU_Nvidia_path      (stage 2, Floyd)
 *   fap/kernel/cuda/cuda_kernel.h:41-42  minplus_NVIDIA_path        (stage 3, min-plus)
 * and the per-part driver fapGraph::run (fap/fap.cpp:92-181) that calls them
 * with the host gather/scatter of fap/utils/util_Myalgorithm.h:30-95.
 * Those three legacy symbols, with their exact C++ signatures, are exported
 * as well (include/fap_legacy_kernel.h).
 *
 * Layout conventions
 *   - Vertex ids are 0-based int32.  Part ids in this ABI are 1-based, like
 *     the reference's graph_id (fap/utils/readIdFile.h:127-131).
 *   - The distance output of a graph is one row-major matrix with n rows and
 *     a leading dimension ld >= n (padded to a multiple of 128 elements).
 *     Row r is the vertex at sorted position r (st2ed[r]); column j is
 *     vertex j.  Part p owns rows ver_offset[p] .. ver_offset[p]+ver_num[p]-1,
 *     its boundary vertices first: exactly the reference's solve() layout
 *     (fap/fap.cpp:184-194).
 *   - Unreachable pairs hold the sentinel 1e8 (100000000 as int32).
 */
#ifndef FAP_B200_H_
#define FAP_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define FAP_API __attribute__((visibility("default")))
#else
#define FAP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define FAP_OK 0
#define FAP_ERR_INVALID (-1)     /* bad argument */
#define FAP_ERR_CUDA (-2)        /* CUDA runtime error */
#define FAP_ERR_NOMEM (-3)       /* device or host allocation failed / too large */
#define FAP_ERR_STATE (-4)       /* call out of order (e.g. solve before parts) */
#define FAP_ERR_NOT_CONVERGED (-5) /* SSSP hit its round bound */
#define FAP_ERR_RANGE (-6)       /* int32 path requested but weights not integral/in range */
#define FAP_ERR_IO (-7)          /* graph file missing or malformed */
#define FAP_ERR_PARTITION (-8)   /* METIS failed or partition invalid */
#define FAP_ERR_DEVICE (-9)      /* a kernel reported a device-side error */

/* ---- distance types ---- */
#define FAP_DTYPE_AUTO (-1) /* int32 when every weight is an integer <= FAP_MAX_INT_WEIGHT */
#define FAP_DTYPE_I32 0
#define FAP_DTYPE_F32 1
#define FAP_MAX_INT_WEIGHT 1000000

/* ---- solve forms ---- */
#define FAP_MODE_PLAIN 0   /* one launch sequence per part */
#define FAP_MODE_BATCHED 1 /* every stage of every requested part in one launch */

#define FAP_INF_I32 100000000
#define FAP_INF_F32 1e8f

typedef struct fap_ctx fap_ctx;
typedef struct fap_dgraph fap_dgraph;

/* Last error message of the calling host thread ("" if none). */
FAP_API const char *fap_last_error(void);
/* ABI version: 0xMMmmpp. */
FAP_API int fap_version(void);

/* ---- context: one CUDA device + one stream ----
 * Destroying a context whose graphs are still alive defers its release
 * until the last of those graphs is destroyed. */
FAP_API int fap_ctx_create(int device, fap_ctx **out);
FAP_API int fap_ctx_destroy(fap_ctx *ctx);
/* Use an external cudaStream_t (passed as void*); NULL = the context's own stream. */
FAP_API int fap_ctx_set_stream(fap_ctx *ctx, void *stream);
FAP_API int fap_ctx_get_stream(fap_ctx *ctx, void **stream);
FAP_API int fap_ctx_sync(fap_ctx *ctx);

/* ---- device-resident graph ----
 * Uploads the CSR (row_offset[n+1], col_val[m], weight[m] as the reference's
 * float weights, fap/fap.h:69-74).  dtype: FAP_DTYPE_AUTO / I32 / F32.
 * Host pointers; copied before return. */
FAP_API int fap_graph_create(fap_ctx *ctx, int32_t n, int64_t m, const int32_t *row_offset,
                     const int32_t *col_val, const float *weight, int dtype,
                     fap_dgraph **out);
FAP_API int fap_graph_destroy(fap_dgraph *g);
FAP_API int fap_graph_dtype(const fap_dgraph *g);

/* Sets the partition and renumbering produced on the host by findBoundry +
 * sort_and_encode (fap/utils/util_preprocess.h:32-106):
 *   graph_id[n]  1-based part of every vertex,
 *   st2ed[n]     vertex at each sorted position,
 *   ver_num[K+1], ver_offset[K+1], bdy_num[K+1]  per part, index 1..K.
 * Checks that they are consistent: st2ed a permutation, each part's block
 * holding only its own vertices, and both ends of every cross-part arc in
 * the first bdy_num[p] places of their part's block (FAP_ERR_PARTITION
 * otherwise).  Host pointers. */
FAP_API int fap_graph_set_parts(fap_dgraph *g, int32_t K, const int32_t *graph_id,
                        const int32_t *st2ed, const int32_t *ver_num,
                        const int32_t *ver_offset, const int32_t *bdy_num);

/* Reserves the output matrix for at most max_rows rows (0 = all n rows, or
 * as many as "max_resident_rows" allows; more than that bound fails with
 * FAP_ERR_NOMEM).  When max_rows < n, each fap_solve call may only request
 * parts whose rows fit; their blocks are packed from row 0 in request order. */
FAP_API int fap_graph_reserve(fap_dgraph *g, int64_t max_rows);

/* Solves the listed parts (1-based ids; parts == NULL means 1..K) into the
 * device-resident output.  mode: FAP_MODE_PLAIN or FAP_MODE_BATCHED.
 * Asynchronous on the context stream; errors from the device are reported by
 * fap_graph_check (or any call that synchronises). */
FAP_API int fap_solve(fap_dgraph *g, const int32_t *parts, int32_t count, int mode);

/* Synchronises and returns FAP_OK or the device-side error of the last solve. */
FAP_API int fap_graph_check(fap_dgraph *g);

/* Where part p's block lives: device pointer to its first row, rows, leading
 * dimension (elements).  Valid until the next fap_solve that reuses rows. */
FAP_API int fap_graph_block(fap_dgraph *g, int32_t part, void **dev_ptr, int64_t *rows, int64_t *ld);

/* Copies part p's block to host memory as a dense rows x n matrix of
 * out_dtype (FAP_DTYPE_F32 gives the reference's float values; I32 requires
 * the int32 path).  Synchronous. */
FAP_API int fap_graph_copy_block(fap_dgraph *g, int32_t part, void *host, int out_dtype);

/* The same copy queued without waiting for it (no counterpart in the
 * reference: its getters return host matrices).  slot (0 or 1) names one of
 * two copies in flight: from int32 to FAP_DTYPE_F32 the conversion runs on
 * the context stream into the slot's own staging buffer and the
 * device-to-host copy on the slot's stream, so that the next block's
 * conversion overlaps this block's copy.  A call on a slot first waits for
 * that slot's previous copy, which frees its host memory for reuse; the
 * staging buffer of a slot is allocated on its first use (cudaMalloc).
 * `host` must stay valid until fap_graph_copy_wait(slot) or the slot's next
 * call returns, and pinned host memory gives the full copy rate.  A copy
 * without conversion runs on the context stream. */
FAP_API int fap_graph_copy_block_async(fap_dgraph *g, int32_t part, void *host, int out_dtype, int32_t slot);
/* Waits for the slot's copy; then FAP_OK or the device-side error of the
 * last solve. */
FAP_API int fap_graph_copy_wait(fap_dgraph *g, int32_t slot);
#define FAP_COPY_SLOTS 2

/* Per-row checksums of part p's block (int32 path only):
 * sum_j uint32(d[r][j]) * (2j+1) mod 2^64, j < n.  host_out[rows]. */
FAP_API int fap_graph_block_checksums(fap_dgraph *g, int32_t part, uint64_t *host_out);

/* Shortest-distance rows from arbitrary sources over the graph's CSR
 * (distance-row requests, self-checks).  Host sources[count]; host
 * out[count * n] receives float distances (the reference's type). */
FAP_API int fap_graph_sssp_rows(fap_dgraph *g, const int32_t *sources, int32_t count, float *host_out);

/* Tuning knobs: "sssp_delta" (bucket width of the near/far SSSP; <= 0 or
 * >= 1e8 means plain frontier Bellman-Ford); "sssp_max_rounds" (round bound
 * after which a source gives up and the solve reports
 * FAP_ERR_NOT_CONVERGED; <= 0 restores the default 8n + 1024);
 * "floyd_per_cta" (non-zero: the batched Floyd closes each part's matrix
 * with one CTA instead of per-tile launches across all parts);
 * "sssp_chain" (hops a thread may follow within one SSSP round; 0 turns
 * chain-following off, the default); "cuda_graph" (non-zero, the default:
 * a batched solve captures its launch sequence in a CUDA graph on first use
 * and replays it while the batch, buffers, parameters and stream are
 * unchanged); "use_cache" (non-zero, the default: batched solves and
 * fap_graph_rows_async use the resident cache once it is built); "paths"
 * (non-zero: later solves also produce the parts' predecessor rows, see
 * fap_graph_path_block; needs every edge weight > 0, else FAP_ERR_RANGE);
 * "stage1" (0 automatic, the default; 1 always SSSP; 2 the boundary graph
 * whenever the graph allows it, whatever its dtype and boundary count; see
 * fap_graph_last_stage1); "bgraph_form" (how the boundary graph is closed
 * and expanded: 0 by size, the default, Floyd up to 8192 boundary vertices
 * and the tiled Bellman-Ford beyond, the staged expansion up to 4096 and the
 * tiled one beyond; 1 Floyd; 2 Bellman-Ford and the tiled expansion; the
 * Bellman-Ford closure checks convergence on the host, so such solves are
 * not captured in a CUDA graph); "sssp_form" (how the SSSP form of stage 1 runs:
 * 0 automatic, the default, tiled when the graph has at least 6 arcs per
 * vertex; 1 one CTA per source, near/far frontier; 2 tiled multi-source
 * Bellman-Ford, 128 sources per pass over the in-edges; the tiled form
 * checks convergence on the host, so a solve that uses it is not captured
 * in a CUDA graph); "tile_mb" (device memory for the 128-source tiles that
 * the tiled SSSP and the Bellman-Ford closure of the boundary graph run side
 * by side, at most 16 of them, at least one; default 384);
 * "minplus_pack16" (int32 graphs, default 1: a min-plus tile of a part with
 * more than 16 boundary vertices runs in packed 16-bit arithmetic, two
 * relaxations per DPX instruction, when its values provably fit: every
 * boundary-row column is shifted by its least finite entry and the part's
 * largest finite inner-to-boundary distance plus the tile's largest shifted
 * entry is below 16383; other tiles run in int32; the results are the same
 * int32 values either way; 0: int32 everywhere); "minplus_prepack" (default
 * 1: the packed tiles read operands packed once per solve, the boundary rows
 * as 16-bit columns and the inner-to-boundary distances with both halves
 * equal, and the packed tiles of the boundary graph's tiled expansion read
 * the dB rows as row pairs and the parts' boundary rows with both halves
 * equal, when those arrays fit in 8 GiB and a quarter of the free device
 * memory; 0, or when they do not fit: each tile converts its int32 stages
 * in shared memory; the same values either way); "floyd_queue" (default 1:
 * the batched Floyd-Warshall as one persistent launch over a device work
 * queue; 0: three launches per pivot block); "floyd_symmetric" (default 1:
 * on parts whose arcs all have reverses of equal weight, the queue computes
 * the local closures' tiles on and above the diagonal and stores their
 * transposes); "thin_max_b" (0..16, default 16: parts with at most this many
 * boundary vertices take the store-shaped thin min-plus kernel, the others
 * the register-tiled one); "max_resident_rows" (>= 1: at most this many
 * output rows are reserved on the device, as when HBM cannot hold all n
 * rows; blocks already reserved beyond it are released; 0, the default: no
 * bound). */
FAP_API int fap_graph_set_param(fap_dgraph *g, const char *key, double value);

/* Diagnostics (no GPU work): builds the Floyd work queue's item list for
 * parts of the given sizes (sym: the symmetric items) and checks that every
 * item's dependencies come earlier in the list and that every item appears
 * once (the persistent launch's waits end only then); FAP_OK when they do,
 * FAP_ERR_STATE otherwise. */
FAP_API int fap_queue_order_check(const int32_t *part_sizes, int32_t nparts, int sym);

/* Min-plus tiles run in the packed 16-bit form and in all, counted over
 * every solve of g so far (see "minplus_pack16").  Synchronous. */
FAP_API int fap_graph_pack16_tiles(fap_dgraph *g, int64_t *packed, int64_t *total);
/* The same for the tiles of the boundary graph's tiled expansion (int32,
 * Bellman-Ford closure of the boundary graph): rows of the closed boundary
 * graph are shifted by their least finite entry per part, and a tile runs
 * packed when that part's largest finite boundary-row distance plus the
 * tile's largest shifted entry is below 16383. */
FAP_API int fap_graph_expand16_tiles(fap_dgraph *g, int64_t *packed, int64_t *total);

/* Tunes the SSSP bucket width: runs the SSSP stage on `sample` boundary
 * sources spread over all parts (0 = one full wave of CTAs) for each of the
 * `count` candidate deltas (>= 1e8 or <= 0 = plain Bellman-Ford), keeps the
 * fastest for later solves and returns it in *best_delta; ms_out[count]
 * (optional) receives each candidate's time.  Needs the partition. */
FAP_API int fap_graph_tune_sssp(fap_dgraph *g, const double *deltas, int32_t count, int32_t sample,
                                double *best_delta, float *ms_out);

/* Mean edge weight of the graph (the scale SSSP bucket widths are tuned in). */
FAP_API double fap_graph_mean_weight(const fap_dgraph *g);

/* ---- sharded boundary-graph form (parts split over ranks, one process
 * per GPU; the multi-GPU form of fap/fap_more_task_mpi.cpp:34-80) ----
 * fap_graph_shard_begin closes this rank's own parts locally (the
 * boundary-graph form's local closures, in the resident cache's Floyd
 * arena) and packs their boundary rows into `send` (device memory of the
 * graph's dtype, send_cap elements): the own parts in ascending order, each
 * part's rows 0..b-1, columns 0..s-1, row-major; *send_elems receives the
 * count.  The caller then gathers every rank's send buffer into one device
 * buffer, rank r's at r * stride (e.g. an NCCL all-gather of buffers padded
 * to `stride` elements).  fap_graph_shard_finish takes that buffer and
 * owner[p] (the rank of part p, p = 1..K; index 0 unused), closes the
 * boundary graph (the same work on every rank), expands the boundary rows of
 * the own parts and makes their closures exact: the resident cache then
 * holds the own parts, and fap_solve(g, own parts, FAP_MODE_BATCHED) runs
 * their min-plus merge (other parts are refused with FAP_ERR_STATE until
 * the cache is built or dropped again).  Needs the boundary-graph form
 * (int32 graph without duplicate arcs inside a part) and "floyd_queue". */
FAP_API int fap_graph_shard_begin(fap_dgraph *g, const int32_t *own_parts, int32_t count, void *send,
                                  int64_t send_cap, int64_t *send_elems);
FAP_API int fap_graph_shard_finish(fap_dgraph *g, const void *recv, int32_t world, const int32_t *owner,
                                   int64_t stride);

/* Frees the output matrix, Floyd arena and scratch of g (the CSR, the
 * partition and the resident cache stay); no block stays resident
 * afterwards. */
FAP_API int fap_graph_release(fap_dgraph *g);
/* Device bytes g holds now. */
FAP_API int fap_graph_device_bytes(const fap_dgraph *g, int64_t *bytes);
/* 1 if part's block is resident in g's output matrix, else 0. */
FAP_API int fap_graph_resident(fap_dgraph *g, int32_t part);
/* Queues, on the context stream, shortest-distance rows from count sources
 * (host ids) into d_out (device, count x n floats, dense); returns without
 * waiting.  Device errors surface in fap_graph_check. */
FAP_API int fap_graph_rows_async(fap_dgraph *g, const int32_t *sources, int32_t count, float *d_out);

/* Predecessor rows of a resident part solved with "paths" on (the
 * reference's subgraph_path, fap/fap.cpp:92-181, is_path_needed): entry
 * (r, j) is the vertex before j on a shortest path from the part's r-th
 * vertex (sorted order), the vertex itself at j = source, -1 when j is
 * unreachable.  Among several shortest paths the one kept is fixed: the
 * in-neighbour u of j with the least dist(r, u) + w(u, j), the smallest u on
 * equal sums (the reference keeps the first its evaluation order finds; the
 * two agree wherever the predecessor is unique).  Same layout as
 * fap_graph_block: int32, rows x ld, ld = ldD. */
FAP_API int fap_graph_path_block(fap_dgraph *g, int32_t part, void **dev_ptr, int64_t *rows, int64_t *ld);
/* rows x n int32 predecessors of the part into host memory. */
FAP_API int fap_graph_copy_path_block(fap_dgraph *g, int32_t part, int32_t *host);

/* Asynchronous forms for pipelines that must not block: queue, on the
 * context stream, the per-row checksums of a resident part's block into
 * device memory (rows x uint64, int32 path), and a copy of the graph's
 * device status word into host memory (pinned for the copy to be
 * asynchronous).  Once the stream has passed the copy, fap_status_code turns
 * the word into FAP_OK or the error code fap_graph_check would return. */
FAP_API int fap_graph_checksums_async(fap_dgraph *g, int32_t part, uint64_t *d_out);
FAP_API int fap_graph_status_async(fap_dgraph *g, int32_t *host_status);
FAP_API int fap_status_code(int32_t device_status);

/* Resident cache for serving (no counterpart in the reference, which
 * recomputes every part's stages 1-2 on each solveSubGraph): computes, on
 * the context stream, the boundary rows of every part (stage 1 for all
 * boundary vertices) and every part's closed Floyd matrix (stage 2), and
 * keeps both in HBM.  Later batched solves then copy the parts' boundary
 * rows and run only the min-plus merge; fap_graph_rows_async computes a
 * row as the min-plus of the source's closed Floyd row with its part's
 * boundary rows.  Both give exactly the values of the uncached path (the
 * same min over the same sums).  Returns once the cache is built (its SSSP
 * scratch is freed again); device errors surface in fap_graph_check; a new
 * partition drops the cache. */
FAP_API int fap_graph_cache_build(fap_dgraph *g);
/* Computes the resident cache again even when it is built, in the same
 * buffers (fap_graph_cache_build returns at once when the cache exists):
 * stages 1-2 of every part, e.g. once per pass of a job whose output is
 * produced in groups of parts. */
FAP_API int fap_graph_cache_rebuild(fap_dgraph *g);
/* Device time of the last cache build's phases, ms4[4]: built with the
 * boundary graph, [local closures (gather + Floyd), boundary-graph closure,
 * expansion into the boundary rows, fix-up of the closures]; built with
 * SSSP, [SSSP, gather, Floyd, 0].  FAP_ERR_STATE without a cache. */
FAP_API int fap_graph_cache_timing(const fap_dgraph *g, float *ms4);
FAP_API int fap_graph_cache_release(fap_dgraph *g);
/* Device bytes the cache holds (*built = 1) or would need to be built,
 * including its SSSP scratch (*built = 0). */
FAP_API int fap_graph_cache_bytes(const fap_dgraph *g, int64_t *bytes, int *built);

/* Device time (ms) of the stages of the last fap_solve, measured with events
 * on the context stream: [sssp, gather, floyd, minplus, total]. */
FAP_API int fap_graph_last_timing(fap_dgraph *g, float *ms5);

/* How the last fap_solve obtained the boundary rows (stage 1): 1 SSSP from
 * every boundary vertex; 2 the boundary graph (every part's local closure,
 * APSP over the boundary vertices, expansion; chosen for batches of all
 * parts of int32 graphs without two arcs joining the same ordered pair
 * inside a part, when they have at most 8192 boundary vertices (closed by
 * Floyd) or when the boundary graph has at most 8 edges per graph edge and
 * at most 65536 vertices (closed by the tiled Bellman-Ford); with "stage1" =
 * 2 also for float32 graphs, whose results then differ from the SSSP form by
 * rounding order, a few ulps); 3 the resident cache; 0 no solve yet. */
FAP_API int fap_graph_last_stage1(const fap_dgraph *g);

/* How stage 1 of the last solve ran, in words: "SSSP, frontier", "SSSP,
 * tiled Bellman-Ford", "boundary graph, Floyd closure", "boundary graph,
 * Bellman-Ford closure", or "resident cache (<how it was built>)"; "" before
 * the first solve.  The string lives until the next solve or cache build. */
FAP_API const char *fap_graph_stage1_name(const fap_dgraph *g);

/* Number of kernels the last fap_solve launched. */
FAP_API int fap_graph_last_launches(fap_dgraph *g, int64_t *count);

/* ---- device-pointer operators (the three stages on their own) ----
 * All pointers are device pointers; run on the context stream. */

/* Stage 1: one shortest-path row per source over the CSR.  out row i
 * (out + i*ld_out) receives the distances from sources[i] to every vertex.
 * weight is int32* for FAP_DTYPE_I32, float* for FAP_DTYPE_F32. */
FAP_API int fap_op_sssp(fap_ctx *ctx, int dtype, int32_t n, int64_t m, const int32_t *row_offset,
                const int32_t *col_val, const void *weight, const int32_t *sources,
                int32_t num_sources, void *out, int64_t ld_out);

/* Stage 2: in-place Floyd-Warshall closure of an s x s matrix (leading
 * dimension ld).  The whole GPU works on the one matrix. */
FAP_API int fap_op_floyd(fap_ctx *ctx, int dtype, int32_t s, void *mat, int64_t ld);

/* Stage 3: C[i][j] = min(1e8, min_k A[i][k] + B[k][j]) for an M x N result,
 * inner dimension K (row-major, leading dimensions lda, ldb, ldc). */
FAP_API int fap_op_minplus(fap_ctx *ctx, int dtype, int32_t M, int32_t N, int32_t K,
                   const void *A, int64_t lda, const void *B, int64_t ldb, void *C,
                   int64_t ldc);

/* ---- allocation-free closure (no counterpart in the reference) ----
 * For callers that may not allocate device memory when they need a closure:
 * a host framework that owns the GPU's memory through its own pool (a
 * database or serving plugin), or a latency-sensitive path where cudaMalloc /
 * cudaFree would implicitly synchronise the device.  Same result as
 * fap_op_floyd (in-place Floyd-Warshall of an s x s device matrix, leading
 * dimension ld, dtype FAP_DTYPE_I32 or FAP_DTYPE_F32), but it allocates
 * nothing and needs no fap_ctx: its padded working copy lives in one 4 MiB
 * device array built into the library, which every GPU that loads the
 * library keeps until the process exits.
 *   - s is limited to FAP_NOALLOC_FLOYD_MAX; larger sizes return
 *     FAP_ERR_RANGE before any GPU work.
 *   - Work is queued on `stream` (a cudaStream_t; NULL = the legacy default
 *     stream) and the call returns without waiting: synchronise the stream
 *     before reading mat.
 *   - Every call on a device uses the same array, so calls whose GPU work
 *     overlaps (different streams, or host threads, on one device) race and
 *     corrupt each other: serialise them.
 *   - Each call outside a stream capture looks up the array's device
 *     address (so a cudaDeviceReset in between is harmless); inside a
 *     capture the last lookup on that device is used, so make the first
 *     call on a device before any stream capture.
 *   - The call returns before the GPU work ends, so a device-side failure (a
 *     bounded TMA wait in the closure that gave up) cannot be its return
 *     value: after synchronising the stream, fap_floyd_noalloc_status()
 *     returns FAP_OK, or FAP_ERR_DEVICE when the last call's closure did not
 *     complete (mat then holds no valid closure).
 * Messages: fap_floyd_noalloc_last_error(). */
#define FAP_NOALLOC_FLOYD_MAX 1024
FAP_API int fap_floyd_noalloc(int dtype, int32_t s, void *mat, int64_t ld, void *stream);
FAP_API const char *fap_floyd_noalloc_last_error(void);
/* Device-side status of the last fap_floyd_noalloc call on the current
 * device (a status word beside the built-in array, cleared by each call).
 * Read it only after that call's stream has been synchronised; it copies
 * 4 bytes to the host and allocates nothing. */
FAP_API int fap_floyd_noalloc_status(void);

/* Measured relaxation throughput of this device (relaxations/s) for the
 * given dtype, from a register-resident microbenchmark. */
FAP_API int fap_measure_relax_peak(fap_ctx *ctx, int dtype, double *relax_per_s);

#ifdef __cplusplus
}
#endif
#endif /* FAP_B200_H_ */
