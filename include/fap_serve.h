/*
 * fap_serve.h -- serving loop over resident graphs (no counterpart in the
 * reference, whose fapGraph solves one part per call on the caller's thread).
 *
 * A server owns one CUDA device.  Graphs are added once (CSR + partition
 * stay resident in HBM).  Clients submit requests from any thread:
 *   FAP_REQ_SUBGRAPH  the block of one part (ver_num[part] x n distances,
 *                     what solveSubGraph computes, fap/fap.cpp:197-207);
 *   FAP_REQ_ROWS      shortest-distance rows from a list of source vertices.
 * A worker thread batches pending requests per graph (all sub-graph requests
 * of a graph that fit one batch run as one batched solve; a request for a
 * part that is still resident from an earlier batch is answered without
 * recomputing), admits a batch only when its estimated device footprint
 * fits the memory budget (idle graphs' output buffers, then their caches,
 * are released first), and runs each graph on its own stream, so batches of
 * different graphs overlap on the GPU while new requests keep arriving
 * (continuous batching).  On a graph's first batch the server builds its
 * resident cache (fap_graph_cache_build: every part's boundary rows and
 * closed Floyd matrix) when it fits, after which sub-graph batches run only
 * the min-plus merge and distance rows come from the cache.
 * Results are copied to the caller's host buffers (float distances) and/or
 * reduced to per-row checksums (int32 graphs).
 */
#ifndef FAP_SERVE_H_
#define FAP_SERVE_H_

#include <stdint.h>

#include "fap_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fap_server fap_server;

#define FAP_REQ_SUBGRAPH 0
#define FAP_REQ_ROWS 1

#define FAP_REQ_PENDING 0
#define FAP_REQ_RUNNING 1
#define FAP_REQ_DONE 2
#define FAP_REQ_FAILED 3

/* budget_bytes: device memory the server may hold for outputs and scratch
 * (<= 0: 60% of the free memory at creation).  max_batch_rows: output rows of
 * one batch (<= 0: no limit beyond the budget). */
FAP_API int fap_server_create(int device, double budget_bytes, int64_t max_batch_rows,
                              fap_server **out);
/* Limits, changeable while the server runs: "max_batch_bytes" (output bytes
 * of one batch beyond its first request, and the size each graph's batch
 * buffers are allocated at once; default 512 MiB, <= 0: no limit),
 * "max_batch_rows" (<= 0: no limit), "budget_bytes" (> 0). */
FAP_API int fap_server_set_option(fap_server *s, const char *key, double value);

/* Waits for the requests in flight, fails the queued ones, frees everything. */
FAP_API int fap_server_destroy(fap_server *s);

/* Adds a resident graph: CSR (weights as float, see fap_graph_create) and
 * its partition / renumbering (see fap_graph_set_parts).  Host pointers,
 * copied.  *index receives the graph's index for fap_server_submit. */
FAP_API int fap_server_add_graph(fap_server *s, int32_t n, int64_t m, const int32_t *row_offset,
                                 const int32_t *col_val, const float *weight, int dtype, int32_t K,
                                 const int32_t *graph_id, const int32_t *st2ed,
                                 const int32_t *ver_num, const int32_t *ver_offset,
                                 const int32_t *bdy_num, int32_t *index);

/* Submits a request.  FAP_REQ_SUBGRAPH: ids = {part} (count 1, 1-based);
 * FAP_REQ_ROWS: ids = source vertices (count >= 1).  host_out (optional)
 * receives rows x n float distances; checksums_out (optional, int32 graphs,
 * either kind) receives one checksum per row (fap_graph_block_checksums'
 * definition).
 * Both must stay valid until the request is done.  *req_id identifies it. */
FAP_API int fap_server_submit(fap_server *s, int32_t graph, int kind, const int32_t *ids,
                              int32_t count, float *host_out, uint64_t *checksums_out,
                              int64_t *req_id);

/* Waits up to timeout_s (< 0: forever) for a request; *state receives
 * FAP_REQ_*.  A done or failed request stays queryable until forgotten. */
FAP_API int fap_server_wait(fap_server *s, int64_t req_id, double timeout_s, int *state);

/* Per-request figures: out4 = [latency ms (submit -> done), queue ms
 * (submit -> start on the GPU), entries (rows x n), status (FAP_* code)]. */
FAP_API int fap_server_request_info(fap_server *s, int64_t req_id, double *out4);

/* Drops a finished request's record. */
FAP_API int fap_server_forget(fap_server *s, int64_t req_id);

/* Waits until every submitted request is done or failed. */
FAP_API int fap_server_drain(fap_server *s);

/* Figures over the requests finished since the last reset; out[i] for
 * i < count (entries past FAP_SERVER_NSTATS read 0):
 *   0 requests completed   1 entries produced      2 p50 latency ms
 *   3 p99 latency ms       4 mean latency ms       5 peak device bytes held
 *   6 batches launched     7 answered from resident blocks
 *   8 requests failed      9 resident caches built 10 device busy ms (sum of
 *   the finished batches' durations, over all graphs' streams)
 *   11-18 the longest single host call of the worker thread, in ms, by kind
 *   (one worker serves every graph, so a slow call delays every graph's next
 *   batch): 11 assembling and queueing one batch (12-18 are parts of it or
 *   follow it), 12 retiring one finished batch, 13 building a resident cache,
 *   14 admission / eviction, 15 output buffer growth, 16 queueing a
 *   sub-graph solve, 17 queueing a distance-row batch, 18 queueing its
 *   checksums and status. */
#define FAP_SERVER_NSTATS 19
FAP_API int fap_server_stats(fap_server *s, double *out, int32_t count);
FAP_API int fap_server_reset_stats(fap_server *s);

/* Message of the last fap_server_* failure on the calling thread. */
FAP_API const char *fap_server_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* FAP_SERVE_H_ */
