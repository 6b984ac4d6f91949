/*
 * fap_host.h -- C wrappers of the drop-in fap::fapGraph (include/fap/fap.h),
 * for FFI callers (ctypes, cgo, JNI ...).  A handle is a fap::fapGraph*.
 *
 * Each wrapper maps one fapGraph member of the reference (fap/fap.h:79-124):
 *   fap_host_from_mtx          fapGraph(file, directed, weighted, K)   fap/fap.cpp:27-59
 *   fap_host_from_csr          fapGraph(n, m, row_offset, col_val, weight, K)  fap/fap.cpp:61-65
 *   fap_host_precondition      preCondition()                          fap/fap.cpp:67-81
 *   fap_host_is_split          isSplit()                               fap/fap.cpp:83-85
 *   fap_host_graph_id          getGraphId()                            fap/fap.cpp:87-89
 *   fap_host_solve             solve(is_path_needed)                   fap/fap.cpp:184-194
 *   fap_host_solve_subgraph    solveSubGraph(id, is_path_needed)       fap/fap.cpp:197-207
 *   fap_host_mapping           getMapping()                            fap/fap.cpp:209-211
 *   fap_host_all_distance      getAllDistance()                        fap/fap.cpp:213-216
 *   fap_host_current_subgraph  getCurrentSubGraphId()                  fap/fap.cpp:231-233
 *   fap_host_subgraph_distance getSubGraphDistance(id)                 fap/fap.cpp:235-238
 *   fap_host_distance_from_one_point getDistanceFromOnePoint(v)        fap/fap.cpp:245-252
 *   fap_host_distance_p2p      getDistanceP2P (TODO in the reference)  fap/fap.cpp:263-265
 *   fap_host_check_result      check_result(...)                       fap/fap.cpp:271-277
 * Status codes are those of fap_b200.h; messages via fap_host_last_error().
 */
#ifndef FAP_HOST_H_
#define FAP_HOST_H_

#include <stdint.h>

#include "fap_b200.h"

#ifdef __cplusplus
namespace fap { class fapGraph; }
typedef fap::fapGraph fap_host_graph;
extern "C" {
#else
typedef struct fap_host_graph fap_host_graph;
#endif

FAP_API const char *fap_host_last_error(void);
/* Reads graph/<kind>/<name>.mtx relative to the working directory. */
FAP_API int fap_host_from_mtx(const char *name, int directed, int weighted, int K, fap_host_graph **out);
FAP_API int fap_host_from_csr(int32_t n, int64_t m, const int32_t *row_offset, const int32_t *col_val,
                              const float *weight, int K, int directed, fap_host_graph **out);
/* Binary graph file (CSR + partition; no counterpart in the reference, which
 * re-reads the text file and re-runs METIS every time): fap_host_save
 * writes the graph as constructed (before or after preCondition);
 * fap_host_load rebuilds it without text parsing or METIS, ready for
 * fap_host_precondition.  A checksum guards the file (FAP_ERR_IO). */
FAP_API int fap_host_save(fap_host_graph *g, const char *path);
FAP_API int fap_host_load(const char *path, fap_host_graph **out);
FAP_API int fap_host_destroy(fap_host_graph *g);
/* 1-based part id per vertex; replaces the METIS result (before precondition). */
FAP_API int fap_host_set_partition(fap_host_graph *g, const int32_t *graph_id);
/* device ordinal, FAP_DTYPE_*, FAP_MODE_* */
FAP_API int fap_host_set_options(fap_host_graph *g, int device, int dtype, int mode);
/* At most `rows` output rows on the device (0 = no bound): solve and
 * solve_subgraph then run the parts in groups whose rows fit, as they do
 * when HBM cannot hold all n rows (no counterpart in the reference, whose
 * split graphs always solve one part per call, fap/fap.cpp:196-208). */
FAP_API int fap_host_set_max_resident_rows(fap_host_graph *g, int64_t rows);
FAP_API int fap_host_precondition(fap_host_graph *g);
FAP_API int fap_host_is_split(fap_host_graph *g);
FAP_API int fap_host_dtype(fap_host_graph *g);
/* The graph's directed / weighted flags (as given or as loaded). */
FAP_API int fap_host_flags(fap_host_graph *g, int *directed, int *weighted);
/* out4 = [n, num_edges (declared arcs), K, stored arcs] */
FAP_API int fap_host_sizes(fap_host_graph *g, int64_t *out4);
/* row_offset[n+1], col_val[stored], weight[stored] */
FAP_API int fap_host_csr(fap_host_graph *g, int32_t *row_offset, int32_t *col_val, float *weight);
FAP_API int fap_host_graph_id(fap_host_graph *g, int32_t *out);
FAP_API int fap_host_mapping(fap_host_graph *g, int32_t *out);
/* ver_num, ver_offset, bdy_num: K+1 entries each (index 1..K) */
FAP_API int fap_host_parts(fap_host_graph *g, int32_t *ver_num, int32_t *ver_offset, int32_t *bdy_num);
FAP_API int fap_host_solve(fap_host_graph *g, int path_needed);
FAP_API int fap_host_solve_subgraph(fap_host_graph *g, int id, int path_needed);
FAP_API int fap_host_current_subgraph(fap_host_graph *g);
/* out: ver_num[id] x n floats */
FAP_API int fap_host_subgraph_distance(fap_host_graph *g, int id, float *out);
/* out: n x n floats (after fap_host_solve) */
FAP_API int fap_host_all_distance(fap_host_graph *g, float *out);
/* out: n floats (vertex v must be in the current part) */
FAP_API int fap_host_distance_from_one_point(fap_host_graph *g, int v, float *out);
FAP_API int fap_host_distance_p2p(fap_host_graph *g, int from, int to, float *out);
/* Predecessors (solved with path_needed): out ver_num[id] x n / n x n / n
 * int32 (see fap_graph_path_block for their meaning). */
FAP_API int fap_host_subgraph_path(fap_host_graph *g, int id, int32_t *out);
FAP_API int fap_host_all_path(fap_host_graph *g, int32_t *out);
FAP_API int fap_host_path_from_one_point(fap_host_graph *g, int v, int32_t *out);
/* Vertices of a shortest path from..to (inclusive) into out[cap]; *len = its
 * length, 0 when `to` is unreachable (no counterpart: a TODO in the
 * reference, fap/fap.cpp:263-269). */
FAP_API int fap_host_path_p2p(fap_host_graph *g, int from, int to, int32_t *out, int32_t cap, int32_t *len);
/* Sampled self-check of part id's block against fresh GPU SSSP rows. */
FAP_API int fap_host_check_result(fap_host_graph *g, int id, int *ok);
/* The device-resident graph behind g (NULL before the first solve). */
FAP_API fap_dgraph *fap_host_device_graph(fap_host_graph *g);

#ifdef __cplusplus
}
#endif
#endif /* FAP_HOST_H_ */
