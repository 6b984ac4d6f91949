/*
 * fap_legacy_kernel.h -- the reference's CUDA kernel ABI, re-implemented on
 * the B200 path so that the reference's own host code (fap/fap.cpp built with
 * -DWITH_CUDA) links against this library unchanged.
 *
 * Signatures and C++ linkage are exactly those of
 * fap/kernel/cuda/cuda_kernel.h:21-42 (Liu-xiandong/FastAPSP), every entry
 * point but batched_sssp_cuGraph (:16-19, the nvGraph build, whose library
 * CUDA no longer ships).  All pointers are host pointers; calls are
 * synchronous, like the reference.
 *
 * Behaviour:
 *   - without predecessor arrays, distances are computed on the GPU in int32
 *     when every input value is an integer (bit-exact with the reference's
 *     float results while finite distances stay below 2^24), else in float32;
 *   - with predecessor arrays (path / mat2_path and res_path / A_path,
 *     diag_path / B_path non-NULL) the GPU computes in float32 with the
 *     reference CPU kernels' own arithmetic and candidate order, and writes
 *     the predecessors the reference's CPU path writes:
 *       floyd_GPU_Nvidia_path   path[i][j] = path[k][j] on every strict
 *                               improvement, pivots in order (floyd_CPU_path,
 *                               fap/kernel/floyd.h:38-49); all entries must
 *                               be non-negative;
 *       minplus_NVIDIA_path     res_path[i][j] = mat2_path[k][j] of the first
 *                               k with the least sum, -1 when none is below
 *                               1e8 (min_plus_path_CPU_advanced,
 *                               fap/kernel/minplus.h:51-65);
 *       floyd_min_plus_Nvidia   the same, starting from res and res_path
 *                               (floyd_min_plus_CPU, fap/kernel/floyd.h:86-102);
 *       floyd_path_A/B_Nvidia   the same, starting from the panel's own value
 *                               and predecessor, candidates from the closed
 *                               diagonal block, computed out of place: equal
 *                               to the reference's in-place CPU panels
 *                               (floyd.h:51-84) in every value, and in every
 *                               predecessor wherever the shortest path is
 *                               unique.  (The reference's CUDA panels start
 *                               from 1e8 and so report diag_path[j][j] where
 *                               the panel entry itself is shortest.)
 *     The SSSP rows carry no predecessors (the reference's CUDA SSSP leaves
 *     them unset too, fap/kernel/cuda/batch_sssp.cu:222-281);
 *   - on an error the outputs are left unchanged, a message goes to stderr
 *     and fap_legacy_last_status() returns the FAP_ERR_* code (the reference
 *     calls exit(EXIT_FAILURE) instead).
 */
#ifndef FAP_LEGACY_KERNEL_H_
#define FAP_LEGACY_KERNEL_H_

#if defined(__GNUC__)
#define FAP_LEGACY_API __attribute__((visibility("default")))
#else
#define FAP_LEGACY_API
#endif

/* Stage 1: shortest-distance rows from st2ed[offset .. offset+bdy_num-1]
 * into subGraph[bdy_num x vertexs].  Replaces cuda_kernel.h:21-24. */
FAP_LEGACY_API void handle_boundry_Nvidia_GPU(float *subGraph, int vertexs, int edges, int bdy_num,
                               int *adj_size, int *row_offset, int *col_val, float *weight,
                               int *st2ed, int offset);

/* Stage 2: in-place Floyd-Warshall of arc[num_node x num_node].
 * Replaces cuda_kernel.h:29. */
FAP_LEGACY_API void floyd_GPU_Nvidia_path(int num_node, float *arc, int *path);

/* Stage 3: res[m x n] = min(1e8, min_k mat1[m x k] + mat2[k x n]).
 * Replaces cuda_kernel.h:41-42. */
FAP_LEGACY_API void minplus_NVIDIA_path(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path,
                         int m, int n, int k);

/* The rest of the reference's kernel header, which fap/fap.cpp also calls
 * (fap/kernel/minplus.h:69-76, fap/kernel/floyd.h:106-139) and so needs at
 * link time.  Same meanings as the reference's CUDA versions; predecessors
 * as above. */

/* Floyd-Warshall of arc[num_node x num_node] in place, no paths.
 * Replaces cuda_kernel.h:27. */
FAP_LEGACY_API void floyd_NVIDIA_GPU(int num_node, float *arc);

/* Blocked Floyd, column panel: A[row x col] = min(1e8, A (x) diag[col x col]).
 * Replaces cuda_kernel.h:31-32. */
FAP_LEGACY_API void floyd_path_A_Nvidia(float *A, int *A_path, const int row, const int col, float *diag,
                                        int *diag_path);

/* Blocked Floyd, row panel: B[row x col] = min(1e8, diag[row x row] (x) B).
 * Replaces cuda_kernel.h:33-34. */
FAP_LEGACY_API void floyd_path_B_Nvidia(float *B, int *B_path, const int row, const int col, float *diag,
                                        int *diag_path);

/* Blocked Floyd, remaining blocks: res[m x n] = min(res, mat1[m x k] (x)
 * mat2[k x n]) (res entries at most 1e8).  Replaces cuda_kernel.h:35-36. */
FAP_LEGACY_API void floyd_min_plus_Nvidia(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path,
                                          int m, int n, int k);

/* res[M x N] = min(1e8, mat1[M x K] (x) mat2[K x N]), no paths.
 * Replaces cuda_kernel.h:39-40. */
FAP_LEGACY_API void minplus_NVIDIA_GPU(float *mat1, float *mat2, float *res, int M, int N, int K);

#ifdef __cplusplus
extern "C" {
#endif
/* Status of the calling thread's last legacy call (FAP_OK or FAP_ERR_*). */
FAP_LEGACY_API int fap_legacy_last_status(void);
#ifdef __cplusplus
}
#endif

#endif /* FAP_LEGACY_KERNEL_H_ */
