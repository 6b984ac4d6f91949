/*
 * Minimal declarations for the METIS 5 k-way partitioner, written for the
 * oracle harness only (test infrastructure, never shipped in the product).
 *
 * The library linked against is the METIS build that the CUDA toolkit ships
 * as libmetis_static.a.  That build uses 64-bit idx_t and 32-bit real_t; the
 * reference calls exactly one entry point (fap/utils/readIdFile.h:118-121)
 * and compares its status with METIS_OK (readIdFile.h:123).
 */
#ifndef FAP_ORACLE_METIS_H_
#define FAP_ORACLE_METIS_H_
#include <stdint.h>

typedef int64_t idx_t;
typedef float real_t;

#ifdef __cplusplus
enum rstatus_et {
  METIS_OK = 1,
  METIS_ERROR_INPUT = -2,
  METIS_ERROR_MEMORY = -3,
  METIS_ERROR = -4
};
extern "C" {
#endif

int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy,
                        idx_t *vwgt, idx_t *vsize, idx_t *adjwgt,
                        idx_t *nparts, real_t *tpwgts, real_t *ubvec,
                        idx_t *options, idx_t *edgecut, idx_t *part);

#ifdef __cplusplus
}
#endif
#endif  // FAP_ORACLE_METIS_H_
