/* Declarations-only stand-in for METIS, so the reference's partitioning
 * and toy-scalar translation units compile when the reference is built as
 * an oracle.  Partitioning is never invoked on a single-zone run. */
#pragma once
#include <stdint.h>
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
#ifdef __cplusplus
extern "C" {
#endif
static inline int METIS_SetDefaultOptions(idx_t *) { return 1; }
static inline int METIS_PartGraphKway(idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *,
                                      real_t *, real_t *, idx_t *, idx_t *, idx_t *) { return 1; }
static inline int METIS_PartGraphRecursive(idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *,
                                           real_t *, real_t *, idx_t *, idx_t *, idx_t *) { return 1; }
#ifdef __cplusplus
}
#endif
