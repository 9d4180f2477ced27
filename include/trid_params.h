/*
 * tridsolver_b200 — solver context, binary compatible with the reference's
 * scalar/include/trid_params.h:31-35 (same members, same order, same types).
 *
 *   mpi_params  distributed-solve parameters, as in the reference's MPI
 *               build: used only when it points at a tridDistParams
 *               registered with tridDistInit (tridsolver_b200.h); any other
 *               value is ignored, as the reference's single-node library
 *               ignores it. The pointer is compared against the registered
 *               ones and never dereferenced otherwise, because the
 *               reference's own tests pass a TridParams whose other members
 *               are left uninitialised (scalar/test/test_cuda.cu:17-21).
 *   opts[d]     per-dimension algorithm hint for solves along dimension d.
 *               0 = autotuned choice (the default and the recommendation).
 *               The reference's values (1..4 for x, 3 for y/z) are accepted
 *               and mapped onto this library's kernel families; every choice
 *               gives the same results to rounding.
 *   sync        reserved in the reference and ignored there; also ignored
 *               here (use tridSetBlocking() from tridsolver_b200.h instead,
 *               because the reference's callers leave it uninitialised).
 *
 * A NULL ctx is accepted everywhere and means "all defaults".
 */
#ifndef TRID_PARAMS_H__
#define TRID_PARAMS_H__

#include "trid_common.h"

struct TridParams {
  void *mpi_params;
  int opts[MAXDIM];
  int sync;
};

#ifndef __cplusplus
typedef struct TridParams TridParams;
#endif

#endif
