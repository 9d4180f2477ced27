/*
 * tridsolver_b200 — common definitions of the drop-in C ABI.
 *
 * Mirrors the reference's scalar/include/trid_common.h:39-75 so that code
 * written against OP-DSL/tridsolver (apps/adi, user codes) compiles unchanged:
 *   - FP / F select float or double from FPPREC (0 = float, 1 = double),
 *     and an undefined FPPREC selects float, as in the reference;
 *   - MAXDIM = 3 is the largest number of array dimensions the API accepts;
 *   - tridStatus_t keeps the reference's numeric codes, which are the
 *     cuSPARSE status values, so status checks in caller code still hold.
 *
 * Unlike the reference (which always returns TRID_STATUS_SUCCESS and aborts
 * the process on CUDA errors), this library returns real status codes:
 *   TRID_STATUS_INVALID_VALUE     bad ndim / solvedim / dims / pads / pointers
 *   TRID_STATUS_ALLOC_FAILED      a scratch allocation failed
 *   TRID_STATUS_ARCH_MISMATCH     no sm_100 device, or the kernels do not load
 *   TRID_STATUS_EXECUTION_FAILED  a kernel launch or the stream sync failed
 *   TRID_STATUS_ZERO_PIVOT        a pivot was zero or non-finite (the result
 *                                 is still written, as the reference would)
 */
#ifndef TRID_COMMON_H__
#define TRID_COMMON_H__

#if !defined(FPPREC) || FPPREC == 0
#  define FP float
#  define F f
#elif FPPREC == 1
#  define FP double
#  define F
#else
#  error "FPPREC must be 0 (float) or 1 (double)"
#endif

#define WARP_SIZE 32
#define ALIGN 32
#define ALIGN_FLOAT (ALIGN / 4)
#define ALIGN_DOUBLE (ALIGN / 8)
#define MAXDIM 3
#define CUDA_ALIGN_BYTE 32

#ifdef __cplusplus
#  define EXTERN_C extern "C"
#else
#  define EXTERN_C
#endif

typedef enum {
  TRID_STATUS_SUCCESS = 0,
  TRID_STATUS_NOT_INITIALIZED = 1,
  TRID_STATUS_ALLOC_FAILED = 2,
  TRID_STATUS_INVALID_VALUE = 3,
  TRID_STATUS_ARCH_MISMATCH = 4,
  TRID_STATUS_MAPPING_ERROR = 5,
  TRID_STATUS_EXECUTION_FAILED = 6,
  TRID_STATUS_INTERNAL_ERROR = 7,
  TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED = 8,
  TRID_STATUS_ZERO_PIVOT = 9
} tridStatus_t;

#endif
