/* Include shim used only when compiling the reference library into oracle/_ref.
 * CUDA 12.9 refuses the legacy <cublas.h> together with <cublas_v2.h>; the
 * reference's include/blasx_common.h:7 names the legacy header, so this file
 * stands in for it and forwards to the v2 API header. No reference source is
 * changed or copied. */
#ifndef BLASX_ORACLE_SHIM_CUBLAS_H
#define BLASX_ORACLE_SHIM_CUBLAS_H
#include <cublas_v2.h>
#endif
