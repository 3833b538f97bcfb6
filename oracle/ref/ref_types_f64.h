/*
 * Pre-included (gcc/nvcc -include) when compiling the reference sources for
 * the oracle build.  The reference selects its scalar type in types.h:4 with a
 * hard-coded `#if 1` (FP32).  Defining the include guard _TYPES_H here first
 * turns the reference's types.h into a no-op and supplies the FP64 branch of
 * types.h:13-22 instead, so the reference compiles unmodified as an FP64 code.
 *
 * Test infrastructure only: this file is part of the oracle recipe.
 */
#ifndef _TYPES_H
#define _TYPES_H

#define FLOTANTE double
#define mdgpu_cublasXsyr cublasDsyr
#define mdgpu_cublasXtrsm cublasDtrsm
#define mdgpu_cublasXgemm cublasDgemm

#define mdgpu_cblasXscal cblas_dscal
#define mdgpu_cblasXsyr cblas_dsyr
#define mdgpu_cblasXtrsm cblas_dtrsm
#define mdgpu_cblasXgemm cblas_dgemm

#endif
