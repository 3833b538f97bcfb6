// Residual and norm kernels used by iterative refinement.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mdgpu {

// Full symmetric pattern of the caller's matrix, rows in original numbering;
// src[p] indexes the caller's lower-triangle value array.
struct SymCsr {
    int n = 0;
    int64_t nnz = 0;
    int* rowptr = nullptr;
    int* col = nullptr;
    int* src = nullptr;
};

void launch_residual(const SymCsr& A, const double* Ax, const double* x, int ldx,
                     const double* b, int ldb, double* r, int ldr, int nrhs, cudaStream_t st);
void launch_anorm(const SymCsr& A, const double* Ax, unsigned long long* out, cudaStream_t st);
void launch_absmax3(int n, int nrhs, const double* r, int ldr, const double* x, int ldx,
                    const double* b, int ldb, unsigned long long* out, cudaStream_t st);
void launch_axpy(int64_t len, const double* d, double* x, cudaStream_t st);

}  // namespace mdgpu
