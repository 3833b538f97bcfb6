/*
 * Linux link shim for the reference's CBLAS wrappers (oracle build only).
 *
 * The reference's cblas.cpp is wrapped in `#ifdef _WIN32` (cblas.cpp:1) and
 * mdgpu.cu includes cblas.h inside `extern "C"` on non-Windows hosts
 * (mdgpu.cu:17-23), so the cblas_* symbols must be compiled with C linkage.
 * This file declares cblas.h with C linkage first (its include guard then
 * keeps cblas.cpp from redeclaring it with C++ linkage) and compiles the
 * reference's cblas.cpp as it lies, with _WIN32 defined for that one file.
 * No system CBLAS exists in this image; the reference's in-tree f2c BLAS
 * (dgemm.cpp, dtrsm.cpp, dsyr.cpp, dscal.cpp) is what these wrappers call.
 */
#include <stddef.h>

#define blasint int
#define _Complex
extern "C" {
#include "cblas.h"
}

#define _WIN32 1
#include "cblas.cpp"
