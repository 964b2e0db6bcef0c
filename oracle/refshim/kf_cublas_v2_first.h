// TEST INFRASTRUCTURE ONLY: force-included before project/src/linear_least_squares.h and
// project/src/icp.cpp.  The reference includes both the legacy <cublas.h>
// (project/src/linear_least_squares.h:5) and, through <cusolverDn.h>, <cublas_v2.h>; the CUDA
// 10 headers it was written for allowed that, the current ones refuse it.  Its calls are the
// handle-based v2 API (cublasCreate, cublasSgemm(handle, ...)), so the v2 header is included
// first and the legacy header's guard is set, which makes its include a no-op.
#pragma once
#include <cublas_v2.h>
#define CUBLAS_H_
