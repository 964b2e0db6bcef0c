"""kf_solve_linear_least_squares_noalloc, called through the C ABI, against the allocating
kf_solve_linear_least_squares on the same device A and b.

The no-allocation entry point keeps its scratch in a static device array of the library and
runs the same kernels with the same block count and reduction order, so both give the same x
bit for bit; the comparison with the allocating entry point is exact, and only the check
against an FP64 solve of the normal equations has a tolerance.  Calls come in a row, a large
system then a smaller one, so the second call runs on a scratch the first one left filled.
This file is named to be collected last: it must pass alone and after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def system(cuda, n, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, 6)).astype(np.float32)
    xt = rng.normal(size=6)
    b = (A.astype(np.float64) @ xt + 1e-3 * rng.normal(size=n)).astype(np.float32)
    return A, b, cuda.from_numpy(A).cuda(), cuda.from_numpy(b).cuda()


def solve(kf, fn, A, b, n, stream=0):
    x = (ctypes.c_float * 6)()
    st = fn(ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(b.data_ptr()), int(n), x, ctypes.c_void_p(stream))
    return st, np.array(x[:], np.float32)


def test_two_calls_in_a_row_match_the_allocating_entry(kf, cuda):
    lib = kf.lib
    stream = cuda.cuda.current_stream().cuda_stream
    for n, seed in ((307200, 11), (5000, 12)):   # 640 x 480 rows, then a smaller system
        A, b, Ad, bd = system(cuda, n, seed)
        st_ref, x_ref = solve(kf, lib.kf_solve_linear_least_squares, Ad, bd, n, stream)
        st_na, x_na = solve(kf, lib.kf_solve_linear_least_squares_noalloc, Ad, bd, n, stream)
        assert st_ref == st_na == kf.KF_OK, (st_ref, st_na)
        np.testing.assert_array_equal(x_na, x_ref)
        # and both solve the FP64 normal equations
        A64 = A.astype(np.float64)
        x64 = np.linalg.solve(A64.T @ A64, A64.T @ b.astype(np.float64))
        np.testing.assert_allclose(x_na, x64, rtol=1e-5, atol=1e-6)


def test_largest_system_and_default_stream(kf, cuda):
    lib = kf.lib
    n = kf._lib.KF_LLS_NOALLOC_MAX_ROWS
    A, b, Ad, bd = system(cuda, n, 13)
    cuda.cuda.synchronize()
    st_ref, x_ref = solve(kf, lib.kf_solve_linear_least_squares, Ad, bd, n)
    st_na, x_na = solve(kf, lib.kf_solve_linear_least_squares_noalloc, Ad, bd, n)
    assert st_ref == st_na == kf.KF_OK
    np.testing.assert_array_equal(x_na, x_ref)


def test_rejects_rows_beyond_the_scratch(kf, cuda):
    lib = kf.lib
    n = kf._lib.KF_LLS_NOALLOC_MAX_ROWS + 1
    Ad = cuda.zeros((8, 6), dtype=cuda.float32, device="cuda")   # never read: rejected before any launch
    bd = cuda.zeros((8,), dtype=cuda.float32, device="cuda")
    st, _ = solve(kf, lib.kf_solve_linear_least_squares_noalloc, Ad, bd, n)
    assert st == kf._lib.KF_ERR_TOO_LARGE
    assert "fixed scratch" in lib.kf_status_string(st).decode()
    assert solve(kf, lib.kf_solve_linear_least_squares_noalloc, Ad, bd, 0)[0] == kf.KF_ERR_ARG
