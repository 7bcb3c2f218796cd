"""rl_radiosity_solve_noalloc: the radiosity solve for callers that cannot
allocate device memory (a plugin whose host application owns every device
allocation, or a bake server that reserved its memory at admission).  It
must give the same radiosity as rl_radiosity_solve, call after call, while
its ping-pong buffer is a fixed device array shared by all calls.

This file is collected last (tests/test_zz_*), and it needs nothing that
other tests set up, so it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# The tolerance of the radiosity tests: fp32 Jacobi within 1e-4 relative.
RTOL, ATOL = 1e-4, 1e-6


def _random_form_factors(n, per_row, seed):
    rng = np.random.default_rng(seed)
    cols = np.sort(rng.integers(0, n, (n, per_row)), axis=1).astype(np.int32)
    vals = rng.random((n, per_row)).astype(np.float32)
    vals *= np.float32(0.95) / vals.sum(1, keepdims=True, dtype=np.float32)
    row = (np.arange(n + 1, dtype=np.int64) * per_row)
    rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    E = np.zeros((n, 3), np.float32)
    E[rng.choice(n, 16, replace=False)] = 1.0
    return row, cols.reshape(-1), vals.reshape(-1), E, rho


def _solve(fn, n, arrays, iters):
    import torch
    dr, dc, dv, dE, drho = arrays
    B = torch.full((n, 3), float("nan"), dtype=torch.float32, device="cuda")
    from relight_b200 import _abi
    _abi.check(fn(n, dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), dE.data_ptr(), drho.data_ptr(), iters,
                  B.data_ptr(), None))
    torch.cuda.synchronize()
    return B.cpu().numpy()


def test_noalloc_solve_matches_allocating_solve_twice(cuda):
    import torch
    from relight_b200 import _abi
    L = _abi.lib()
    results = []
    for call, (n, seed, iters) in enumerate(((3000, 1, 50), (4096, 2, 37))):
        row, cols, vals, E, rho = _random_form_factors(n, 24, seed)
        arrays = [torch.from_numpy(a).cuda() for a in (row, cols, vals, E, rho)]
        want = _solve(L.rl_radiosity_solve, n, arrays, iters)
        got = _solve(L.rl_radiosity_solve_noalloc, n, arrays, iters)
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)
        results.append(got)
    # the second call reused the shared array left over by the first
    assert results[0].shape != results[1].shape


def test_noalloc_solve_rejects_oversized_input(cuda):
    from relight_b200 import _abi
    n = _abi.SOLVE_NOALLOC_MAX_PATCHES + 1
    rc = _abi.lib().rl_radiosity_solve_noalloc(n, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                               C.c_void_p(16), C.c_void_p(16), 1, C.c_void_p(16), None)
    assert rc == _abi.RL_INVALID_CALL
    buf = C.create_string_buffer(512)
    _abi.lib().rl_last_error(buf, 512)
    assert b"fixed maximum" in buf.value
