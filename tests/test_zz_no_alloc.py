"""rl_radiosity_solve_noalloc: the radiosity solve for callers that cannot
allocate device memory (a plugin whose host application owns every device
allocation, or a bake server that reserved its memory at admission).  It
runs rl_radiosity_solve's kernels in the same order, so it must give the
same bits, call after call, while its ping-pong iterates live in one fixed
device array shared by all calls — and it must not change the device's free
memory once its module is loaded.

This file is collected last (tests/test_zz_*), and it needs nothing that
other tests set up, so it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _call(fn, n, arrays, iters, B):
    import torch
    from relight_b200 import _abi
    dr, dc, dv, dE, drho = arrays
    _abi.check(fn(n, dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), dE.data_ptr(), drho.data_ptr(), iters,
                  B.data_ptr(), None))
    torch.cuda.synchronize()
    return B.cpu().numpy().copy()


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_noalloc_solve_matches_allocating_solve_twice(cuda):
    """Two calls in a row with the same n and different data (the second
    finds the first one's iterates in the shared array), each bit-identical
    to rl_radiosity_solve, with the device's free memory unchanged across
    them; iters = 0 copies E."""
    import torch
    from relight_b200 import _abi
    L = _abi.lib()
    n = 4096
    inputs = []
    for seed in (1, 2):
        row, cols, vals, E, rho = _random_form_factors(n, 24, seed)
        inputs.append([torch.from_numpy(a).cuda() for a in (row, cols, vals, E, rho)])
    outs = [torch.full((n, 3), float("nan"), dtype=torch.float32, device="cuda") for _ in range(4)]
    # first call: loads the solver module (which commits the fixed array)
    # and the kernels; an n = 0 call alone must already find the array
    _abi.check(L.rl_radiosity_solve_noalloc(0, None, None, None, None, None, 1, None, None))
    got = [_call(L.rl_radiosity_solve_noalloc, n, inputs[0], 50, outs[0])]
    free0 = torch.cuda.mem_get_info()[0]
    got.append(_call(L.rl_radiosity_solve_noalloc, n, inputs[1], 37, outs[1]))
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    for k, iters in ((0, 50), (1, 37)):
        want = _call(L.rl_radiosity_solve, n, inputs[k], iters, outs[2 + k])
        assert np.isfinite(got[k]).all()
        assert np.array_equal(_bits(got[k]), _bits(want))
    assert not np.array_equal(got[0], got[1])
    # iters = 0: B = E
    z = _call(L.rl_radiosity_solve_noalloc, n, inputs[1], 0, outs[0])
    assert np.array_equal(_bits(z), _bits(inputs[1][3].cpu().numpy()))


def test_noalloc_solve_in_place_on_E(cuda):
    """d_B may alias d_E: the result is written after the last read of E."""
    import torch
    from relight_b200 import _abi
    L = _abi.lib()
    n = 3000
    row, cols, vals, E, rho = _random_form_factors(n, 24, 3)
    arrays = [torch.from_numpy(a).cuda() for a in (row, cols, vals, E, rho)]
    want = _call(L.rl_radiosity_solve, n, arrays, 50, torch.empty((n, 3), dtype=torch.float32, device="cuda"))
    dE = arrays[3].clone()
    got = _call(L.rl_radiosity_solve_noalloc, n, arrays[:3] + [dE, arrays[4]], 50, dE)
    assert np.array_equal(_bits(got), _bits(want))


def test_noalloc_solve_rejects_oversized_input(cuda):
    from relight_b200 import _abi
    n = _abi.SOLVE_NOALLOC_MAX_PATCHES + 1
    rc = _abi.lib().rl_radiosity_solve_noalloc(n, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                               C.c_void_p(16), C.c_void_p(16), 1, C.c_void_p(16), None)
    assert rc == _abi.RL_INVALID_CALL
    buf = C.create_string_buffer(512)
    _abi.lib().rl_last_error(buf, 512)
    assert b"fixed maximum" in buf.value
