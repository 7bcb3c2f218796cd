"""The lightmap denoiser: a 4-level convolutional encoder-decoder over BF16
activations, trained on (low, high) sample-count final-gather pairs that
the baker itself produces, run on the tensor cores (rl_dn_* in
librelight_b200.so).  torch provides device memory and streams only.

Layer primitives (`conv3x3`, `conv3x3_wgrad`) take torch tensors in NHWC
BF16 with channel strides padded to 16.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

from ._abi import check, lib


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def conv3x3(in0, weights, ncols, bias=None, relu=False, in1=None, out0=None, out0_c0=0, out0_cn=None,
            mask0=None, out1=None, out1_c0=0, out1_cn=0, mask1=None, err=None, stream=None):
    """One 3x3 'same' convolution (rl_dn_conv3x3); in/out [n][h][w][c]."""
    n, h, w, c0 = in0.shape
    c1 = 0 if in1 is None else in1.shape[-1]
    out0_cn = ncols if out0_cn is None else out0_cn
    check(lib().rl_dn_conv3x3(_p(in0), c0, _p(in1), c1, w, h, n, _p(weights), ncols, _p(bias), int(relu), _p(out0),
                              out0_c0, out0_cn, out0.shape[-1], _p(mask0), _p(out1), out1_c0, out1_cn,
                              0 if out1 is None else out1.shape[-1], _p(mask1), _p(err), stream))


def conv3x3_wgrad(grad, cout, inp, cin, dw, ci_off=0, ci_total=None, err=None, stream=None):
    """dw[co][tap][ci_off + ci] += sum_p grad[p][co] * inp[p + off(tap)][ci] (rl_dn_conv3x3_wgrad)."""
    n, h, w, gcs = grad.shape
    ci_total = dw.shape[-1] if ci_total is None else ci_total
    check(lib().rl_dn_conv3x3_wgrad(_p(grad), cout, gcs, _p(inp), cin, inp.shape[-1], w, h, n, _p(dw), ci_off,
                                    ci_total, _p(err), stream))
