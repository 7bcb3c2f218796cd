"""Lightmap post-processing and output formats: Lightmap::expand, ::blur and
::save (RawHdr, TgaDoubleLdr, TgaRgbm; Lightmap.cpp:167-349).

  - the oracle equals the reference's outputs committed in golden/post.npz
    (and the live reference build, where present) bit for bit;
  - the CUDA kernels (rl_map_expand / rl_map_blur / rl_map_encode /
    rl_map_save) equal the oracle bit for bit, files byte for byte.

Lightmap::toRgbmLdr writes pixels at offset x*3 in rows of w*4 bytes and
leaves the rest of each row uninitialised, so RGBM buffers and files are
compared on the bytes the reference determines (those are 0 here).
Colour comparisons are bit for bit with NaN payloads aside (the inputs
include NaN, inf and -1e10 colours).
"""
import os
import sys

import numpy as np
import pytest

import oracle_bind as ob

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import POST_SHAPES, post_inputs  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "post.npz"))


def _lm(W, H, flags, color):
    lm = ob.LumelMap(W, H)
    lm.flags[:] = flags
    lm.color[:] = color
    return lm


def _same(a, b):
    """Bit-identical, except that NaN payloads may differ (x86 propagates an
    input NaN's bits, the GPU returns its canonical NaN): NaNs must sit at
    the same places."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


@pytest.mark.parametrize("case", range(len(POST_SHAPES)))
def test_oracle_postprocess_matches_golden(case):
    W, H, dens = POST_SHAPES[case]
    flags, color = post_inputs(W, H, dens, 100 + case)
    for op in ("expand", "blur"):
        lm = _lm(W, H, flags, color)
        getattr(ob, op)(lm)
        assert _same(lm.color, GOLD[f"{op}{case}"]), op
    for fmt in (0, 1, 2):
        mine = np.frombuffer(ob.save_bytes(_lm(W, H, flags, color), fmt), np.uint8)
        want = GOLD[f"file{case}_{fmt}"]
        mask = ob.tga_written_mask(W, H, fmt)
        assert mine.size == want.size
        assert np.array_equal(mine[mask], want[mask]), fmt


def test_f2u8_models_x86_float_to_uchar():
    f = ob.oracle_lib().oro_f2u8
    assert f(255.9) == 255 and f(0.99) == 0 and f(-1.5) == 255 and f(-256.0) == 0
    assert f(float("nan")) == 0 and f(float("-inf")) == 0 and f(-1e10) == 0


@pytest.mark.skipif(not os.path.exists(ob.REF_LIB), reason="reference build absent")
def test_oracle_postprocess_matches_live_reference():
    from relight_b200 import scenes
    ref = ob.RefScene(scenes.room_scene(size=16).scene)
    rng = np.random.default_rng(7)
    for W, H in ((131, 77), (200, 200), (3, 3), (1, 9)):
        flags = (rng.random(W * H) < 0.5).astype(np.int32)
        color = rng.uniform(-1, 4, (W * H, 3)).astype(np.float32)
        for op in ("expand", "blur"):
            k = ref.post_map(W, H, flags, color)
            getattr(ref.lib, "ref_map_" + op)(ref.h, k)
            lm = _lm(W, H, flags, color)
            getattr(ob, op)(lm)
            assert _same(lm.color, ref.map_colors(k, W, H)), (W, H, op)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(POST_SHAPES)))
def test_gpu_postprocess_matches_oracle(cuda, case, tmp_path):
    from relight_b200.device import DeviceMap
    W, H, dens = POST_SHAPES[case]
    flags, color = post_inputs(W, H, dens, 100 + case)
    for op in ("expand", "blur"):
        m = DeviceMap(0, W, H)
        m.upload(flags=flags, color=color)
        getattr(m, op)()
        got = m.download(fields=("color",))["color"]
        assert _same(got, GOLD[f"{op}{case}"]), op
        m.close()
    m = DeviceMap(0, W, H)
    m.upload(flags=flags, color=color)
    lm = _lm(W, H, flags, color)
    assert np.array_equal(m.encode(1), ob.to_double_ldr(lm))
    mask = ob.rgbm_written_mask(W, H)
    enc = m.encode(2)
    assert np.array_equal(enc[mask], ob.to_rgbm(lm)[mask]) and not enc[~mask].any()
    for fmt in (0, 1, 2):
        path = tmp_path / f"lm{fmt}.bin"
        m.save(str(path), fmt)
        got = np.frombuffer(path.read_bytes(), np.uint8)
        want = GOLD[f"file{case}_{fmt}"]
        fmask = ob.tga_written_mask(W, H, fmt)
        assert got.size == want.size and np.array_equal(got[fmask], want[fmask]), fmt
    m.close()


@pytest.mark.gpu
def test_gpu_blur_expand_large_maps(cuda):
    """Full-size maps (the wavefront blur over 1024 rows and beyond one
    thread per row) against the oracle."""
    from relight_b200.device import DeviceMap
    rng = np.random.default_rng(3)
    for W, H in ((1024, 1024), (300, 2100)):
        flags = (rng.random(W * H) < 0.7).astype(np.int32)
        color = rng.random((W * H, 3)).astype(np.float32)
        for op in ("expand", "blur"):
            m = DeviceMap(0, W, H)
            m.upload(flags=flags, color=color)
            getattr(m, op)()
            got = m.download(fields=("color",))["color"]
            lm = _lm(W, H, flags, color)
            getattr(ob, op)(lm)
            assert _same(got, lm.color), (W, H, op)
            m.close()
