"""The k-nearest-neighbour photon estimate (rl_emit_photons_records +
rl_photonmap_gather_knn) against the brute-force checker in
oracle/knn_ref.py, on the deposits the GPU kept.

Tolerances: the exact checker repeats the kernel's arithmetic (float32
distances, the fixed-point colour sum, the double-precision mean), so valid
lumels agree bit for bit; the FP64 checker within 1e-5 relative (of the
largest gathered value).  Lumels that are not valid keep the disc
gather's value exactly.  The records are the photonmap's deposits: their
number equals the stored count and their colour sum the accumulators' sum
(float atomics in arbitrary order: 1e-5 relative).
"""
import numpy as np
import pytest

from knn_ref import knn_gather
from relight_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup(passes=1):
    from relight_b200.device import PhotonRecords, Relight
    w = scenes.terrain_scene(seed=5, verts=48, n_boxes=60, size=64, tiles=2, passes=passes)
    rl = Relight(builder=0)
    ds = rl.device_scene(w.scene)
    rec = PhotonRecords(1 << 20)
    return w, rl, ds, rec


@pytest.mark.parametrize("k,radius", [(100, 3.0), (7, 0.6), (128, 1.5)])
def test_knn_matches_brute_force(cuda, k, radius):
    import ctypes as C
    import torch
    from relight_b200._abi import check, lib
    from relight_b200.device import _map_array
    w, rl, ds, rec = _setup()
    pm = w.photonmap._device
    f = w.scene.flat
    st = w.settings
    stored = C.c_int64()
    check(lib().rl_emit_photons_records(ds.handle, _map_array([pm]), 1, C.c_void_p(f.lights.ctypes.data),
                                        len(f.lights), st.photon_pass_count, st.photon_bounce_count,
                                        st.photon_energy_threshold, st.photon_max_distance, 77, rec.handle,
                                        C.byref(stored), None))
    check(lib().rl_photonmap_gather(pm.handle, st.final_gather_radius, None))
    disc = pm.download(fields=("gathered",))["gathered"]
    rec.gather_knn(pm, 0, k, radius)
    torch.cuda.synchronize()
    got = pm.download(fields=("flags", "position", "gathered", "photons", "color"))
    xyz, ph, depth, slot = rec.download()
    assert rec.count() == len(xyz) == stored.value == int(got["photons"].sum())
    assert np.allclose(xyz[:, 3:6].astype(np.float64).sum(0), got["color"].astype(np.float64).sum(0), rtol=1e-5)
    valid = (got["flags"] & 1).astype(bool)
    want = knn_gather(got["position"], valid, xyz, ph, depth, slot, 0, k, radius)
    assert np.array_equal(got["gathered"][valid].view(np.uint32), want[valid].view(np.uint32))
    assert np.array_equal(got["gathered"][~valid], disc[~valid])
    w64 = knn_gather(got["position"], valid, xyz, ph, depth, slot, 0, k, radius, exact32=False)
    assert np.abs(got["gathered"][valid] - w64[valid]).max() <= 1e-5 * max(np.abs(w64).max(), 1e-30)
    rec.close()


def test_knn_final_gather_runs(cuda):
    """The kNN estimate feeds the final gather like the disc's."""
    import torch
    from relight_b200.device import Relight
    w, rl, ds, rec = _setup()
    rl.emit_photons(w.scene, w.settings, seed=3, knn=(100, 3.0), records=rec)
    rl.bake_indirect_light(w.scene, w.meshes[0], None, w.settings)
    torch.cuda.synchronize()
    c = w.lightmap._device.download(fields=("flags", "color"))
    v = (c["flags"] & 1).astype(bool)
    assert np.isfinite(c["color"][v]).all() and c["color"][v].sum() > 0
    rec.close()


def _planted(seed, n=20_000, slots=3, outlier=False):
    """Synthetic records: a plane, points on a 0.25 lattice (exact distance
    ties and points on cell edges), repeated positions, non-finite
    coordinates and colours, a colour that sets the fixed-point scale and
    one below its resolution, several slots; ids unique (photon number x16
    + bounce)."""
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    xyz[: n // 4, 1] = 0.0
    xyz[n // 4: n // 2] = np.round(xyz[n // 4: n // 2] * 4) / 4
    xyz[n // 2: n // 2 + 500] = xyz[n // 2 + 500: n // 2 + 1000]
    xyz[7, 0] = np.nan
    xyz[8, 2] = np.inf
    xyz[9, 1] = -np.inf
    if outlier:
        xyz[10] = (1.0e6, -3.0e5, 2.0e5)
    rgb = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    rgb[11, 1] = np.nan
    rgb[12, 2] = np.inf
    rgb[13] = (3.0, 0.0, 5e-30)
    photon = rng.permutation(n * 3)[:n].astype(np.uint32)
    depth = rng.integers(0, 16, n).astype(np.int32)
    slot = rng.integers(0, slots, n).astype(np.int32)
    return np.concatenate([xyz, rgb], 1), photon, depth, slot


def _planted_map(seed, w=48, h=40):
    """Lumel positions near and on the lattice, far from every record, and
    invalid lumels holding a value the gather must keep."""
    rng = np.random.default_rng(seed + 1)
    n = w * h
    pos = rng.uniform(-6, 6, (n, 3)).astype(np.float32)
    pos[: n // 3] = np.round(pos[: n // 3] * 4) / 4
    pos[n // 3: n // 3 + 40] = (40.0, 40.0, 40.0)
    flags = (rng.uniform(size=n) < 0.85).astype(np.int32)
    gathered = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    return pos, flags, gathered


@pytest.mark.parametrize("k,radius,slot,outlier", [
    (100, 1.0, 0, False), (1, 0.25, 1, False), (128, 3.0, 2, False), (5, 0.1, 0, False),
    (16, 0.75, 5, False), (100, 1.0, 0, True), (64, 2.0, 1, True)])
def test_knn_planted_records(cuda, k, radius, slot, outlier):
    """Bit for bit against the float32 brute force on planted records; slot 5
    holds no records (every valid lumel gets 0); the outlier record makes the
    grid grow its cells."""
    import torch
    from relight_b200.device import DeviceMap, PhotonRecords
    xyzrgb, photon, depth, slot_of = _planted(3 + k)
    if outlier:
        xyzrgb, photon, depth, slot_of = _planted(3 + k, outlier=True)
        slot_of[10] = slot
    pos, flags, pre = _planted_map(k)
    w, h = 48, 40
    pm = DeviceMap(1, w, h)
    pm.upload(flags=flags, position=pos, gathered=pre)
    rec = PhotonRecords(1 << 16)
    rec.upload(xyzrgb, photon, depth, slot_of)
    assert rec.count() == len(photon)
    rec.gather_knn(pm, slot, k, radius)
    torch.cuda.synchronize()
    got = pm.download(fields=("gathered",))["gathered"]
    valid = flags.astype(bool)
    want = knn_gather(pos, valid, xyzrgb, photon, depth, slot_of, slot, k, radius)
    assert np.array_equal(got[valid].view(np.uint32), want[valid].view(np.uint32))
    assert np.array_equal(got[~valid], pre[~valid])
    if slot == 5:
        assert not got[valid].any()
    else:
        assert got[valid].any()
    rec.close()


def test_knn_no_records(cuda):
    import torch
    from relight_b200.device import DeviceMap, PhotonRecords
    pos, flags, pre = _planted_map(1, 16, 8)
    pm = DeviceMap(1, 16, 8)
    pm.upload(flags=flags, position=pos, gathered=pre)
    rec = PhotonRecords(1024)
    rec.upload(np.zeros((0, 6), np.float32), np.zeros(0, np.uint32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    rec.gather_knn(pm, 0, 10, 1.0)
    torch.cuda.synchronize()
    got = pm.download(fields=("gathered",))["gathered"]
    valid = flags.astype(bool)
    assert not got[valid].any() and np.array_equal(got[~valid], pre[~valid])
    rec.close()


def test_knn_rejects_bad_arguments(cuda):
    from relight_b200._abi import RelightCudaError as RelightError
    from relight_b200.device import DeviceMap, PhotonRecords
    pm = DeviceMap(1, 8, 8)
    rec = PhotonRecords(16)
    xyz = np.zeros((17, 6), np.float32)
    with pytest.raises(RelightError):
        rec.upload(xyz, np.arange(17, dtype=np.uint32), np.zeros(17, np.int32), np.zeros(17, np.int32))
    with pytest.raises(RelightError):
        rec.upload(xyz[:2], np.arange(2, dtype=np.uint32), np.array([0, 70000], np.int32), np.zeros(2, np.int32))
    for k, r in ((0, 1.0), (129, 1.0), (4, 0.0), (4, float("inf")), (4, float("nan"))):
        with pytest.raises(RelightError):
            rec.gather_knn(pm, 0, k, r)
    rec.close()


@pytest.mark.parametrize("cell", [8, 45, 128])
def test_knn_cell_widths(cuda, cell):
    """Any cell width gives the same bits: narrow cells send most lumels to
    the second pass, cells twice the radius settle every lumel in the first."""
    import torch
    from relight_b200 import autotune
    from relight_b200.device import DeviceMap, PhotonRecords
    xyzrgb, photon, depth, slot_of = _planted(11)
    pos, flags, pre = _planted_map(11)
    pm = DeviceMap(1, 48, 40)
    pm.upload(flags=flags, position=pos, gathered=pre)
    rec = PhotonRecords(1 << 16)
    rec.upload(xyzrgb, photon, depth, slot_of)
    old = autotune.get_knn_cell()
    try:
        autotune.set_knn_cell(cell)
        rec.gather_knn(pm, 1, 40, 0.8)
        torch.cuda.synchronize()
    finally:
        autotune.set_knn_cell(old)
    got = pm.download(fields=("gathered",))["gathered"]
    valid = flags.astype(bool)
    want = knn_gather(pos, valid, xyzrgb, photon, depth, slot_of, 1, 40, 0.8)
    assert np.array_equal(got[valid].view(np.uint32), want[valid].view(np.uint32))
    rec.close()
