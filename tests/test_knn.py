"""The k-nearest-neighbour photon estimate (rl_emit_photons_records +
rl_photonmap_gather_knn) against the brute-force checker in
oracle/knn_ref.py, on the deposits the GPU kept.

Tolerances: the float32 checker repeats the kernel's operation order, so
valid lumels agree bit for bit; the FP64 checker within 1e-5 relative (of
the largest gathered value).  Lumels that are not valid keep the disc
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
