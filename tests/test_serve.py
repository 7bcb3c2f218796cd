"""The bake-serving loop: slice planning and arrivals on the CPU; on the GPU,
every request's lightmap is bit-identical whether baked alone through the
single-job calls or sliced across iterations in the mix with others, and the
HBM budget holds."""
import numpy as np
import pytest

from relight_b200 import scenes, serve


def test_plan_slices_water_filling():
    assert serve.plan_slices([], 1024) == []
    # small requests get everything they need, the big one the rest
    assert serve.plan_slices([64, 5000, 100], 1024) == [64, 832, 100]
    # equal shares in multiples of 32
    s = serve.plan_slices([10_000] * 3, 1000)
    assert sum(s) <= 1000 and all(x % 32 == 0 and 320 <= x <= 352 for x in s)
    # everyone progresses even when the quantum is smaller than the crowd
    s = serve.plan_slices([500] * 10, 64)
    assert all(x >= 32 for x in s)
    # finished requests get nothing; a remainder below the alignment is taken whole
    assert serve.plan_slices([0, 7], 1024) == [0, 7]


def test_plan_slices_never_exceed_remaining():
    rng = np.random.default_rng(0)
    for _ in range(200):
        rem = [int(x) for x in rng.integers(0, 5000, rng.integers(1, 30))]
        q = int(rng.integers(32, 20000))
        s = serve.plan_slices(rem, q)
        assert all(0 <= a <= r for a, r in zip(s, rem))
        assert all(a > 0 for a, r in zip(s, rem) if r > 0)
        assert all(a % 32 == 0 or a == r for a, r in zip(s, rem))


def test_poisson_arrivals_rate():
    t = serve.poisson_arrivals(50.0, 20000, 1)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 50.0) < 1.5


def test_make_requests_distribution():
    wl = scenes.batch_workload(n_jobs=1, n_scenes=4, tris=(1000, 2000), sides=(32, 64), photon_map=32)
    reqs = serve.make_requests(wl, 100.0, 2000, seed=2)
    sides = np.array([r.side for r in reqs])
    assert sides.min() >= 32 and sides.max() <= 1024
    # log-uniform: the median side is near sqrt(32 * 1024) = 181
    assert 150 < np.median(sides) < 215
    assert set(r.scene for r in reqs) == {0, 1, 2, 3}


@pytest.mark.gpu
def test_serve_alone_equals_mix(cuda):
    from relight_b200 import batch
    from relight_b200.device import DeviceMap
    wl = scenes.batch_workload(n_jobs=1, n_scenes=3, seed=11, tris=(1_000, 20_000), sides=(24, 96),
                               ao_samples=8, fg_samples=16, photon_map=64)
    rs = batch.make_resident_scenes(wl)
    reqs = serve.make_requests(wl, rate=2000.0, n=12, seed=3, sides=(24, 160))
    budget = 3 * DeviceMap.nbytes(160, 160)
    srv = serve.BakeServer(rs, budget_bytes=budget, quantum=4096, fg_samples=16)
    stats = srv.run(reqs)
    srv.close()
    assert stats.requests == len(reqs)
    assert stats.peak_bytes <= budget
    assert stats.iterations > len(reqs) // 3  # slices spread over many iterations
    assert stats.mean_active > 1.0            # requests overlapped on the device
    for r in reqs:
        want = serve.bake_alone(rs, r, fg_samples=16)
        assert np.array_equal(r.result.view(np.uint32), want.view(np.uint32)), f"request {r.rid}"
        assert r.t_admit >= r.arrival and r.t_done >= r.t_admit


@pytest.mark.gpu
def test_serve_denoised_alone_equals_mix(cuda):
    """With the denoiser in the loop (final gather to its own map, denoised
    onto direct + AO at completion) each result is still the same bits alone
    and in the mix."""
    from relight_b200 import batch
    from relight_b200.denoise import Denoiser
    from relight_b200.device import DeviceMap
    wl = scenes.batch_workload(n_jobs=1, n_scenes=2, seed=12, tris=(1_000, 10_000), sides=(24, 96),
                               ao_samples=8, fg_samples=16, photon_map=64)
    rs = batch.make_resident_scenes(wl)
    dn = Denoiser(seed=2)
    reqs = serve.make_requests(wl, rate=2000.0, n=8, seed=4, sides=(24, 130))
    srv = serve.BakeServer(rs, budget_bytes=6 * DeviceMap.nbytes(130, 130), quantum=4096, denoiser=dn, max_side=130)
    stats = srv.run(reqs)
    srv.close()
    assert stats.requests == len(reqs) and dn.status() == 0
    for r in reqs:
        want = serve.bake_alone(rs, r, fg_samples=16, denoiser=dn)
        assert np.array_equal(r.result.view(np.uint32), want.view(np.uint32)), f"request {r.rid}"
    dn.close()
