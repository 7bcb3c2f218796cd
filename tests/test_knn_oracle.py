"""The brute-force kNN checker (oracle/knn_ref.py) on its own, CPU only:
its fixed-point mean against a float64 mean, its (distance, id) order on
exact ties, and its exclusions.  The GPU kernel is compared with it bit for
bit in test_knn.py."""
import numpy as np

from knn_ref import fixed_shift, knn_gather


def test_fixed_point_mean_matches_float64_mean():
    rng = np.random.default_rng(4)
    n = 3000
    rec = np.concatenate([rng.uniform(-3, 3, (n, 3)), rng.exponential(0.01, (n, 3))], 1).astype(np.float32)
    ph = np.arange(n, dtype=np.uint32)
    dep = np.zeros(n, np.int32)
    sl = np.zeros(n, np.int32)
    pos = rng.uniform(-3, 3, (200, 3)).astype(np.float32)
    valid = np.ones(200, bool)
    a = knn_gather(pos, valid, rec, ph, dep, sl, 0, 50, 1.0)
    b = knn_gather(pos, valid, rec, ph, dep, sl, 0, 50, 1.0, exact32=False)
    assert a.any()
    np.testing.assert_allclose(a, b, rtol=2 ** -22, atol=0)


def test_fixed_shift_keeps_sums_in_range():
    for m in (1e-30, 1e-6, 0.37, 1.0, 3.0, 1e6, 3e20):
        s = fixed_shift(np.array([[m, 0, 0]], np.float32))
        assert 128 * m * 2.0 ** s < 2.0 ** 62
        assert m * 2.0 ** s >= 2.0 ** 40 or s == 100
    assert fixed_shift(np.zeros((0, 3), np.float32)) == 0
    assert fixed_shift(np.zeros((4, 3), np.float32)) == 0


def test_ties_break_by_photon_then_bounce():
    # four records at the same distance from the lumel; k = 2 keeps the two
    # smallest ids (photon * 16 + bounce): photon 3 bounce 1, photon 3 bounce 2
    rec = np.array([[1, 0, 0, 1, 0, 0], [0, 1, 0, 0, 1, 0], [0, 0, 1, 0, 0, 1], [-1, 0, 0, 1, 1, 1]], np.float32)
    ph = np.array([5, 3, 3, 4], np.uint32)
    dep = np.array([0, 2, 1, 0], np.int32)
    sl = np.zeros(4, np.int32)
    got = knn_gather(np.zeros((1, 3), np.float32), np.ones(1, bool), rec, ph, dep, sl, 0, 2, 1.5)
    np.testing.assert_array_equal(got[0], np.array([0, 0.5, 0.5], np.float32))


def test_records_that_do_not_count():
    # another slot, a non-finite position, a non-finite colour: none counts
    rec = np.array([[0, 0, 0, 1, 1, 1], [0.1, 0, 0, 7, 7, 7], [np.nan, 0, 0, 7, 7, 7], [0, 0.1, 0, np.inf, 7, 7]],
                   np.float32)
    ph = np.arange(4, dtype=np.uint32)
    z = np.zeros(4, np.int32)
    sl = np.array([0, 1, 0, 0], np.int32)
    got = knn_gather(np.zeros((2, 3), np.float32), np.array([True, False]), rec, ph, z, sl, 0, 8, 1.0)
    np.testing.assert_array_equal(got, np.array([[1, 1, 1], [0, 0, 0]], np.float32))
