"""Brute-force k-nearest-neighbour photon estimate: the checker of
rl_photonmap_gather_knn.  Test infrastructure only.

For each valid lumel: the mean colour of the k photon records of the
photonmap nearest to the lumel position within `radius` (squared distance
ex*ex + ey*ey + ez*ez <= radius*radius in float32, ties by photon number *
16 + bounce).  Records count when their slot matches and their position
and colour are finite.  `exact32` repeats the kernel's arithmetic so that
results compare bit for bit: float32 distances; each colour component
rounded to a 64-bit integer at 2^s per unit, with s = 54 - e where
2^(e-1) <= max |colour| < 2^e over the counted records (clamped to
[-100, 100]); the integer sum over the selection; then
float32(float64(sum) * 2^-s / count).  `exact32=False` is the same
selection with the mean in double precision.  The estimator is the
world-space counterpart of Photonmap::gather (Lightmap.cpp:376-413): a mean
photon colour, not a density.
"""
import numpy as np


def fixed_shift(colours):
    """s of the fixed-point colour sums for these counted colours [m][3]."""
    m = float(np.abs(colours).max()) if colours.size else 0.0
    if m == 0.0:
        return 0
    e = int(np.frexp(np.float64(m))[1])  # m < 2^e
    return min(100, max(-100, 54 - e))


def knn_gather(positions, valid, records, photon, depth, slot_of, slot, k, radius, exact32=True):
    """positions [n][3], valid [n] bool, records [m][6] (xyz rgb), photon [m],
    depth [m], slot_of [m]  ->  gathered [n][3] (0 where invalid)."""
    records = np.asarray(records, np.float32)
    sel = (slot_of == slot) & np.isfinite(records).all(axis=1)
    rec = records[sel]
    ids = photon[sel].astype(np.uint64) * np.uint64(16) + (depth[sel].astype(np.uint64) & np.uint64(15))
    r2 = np.float32(radius) * np.float32(radius)
    s = fixed_shift(rec[:, 3:6])
    fx = np.rint(rec[:, 3:6] * np.float32(2.0 ** s)).astype(np.int64)
    out = np.zeros((positions.shape[0], 3), np.float32)
    pos = positions.astype(np.float32)
    for i in np.nonzero(valid)[0]:
        ex = rec[:, 0] - pos[i, 0]
        ey = rec[:, 1] - pos[i, 1]
        ez = rec[:, 2] - pos[i, 2]
        d2 = ex * ex + ey * ey + ez * ez
        m = np.nonzero(d2 <= r2)[0]
        if m.size == 0:
            continue
        order = m[np.lexsort((ids[m], d2[m]))][:k]
        if exact32:
            tot = fx[order].sum(axis=0)
            out[i] = (tot.astype(np.float64) * 2.0 ** -s / order.size).astype(np.float32)
        else:
            out[i] = (rec[order, 3:6].astype(np.float64).sum(axis=0) / order.size).astype(np.float32)
    return out
