"""Brute-force k-nearest-neighbour photon estimate: the checker of
rl_photonmap_gather_knn.  Test infrastructure only.

For each valid lumel: the mean colour of the k photon records of the
photonmap nearest to the lumel position within `radius` (squared distance
ex*ex + ey*ey + ez*ez <= radius*radius, ties by photon number * 16 +
bounce).  `exact32` repeats the kernel's float32 operation order (the
distance, the ascending-order sum, the division) so results compare bit for
bit; `fp64` is the same selection in double precision.  The estimator is the
world-space counterpart of Photonmap::gather (Lightmap.cpp:376-413): a mean
photon colour, not a density.
"""
import numpy as np


def knn_gather(positions, valid, records, photon, depth, slot_of, slot, k, radius, exact32=True):
    """positions [n][3], valid [n] bool, records [m][6] (xyz rgb), photon [m],
    depth [m], slot_of [m]  ->  gathered [n][3] (0 where invalid)."""
    f = np.float32 if exact32 else np.float64
    sel = slot_of == slot
    rec = records[sel].astype(f)
    ids = photon[sel].astype(np.uint64) * np.uint64(16) + (depth[sel].astype(np.uint64) & np.uint64(15))
    r2 = f(radius) * f(radius)
    out = np.zeros((positions.shape[0], 3), f)
    pos = positions.astype(f)
    for i in np.nonzero(valid)[0]:
        ex = rec[:, 0] - pos[i, 0]
        ey = rec[:, 1] - pos[i, 1]
        ez = rec[:, 2] - pos[i, 2]
        d2 = ex * ex + ey * ey + ez * ez
        m = np.nonzero(d2 <= r2)[0]
        if m.size == 0:
            continue
        order = m[np.lexsort((ids[m], d2[m]))][:k]
        c = rec[order, 3:6]
        s = np.cumsum(c, axis=0, dtype=f)[-1]
        out[i] = s / f(order.size)
    return out
