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
    if t is None:
        return None
    if isinstance(t, int):
        return C.c_void_p(t)
    return C.c_void_p(t.data_ptr())


def conv3x3(in0, weights, ncols, bias=None, relu=False, in1=None, out0=None, out0_c0=0, out0_cn=None,
            mask0=None, out1=None, out1_c0=0, out1_cn=0, mask1=None, err=None, stream=None, slope=0.0):
    """One 3x3 'same' convolution (rl_dn_conv3x3); in/out [n][h][w][c]."""
    n, h, w, c0 = in0.shape
    c1 = 0 if in1 is None else in1.shape[-1]
    out0_cn = ncols if out0_cn is None else out0_cn
    check(lib().rl_dn_conv3x3(_p(in0), c0, _p(in1), c1, w, h, n, _p(weights), ncols, _p(bias), int(relu),
                              float(slope), _p(out0),
                              out0_c0, out0_cn, out0.shape[-1], _p(mask0), _p(out1), out1_c0, out1_cn,
                              0 if out1 is None else out1.shape[-1], _p(mask1), _p(err), stream))


def conv3x3_wgrad(grad, cout, inp, cin, dw, ci_off=0, ci_total=None, err=None, stream=None):
    """dw[co][tap][ci_off + ci] += sum_p grad[p][co] * inp[p + off(tap)][ci] (rl_dn_conv3x3_wgrad)."""
    n, h, w, gcs = grad.shape
    ci_total = dw.shape[-1] if ci_total is None else ci_total
    check(lib().rl_dn_conv3x3_wgrad(_p(grad), cout, gcs, _p(inp), cin, inp.shape[-1], w, h, n, _p(dw), ci_off,
                                    ci_total, _p(err), stream))


# ------------------------------------------------------------------ network

# (cout, input segment channel counts) per convolution, as built by
# rl_denoiser_create; k = sum of segments padded to 64.
LAYERS = [(32, (16,)), (64, (32,)), (96, (64,)), (128, (96,)), (96, (128, 96)), (64, (96, 64)), (32, (64, 32)),
          (3, (32,))]
FEATURES = 16


def _pad64(c):
    return (c + 63) // 64 * 64


def _pad16(c):
    return (c + 15) // 16 * 16


def pack_conv_weights(w, segs, ncols):
    """torch fp32 weights [co][sum(segs)][3][3] -> the BF16 operand that
    rl_dn_conv3x3 takes: [9][K/8][ncols][8] (tap = 3*ky + kx), K = the input
    segments' channels each padded to 16, rows past co zero."""
    import torch
    co = w.shape[0]
    k = sum(_pad16(c) for c in segs)
    full = torch.zeros(ncols, 9, k, device=w.device)
    src = w.permute(0, 2, 3, 1).reshape(co, 9, -1)
    off = o2 = 0
    for c in segs:
        full[:co, :, o2:o2 + c] = src[:, :, off:off + c]
        off += c
        o2 += _pad16(c)
    return full.reshape(ncols, 9, k // 8, 8).permute(1, 2, 0, 3).contiguous().to(torch.bfloat16)


class Denoiser:
    """rl_denoiser: the BF16 tensor-core encoder-decoder."""

    def __init__(self, seed: int = 1):
        self.handle = C.c_void_p()
        check(lib().rl_denoiser_create(seed, C.byref(self.handle)))
        n = C.c_int64()
        check(lib().rl_denoiser_param_count(self.handle, C.byref(n)))
        self.nparam = n.value

    # parameters ------------------------------------------------------
    def params(self):
        import numpy as np
        out = np.zeros(self.nparam, np.float32)
        check(lib().rl_denoiser_get_params(self.handle, C.c_void_p(out.ctypes.data)))
        return out

    def set_params(self, arr):
        import numpy as np
        arr = np.ascontiguousarray(arr, np.float32)
        assert arr.size == self.nparam
        check(lib().rl_denoiser_set_params(self.handle, C.c_void_p(arr.ctypes.data)))

    def grads(self):
        import numpy as np
        out = np.zeros(self.nparam, np.float32)
        check(lib().rl_denoiser_get_grads(self.handle, C.c_void_p(out.ctypes.data)))
        return out

    @staticmethod
    def unflatten(flat):
        """[(w [cout][9][k], b [cout])] per layer from a flat parameter array."""
        out, o = [], 0
        for cout, segs in LAYERS:
            k = sum(_pad64(s) for s in segs)
            w = flat[o:o + cout * 9 * k].reshape(cout, 9, k)
            o += cout * 9 * k
            out.append((w, flat[o:o + cout]))
            o += cout
        return out

    def save(self, path):
        import numpy as np
        np.save(path, self.params())

    def load(self, path):
        import numpy as np
        self.set_params(np.load(path))

    # compute ---------------------------------------------------------
    def train_step(self, x, t, lr, loss=None, stream=None):
        """One Adam step on a batch: x BF16 [b][p][p][16], t FP32 [b][p][p][4]."""
        b, p = x.shape[0], x.shape[1]
        check(lib().rl_denoiser_train_step(self.handle, _p(x), _p(t), b, p, float(lr), _p(loss), stream))

    def forward(self, x, stream=None):
        import torch
        y = torch.empty_like(x)
        n, h, w, _ = x.shape
        check(lib().rl_denoiser_forward(self.handle, _p(x), n, h, w, _p(y), stream))
        return y

    def apply(self, scene, lightmap, base=None, stream=None):
        """Denoise a baked lightmap (DeviceMap) of a DeviceScene in place."""
        check(lib().rl_denoiser_apply(self.handle, scene.handle, lightmap.handle, _p(base), stream))

    def reserve(self, images, height, width, train=False):
        """Pre-size the working buffers (rl_denoiser_reserve)."""
        check(lib().rl_denoiser_reserve(self.handle, images, height, width, int(train)))

    def status(self) -> int:
        f = C.c_int()
        check(lib().rl_denoiser_status(self.handle, C.byref(f)))
        return f.value

    def close(self):
        if self.handle:
            check(lib().rl_denoiser_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def features(scene, lightmap, stream=None):
    """BF16 [h][w][16] input features of a baked lightmap (rl_denoiser_features)."""
    import torch
    x = torch.empty(lightmap.height, lightmap.width, FEATURES, dtype=torch.bfloat16, device="cuda")
    check(lib().rl_denoiser_features(scene.handle, lightmap.handle, _p(x), stream))
    return x


def targets(lightmap, stream=None):
    """FP32 [h][w][4] training targets (log1p rgb, valid) of a baked lightmap."""
    import torch
    t = torch.empty(lightmap.height, lightmap.width, 4, dtype=torch.float32, device="cuda")
    check(lib().rl_denoiser_targets(lightmap.handle, _p(t), stream))
    return t


# ---------------------------------------------------------------- training data

def bake_fg(relight, ds, lightmap, photonmaps, settings, spp, seed, stream=None):
    """The final-gather component alone at `spp` samples (colours cleared first)."""
    from .device import _map_array
    lightmap.clear(colors=True, photons=False, stream=stream)
    sky = (C.c_float * 3)(*[float(v) for v in settings.sky_color])
    amb = (C.c_float * 3)(*[float(v) for v in settings.ambient_color])
    check(lib().rl_bake_indirect(ds.handle, lightmap.handle, _map_array(photonmaps), len(photonmaps), int(spp),
                                 float(settings.final_gather_distance), sky, amb, int(seed), None, stream))


def training_scenes(n, seed=100, sides=(256, 384, 512)):
    """Seeded terrain-and-boxes scenes (the bench scene's recipe at varied
    sizes) for (low, high) sample-count pairs."""
    import numpy as np
    from . import scenes
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        verts = int(rng.integers(48, 160))
        boxes = int(rng.integers(20, 600))
        side = int(rng.choice(sides))
        recipe = dict(seed=seed * 1000 + k, verts=verts, n_boxes=boxes, size=side, tiles=1, passes=2)
        wl = scenes.terrain_scene(**recipe)
        wl.recipe = recipe  # scenes.terrain_scene(**recipe) rebuilds it (e.g. in another process)
        out.append(wl)
    return out


def make_pairs(workloads, spp_lo=16, spp_hi=1024, seed=7, stream=None, builder=0):
    """Bake each workload's lightmap twice (final gather only, different
    seeds): features of the low-sample bake and targets of the high-sample
    one.  Returns [(x [h][w][16], t [h][w][4])] on the device."""
    from .device import Relight
    pairs = []
    for k, wl in enumerate(workloads):
        rl = Relight(stream, seed=seed + 31 * k, builder=builder)
        ds = rl.device_scene(wl.scene)
        rl.emit_photons(wl.scene, wl.settings)
        lm = wl.lightmap._device
        pms = [m._device for m in wl.scene.flat.photonmaps]
        bake_fg(rl, ds, lm, pms, wl.settings, spp_lo, seed * 7 + 2 * k + 1, stream)
        x = features(ds, lm, stream)
        bake_fg(rl, ds, lm, pms, wl.settings, spp_hi, seed * 7 + 2 * k + 2, stream)
        t = targets(lm, stream)
        pairs.append((x, t))
    return pairs


def make_patches(pairs, count, patch=64, seed=11, min_valid=0.3):
    """`count` random patch crops (at least `min_valid` valid texels) from
    the pairs: x BF16 [count][p][p][16], t FP32 [count][p][p][4]."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    xs, ts = [], []
    tries = 0
    while len(xs) < count and tries < 50 * count:
        tries += 1
        x, t = pairs[int(rng.integers(0, len(pairs)))]
        h, w = x.shape[0], x.shape[1]
        y0, x0 = int(rng.integers(0, h - patch + 1)), int(rng.integers(0, w - patch + 1))
        tt = t[y0:y0 + patch, x0:x0 + patch]
        if float(tt[..., 3].mean()) < min_valid:
            continue
        xs.append(x[y0:y0 + patch, x0:x0 + patch])
        ts.append(tt)
    return torch.stack(xs).contiguous(), torch.stack(ts).contiguous()


def train(dn, xs, ts, steps, batch=16, lr=2e-3, seed=5, stream=None, warmup=200):
    """Adam on random batches of the patch set: linear learning-rate warmup
    over `warmup` steps, then cosine decay; returns the per-step losses
    (mean L1 in log space)."""
    import math
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    loss = torch.zeros(steps, dtype=torch.float32, device="cuda")
    n = xs.shape[0]
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
        rate = lr * 0.5 * (1 + math.cos(math.pi * s / steps)) * min(1.0, (s + 1) / max(warmup, 1))
        dn.train_step(xs[idx].contiguous(), ts[idx].contiguous(), rate, loss=loss[s:s + 1], stream=stream)
    return loss.cpu().numpy() * 1.0


def rmse(a, b, valid):
    """Per-texel RMSE over valid lumels (linear colour)."""
    import numpy as np
    d = (np.asarray(a, np.float64) - np.asarray(b, np.float64))[valid]
    return float(np.sqrt((d * d).mean()))


def evaluate(dn, workloads, spp_lo=16, spp_ref=8192, plain=(16, 64, 256, 1024), seed=900, stream=None,
             truth=None):
    """Per-texel RMSE against a reference (linear colour) of the plain final
    gather at each sample count in `plain` and of the `spp_lo` bake after the
    denoiser, with the device time of each (bake, and bake + denoise).  The
    reference is truth(i, workload) -> (texel indices, expected colours
    [n][3][, the estimate's own noise variance per colour value]) when given
    (an FP64 high-sample estimate, called after the workload's photons are
    gathered on the device; its noise variance, when returned, is taken out
    of every mean squared error), else a `spp_ref` bake over all valid
    lumels.  The plain bake's sample count of equal RMSE is
    interpolated (log-log) inside the measured range, or past its end from
    the fit RMSE^2 = a / spp + c (c: the reference's own noise and any
    bias).  Returns {"plain": {spp: (rmse, ms)}, "denoised": (rmse, ms),
    "denoised_max_err", "equal_rmse_spp", "extrapolated",
    "plain_ms_at_equal_rmse", "speedup"}."""
    import numpy as np
    import torch
    from .device import Relight
    ev = lambda: torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream()
    acc_plain = {k: [0.0, 0.0, 0] for k in plain}
    acc_dn = [0.0, 0.0, 0]
    max_err = 0.0
    # working buffers sized up front, so no timed call allocates
    dn.reserve(1, max(w.lightmap.height for w in workloads), max(w.lightmap.width for w in workloads))
    for i, wl in enumerate(workloads):
        rl = Relight(stream, seed=seed + i)
        ds = rl.device_scene(wl.scene)
        rl.emit_photons(wl.scene, wl.settings)
        lm = wl.lightmap._device
        pms = [m._device for m in wl.scene.flat.photonmaps]
        noise_var = 0.0
        if truth is not None:
            torch.cuda.synchronize()
            t = truth(i, wl)
            texels, expect = t[0], t[1]
            noise_var = float(t[2]) if len(t) > 2 else 0.0
            n = wl.lightmap.width * wl.lightmap.height
            ref = np.zeros((n, 3), np.float64)
            ref[texels] = expect
            valid = np.zeros(n, bool)
            valid[texels] = True
        else:
            bake_fg(rl, ds, lm, pms, wl.settings, spp_ref, seed * 13 + i, stream)
            d = lm.download(stream, fields=("flags", "color"))
            valid = (d["flags"] & 1).astype(bool)
            ref = d["color"]

        def timed(fn):
            e0, e1 = ev(), ev()
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            return e0.elapsed_time(e1)

        for k in plain:
            ms = timed(lambda: bake_fg(rl, ds, lm, pms, wl.settings, k, seed * 17 + i * 31 + k, stream))
            c = lm.download(stream, fields=("color",))["color"]
            acc_plain[k][0] += rmse(c, ref, valid) ** 2 - noise_var
            acc_plain[k][1] += ms
            acc_plain[k][2] += 1

        def lo_and_denoise():
            bake_fg(rl, ds, lm, pms, wl.settings, spp_lo, seed * 19 + i, stream)
            dn.apply(ds, lm, stream=stream)

        if i == 0:
            lo_and_denoise()  # untimed warm-up of the denoiser's kernels
        ms = timed(lo_and_denoise)
        c = lm.download(stream, fields=("color",))["color"]
        acc_dn[0] += rmse(c, ref, valid) ** 2 - noise_var
        acc_dn[1] += ms
        acc_dn[2] += 1
        max_err = max(max_err, float(np.abs(c - ref)[valid].max()) if valid.any() else 0.0)
    res_plain = {k: (float(np.sqrt(max(v[0], 0.0) / v[2])), v[1] / v[2]) for k, v in acc_plain.items()}
    dn_rmse, dn_ms = float(np.sqrt(max(acc_dn[0], 0.0) / acc_dn[2])), acc_dn[1] / acc_dn[2]
    ks = sorted(res_plain)
    r = np.array([res_plain[k][0] for k in ks])
    extrapolated = False
    if dn_rmse >= r[0]:
        s_eq = float(ks[0])
    elif dn_rmse >= r[-1]:
        j = int(np.argmax(r <= dn_rmse))
        lk0, lk1 = np.log(ks[j - 1]), np.log(ks[j])
        f = (np.log(dn_rmse) - np.log(r[j - 1])) / (np.log(r[j]) - np.log(r[j - 1]))
        s_eq = float(np.exp(lk0 + f * (lk1 - lk0)))
    else:
        # least squares of RMSE^2 = a / spp + c over the measured counts
        A = np.stack([1.0 / np.array(ks, float), np.ones(len(ks))], 1)
        (a, c0), *_ = np.linalg.lstsq(A, r * r, rcond=None)
        extrapolated = True
        s_eq = float(a / (dn_rmse ** 2 - c0)) if dn_rmse ** 2 > c0 and a > 0 else float("inf")
    ms = np.array([res_plain[k][1] for k in ks])
    a1, b1 = np.polyfit(np.array(ks, float), ms, 1)  # bake time is linear in samples
    plain_ms_eq = float(a1 * s_eq + b1) if np.isfinite(s_eq) else float("inf")
    return {"plain": res_plain, "denoised": (dn_rmse, dn_ms), "denoised_max_err": max_err,
            "equal_rmse_spp": s_eq, "extrapolated": extrapolated, "plain_ms_at_equal_rmse": plain_ms_eq,
            "speedup": plain_ms_eq / dn_ms}


def _main():
    """Time the network's forward pass on a synthetic side x side feature map
    (CUDA events, after one warm-up pass): the inference a bake request
    pays.  Used as the profiling target of the convolution kernels."""
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.zeros(1, args.side, args.side, FEATURES, device="cuda")
    x[..., :10] = torch.rand(1, args.side, args.side, 10, device="cuda", generator=g)
    x = x.to(torch.bfloat16)
    dn = Denoiser(seed=1)
    dn.forward(x)
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dn.forward(x)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    # multiply-adds of the 8 convolutions as the MMAs run them (K padded to
    # 16 per input segment, N to 16) and as the network defines them
    flops, real, s = 0, 0, args.side
    sizes = [s, (s + 1) // 2, (s + 3) // 4, (s + 7) // 8]
    levels = [0, 1, 2, 3, 2, 1, 0, 0]
    for (cout, segs), lv in zip(LAYERS, levels):
        flops += 2 * sizes[lv] ** 2 * _pad16(cout) * 9 * sum(_pad16(c) for c in segs)
        real += 2 * sizes[lv] ** 2 * cout * 9 * sum(segs)
    print(json.dumps({"side": args.side, "forward_ms": min(ms), "mma_tflops": flops / (min(ms) / 1e3) / 1e12,
                      "network_tflops": real / (min(ms) / 1e3) / 1e12, "status": dn.status()}))


if __name__ == "__main__":
    _main()
