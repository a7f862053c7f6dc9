"""Uneven batch: 16 raw frames of mixed sizes and sensors through the colour +
film model, forward and adjoint, grain off.

Frame i is drawn from seed 1000 + i: an area uniform in 12-45 MP at aspect
3:2 (at most 8256x5504), and a Bayer (RGGB, AMaZE) or X-Trans (6x6, the
reference's 3x3-mean demosaic) sensor with equal odds.  Width and height are
multiples of 6 (the X-Trans period); Bayer frames step down by 6 until AMaZE's
tiling accepts them.  Per frame and per pass:

  develop   u16 frame -> camera RGB (scale, demosaic)         imops_develop_u16
  forward   24-parameter colour + film model                  imops_param_forward
  backward  its adjoint against a target (loss + 24 grads)    imops_param_backward

Targets are rendered once with perturbed parameters.  Each stage is timed
with CUDA events on the launching stream and summed over the batch; the
output is one JSON line with per-stage MP/s, the algorithmic HBM bytes per
pixel and their fraction of the measured copy bandwidth, and the SM clocks
sampled during the timed passes.

  python -m experiments.uneven_batch [--images 16] [--passes 3] [--warmup 1]
"""
from __future__ import annotations

import argparse
import json
import math
import os

import numpy as np

MIN_MP, MAX_MP = 12e6, 45e6
MAX_W, MAX_H = 8256, 5504
PERIOD = 6

# algorithmic HBM bytes per pixel: develop reads the u16 frame and writes f32
# RGB; forward reads and writes f32 RGB; backward reads the frame's RGB and the
# target (its gradients are block reductions, a few bytes per block)
BYTES_PER_PX = {"develop": 2 + 12, "forward": 12 + 12, "backward": 12 + 12}


def frame_spec(i: int, amaze_ok) -> dict:
    """Size and sensor of frame i.  `amaze_ok(W, H)` is AMaZE's size rule
    (imops_amaze_size_supported)."""
    rng = np.random.default_rng(1000 + i)
    area = rng.uniform(MIN_MP, MAX_MP)
    xtrans = bool(rng.random() < 0.5)
    W = min(MAX_W, int(math.sqrt(area * 1.5)) // PERIOD * PERIOD)
    H = min(MAX_H // PERIOD * PERIOD, int(round(W / 1.5)) // PERIOD * PERIOD)
    if not xtrans:
        while not amaze_ok(W, H):
            if not amaze_ok(W, 96):
                W -= PERIOD
            else:
                H -= PERIOD
    return {"seed": 1000 + i, "W": W, "H": H, "sensor": "xtrans" if xtrans else "bayer"}


def _mosaic(spec):
    from imops_b200 import synthetic
    pattern = synthetic.XTRANS if spec["sensor"] == "xtrans" else "RGGB"
    return synthetic.mosaic_u16(spec["H"], spec["W"], spec["seed"], pattern)


def make_mosaics(specs, workers: int):
    """Synthetic frames on a spawn pool (started before any CUDA call)."""
    if workers <= 1:
        return [_mosaic(s) for s in specs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_mosaic, specs))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=16)
    ap.add_argument("--passes", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()

    import imops_b200 as im
    from imops_b200 import synthetic

    specs = [frame_spec(i, im.amaze_size_supported) for i in range(a.images)]
    mosaics = make_mosaics(specs, min(16, os.cpu_count() or 1))

    import torch

    from bench import Clocks, peaks

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    theta = im.FilmGradParams.from_vector(synthetic.film_grad_base())
    truth = im.FilmGradParams.from_vector(synthetic.film_grad_perturbed(2))

    frames = []
    for s, m in zip(specs, mosaics):
        xt = s["sensor"] == "xtrans"
        p = im.DevelopParams()
        p.demosaic = im.DEMOSAIC_MARKESTEIJN if xt else im.DEMOSAIC_AMAZE
        p.cfa = (synthetic.XTRANS if xt else "RGGB").encode()
        p.clip_pt, p.target, p.film, p.n_gain = 1.0, im.CS_CAMERA, 0, 0
        for k in range(4):
            p.wb[k] = 1.0
        raw = torch.from_numpy(m.view(np.int16)).to(dev)
        cam = torch.empty((s["H"], s["W"], 3), device=dev)
        period = (6, 6) if xt else (2, 2)
        im.develop_u16(raw, (0, 0, s["W"], s["H"]), synthetic.BLACK, synthetic.WHITE, p, period=period, out=cam)
        target = im.param_forward(cam, truth)
        frames.append({"raw": raw, "p": p, "period": period, "cam": cam, "out": torch.empty_like(cam),
                       "target": target, **s})
    del mosaics
    total_px = sum(f["W"] * f["H"] for f in frames)
    loss_scale = 1.0 / (3 * total_px)
    grad = torch.zeros(25, dtype=torch.float64, device=dev)

    def one_pass(ev=None):
        grad.zero_()
        for j, f in enumerate(frames):
            if ev:
                ev[j][0].record(stream)
            im.develop_u16(f["raw"], (0, 0, f["W"], f["H"]), synthetic.BLACK, synthetic.WHITE, f["p"],
                           period=f["period"], out=f["cam"], stream=stream)
            if ev:
                ev[j][1].record(stream)
            im.param_forward(f["cam"], theta, out=f["out"], stream=stream)
            if ev:
                ev[j][2].record(stream)
            im.param_backward(f["cam"], theta, grad, target=f["target"], loss_scale=loss_scale, stream=stream)
            if ev:
                ev[j][3].record(stream)

    for _ in range(a.warmup):
        one_pass()
    torch.cuda.synchronize()
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in frames] for _ in range(a.passes)]
    launches0 = im.launch_count()
    with Clocks(0) as clk:
        torch.cuda.synchronize()
        for ev in evs:
            one_pass(ev)
        torch.cuda.synchronize()
    launches = im.launch_count() - launches0
    g = grad.cpu().numpy()
    assert np.isfinite(g).all()

    hbm, hbm_kind = peaks()
    names = ["develop", "forward", "backward"]
    t = {n: 0.0 for n in names}
    t_dev = {"bayer": [0.0, 0], "xtrans": [0.0, 0]}
    for ev in evs:
        for f, e in zip(frames, ev):
            for k, n in enumerate(names):
                t[n] += e[k].elapsed_time(e[k + 1]) / a.passes
            t_dev[f["sensor"]][0] += e[0].elapsed_time(e[1]) / a.passes
    for f in frames:
        t_dev[f["sensor"]][1] += f["W"] * f["H"]
    t_pass = sum(e[0][0].elapsed_time(e[-1][3]) for e in evs) / a.passes
    stages = {}
    for n in names:
        mp_s = total_px / (t[n] / 1e3) / 1e6
        gbs = BYTES_PER_PX[n] * total_px / (t[n] / 1e3) / 1e9
        stages[n] = {"ms": round(t[n], 3), "mp_s": round(mp_s, 1), "bytes_per_px": BYTES_PER_PX[n],
                     "hbm_gbs": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4)}
    for sensor, (ms, px) in t_dev.items():
        if px:
            stages[f"develop_{sensor}"] = {"ms": round(ms, 3), "mp_s": round(px / (ms / 1e3) / 1e6, 1),
                                           "megapixels": round(px / 1e6, 2)}
    print(json.dumps({
        "workload": "uneven batch: 16 frames 12-45 MP 3:2, mixed Bayer/X-Trans, develop + colour/film fwd+bwd, "
                    "grain off",
        "frames": [{k: f[k] for k in ("seed", "W", "H", "sensor")} for f in frames],
        "megapixels": round(total_px / 1e6, 2), "passes": a.passes, "warmup": a.warmup,
        "ms_per_pass": round(t_pass, 3), "mp_s": round(total_px / (t_pass / 1e3) / 1e6, 1),
        "stages": stages, "hbm_peak_gbs": hbm, "hbm_peak_kind": hbm_kind, "gpu_launches": launches, "loss": float(g[24]),
        "clocks": clk.summary()}))


if __name__ == "__main__":
    main()
