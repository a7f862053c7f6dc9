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

Under torchrun (one rank per GPU) the frames are split into size-balanced
bins, one per rank (balanced_bins: largest estimated cost first, each to the
least-loaded rank); every rank develops and differentiates its own frames
and the 24 gradients + loss are summed with one all-reduce per pass, the
only collective.  The pass time is the max over ranks.

  python -m experiments.uneven_batch [--images 16] [--passes 3] [--warmup 1]
  torchrun --nproc-per-node N --master-addr 127.0.0.1 -m experiments.uneven_batch
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


# estimated device time per pixel (ns) of a frame's develop + forward +
# backward, from the single-GPU stage rates of this workload: forward 22 and
# backward 7.6 GP/s for every frame, develop 7.7 GP/s through AMaZE (Bayer)
# and 133 GP/s through the 3x3 mean (X-Trans)
NS_PER_PX = {"bayer": 1 / 22.0 + 1 / 7.6 + 1 / 7.7, "xtrans": 1 / 22.0 + 1 / 7.6 + 1 / 133.0}


def frame_cost(spec) -> float:
    return spec["W"] * spec["H"] * NS_PER_PX[spec["sensor"]]


def balanced_bins(specs, world: int) -> list[list[int]]:
    """Frame indices per rank: frames in order of decreasing estimated cost,
    each to the rank with the least cost so far (ties to the lower rank).
    Deterministic, so every rank computes the same split."""
    order = sorted(range(len(specs)), key=lambda i: (-frame_cost(specs[i]), i))
    load = [0.0] * world
    bins = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        bins[r].append(i)
        load[r] += frame_cost(specs[i])
    return [sorted(b) for b in bins]


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

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    all_specs = [frame_spec(i, im.amaze_size_supported) for i in range(a.images)]
    mine = balanced_bins(all_specs, world)[rank]
    specs = [all_specs[i] for i in mine]
    # the spawn pool starts before any CUDA call
    mosaics = make_mosaics(specs, max(1, min(16, (os.cpu_count() or 1) // world)))

    import torch

    from bench import Clocks, init_ranks, peaks
    from experiments.fit_params import reduce_grad

    torch.cuda.set_device(local)
    dist = init_ranks(world, "nccl")
    dev = torch.device("cuda", local)
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
    total_px = sum(s["W"] * s["H"] for s in all_specs)  # the whole batch: the loss is over every frame
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
        if ev:
            ev[-1][0].record(stream)
        reduce_grad(grad, dist)  # the batch gradient: one all-reduce of 25 doubles
        if ev:
            ev[-1][1].record(stream)

    for _ in range(a.warmup):
        one_pass()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # per pass: 4 events per frame, then a pair around the all-reduce
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in frames] +
           [[torch.cuda.Event(enable_timing=True) for _ in range(2)]] for _ in range(a.passes)]
    launches0 = im.launch_count()
    with Clocks(local) as clk:
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
    my_px = sum(f["W"] * f["H"] for f in frames)
    for ev in evs:
        for f, e in zip(frames, ev):
            for k, n in enumerate(names):
                t[n] += e[k].elapsed_time(e[k + 1]) / a.passes
            t_dev[f["sensor"]][0] += e[0].elapsed_time(e[1]) / a.passes
    for f in frames:
        t_dev[f["sensor"]][1] += f["W"] * f["H"]
    t_pass = sum(e[0][0].elapsed_time(e[-1][1]) for e in evs) / a.passes
    t_allreduce = sum(e[-1][0].elapsed_time(e[-1][1]) for e in evs) / a.passes
    t_rank = t_pass
    if dist:
        tt = torch.tensor([t_pass], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_pass = float(tt.item())
    stages = {}
    for n in names:
        mp_s = my_px / (t[n] / 1e3) / 1e6
        gbs = BYTES_PER_PX[n] * my_px / (t[n] / 1e3) / 1e9
        stages[n] = {"ms": round(t[n], 3), "mp_s": round(mp_s, 1), "bytes_per_px": BYTES_PER_PX[n],
                     "hbm_gbs": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4)}
    for sensor, (ms, px) in t_dev.items():
        if px:
            stages[f"develop_{sensor}"] = {"ms": round(ms, 3), "mp_s": round(px / (ms / 1e3) / 1e6, 1),
                                           "megapixels": round(px / 1e6, 2)}
    if rank == 0:
        print(json.dumps({
            "workload": "uneven batch: 16 frames 12-45 MP 3:2, mixed Bayer/X-Trans, develop + colour/film fwd+bwd, "
                        "grain off",
            "frames": [{k: s[k] for k in ("seed", "W", "H", "sensor")} for s in all_specs],
            "n_gpus": world, "bins": balanced_bins(all_specs, world),
            "megapixels": round(total_px / 1e6, 2), "passes": a.passes, "warmup": a.warmup,
            "ms_per_pass": round(t_pass, 3), "mp_s": round(total_px / (t_pass / 1e3) / 1e6, 1),
            "rank0": {"ms_per_pass": round(t_rank, 3), "allreduce_ms": round(t_allreduce, 4),
                      "megapixels": round(my_px / 1e6, 2), "stages": stages},
            "hbm_peak_gbs": hbm, "hbm_peak_kind": hbm_kind, "gpu_launches_rank0": launches, "loss": float(g[24]),
            "clocks_rank0": clk.summary()}))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
