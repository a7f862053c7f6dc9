"""Parameter-fit workload (8 x 2048x1365 Bayer frames): a batch of mosaics, loss
= MSE to targets rendered with perturbed parameters, gradients w.r.t. the 24
parameters (WB 3, colour matrix 9, exposure 1, curves 3x3, halation
strength/sigma 2), Adam with a step of lr x (|initial value| + 0.01) per
parameter (the parameters differ in scale by orders of magnitude).  The loss
is the convergence figure: WB gains and matrix columns can trade off exactly,
and the halation sigma barely moves the loss, so the parameters themselves
need not return to the values the targets were rendered with.

  python -m experiments.fit_params [--images 8] [--width 2048] [--height 1365] [--steps 20]

Under torchrun each rank develops its share of the batch (images are
independent) and the 24 gradients + loss are summed across ranks with one
all-reduce per step -- the only collective of the path.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np


def shard(n_images: int, rank: int, world: int) -> list[int]:
    """Images of the batch this rank owns (round robin, independent units)."""
    return list(range(rank, n_images, world))


def reduce_grad(grad, dist=None):
    """Sum the per-rank gradient vector (24 params + loss) across ranks."""
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM)
    return grad


def batch_gradient(images, targets, theta, scale, backward_fn, grad_buffer, dist=None):
    """Accumulate backward_fn(image, target, theta, scale, grad) over this
    rank's images, then all-reduce.  backward_fn adds into grad_buffer."""
    grad_buffer.zero_()
    for x, t in zip(images, targets):
        backward_fn(x, t, theta, scale, grad_buffer)
    return reduce_grad(grad_buffer, dist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=8)
    ap.add_argument("--width", type=int, default=2048)
    ap.add_argument("--height", type=int, default=1365)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--lr", type=float, default=0.01)
    a = ap.parse_args()

    import torch

    import imops_b200 as im
    from imops_b200 import synthetic

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    H, W = a.height, a.width
    base = synthetic.film_grad_base()
    truth = synthetic.film_grad_perturbed(7)

    mine = shard(a.images, rank, world)
    cams, targets = [], []
    for i in mine:
        raw = torch.from_numpy(synthetic.mosaic_u16(H, W, seed=1000 + i).view(np.int16)).to(dev)
        p = im.DevelopParams()
        p.demosaic, p.cfa, p.clip_pt, p.target, p.film = 0, b"RGGB", 1.0, im.CS_CAMERA, 0
        for k in range(4):
            p.wb[k] = 1.0
        cam = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, p)
        cams.append(cam)
        targets.append(im.param_forward(cam, im.FilmGradParams.from_vector(truth)).clone())
    scale = 1.0 / (a.images * H * W * 3)
    grad = torch.zeros(25, dtype=torch.float64, device=dev)

    def backward_fn(x, t, theta, s, g):
        im.param_backward(x, im.FilmGradParams.from_vector(theta), g, target=t, loss_scale=s)

    theta = base.copy()
    m1, m2 = np.zeros(24), np.zeros(24)
    lr = a.lr * (np.abs(base) + 1e-2)
    for step in range(a.steps):
        t0 = time.perf_counter()
        g = batch_gradient(cams, targets, theta, scale, backward_fn, grad, dist).cpu().numpy()
        dt = time.perf_counter() - t0
        m1 = 0.9 * m1 + 0.1 * g[:24]
        m2 = 0.999 * m2 + 0.001 * g[:24] ** 2
        k = step + 1
        theta = theta - lr * (m1 / (1 - 0.9 ** k)) / (np.sqrt(m2 / (1 - 0.999 ** k)) + 1e-12)
        if rank == 0:
            err = np.abs(theta - truth).max()
            print(f"step {step:3d} loss {g[24]:.6e} |grad| {np.linalg.norm(g[:24]):.3e} max|theta-truth| {err:.3e} "
                  f"{dt * 1e3:.1f} ms", flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
