"""The data-parallel gradient path of experiments/fit_params.py on CPU with
two gloo ranks: sharded per-image gradients summed by the all-reduce equal
the single-process batch gradient.  The per-image gradient here is the FP64
oracle (no GPU needed); on GPUs the same code runs imops_param_backward."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from adjoint_setup import base_vector, camera_rgb, perturbed_vector


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _images(n):
    import oracle
    xs, ts = [], []
    for i in range(n):
        x = camera_rgb(72, 80, seed=300 + i).astype(np.float64)
        t = oracle.param_forward(x, oracle.OracleGrad.from_vector(perturbed_vector(i)))
        xs.append(x)
        ts.append(t)
    return xs, ts


def _backward(x, t, theta, scale, g):
    import oracle
    fixed = oracle.baseline_params(grain_on=0, hal_radius=16, hal_sigma=5.0)
    out = oracle.param_grad(x, t, oracle.OracleGrad.from_vector(theta), scale, fixed)
    g += torch.from_numpy(out)


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from experiments.fit_params import batch_gradient, shard
    n = 4
    xs, ts = _images(n)
    mine = shard(n, rank, world)
    g = torch.zeros(25, dtype=torch.float64)
    theta = base_vector().copy()
    theta[23] = 5.0
    batch_gradient([xs[i] for i in mine], [ts[i] for i in mine], theta, 1e-4, _backward, g, dist)
    if rank == 0:
        q.put(g.numpy().copy())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_gradient_allreduce_matches_single_process():
    from experiments.fit_params import batch_gradient, shard
    assert shard(8, 0, 2) == [0, 2, 4, 6] and shard(8, 1, 2) == [1, 3, 5, 7]
    xs, ts = _images(4)
    theta = base_vector().copy()
    theta[23] = 5.0
    ref = torch.zeros(25, dtype=torch.float64)
    batch_gradient(xs, ts, theta, 1e-4, _backward, ref, None)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    np.testing.assert_allclose(got, ref.numpy(), rtol=1e-12, atol=0)
