"""GPU adjoint kernels against the FP64 oracle (forward, analytic
gradients) and against central finite differences (h = 1e-3)."""
import numpy as np
import pytest

from adjoint_setup import base_vector, camera_rgb, perturbed_vector

pytestmark = pytest.mark.gpu


def _setup(gpu, H=128, W=160, seed=61):
    import torch
    import oracle
    x = camera_rgb(H, W, seed)
    tgt = oracle.param_forward(x.astype(np.float64), oracle.OracleGrad.from_vector(perturbed_vector(2)))
    return x, tgt, torch.from_numpy(x).to(gpu), torch.from_numpy(tgt.astype(np.float32)).to(gpu)


def test_param_forward_matches_fp64(gpu):
    import imops_b200 as im
    import oracle
    x, _, xd, _ = _setup(gpu)
    v = base_vector()
    out = im.param_forward(xd, im.FilmGradParams.from_vector(v)).cpu().numpy()
    ref = oracle.param_forward(x.astype(np.float64), oracle.OracleGrad.from_vector(v))
    assert np.abs(out - ref).max() < 1e-4


def test_param_gradient_matches_fp64_oracle(gpu):
    import torch
    import imops_b200 as im
    import oracle
    x, tgt, xd, td = _setup(gpu)
    v = np.array(oracle.OracleGrad.from_vector(base_vector()).to_vector())
    scale = 1.0 / x.size
    grad = torch.zeros(25, dtype=torch.float64, device=gpu)
    im.param_backward(xd, im.FilmGradParams.from_vector(v), grad, target=td, loss_scale=scale)
    g = grad.cpu().numpy()
    ref = oracle.param_grad(x.astype(np.float64), tgt.astype(np.float32).astype(np.float64),
                            oracle.OracleGrad.from_vector(v), scale)
    rel = np.abs(g - ref) / np.maximum(np.abs(ref), 1e-3 * np.abs(ref[:24]).max())
    assert rel.max() < 1e-3, f"worst {int(rel.argmax())}: gpu {g[rel.argmax()]} fp64 {ref[rel.argmax()]}"


def test_param_gradient_matches_central_differences(gpu):
    import torch
    import imops_b200 as im
    import oracle
    x, tgt, xd, td = _setup(gpu, seed=62)
    G = oracle.OracleGrad
    v0 = np.array(G.from_vector(base_vector()).to_vector())
    scale = 1.0 / x.size
    grad = torch.zeros(25, dtype=torch.float64, device=gpu)
    im.param_backward(xd, im.FilmGradParams.from_vector(v0), grad, target=td, loss_scale=scale)
    g = grad.cpu().numpy()[:24]
    tgt64 = tgt.astype(np.float32).astype(np.float64)
    def loss(v):
        o = oracle.param_forward(x.astype(np.float64), G.from_vector(v))
        return scale * ((o - tgt64) ** 2).sum()
    h = 1e-3
    fd = np.zeros(24)
    for i in range(24):
        vp, vm = v0.copy(), v0.copy()
        vp[i] += h
        vm[i] -= h
        sp = G.from_vector(vp).to_vector()[i] - v0[i]
        sm = v0[i] - G.from_vector(vm).to_vector()[i]
        fd[i] = (loss(vp) - loss(vm)) / (sp + sm)
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    assert rel.max() < 1e-3, f"worst {int(rel.argmax())}: gpu {g[rel.argmax()]} fd {fd[rel.argmax()]}"


def test_param_backward_accumulates_over_a_batch(gpu):
    import torch
    import imops_b200 as im
    _, _, xa, ta = _setup(gpu, seed=63)
    _, _, xb, tb = _setup(gpu, seed=64)
    p = im.FilmGradParams.from_vector(base_vector())
    ga = torch.zeros(25, dtype=torch.float64, device=gpu)
    gb = torch.zeros(25, dtype=torch.float64, device=gpu)
    both = torch.zeros(25, dtype=torch.float64, device=gpu)
    im.param_backward(xa, p, ga, target=ta, loss_scale=1e-5)
    im.param_backward(xb, p, gb, target=tb, loss_scale=1e-5)
    im.param_backward(xa, p, both, target=ta, loss_scale=1e-5)
    im.param_backward(xb, p, both, target=tb, loss_scale=1e-5)
    assert torch.allclose(both, ga + gb, rtol=1e-12, atol=0)


def test_param_backward_with_upstream_gradient(gpu):
    import torch
    import imops_b200 as im
    _, _, xd, td = _setup(gpu, seed=65)
    p = im.FilmGradParams.from_vector(base_vector())
    out = im.param_forward(xd, p)
    scale = 1.0 / xd.numel()
    g_out = (2 * scale * (out - td)).contiguous()
    g1 = torch.zeros(25, dtype=torch.float64, device=gpu)
    g2 = torch.zeros(25, dtype=torch.float64, device=gpu)
    im.param_backward(xd, p, g1, g_out=g_out)
    im.param_backward(xd, p, g2, target=td, loss_scale=scale)
    assert torch.allclose(g1[:24], g2[:24], rtol=1e-5, atol=1e-12)


def test_autograd_function_matches_adjoint(gpu):
    import sys
    import torch
    import imops_b200 as im
    sys.path.insert(0, __import__("os").path.dirname(__import__("os").path.dirname(__file__)))
    from experiments.film_autograd import film_model
    _, _, xd, td = _setup(gpu, seed=66)
    theta = torch.tensor(base_vector(), dtype=torch.float64, requires_grad=True)
    out = film_model(xd, theta)
    loss = ((out.double() - td.double()) ** 2).mean()
    loss.backward()
    ref = torch.zeros(25, dtype=torch.float64, device=gpu)
    im.param_backward(xd, im.FilmGradParams.from_vector(base_vector()), ref, target=td, loss_scale=1.0 / xd.numel())
    assert torch.allclose(theta.grad, ref[:24].cpu(), rtol=1e-4, atol=1e-12)
