"""Shared setup of the adjoint tests: camera RGB, the base parameters of the
differentiable model (the 8 x 2048x1365 fitting workload) and a target rendered with
perturbed parameters (+-5% WB, +-0.02 matrix, +-0.1 EV, +-5% curves,
+-10% halation)."""
import numpy as np

from imops_b200 import synthetic


def camera_rgb(H, W, seed):
    import oracle
    m = synthetic.mosaic_f32(H, W, seed=seed)
    return oracle.amaze(m, "RGGB").astype(np.float32)


def base_vector():
    return synthetic.film_grad_base()


def perturbed_vector(seed=0):
    return synthetic.film_grad_perturbed(seed)
