"""Shared setup of the adjoint tests: camera RGB, the base parameters of the
differentiable model and a target rendered with
perturbed parameters (+-5% WB, +-0.02 matrix, +-0.1 EV, +-5% curves,
+-10% halation)."""
import numpy as np

from imops_b200 import synthetic

XYZ2AP1 = np.array([[1.6410233797, -0.3248032942, -0.2364246952], [-0.6636628587, 1.6153315917, 0.0167563477],
                    [0.0117218943, -0.0082844165, 0.9883948585]])


def camera_rgb(H, W, seed):
    import oracle
    m = synthetic.mosaic_f32(H, W, seed=seed)
    return oracle.amaze(m, "RGGB").astype(np.float32)


def base_vector():
    import oracle
    F = oracle.camera_forward_matrix(synthetic.CALIB_D65, precision="f64")
    C = (XYZ2AP1 @ F).reshape(9)
    return np.array([2.0, 1.0, 1.5, *C, 0.0, 2.0, 2.1, 2.2, 2.3, 2.5, 2.7, -0.70, -0.73, -0.76, 0.15, 20.0])


def perturbed_vector(seed=0):
    rng = np.random.default_rng(seed)
    v = base_vector().copy()
    v[0:3] *= 1 + rng.uniform(-0.05, 0.05, 3)
    v[3:12] += rng.uniform(-0.02, 0.02, 9)
    v[12] += rng.uniform(-0.1, 0.1)
    v[13:22] *= 1 + rng.uniform(-0.05, 0.05, 9)
    v[22:24] *= 1 + rng.uniform(-0.1, 0.1, 2)
    return v
