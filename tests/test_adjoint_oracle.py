"""FP64 oracle of the adjoint: analytic gradients against central finite
differences (h = 1e-3) of the FP64 forward, for all 24 parameters."""
import numpy as np

from adjoint_setup import base_vector, camera_rgb, perturbed_vector


def test_fp64_gradient_matches_central_differences(oracle_lib):
    x = camera_rgb(96, 112, seed=51).astype(np.float64)
    G = oracle_lib.OracleGrad
    target = oracle_lib.param_forward(x, G.from_vector(perturbed_vector(1)))
    v0 = base_vector()
    # float32 parameters: evaluate at the f32-rounded point
    v0 = np.array(G.from_vector(v0).to_vector())
    scale = 1.0 / x.size
    g = oracle_lib.param_grad(x, target, G.from_vector(v0), scale)
    def loss(v):
        o = oracle_lib.param_forward(x, G.from_vector(v))
        return scale * ((o - target) ** 2).sum()
    assert abs(g[24] - loss(v0)) < 1e-12 * max(1.0, abs(g[24]))
    h = 1e-3
    fd = np.zeros(24)
    for i in range(24):
        vp, vm = v0.copy(), v0.copy()
        vp[i] += h
        vm[i] -= h
        # parameters are f32 in the model: use the actually representable step
        sp = G.from_vector(vp).to_vector()[i] - v0[i]
        sm = v0[i] - G.from_vector(vm).to_vector()[i]
        fd[i] = (loss(vp) - loss(vm)) / (sp + sm)
    rel = np.abs(g[:24] - fd) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    assert rel.max() < 1e-3, f"worst parameter {int(rel.argmax())}: analytic {g[rel.argmax()]} fd {fd[rel.argmax()]}"
