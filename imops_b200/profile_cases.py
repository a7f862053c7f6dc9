"""Single-launch cases for profiling one kernel of the path under ncu.

  python -m imops_b200.profile_cases amaze --width 4096 --height 3072
  python -m imops_b200.profile_cases film81 --width 4096 --height 3072 [--scan bf16_tc]
  python -m imops_b200.profile_cases fwdbwd --width 6048 --height 4024
  python -m imops_b200.profile_cases display --width 6048 --height 4024
  python -m imops_b200.profile_cases xtrans --width 6032 --height 4032

Each case builds a seeded synthetic input, runs the stage once and
synchronises, so `ncu -k regex:<kernel> -c 1` captures exactly one launch.
"""
from __future__ import annotations

import argparse

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["amaze", "film81", "develop", "fwdbwd", "display", "xtrans"])
    ap.add_argument("--width", type=int, default=4096)
    ap.add_argument("--height", type=int, default=3072)
    ap.add_argument("--scan", choices=["fp32", "bf16_tc"], default="fp32",
                    help="the 81-bin scan's contractions: CUDA cores (FP32) or tensor cores (BF16 hi/lo)")
    a = ap.parse_args()

    import torch

    import imops_b200 as im
    from imops_b200 import synthetic

    W, H = a.width, a.height
    if a.case == "xtrans":
        # the 24 MP X-Trans frame: the reference's 3x3 mean, then the 3-pass
        # directional demosaic
        m = torch.from_numpy(synthetic.mosaic_f32(H, W, seed=1001, pattern=synthetic.XTRANS)).cuda()
        mean = im.demosaic_markesteijn(m, synthetic.XTRANS)
        out = im.demosaic_markesteijn3(m, synthetic.XTRANS)
        torch.cuda.synchronize()
        print(f"{a.case} {W}x{H} ok, mean {float(mean.mean()):.6f} {float(out.mean()):.6f}")
        return
    raw = torch.from_numpy(synthetic.mosaic_u16(H, W, seed=5).view(np.int16)).cuda()
    if a.case == "fwdbwd":
        # the differentiable model: AMaZE to camera RGB, forward, adjoint
        # against a target rendered with perturbed parameters
        p = im.DevelopParams()
        p.demosaic, p.cfa, p.clip_pt, p.target, p.film = im.DEMOSAIC_AMAZE, b"RGGB", 1.0, im.CS_CAMERA, 0
        for i in range(4):
            p.wb[i] = 1.0
        cam = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, p)
        target = im.param_forward(cam, im.FilmGradParams.from_vector(synthetic.film_grad_perturbed(2)))
        theta = im.FilmGradParams.from_vector(synthetic.film_grad_base())
        out = im.param_forward(cam, theta)
        grad = torch.zeros(25, dtype=torch.float64, device=cam.device)
        im.param_backward(cam, theta, grad, target=target, loss_scale=1.0 / (H * W * 3))
        torch.cuda.synchronize()
        print(f"{a.case} {W}x{H} ok, loss {float(grad[24]):.6e}")
        return
    p = im.DevelopParams()
    p.demosaic, p.cfa, p.clip_pt = im.DEMOSAIC_AMAZE, b"RGGB", 1.0
    for i in range(4):
        p.wb[i] = synthetic.WB[i]
    p.target = im.CS_ACESCG
    for i in range(9):
        p.calib_d65[i] = synthetic.CALIB_D65[i]
    p.film = 1 if a.case in ("develop", "display") else 0
    p.film_params = im.FilmParams(im.STOCK_BASELINE81, 0, 1, 0, -1.0, 1)
    scan = im.SCAN_BF16_TC if a.scan == "bf16_tc" else im.SCAN_FP32
    p.baseline = im.baseline_film_defaults(scan=scan)
    out = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, p)
    if a.case == "film81":
        torch.cuda.synchronize()
        im.film_process(out, stock=im.STOCK_BASELINE81, baseline=im.baseline_film_defaults(scan=scan))
    if a.case == "display":
        # the display modules after the scan, one chain launch through the
        # pipeline C-ABI: Exp -> SigmoidToneMap -> CST LinearSrgb -> Gamma
        from imops_b200.pipeline import Image, make_meta, parse_config, run_pixel_pipeline
        img = Image.from_rgb(out.cpu().numpy().reshape(H, W, 3), im.CS_ACESCG, make_meta())
        cfg = parse_config('[[pipeline_modules]]\nname = "Exp"\nev = 0.5\n'
                           '[[pipeline_modules]]\nname = "SigmoidToneMap"\n'
                           '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "LinearSrgb"\n'
                           '[[pipeline_modules]]\nname = "Gamma"\ngamma = 2.2\n')
        run_pixel_pipeline(img, cfg)
        out = torch.from_numpy(img.rgb_f32())
    torch.cuda.synchronize()
    print(f"{a.case} {W}x{H} ok, mean {float(out.mean()):.6f}")


if __name__ == "__main__":
    main()
