"""Benchmark of the raw-development hot path on B200.

Workload (one step): the 24 MP Bayer forward -- a 6048x4024 RGGB 14-bit
(black 600, white 16383) synthetic mosaic, black/white scaling to f32, the
AMaZE demosaic with WB (2, 1, 1.5) + camera matrix to ACEScg fused into its
output, then the 81-bin spectral film simulation (3 layers,
logistic curves, halation sigma 20 px / 0.15 on R > 0.8, seeded grain
sigma 0.02).  Metric: megapixels per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one rank per GPU, each developing its own frame (weak scaling,
no collective on the data path); time = max over ranks.  Started under
torchrun the ranks come from its environment; started plainly with
--gpus N > 1, bench.py launches the N ranks itself (torchrun on this node,
127.0.0.1).  --dry-run runs the launch and rank plumbing (gloo, barrier,
max-over-ranks reduction, rank 0's JSON line) without touching a GPU.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import queue
import signal
import socket
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

H, W = 4024, 6048
SEED = 1002
METRIC = "MP/s fwd, 24MP AMaZE+colour+film on 1xB200"
L2_FLUSH_BYTES = 256 << 20
PIPELINE_CONFIG = """
[[pipeline_modules]]
name = "Demosaic"
algorithm = "amaze"
[[pipeline_modules]]
name = "CFACoeffs"
[[pipeline_modules]]
name = "CST"
target_color_space = "AcesCg"
[[pipeline_modules]]
name = "Film"
stock = "Baseline81"
film_format = "Film35mm"
seed = 1002
output = "NegativeLinear"
"""


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="imops_b200", choices=["imops_b200", "reference"])
    ap.add_argument("--dry-run", action="store_true",
                    help="launch and rank plumbing only (gloo, no GPU work); prints a line with dry_run: true")
    return ap.parse_args()


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


LAUNCH_TIMEOUT_S = 1800  # last bound on a self-launched run, far above the process groups' 120 s timeout


def launch_ranks(args) -> int:
    """--gpus N (N > 1) outside torchrun: run N ranks of this script, one per
    GPU, under torchrun on this node and return its exit status.  Rank 0
    prints the JSON line."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.abspath(__file__),
           *sys.argv[1:]]
    proc = subprocess.Popen(cmd, start_new_session=True)
    try:
        return proc.wait(timeout=LAUNCH_TIMEOUT_S)
    except subprocess.TimeoutExpired:
        os.killpg(proc.pid, signal.SIGKILL)  # torchrun and its ranks: the group this call started
        proc.wait()
        print(f"bench.py: {args.gpus} ranks did not finish within {LAUNCH_TIMEOUT_S} s", file=sys.stderr)
        return 124


def init_ranks(world: int, backend: str):
    """The process group of a multi-rank run (short timeout, so ranks that
    wait for one another end with an error), or None for one rank."""
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def dry_run(args, rank, world):
    """The launch and rank plumbing without a GPU: every rank times a small
    host computation, the time is reduced to the max over ranks, and rank 0
    prints the line with n_gpus = the number of ranks that took part."""
    import numpy as np
    import torch

    dist = init_ranks(world, "gloo")
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.warmup + args.steps):
        np.sort(np.random.default_rng(rank * 1000 + k).random(1 << 16))
    t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64)
    ranks = torch.ones(1, dtype=torch.float64)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(ranks, op=dist.ReduceOp.SUM)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": "MP/s", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "dry_run": True, "impl": args.impl, "ranks_reporting": int(ranks.item()),
                          "max_rank_s": round(float(t.item()), 6), "config": workload_config(world)}), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_figure(key):
    """A per-launch figure of the dominant kernel (`traffic_bytes_per_launch`,
    `warp_instructions_per_launch`) from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "amaze_develop_6048x4024_ncu.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            try:
                return int(line.split(":")[1].strip().split()[0])
            except ValueError:
                return None
    return None


def ncu_traffic():
    return ncu_figure("traffic_bytes_per_launch")


def issue_fraction(t_ms, clk):
    """The dominant kernel against the SM issue rate: its warp instructions
    per launch (ncu count, scaled to the frame) over its CUDA-event time,
    divided by SMs x 4 schedulers x the SM clock (the sampled maximum, else
    1965 MHz)."""
    import torch
    inst = ncu_figure("warp_instructions_per_launch")
    if not inst or not t_ms:
        return None
    mhz = (clk or {}).get("sm_max_mhz") or 1965.0
    peak = torch.cuda.get_device_properties(0).multi_processor_count * 4 * mhz * 1e6
    achieved = inst / (t_ms / 1e3)
    return {"achieved": round(achieved / 1e9, 1), "peak": round(peak / 1e9, 1), "unit": "G warp-instr/s",
            "frac": round(achieved / peak, 4), "instructions_per_launch": inst}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 6:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def develop_params(im, film: bool):
    from imops_b200 import synthetic
    p = im.DevelopParams()
    p.demosaic = im.DEMOSAIC_AMAZE
    p.cfa = b"RGGB"
    p.clip_pt = 1.0
    for i in range(4):
        p.wb[i] = synthetic.WB[i]
    p.n_gain = 0
    p.target = im.CS_ACESCG
    for i in range(9):
        p.calib_d65[i] = synthetic.CALIB_D65[i]
    p.film = 1 if film else 0
    p.film_params = im.FilmParams(im.STOCK_BASELINE81, 0, 1, 0, -1.0, 1)
    p.baseline = im.baseline_film_defaults(seed=SEED)
    return p


def cpu_sample(threads: int):
    """The oracle port on the host: AMaZE + colour + 81-bin film on a
    1536x1024 crop of the workload's frame (same generator, same seed)."""
    import numpy as np

    import oracle
    from imops_b200 import synthetic
    h, w = 1024, 1536
    m = synthetic.mosaic_f32(h, w, seed=SEED)
    t0 = time.perf_counter()
    rgb = oracle.amaze(m, "RGGB", threads=threads)
    rgb = oracle.wb(rgb, synthetic.WB)
    rgb = oracle.camera_cst(rgb, synthetic.CALIB_D65, oracle.CS_ACESCG)
    out = oracle.film_baseline(rgb, oracle.baseline_params(seed=SEED), precision="f32", threads=threads)
    dt = time.perf_counter() - t0
    assert np.isfinite(out).all()
    return h * w / 1e6 / dt, f"{w}x{h} crop of the 6048x4024 frame: AMaZE + WB + CST + 81-bin film (f32 oracle)"


def cpu_check_error(raw_np, colour, film, film_other_scan=None):
    """Error of this rank's frame against FP64, whole frame: max and RMS
    absolute error in linear [0, 1] and in 16-bit LSB of
      colour      the colour forward (AMaZE + WB + camera matrix) against the
                  FP64 colour chain; AMaZE decision flips (more than 8 LSB from
                  FP64, where a comparison resolves differently in f32) apart;
      film_stage  the film output against the FP64 film of the same colour;
      film_chain  the film output against the FP64 chain end to end (flips
                  apart): the film's curves amplify the colour stage's error.
    Host cores, after the timed regions; the oracle is the checker here."""
    import oracle
    from imops_b200 import synthetic
    t0 = time.perf_counter()
    r = lambda d: {k: (round(v, 9) if k.endswith("abs") else round(v, 4)) for k, v in d.items()}
    bp = oracle.baseline_params(seed=SEED)
    stage64 = oracle.film_baseline(colour, bp, precision="f64")
    out = {"vs": "FP64 oracle (scaling, AMaZE, WB, camera matrix, 81-bin film with grain), whole frame",
           "pixels": int(raw_np.size), "film_stage": r(oracle.error_figures(film, stage64))}
    if film_other_scan is not None:
        out["film_stage_other_scan"] = r(oracle.error_figures(film_other_scan, stage64))
    del stage64
    c64 = oracle.colour_chain(raw_np, synthetic.BLACK, synthetic.WHITE, synthetic.WB, synthetic.CALIB_D65)
    flips = oracle.decision_flips(colour, c64)
    out["amaze_decision_flips"] = int(flips.sum())
    out["colour"] = r(oracle.error_figures(colour, c64, skip=flips))
    chain64 = oracle.film_baseline(c64, bp, precision="f64")
    out["film_chain"] = r(oracle.error_figures(film, chain64, skip=flips))
    out["film_chain_incl_flips_max_lsb"] = round(oracle.error_figures(film, chain64)["max_lsb"], 2)
    out["check_s"] = round(time.perf_counter() - t0, 1)
    return out


def workload_config(world):
    """The workload both arms report (the reference arm times a bounded sample
    of it, described in its cpu_baseline.sample)."""
    return {"workload": "24MP Bayer forward: 6048x4024 RGGB u16 14-bit -> AMaZE -> WB+CST(ACEScg) -> "
                        "81-bin film (halation, grain)", "global_batch": world, "frames_per_gpu": 1,
            "parallelism": f"replicas x{world}", "l2": "256 MB buffer written between timed steps"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, sample = cpu_sample(threads)
        if i >= args.warmup:
            vals.append(v)
    value = sum(vals) / len(vals)
    line = {"metric": METRIC, "value": round(value, 3), "unit": "MP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1536 * 1024 / 1e3 / value, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(world),
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 3), "unit": "MP/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "MP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.dry_run:
        return dry_run(args, rank, world)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch

    import imops_b200 as im
    from imops_b200 import synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_ranks(world, "nccl")

    raw_np = synthetic.mosaic_u16(H, W, seed=SEED + rank)
    raw = torch.from_numpy(raw_np.view(np.int16)).to(dev)
    rgb = torch.empty((H, W, 3), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev)
    black = (ctypes.c_float * 4)(*([synthetic.BLACK] * 4))
    white = (ctypes.c_float * 4)(*([synthetic.WHITE] * 4))
    p_dem = develop_params(im, film=False)
    p_all = develop_params(im, film=True)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    L = im.lib()
    L.imops_develop_u16.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(im.DevelopParams),
        ctypes.c_void_p, ctypes.c_void_p]
    L.imops_film_process.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(im.FilmParams), ctypes.c_void_p, ctypes.c_void_p]
    L.imops_launch_count.restype = ctypes.c_uint64

    def step_device(events=None):
        if events:
            events[0].record(stream)
        im.check(L.imops_develop_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                                     ctypes.byref(p_dem), ctypes.c_void_p(rgb.data_ptr()), sp))
        if events:
            events[1].record(stream)
        im.check(L.imops_film_process(ctypes.c_void_p(rgb.data_ptr()), W, H, im.CS_ACESCG,
                                      ctypes.byref(p_all.film_params), ctypes.byref(p_all.baseline), sp))
        if events:
            events[2].record(stream)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    launches0 = L.imops_launch_count()
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(float(k))  # evict the previous step's data from L2
            step_device(ev[k])
        torch.cuda.synchronize()
    launches = L.imops_launch_count() - launches0
    if dist:
        dist.barrier()
    t_total = sum(e[0].elapsed_time(e[2]) for e in ev)  # ms over K steps
    t_dem = sum(e[0].elapsed_time(e[1]) for e in ev) / args.steps
    t_film = sum(e[1].elapsed_time(e[2]) for e in ev) / args.steps
    if dist:
        t = torch.tensor([t_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_total = float(t.item())

    # the film stage with each of the 81-bin scan's two forms (contractions on
    # the CUDA cores in FP32, or on the tensor cores in BF16 hi/lo), timed
    # alike on the same colour output: K steps each, L2 flushed between
    colour_d = rgb.clone()
    im.check(L.imops_develop_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                                 ctypes.byref(p_dem), ctypes.c_void_p(colour_d.data_ptr()), sp))
    arm_ms = {}
    for arm_name, arm in (("fp32", im.SCAN_FP32), ("bf16_tc", im.SCAN_BF16_TC)):
        p_arm = im.baseline_film_defaults(seed=SEED, scan=arm)

        def film_arm(events=None):
            rgb.copy_(colour_d)
            if events:
                events[0].record(stream)
            im.check(L.imops_film_process(ctypes.c_void_p(rgb.data_ptr()), W, H, im.CS_ACESCG,
                                          ctypes.byref(p_all.film_params), ctypes.byref(p_arm), sp))
            if events:
                events[1].record(stream)

        for _ in range(args.warmup):
            film_arm()
        eva = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(float(k))
            film_arm(eva[k])
        torch.cuda.synchronize()
        arm_ms[arm_name] = sum(e[0].elapsed_time(e[1]) for e in eva) / args.steps
    del colour_d

    # the dominant kernel alone for the roofline: AMaZE with the colour
    # epilogue on the scaled f32 mosaic (imops_develop_f32 launches exactly
    # that one kernel), K launches, L2 flushed between
    mosaic = torch.empty((H, W), device=dev)
    L.imops_scale_u16.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p,
                                                                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                                            ctypes.c_void_p]
    L.imops_develop_f32.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(im.DevelopParams), ctypes.c_void_p, ctypes.c_void_p]
    im.check(L.imops_scale_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                               ctypes.c_void_p(mosaic.data_ptr()), sp))

    def amaze_alone(events=None):
        if events:
            events[0].record(stream)
        im.check(L.imops_develop_f32(ctypes.c_void_p(mosaic.data_ptr()), W, H, 0, 0, ctypes.byref(p_dem),
                                     ctypes.c_void_p(rgb.data_ptr()), sp))
        if events:
            events[1].record(stream)

    for _ in range(args.warmup):
        amaze_alone()
    evk = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(float(k))
        amaze_alone(evk[k])
    torch.cuda.synchronize()
    t_amaze = sum(e[0].elapsed_time(e[1]) for e in evk) / args.steps
    del mosaic

    # forward + backward of the differentiable colour + film model (24
    # parameters: WB, camera->ACEScg matrix, EV, curves, halation) on the same
    # frame: AMaZE to camera RGB, the model's forward, and its adjoint
    # against a target rendered once with perturbed parameters.
    p_cam = develop_params(im, film=False)
    p_cam.target = im.CS_CAMERA
    for i in range(4):
        p_cam.wb[i] = 1.0
    theta = im.FilmGradParams.from_vector(synthetic.film_grad_base())
    cam = torch.empty((H, W, 3), device=dev)
    fwd_out = torch.empty((H, W, 3), device=dev)
    grad = torch.zeros(25, dtype=torch.float64, device=dev)
    im.check(L.imops_develop_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                                 ctypes.byref(p_cam), ctypes.c_void_p(cam.data_ptr()), sp))
    target = im.param_forward(cam, im.FilmGradParams.from_vector(synthetic.film_grad_perturbed(2)), stream=stream)
    loss_scale = 1.0 / (H * W * 3)

    def step_fwd_bwd(events=None):
        if events:
            events[0].record(stream)
        im.check(L.imops_develop_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                                     ctypes.byref(p_cam), ctypes.c_void_p(cam.data_ptr()), sp))
        im.param_forward(cam, theta, out=fwd_out, stream=stream)
        if events:
            events[1].record(stream)
        grad.zero_()
        im.param_backward(cam, theta, grad, target=target, loss_scale=loss_scale, stream=stream)
        if events:
            events[2].record(stream)

    for _ in range(args.warmup):
        step_fwd_bwd()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    evb = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.fill_(float(k))
        step_fwd_bwd(evb[k])
    torch.cuda.synchronize()
    t_fb = sum(e[0].elapsed_time(e[2]) for e in evb)
    t_fb_fwd = sum(e[0].elapsed_time(e[1]) for e in evb) / args.steps
    t_fb_bwd = sum(e[1].elapsed_time(e[2]) for e in evb) / args.steps
    assert np.isfinite(grad.cpu().numpy()).all()
    if dist:
        t = torch.tensor([t_fb], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_fb = float(t.item())

    # end to end through the reference-facing C-ABI (extern_pipeline.rs names):
    # per frame, host u16 frame in (new_raw_image_u16_c returns once uploaded),
    # pipeline run (returns once queued), host f32 RGB out, image freed.  A
    # batch submits frame k before reading back frame k-1, so one frame's
    # download overlaps the next frame's compute; every frame's copies and
    # compute are inside the timed region, on the host clock.
    from imops_b200.pipeline import Image, make_meta, parse_config, run_pixel_pipeline
    raw_h = torch.from_numpy(raw_np.view(np.int16)).pin_memory()
    rgb_h = torch.empty((H, W, 3), dtype=torch.float32).pin_memory()
    cfg = parse_config(PIPELINE_CONFIG)
    meta = make_meta(cfa="RGGB", wb=synthetic.WB, calibration=synthetic.CALIB_D65, black=synthetic.BLACK,
                     white=synthetic.WHITE)
    Lp = im.lib()

    host_ms = {"upload": [], "submit": [], "download": []}  # per call, host clock

    def e2e_batch(frames, log=False):
        """Two host threads, as an application that streams frames would use
        the C-ABI: this one uploads each frame and submits its pipeline
        (new_raw_image_u16_c returns once the upload is done,
        run_pixel_pipeline_c once the work is queued); a reader thread
        downloads the finished frames in order (get_image_rgb_f32_c waits for
        its frame).  So frame k+1's upload, frame k's kernels and frame k-1's
        download overlap on the two copy engines and the SMs.  At most two
        frames wait for the reader."""
        pending = queue.Queue(maxsize=2)
        errors = []

        def reader():
            while True:
                img = pending.get()
                if img is None:
                    return
                try:
                    t_a = time.perf_counter()
                    im.check(Lp.get_image_rgb_f32_c(img._h, ctypes.c_void_p(rgb_h.data_ptr()), H * W * 3))
                    if log:
                        host_ms["download"].append((time.perf_counter() - t_a) * 1e3)
                except Exception as e:  # reported by the submitting thread
                    errors.append(e)
                del img

        t = threading.Thread(target=reader)
        t.start()
        try:
            for _ in range(frames):
                t_a = time.perf_counter()
                img = Image(Lp.new_raw_image_u16_c(ctypes.c_void_p(raw_h.data_ptr()), W, H, ctypes.byref(meta)))
                t_b = time.perf_counter()
                run_pixel_pipeline(img, cfg)
                if log:
                    host_ms["upload"].append((t_b - t_a) * 1e3)
                    host_ms["submit"].append((time.perf_counter() - t_b) * 1e3)
                pending.put(img)
                del img
        finally:
            pending.put(None)
            t.join()
        if errors:
            raise errors[0]

    # warm-up: a frame on each of the library's image streams (six a device),
    # so that every stream's film working set exists before the timed frames
    e2e_batch(6)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_batch(args.steps, log=True)
    t_e2e = (time.perf_counter() - t0) * 1e3
    if dist:
        t = torch.tensor([t_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())

    # the box's host link: plain pinned copies of one frame's RGB in each
    # direction (CUDA events on a side stream), and the frame rate they and
    # the kernels allow when upload, kernels and download overlap
    def link_gbs(dst, src):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            dst.copy_(src, non_blocking=True)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            for _ in range(3):
                dst.copy_(src, non_blocking=True)
            b.record(s)
        b.synchronize()
        return 3 * src.numel() * src.element_size() / (a.elapsed_time(b) / 1e3) / 1e9

    rgb_d = torch.empty(H * W * 3, dtype=torch.float32, device=dev)
    d2h_gbs = link_gbs(rgb_h.view(-1), rgb_d)
    h2d_gbs = link_gbs(rgb_d, rgb_h.view(-1))
    del rgb_d
    t_frame = max(H * W * 12 / (d2h_gbs * 1e9), H * W * 2 / (h2d_gbs * 1e9), t_total / args.steps / 1e3)

    mp = H * W / 1e6
    value = world * mp * args.steps / (t_total / 1e3)
    e2e = world * mp * args.steps / (t_e2e / 1e3)
    e2e_bound = world * mp / t_frame
    fwd_bwd = world * mp * args.steps / (t_fb / 1e3)
    bw, peak_kind = peaks()
    dom_bytes = H * W * 16  # f32 mosaic in (4 B) + f32 RGB out (12 B) per pixel
    achieved = dom_bytes / (t_amaze / 1e3) / 1e9
    if rank == 0:
        clk_summary = clk.summary()
        # this frame's outputs for the error check: the colour forward, then the film
        im.check(L.imops_develop_u16(ctypes.c_void_p(raw.data_ptr()), W, H, 0, 0, W, H, black, white, 2, 2,
                                     ctypes.byref(p_dem), ctypes.c_void_p(rgb.data_ptr()), sp))
        colour_np = rgb.cpu().numpy()
        im.check(L.imops_film_process(ctypes.c_void_p(rgb.data_ptr()), W, H, im.CS_ACESCG,
                                      ctypes.byref(p_all.film_params), ctypes.byref(p_all.baseline), sp))
        film_np = rgb.cpu().numpy()
        p_other = im.baseline_film_defaults(seed=SEED)
        p_other.scan = im.SCAN_BF16_TC if p_all.baseline.scan == im.SCAN_FP32 else im.SCAN_FP32
        rgb.copy_(torch.from_numpy(colour_np).to(dev))
        im.check(L.imops_film_process(ctypes.c_void_p(rgb.data_ptr()), W, H, im.CS_ACESCG,
                                      ctypes.byref(p_all.film_params), ctypes.byref(p_other), sp))
        other_np = rgb.cpu().numpy()
        error = cpu_check_error(raw_np, colour_np, film_np, other_np)
        cpu_v, cpu_sample_desc = cpu_sample(os.cpu_count() or 1)
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_total / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(world),
            "stages_ms": {"scale_amaze_colour": round(t_dem, 4), "film": round(t_film, 4),
                          "amaze_kernel": round(t_amaze, 4)},
            "scan": {"in_value": "fp32" if p_all.baseline.scan == im.SCAN_FP32 else "bf16_tc",
                     "film_ms": {k: round(v, 4) for k, v in arm_ms.items()},
                     "note": "film stage alone per arm, K steps each with the L2 flushed between; the 81-bin scan's "
                             "contractions in FP32 on the CUDA cores, or BF16 hi/lo with FP32 accumulation on the "
                             "tensor cores (tcgen05); error.film_stage_other_scan is the arm not in value"},
            "fwd_bwd": {"value": round(fwd_bwd, 2), "unit": "MP/s", "ms_per_step": round(t_fb / args.steps, 4),
                        "stages_ms": {"amaze_cam_plus_model_fwd": round(t_fb_fwd, 4),
                                      "model_bwd": round(t_fb_bwd, 4)},
                        "model": "24 params: WB 3, camera->ACEScg 9, EV, dmax/k/x0 per layer, halation strength/sigma; "
                                 "81-bin scan, grain off; MSE to a perturbed-parameter target"},
            "roofline": {"bound": "hbm", "kernel": "amaze (f32 mosaic in, colour epilogue)",
                         "achieved": round(achieved, 2), "peak": bw, "unit": "GB/s",
                         "frac": round(achieved / bw, 5), "traffic": ncu_traffic(), "peak_kind": peak_kind,
                         "bytes_per_launch": dom_bytes,
                         "traffic_note": "ncu dram__bytes_read + dram__bytes_write of one launch (scaled from the "
                                         "committed capture): a lower bound, since output lines still dirty in L2 "
                                         "when the kernel ends are written back after it",
                         "note": "AMaZE is FP32-issue bound (~25 IEEE divides/px on 1.78x overlapping tiles); "
                                 "the HBM fraction is reported against its 16 B/px compulsory traffic, the time is "
                                 "stages_ms.amaze_kernel (the kernel alone, CUDA events)",
                         "issue": issue_fraction(t_amaze, clk_summary)},
            "cpu_baseline": {"value": round(cpu_v, 3), "unit": "MP/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": cpu_sample_desc},
            "e2e": {"value": round(e2e, 2), "unit": "MP/s", "h2d_bytes_per_step": H * W * 2,
                    "d2h_bytes_per_step": H * W * 12, "api": "new_raw_image_u16_c + run_pixel_pipeline_c + "
                    "get_image_rgb_f32_c per frame; one host thread uploads and submits, a second reads the frames "
                    "back, so upload, kernels and download of consecutive frames overlap (pinned host buffers, host "
                    "clock)",
                    "host_ms": {k: {"median": round(statistics.median(v), 3), "max": round(max(v), 3),
                                    "max_frame": v.index(max(v))} for k, v in host_ms.items() if v},
                    "link": {"d2h_gbs": round(d2h_gbs, 2), "h2d_gbs": round(h2d_gbs, 2),
                             "bound_mp_s": round(e2e_bound, 2), "frac_of_bound": round(e2e / e2e_bound, 3),
                             "note": "plain pinned copies of one frame's f32 RGB on this box; the bound is the "
                                     "slowest of download, upload and kernels per frame"}},
            "error": error,
            "gpu_launches": int(launches),
            "clocks": clk_summary,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
