#!/usr/bin/env python
"""bench.py -- photon paths/s of the B200 photon march.

Workload (the precision scale-up configuration): cylindrical Bessel mode 1 field, dn 2e-3 at
848 kHz, 10 mm cube, sigma_s 1/mm, albedo 0.95, HG g 0.85, 64x64 Bernoulli(0.5) texture (seed 1),
512x512 px x 128 path-length bins over 0-100 mm, FP32 march with FP64 path length and film.
One step traces 1e7 photons (1/10 of the 1e8-photon render) into the resident film: the slot
pool of the two-kernel march is refilled until the step's photons run out, then drained.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank traces its own photon range (counter-based streams keyed by the global
photon index, so the render is the same for any GPU count) and the film is reduced to rank 0 over
NCCL every step. Prints one JSON line (rank 0). On one GPU the line also carries `plain` (the plain
one-thread-per-photon kernel on the same workload), `image_rmse_vs_fp64` (the films against the FP64
oracle on the same photons) and `batched_form`: the north star's batched form, the 256-instance
sweep with ER steps from the step-size autotuner, against the plain kernel on the same instances,
with its own image check against the FP64 oracle (`--workload sweep` prints it as its own line,
with the nominal-step sweep and the one-render-per-instance loop beside it).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import simpler_b200 as sb  # noqa: E402
from simpler_b200 import _lib as L  # noqa: E402
from simpler_b200.roofline import flop_per_point_adjoint, flop_per_step  # noqa: E402

METRIC = "photon paths/s"
RENDER_PHOTONS = 100_000_000
PHOTONS_PER_STEP = 10_000_000
WORKLOAD = "precision scale-up: Bessel mode 1, dn 2e-3, sigma_s 1/mm, albedo 0.95, g 0.85, 1e8-photon render"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--photons-per-step", type=int, default=PHOTONS_PER_STEP)
    ap.add_argument("--workload", choices=["precision", "sweep", "plain", "planewave", "spline", "sources", "adjoint",
                                           "adjoint-spline", "adjoint-bessel"], default="precision",
                    help="precision: the headline line (default); sweep: the batched 256-instance sweep "
                         "against the same instances rendered one by one; adjoint / adjoint-spline: gradients "
                         "of the central 32x32 px ROI throughput")
    ap.add_argument("--sweep-scale", type=float, default=1.0,
                    help="sweep: multiply every instance's photon budget")
    ap.add_argument("--step-budget", type=float, default=2e-3,
                    help="sweep: relative image RMSE the step-size autotuner may spend per instance, against "
                         "the instance's film at its own 0.01 mm step on the same photons")
    return ap.parse_args()


# secondary workloads (--workload): the other configurations of the same path, one JSON line each
OTHER = {
    "plain": (lambda d: sb.config_plain_small(device=d), 1_000_000, 1_000_000,
              "plain small: Bessel mode 0, dn 1e-3 at 848 kHz, sigma_s 0.1/mm, albedo 0.9, g 0.9, "
              "0.5 mm beam, 128x128 x 32 bins, fp32, 1e6 photons"),
    "planewave": (lambda d: sb.config_planewave(device=d), 10_000_000, 10_000_000,
                  "two plane waves a = 1e-3 at 1 MHz along +y and +z, phases U[0, 2 pi) (seed 3), "
                  "sigma_s 0.5/mm, albedo 0.9, g 0.9, 128x128 x 32 bins, fp32, 1e7 photons"),
    "sources": (lambda d: _sources_grid(d), 2_000_000, 10_000_000,
                "focused-ultrasound point sources (two 2 in arcs of 100 x 501 sources, first harmonic) sampled "
                "once on a 96^3 tricubic grid (sources_to_spline, grad n within 7e-4 of the direct sum), medium "
                "and 128x128 x 32 film of the plain small configuration, fp32; 2e6-photon steps"),
    "spline": (lambda d: sb.config_spline(device=d), 10_000_000, 1_000_000_000,
               "tricubic spline 64^3 over the 10 mm cube (Gaussian-filtered noise, max dn 1e-3, seed 4), "
               "sigma_s 1/mm, albedo 0.95, g 0.8, 256x256 x 64 bins, fp32; 1e7-photon steps of a "
               "1e9-photon render"),
}


# adjoint workloads: (setup, photons per gradient, description)
ADJOINT = {
    "adjoint": (lambda d: sb.config_planewave(device=d), 10_000_000,
                "traveling-wave adjoint: two plane waves a = 1e-3 at 1 MHz along +y and +z, phases U[0, 2 pi) "
                "(seed 3), sigma_s 0.5/mm, albedo 0.9, g 0.9, 128x128 x 32 bins, fp32, 1e7 photons; gradient "
                "of the central 32x32 px ROI throughput w.r.t. (a_i, phase_i)"),
    "adjoint-bessel": (lambda d: sb.config_plain_small(device=d, n_clip=2e-3), 1_000_000,
                       "transducer adjoint: Bessel mode 0, n_max 1e-3 (n_clip 2e-3: no scaling clamped) at 848 kHz, "
                       "sigma_s 0.1/mm, albedo 0.9, g 0.9, 128x128 x 32 bins, fp32, 1e6 photons; gradient of the "
                       "central 32x32 px ROI throughput w.r.t. (n_max, phi_min, phi_max)"),
    "adjoint-spline": (lambda d: sb.config_spline(device=d), 1_000_000,
                       "spline adjoint: 64^3 tricubic coefficients over the 10 mm cube (Gaussian-filtered noise, "
                       "max dn 1e-3, seed 4), sigma_s 1/mm, albedo 0.95, g 0.8, 256x256 x 64 bins, fp32; "
                       "gradient of the central 32x32 px ROI throughput w.r.t. all 262144 coefficients over "
                       "1e6-photon steps of the 1e9-photon render"),
}

_ARGS = None           # the parsed command line (set in main)
_GRIDS = {}


def _sources_grid(device: int) -> sb.Setup:
    """The point-source workload's field on its 96^3 grid, sampled once per device."""
    if device not in _GRIDS:
        _GRIDS[device] = sb.sources_to_spline(sb.config_sources(device=device), 96)
    return _GRIDS[device]


def workload(args=None, device: int = 0) -> sb.Setup:
    args = args or _ARGS
    if args is not None and args.workload in OTHER:
        return OTHER[args.workload][0](device)
    return sb.config_precision(device=device)


def render_photons(args=None) -> int:
    args = args or _ARGS
    return OTHER[args.workload][2] if args is not None and args.workload in OTHER else RENDER_PHOTONS


def config_json(args, per_step: int) -> dict:
    s = workload(args)
    if args.workload in OTHER:
        return {"workload": OTHER[args.workload][3], "photons_per_step_per_gpu": per_step,
                "render_photons": render_photons(args), "film": [s.spatial_x, s.spatial_y, s.path_length_bins],
                "er_stepsize_m": s.er_stepsize, "precision_levels": s.precision,
                "rng": "philox-4x32-10 keyed by global photon index"}
    return {
        "workload": WORKLOAD,
        "photons_per_step_per_gpu": per_step,
        "render_photons": RENDER_PHOTONS,
        "field": "bessel", "mode": s.mode, "n_max": s.n_max, "f_u": s.f_u,
        "medium_mm": 10.0, "sigma_s_per_mm": 1.0, "albedo": s.albedo, "g": s.g,
        "film": [s.spatial_x, s.spatial_y, s.path_length_bins],
        "er_stepsize_m": s.er_stepsize, "precision_levels": s.precision,
        "rng": "philox-4x32-10 keyed by global photon index",
        "precision": "fp32 march, fp64 path length + fp64 film",
        "l2": "film 256 MiB (fp64) exceeds the 126 MB L2; no flush needed",
    }


# ---- clocks ---------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- CPU baseline: the oracle port on the host cores ----------------------------------------------
def _oracle_lib(fast: bool = True):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle_fast.so" if fast else "liboracle.so"))
    P = C.POINTER
    vp = C.c_void_p
    lib.orc_render.argtypes = [P(L.SceneDesc), P(L.MediumDesc), P(L.FieldDesc), P(L.RenderOpts), C.c_int, C.c_int,
                               C.c_int64, C.c_int64, C.c_int64, vp, vp, vp, vp]
    lib.orc_render_films.argtypes = [P(L.SceneDesc), P(L.MediumDesc), P(L.FieldDesc), P(L.RenderOpts), C.c_int,
                                     C.c_int, C.c_int64, C.c_int64, C.c_int64, vp]
    return lib


class ThreadFilms:
    """The CPU restatement's per-thread films, as the reference's renderImage keeps one image per
    thread through its photon loop and merges them at the end (photon.cpp:290-291, 337): allocated
    and written once before any timing (so that no page is first touched inside a timed call),
    accumulated into by every timed trace, merged once at the end. Threads are capped so that the
    films take at most half of the host's available memory."""

    def __init__(self, setup: sb.Setup, threads: int):
        import psutil
        self.dtype = np.float64 if setup.precision_mode == L.PREC_MIXED else np.float32
        self.npix = setup.spatial_x * setup.spatial_y * setup.path_length_bins
        per = self.npix * np.dtype(self.dtype).itemsize
        avail = psutil.virtual_memory().available
        self.threads = max(1, min(threads, int(0.5 * avail // per)))
        self.films = np.zeros((self.threads, self.npix), dtype=self.dtype)
        self.films.fill(0)
        self.bytes = self.films.nbytes

    def merge(self):
        """(film, seconds): the sum of the thread films, as the reference's final merge."""
        t0 = time.perf_counter()
        img = self.films.sum(axis=0, dtype=np.float64)
        return img, time.perf_counter() - t0


def fp32_peak_from_clock(device: int) -> dict:
    """The FP32 peak from the chip's figures, beside the live-measured one: SMs x 128 FP32 lanes x
    2 FLOP (FMA) x the maximum SM clock (nvidia-smi clocks.max.sm)."""
    import torch
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = None
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(device), "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=20).stdout.strip()
        mhz = float(out.splitlines()[0])
    except Exception:
        mhz = None
    if not mhz:
        return {"tflops": None, "how": "clocks.max.sm unavailable"}
    return {"tflops": sms * 128 * 2 * mhz * 1e6 / 1e12, "how": f"{sms} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz"}


def cpu_trace(n: int, first: int, films: ThreadFilms) -> float:
    """Trace n photons of the workload with the CPU restatement on films.threads host threads, each
    accumulating its splats into its own film; returns seconds (wall)."""
    lib = _oracle_lib()
    s = workload()
    sc, md, fd, op = s.descs()
    t0 = time.perf_counter()
    rc = lib.orc_render_films(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 32, films.threads, first, n,
                              render_photons(), C.c_void_p(films.films.ctypes.data))
    dt = time.perf_counter() - t0
    assert rc == 0
    return dt


def cpu_baseline(target_s: float = 12.0) -> dict:
    """Trace batches of the workload on all host threads until about target_s of wall time: one
    photon per thread first, then batches doubling while the next one fits in the time left (a
    photon of the point-source field costs seconds on the CPU). Every splat is accumulated into the
    thread's film; the films' one-time merge is timed apart and reported."""
    films = ThreadFilms(workload(), os.cpu_count() or 1)
    threads = films.threads
    batch = threads
    done, dt, first = 0, 0.0, 0
    while dt < target_s and done < 2_000_000:
        t = cpu_trace(batch, first, films)
        dt += t
        done += batch
        first += batch
        if 2.0 * t < target_s - dt:
            batch *= 2
    _, merge_s = films.merge()
    return {"value": done / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"photons 0..{done} of the same workload ({done} photon paths) in {dt:.1f} s on "
                      f"{threads} host threads, CPU restatement built with the reference's -O3 -ffast-math "
                      f"flags, each splat accumulated into its thread's film ({threads} films, "
                      f"{films.bytes / 2**30:.2f} GiB); the films' merge, once per render, took {merge_s:.2f} s "
                      f"and is not in the rate"}


def image_check(setup: sb.Setup, n: int, threads: int = 8) -> dict:
    """The cpu_baseline leg's check of the image error (the oracle as the checker): photons 0..n-1 of
    the workload on the same Philox streams, rendered by this library's default path (FP32 march,
    the workload's precision form) and by the plain kernel in the reference GPU's FP32 form (FP32
    path length and float film), each against the FP64 restatement on the CPU; beside them the FP32
    restatement on the CPU against the same FP64 one, the error that FP32 marching itself makes.
    Relative RMSE sqrt(sum (film - ref)^2 / sum ref^2) at the workload's film and with bins merged
    4x4x4 and 16x16x16; and the fraction of photons whose discrete events (end, draws, depth, splat
    count) are the same in the FP32 GPU march and the FP64 oracle."""
    import dataclasses
    lib = _oracle_lib(fast=False)
    ours, _ = sb.render(setup, n)
    plain_setup = dataclasses.replace(setup, kernel=L.KERNEL_PLAIN, precision_mode=L.PREC_FP32)
    plain, _ = sb.render(plain_setup, n)
    recs, _ = sb.trace_photons(setup, 0, n, n, with_image=False)
    recs = sb.records_to_arrays(recs)
    sc, md, fd, op = setup.descs()

    def oracle(bits):
        img = np.zeros(setup.film_shape(), dtype=np.float64)
        rr = (L.PhotonRecord * n)()
        t0 = time.perf_counter()
        rc = lib.orc_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), bits, threads, 0, n, n, None, None,
                            C.cast(rr, C.c_void_p), C.c_void_p(img.ctypes.data))
        assert rc == 0
        return img, sb.records_to_arrays(rr), time.perf_counter() - t0

    ref, orecs, dt = oracle(64)
    cpu32, _, _ = oracle(32)
    same = ((recs["end"] == orecs["end"]) & (recs["draws"] == orecs["draws"]) & (recs["depth"] == orecs["depth"])
            & (recs["n_splats"] == orecs["n_splats"]))

    def binned(a, f):
        z, y, x = a.shape
        fz, fy, fx = min(f, z), min(f, y), min(f, x)
        return a.reshape(z // fz, fz, y // fy, fy, x // fx, fx).sum(axis=(1, 3, 5))

    def rmse(a, f):
        a, b = binned(a, f), binned(ref, f)
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))

    out = {"photons": n, "film": [setup.spatial_x, setup.spatial_y, setup.path_length_bins],
           "same_events_fraction": float(same.mean()),
           "reference": f"FP64 CPU restatement (oracle/liboracle.so, {threads} threads, {dt:.1f} s), same Philox photons"}
    for f in (1, 4, 16):
        key = "" if f == 1 else f"_binned_{f}x{f}x{f}"
        out["ours" + key] = rmse(ours, f)
        out["plain_fp32" + key] = rmse(plain, f)
        out["cpu_fp32_restatement" + key] = rmse(cpu32, f)
    return out


# ---- reference arm ---------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    films = ThreadFilms(workload(args), os.cpu_count() or 1)
    threads = films.threads
    # 64 photons per thread: a step waits for its slowest photon, so small steps understate the
    # CPU's throughput
    per_step = max(threads * 64, 1024)
    for i in range(args.warmup):
        cpu_trace(per_step, i * per_step, films)
    times = []
    for i in range(args.steps):
        times.append(cpu_trace(per_step, (args.warmup + i) * per_step, films))
    tot = sum(times)
    _, merge_s = films.merge()
    v = per_step * args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": config_json(args, per_step),
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{per_step} photons per step of the same workload on {threads} host threads "
                                   f"(the reference does not build here; CPU restatement with its -O3 -ffast-math "
                                   f"flags), each splat accumulated into its thread's film ({films.bytes / 2**30:.2f} "
                                   f"GiB of films); their merge, once per render, took {merge_s:.2f} s, not in the rate"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm -------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    per_step = args.photons_per_step if args.workload not in OTHER or args.photons_per_step != PHOTONS_PER_STEP \
        else OTHER[args.workload][1]
    setup = workload(args, local)
    plan = sb.Plan(setup)
    # the project's autotuner picks the slot pool's schedule (march-kernel block size, slots per
    # lane, chunk) from trial traces before anything is timed
    t0 = time.perf_counter()
    tuning = plan.tune(min(per_step, 5_000_000))
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    h = stream.cuda_stream
    nz, ny, nx = setup.film_shape()
    film = torch.zeros((nz, ny, nx), dtype=torch.float64, device=f"cuda:{local}") if world > 1 else None

    def step(i):
        first = (i * world + rank) * per_step
        plan.trace(first, per_step, render_photons(args), stream=h)
        if world > 1:
            plan.read_image_device(film.data_ptr(), stream=h)
            dist.reduce(film, dst=0)

    plan.clear(h)
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    st0 = plan.stats()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    st1 = plan.stats()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    steps_timed = st1.er_steps - st0.er_steps
    march_ms = st1.march_ms - st0.march_ms
    march_steps = st1.march_steps - st0.march_steps
    launches = st1.launches - st0.launches
    value = per_step * args.steps * world / (ms / 1e3)

    out = None
    if rank == 0:
        peak = C.c_double()
        L.check(L.load().smp_fp32_peak(local, C.byref(peak)))
        fps = flop_per_step(setup)
        # the dominant kernel is the ER-march kernel: its launches are timed with CUDA events on
        # this stream inside the library, and it counts the steps it executes
        n_march = max(1, st1.march_launches - st0.march_launches)
        achieved = fps * march_steps / (march_ms / 1e3) / 1e12
        kname = {L.FIELD_PLANEWAVE: "FK_PLANEWAVE", L.FIELD_SPLINE: "FK_SPLINE", L.FIELD_SOURCES: "FK_SOURCES"}.get(
            setup.field_type, f"FK_BESSEL{setup.mode}")
        form = "fp64 path length" if setup.precision_mode == L.PREC_MIXED else "fp32"
        roof = {"bound": "fp32", "kernel": f"wf_march_kernel<{kname}, {form}>",
                "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value,
                "traffic": _profile_traffic(tuning.slots_per_lane) if args.workload == "precision" else None,
                "traffic_source": "profiles/wf_march_kernel_precision_traffic.txt: one captured steady-state "
                                  "launch, scaled to this run's slots per lane",
                "flop_per_er_step": fps, "er_steps_per_launch": march_steps / n_march,
                "march_kernel_share_of_step_time": march_ms / ms,
                "peak_source": "FP32 FMA throughput measured live on this GPU (smp_fp32_peak)"}
        clk_peak = fp32_peak_from_clock(local)
        roof["peak_clock_derived"] = clk_peak["tflops"]
        roof["peak_clock_derived_how"] = clk_peak["how"]
        roof["frac_of_clock_derived"] = achieved / clk_peak["tflops"] if clk_peak["tflops"] else None
        e2e = run_e2e(args, setup, min(args.steps, 3), per_step)
        out = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": dict(config_json(args, per_step), schedule={
                "march_block": tuning.march_block, "slots_per_lane": tuning.slots_per_lane, "chunk": tuning.chunk,
                "tuner_trials": tuning.trials, "tuner_sample_photons": min(per_step, 5_000_000),
                "tuner_seconds": round(tune_s, 2)}),
            "roofline": roof, "cpu_baseline": cpu_baseline() if world == 1 else None, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk,
            "er_steps_per_s": steps_timed * world / (ms / 1e3),
        }
    plan.close()
    if rank == 0:
        # the plain GPU kernel (one thread per photon, FP32 form) on the same workload and step size
        plain = run_plain(args, setup, per_step, local, first_step=args.warmup + args.steps)
        out["plain"] = plain
        out["speedup_vs_plain"] = value / world / plain["value"]
        if world == 1 and args.workload in ("precision", "plain"):
            out["image_rmse_vs_fp64"] = image_check(setup, 20_000 if args.workload == "precision" else 100_000)
        if world == 1 and args.workload == "precision":
            # the north star's batched form against the plain kernel, beside the headline
            out["batched_form"] = batched_form(args, False)
        if world == 1 and args.workload == "plain":
            out["tuned_step"] = plan_tuned_step(args, setup, per_step)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


def run_plain(args, setup, per_step: int, device: int, first_step: int, steps: int = 2) -> dict:
    """The plain kernel (the reference GPU renderer's structure: one thread per photon, one launch,
    no regeneration, float atomics; this library's per-photon arithmetic) in the reference GPU's FP32
    form on the same workload, device-timed over `steps` steps of per_step photons after one
    warm-up step."""
    import dataclasses
    import torch
    ps = dataclasses.replace(setup, kernel=L.KERNEL_PLAIN, precision_mode=L.PREC_FP32)
    plan = sb.Plan(ps)
    stream = torch.cuda.current_stream()
    h = stream.cuda_stream
    plan.clear(h)
    plan.trace(first_step * per_step, per_step, render_photons(args), stream=h)
    torch.cuda.synchronize()
    st0 = plan.stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        plan.trace((first_step + 1 + i) * per_step, per_step, render_photons(args), stream=h)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = plan.stats()
    plan.close()
    return {"value": per_step * steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / steps, "steps": steps,
            "kernel": "plain_kernel: one thread per photon, one launch per step (cuda_renderer.cu:681-725 structure)",
            "precision": "fp32 march, fp32 path length, fp32 film atomics",
            "er_steps_per_s": (st.er_steps - st0.er_steps) / (ms / 1e3)}


def plan_tuned_step(args, setup, per_step: int) -> dict:
    """The same workload with the plan's ER step from the step-size autotuner (smp_plan_tune_step on
    the render's first 2e4 photons, within --step-budget of the film at the workload's own step),
    device-timed over --steps renders of per_step photons, and its image against the FP64 oracle at
    the own step on 2e4 photons (the oracle as the checker)."""
    plan = sb.Plan(setup)
    plan.tune(min(per_step, 5_000_000))
    t0 = time.perf_counter()
    step, rmse = plan.tune_step(20000, args.step_budget)
    t_tune = time.perf_counter() - t0
    ms = 0.0
    for i in range(args.steps):
        plan.clear(0)
        st0 = plan.stats()
        plan.trace((args.warmup + i) * per_step, per_step, render_photons(args), 0)
        ms += plan.stats().kernel_ms - st0.kernel_ms
    n = 20000
    film, _ = plan.render(n)
    plan.close()
    sc, md, fd, op = setup.descs()
    lib = _oracle_lib(fast=False)
    ref = np.zeros(setup.film_shape(), dtype=np.float64)
    assert lib.orc_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 64, os.cpu_count() or 1, 0, n, n,
                          None, None, None, C.c_void_p(ref.ctypes.data)) == 0
    return {"value": per_step * args.steps / (ms / 1e3), "unit": METRIC, "step_m": step,
            "step_multiple": step / setup.er_stepsize, "tuner_seconds": t_tune, "tuner_rmse": rmse,
            "image_rmse_vs_fp64": float(np.sqrt(((film - ref) ** 2).sum() / (ref ** 2).sum())),
            "image_photons": n, "call": "Plan.tune_step then device-timed traces (smp_plan_trace)"}


def _profile_traffic(slots_per_lane: int):
    """DRAM bytes of one steady-state march-kernel launch (every slot of the pool live) from the
    committed ncu capture, scaled from the capture's slots per lane to this run's: a launch moves
    each live slot's march state, so its traffic follows the live slots."""
    path = os.path.join(ROOT, "profiles", "wf_march_kernel_precision_traffic.txt")
    vals = {}
    try:
        with open(path) as f:
            for line in f:
                if "=" in line and not line.startswith("#"):
                    k, v = line.split("=")
                    vals[k.strip()] = float(v)
    except OSError:
        return None
    if "dram_bytes_per_launch" not in vals:
        return None
    return vals["dram_bytes_per_launch"] * slots_per_lane / vals.get("slots_per_lane", slots_per_lane)


def run_e2e(args, setup, steps: int, per_step: int) -> dict:
    """The same metric through the one-shot C-ABI call with a host film (CudaRenderer::renderImage's
    contract): scene upload, trace, FP64 film read back to host memory, every step."""
    lib = L.load()
    sc, md, fd, op = setup.descs()
    img = np.zeros(setup.film_shape(), dtype=np.float64)
    stt = L.Stats()
    t_total = 0.0
    for i in range(steps + 1):
        t0 = time.perf_counter()
        L.check(lib.smp_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), per_step,
                               C.c_void_p(img.ctypes.data), C.byref(stt)))
        dt = time.perf_counter() - t0
        if i > 0:
            t_total += dt
    tex = setup.texture.size
    h2d = (tex + 1) * 4 + 2050 * 16 + 1024          # texture CDF + Bessel table + parameters
    d2h = img.nbytes + 64
    return {"value": per_step * steps / t_total, "unit": METRIC, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps,
            "call": "smp_render (one-shot plan, host film) per step, wall clock"}


def sweep_image_check(setup, insts, steps, n: int, threads: int) -> list:
    """The sweep's image check (the oracle as the checker): for the instances given, photons 0..n-1 on
    their own Philox streams rendered by the batched form at its tuned step, by the batched form at
    the nominal 0.01 mm step and by the plain kernel (FP32, nominal step), each against the FP64
    restatement on the CPU at the nominal step; relative RMSE sqrt(sum (film - ref)^2 / sum ref^2)."""
    import dataclasses
    lib = _oracle_lib(fast=False)
    out = []
    for i, h in steps:
        inst = dict(insts[i], n_photons=n)
        over = {k: v for k, v in inst.items() if k != "n_photons"}
        s = dataclasses.replace(setup, **over)
        tuned, _ = sb.render_batch(setup, [dict(inst, er_stepsize=float(h))])
        nominal, _ = sb.render_batch(setup, [inst])
        plain, _ = sb.render(dataclasses.replace(s, kernel=L.KERNEL_PLAIN), n)
        sc, md, fd, op = s.descs()
        ref = np.zeros(s.film_shape(), dtype=np.float64)
        rc = lib.orc_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 64, threads, 0, n, n, None, None,
                            None, C.c_void_p(ref.ctypes.data))
        assert rc == 0

        def rel(a):
            return float(np.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum()))
        out.append({"instance": i, "mode": inst["mode"], "f_u": inst["f_u"], "n_max": inst["n_max"],
                    "step_m": float(h), "step_multiple": round(float(h) / setup.er_stepsize),
                    "batched_tuned_step": rel(tuned[0]), "batched_nominal_step": rel(nominal[0]),
                    "plain_fp32_nominal_step": rel(plain)})
    return out


SWEEP_DESC = ("batched sweep: 256 Bessel instances (n_max U[0,2e-3], f U[0.5,2] MHz, mode 0-2, duty U[1,100]%, "
              "budgets log-uniform 1e5-1e7 x scale), medium and film of the plain small configuration, seed 2")


def batched_form(args, with_reference_legs: bool) -> dict:
    """The batched form against the plain kernel (the north star's target): the 256-instance sweep
    with each instance's ER step from the step-size autotuner (smp_batch_tune_steps within
    --step-budget of the instance's film at its own step; the tuner inside the timed region),
    rendered in one slot pool by smp_render_batch; the plain kernel (one thread per photon, FP32,
    0.01 mm) over every 8th instance, one render each; and the image check of three instances
    against the FP64 oracle at 0.01 mm. With with_reference_legs also the sweep at the nominal step
    and the one-smp_render-per-instance loop. All host-timed end to end (films read back)."""
    import dataclasses
    setup, insts = sb.config_batch_sweep(n_inst=256, seed=2, scale=args.sweep_scale)
    total = sum(i["n_photons"] for i in insts)
    # warm-up: module load, first allocations, and the schedule tuner's trials (2e6 photons of this
    # scene), whose schedule the timed sweeps take from the process-wide cache (keyed by the scene and
    # the first instance's field and step, so once for the nominal and once for the tuned steps)
    w_steps, _, _ = sb.tune_batch_steps(setup, insts[:16], args.step_budget, n_sample=20000)
    sb.render_batch(setup, [dict(inst, er_stepsize=float(h)) for inst, h in zip(insts[:16], w_steps)])
    if with_reference_legs:
        sb.render_batch(setup, insts[:16])
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    steps, rmse, rounds = sb.tune_batch_steps(setup, insts, args.step_budget, n_sample=20000)
    t_tune = time.perf_counter() - t0
    t0 = time.perf_counter()
    films_t, st_t = sb.render_batch(setup, [dict(inst, er_stepsize=float(h)) for inst, h in zip(insts, steps)])
    t_tuned = time.perf_counter() - t0
    extra = {}
    if with_reference_legs:
        t0 = time.perf_counter()
        films, st = sb.render_batch(setup, insts)
        t_batch = time.perf_counter() - t0
        t0 = time.perf_counter()
        serial_sum = 0.0
        for i, inst in enumerate(insts):
            over = {k: v for k, v in inst.items() if k != "n_photons"}
            img, _ = sb.render(dataclasses.replace(setup, **over), inst["n_photons"])
            serial_sum += float(img.sum())
        t_serial = time.perf_counter() - t0
        extra = {"nominal_step": {"value": total / t_batch, "unit": METRIC, "seconds": t_batch, "er_steps": st.er_steps,
                                  "call": "smp_render_batch with every instance at 0.01 mm"},
                 "serial": {"value": total / t_serial, "unit": METRIC, "seconds": t_serial,
                            "call": "one smp_render per instance, host film, nominal step"},
                 "speedup_vs_serial": t_serial / (t_tuned + t_tune),
                 "film_sum_relative_difference": abs(float(films.sum()) - serial_sum) / max(serial_sum, 1e-300)}
    # the plain kernel (one thread per photon, FP32, nominal step) over every 8th instance, one render each
    t0 = time.perf_counter()
    plain_photons = 0
    plain_dev_ms = 0.0
    for i, inst in enumerate(insts[::8]):
        over = {k: v for k, v in inst.items() if k != "n_photons"}
        _, pst = sb.render(dataclasses.replace(setup, kernel=L.KERNEL_PLAIN, **over), inst["n_photons"])
        plain_photons += inst["n_photons"]
        plain_dev_ms += pst.kernel_ms
    t_plain = time.perf_counter() - t0
    clk = clocks.stop()
    mults = steps / setup.er_stepsize
    plain_rate = plain_photons / t_plain
    value = total / (t_tuned + t_tune)
    if with_reference_legs:
        extra["nominal_step"]["speedup_vs_plain"] = extra["nominal_step"]["value"] / plain_rate
    # image check against the FP64 oracle: the hardest field (largest n_max x f), the instance with
    # the largest multiple, the one with the largest error the tuner measured, and instance 0
    hard = max(range(len(insts)), key=lambda i: insts[i]["n_max"] * insts[i]["f_u"])
    big = int(np.argmax(mults))
    worst = int(np.argmax(rmse))                # the largest error the tuner measured
    check = sweep_image_check(setup, insts, [(i, steps[i]) for i in sorted({hard, big, worst, 0})], 10000,
                              os.cpu_count() or 1)
    hist = {str(m): int((np.rint(mults) == m).sum()) for m in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32)}
    out = {
        "value": value, "unit": METRIC, "seconds": t_tuned + t_tune,
        "config": {"workload": SWEEP_DESC + "; ER step per instance from the step-size autotuner (its trial renders "
                                           "inside the timed region)", "photons": total, "scale": args.sweep_scale,
                   "film": list(setup.film_shape()), "step_budget": args.step_budget},
        "step_tuner": {"seconds": t_tune, "rounds": rounds, "sample_photons_per_instance": 20000,
                       "multiples_histogram": hist, "mean_multiple_by_photons":
                           float(sum(m * i["n_photons"] for m, i in zip(mults, insts)) / total),
                       "max_measured_rmse": float(rmse.max())},
        "tuned_render_seconds": t_tuned, "er_steps_per_s": st_t.er_steps / t_tuned, "er_steps": st_t.er_steps,
        "plain": {"value": plain_rate, "unit": METRIC, "seconds": t_plain, "photons": plain_photons,
                  "call": "one smp_render per instance with the plain kernel (one thread per photon, fp32, "
                          "0.01 mm step), every 8th instance (32 of 256)"},
        "speedup_vs_plain": value / plain_rate,
        # the same comparison on device time alone (the render's traces against the plain kernel's
        # launches; the step tuner's renders are host-timed only and left out here)
        "device": {"tuned_render_seconds": st_t.kernel_ms / 1e3, "plain_seconds": plain_dev_ms / 1e3,
                   "value": total / (st_t.kernel_ms / 1e3), "plain_value": plain_photons / (plain_dev_ms / 1e3),
                   "speedup_vs_plain": (total / st_t.kernel_ms) / (plain_photons / plain_dev_ms)},
        "image_rmse_vs_fp64": {"photons": 10000, "reference": "FP64 CPU restatement at the nominal 0.01 mm step, "
                                                              "same Philox photons", "instances": check},
        "gpu_launches": st_t.launches, "clocks": clk,
        "schedule": {"march_block": st_t.march_block, "slots_per_lane": st_t.slots_per_lane, "chunk": st_t.chunk,
                     "tuned": bool(st_t.tuned), "cuda_graph": True},
    }
    out.update(extra)
    return out


def run_sweep(args):
    """The batched sweep as its own JSON line (batched_form with the nominal-step and
    one-render-per-instance legs)."""
    import torch
    torch.cuda.set_device(0)
    b = batched_form(args, True)
    out = {"metric": METRIC, "value": b.pop("value"), "unit": METRIC, "n_gpus": 1, "steps": 1, "warmup": 1,
           "ms_per_step": b.pop("seconds") * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32", "data": "synthetic"}
    out.update(b)
    print(json.dumps(out), flush=True)


def run_adjoint(args):
    """Gradients of the central 32x32 px ROI throughput per second, on one GPU (under torchrun only
    rank 0 runs it). Each step differentiates its own
    photon range (photons [i N, (i+1) N)); device time from CUDA events around the adjoint launch.
    Beside it: the forward render of the same photons, and central finite differences, which cost
    two forward renders per parameter."""
    import torch
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    make, n, desc = ADJOINT[args.workload]
    setup = make(0)
    G = sb.roi_weights(setup, 32)
    npar = sb.param_count(setup)
    plan = sb.Plan(setup)
    for i in range(args.warmup):
        plan.adjoint(G, i * n, n, n)
    clocks = ClockSampler(0)
    clocks.start()
    ms, tot = [], {k: 0 for k in ("er_steps_forward", "er_steps_replay", "points", "splats", "dropped", "skipped",
                                  "replay_mismatch", "photons", "trace_ms", "replay_ms", "sweep_ms",
                                  "launches")}
    for i in range(args.steps):
        _, st = plan.adjoint(G, (args.warmup + i) * n, n, n)
        ms.append(st.kernel_ms)
        for k in tot:
            tot[k] += getattr(st, k)
    clk = clocks.stop()
    # the forward render of the same photon ranges, device-timed
    fwd = []
    for i in range(args.steps):
        plan.clear(0)
        plan.trace((args.warmup + i) * n, n, n, 0)
        fwd.append(plan.stats().kernel_ms)
    plan.close()
    adj_ms = sum(ms) / len(ms)
    fwd_ms = sum(fwd) / len(fwd)
    # e2e: the one-shot C-ABI call with host dJ/dfilm and host gradient, wall clock
    t0 = time.perf_counter()
    sb.adjoint(setup, n, G)
    e2e_s = time.perf_counter() - t0
    peak = C.c_double()
    L.check(L.load().smp_fp32_peak(0, C.byref(peak)))
    flop = (tot["er_steps_forward"] + tot["er_steps_replay"]) * flop_per_step(setup) + \
        tot["points"] * flop_per_point_adjoint(setup)
    achieved = flop / (sum(ms) / 1e3) / 1e12
    out = {
        "metric": "adjoint gradients/s", "value": 1e3 / adj_ms, "unit": "gradients/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": adj_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": desc, "photons_per_gradient": n, "parameters": npar,
                   "objective": "sum of the film over the central 32x32 px, all bins"},
        "photon_paths_per_s": n / (adj_ms / 1e3),
        "forward_ms": fwd_ms, "cost_vs_forward": adj_ms / fwd_ms,
        "finite_differences": {"renders": 2 * npar, "ms": 2 * npar * fwd_ms,
                               "speedup_of_adjoint": 2 * npar * fwd_ms / adj_ms},
        "roofline": {"bound": "fp32", "kernel": "adjoint_{trace,replay,sweep}_kernel<"
                     + {L.FIELD_PLANEWAVE: "FK_PLANEWAVE", L.FIELD_SPLINE: "FK_SPLINE"}.get(
                         setup.field_type, f"FK_BESSEL{setup.mode}") + ">",
                     "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s", "frac": achieved / peak.value,
                     "traffic": None,
                     "flop_model": "er_steps (checkpointing trace + replays) x flop_per_step + swept points x "
                                   "flop_per_point_adjoint (simpler_b200/roofline.py)",
                     "peak_source": "FP32 FMA throughput measured live on this GPU (smp_fp32_peak)"},
        "counts_per_step": {k: v / args.steps for k, v in tot.items()},
        "e2e": {"value": 1.0 / e2e_s, "unit": "gradients/s", "h2d_bytes_per_step": G.nbytes + 4096,
                "d2h_bytes_per_step": npar * 8 + 80, "call": "smp_render_adjoint (one-shot plan, host dJ/dfilm "
                                                            "and gradient), wall clock"},
        "gpu_launches": int(tot["launches"]), "clocks": clk,
    }
    print(json.dumps(out), flush=True)


def main():
    global _ARGS
    args = parse()
    _ARGS = args
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "sweep":
        run_sweep(args)
    elif args.workload in ADJOINT:
        run_adjoint(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
