#!/usr/bin/env python
"""Benchmark of the hologram -> refractive-index path on B200.

Workload (one "step" = one reconstruction): 49 off-axis holograms of 512^2 float32 of a synthetic
cell (ellipsoidal body n=1.360 of 12 x 10 x 8 um, nucleus n=1.375, two vesicles n=1.390, medium
1.337; first-order Rytov fields; Gaussian noise sigma = 0.02 = 1% of the mean intensity, seeds 1 and
2) plus matching backgrounds -> fields of 256^2 (carrier 141,141 px, crop radius 65) -> Rytov ->
Ewald mapping -> 256^3 FISTA-TV, 20 outer x 10 FGP iterations, TV weight 1e-2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Ours: `value` = reconstructions/s of the device-resident pipeline (holograms already in HBM,
volume left in HBM), timed per step with CUDA events on the pipeline's stream, L2 flushed between
steps; `e2e` = the same through the public Python API (qoraholo_b200.Pipeline.run_stream over the
steps' stacks: pageable numpy in, pinned staging, H2D, compute, D2H, numpy out, each stack's transfers
overlapping a neighbour's solve; `per_call_value` is Pipeline.run called once per stack). Under torchrun each rank runs the same workload
on its GPU (replicas; the path has no data exchange); times are the max over ranks.

Both arms reconstruct the same holograms, made with numpy only (make_inputs), so neither arm loads
the other's libraries to build its inputs.

Reference arm (--impl reference): the reference's own CPU implementation (oracle/_ref, its sources
compiled unmodified) on this host's cores through its public Pipeline API, every step one full
reconstruction (Pipeline::run, all 20 x 10 iterations). The GPU arm's `cpu_baseline` is two such
runs; their volume is the parity reference: `parity` gives our error against it (index contrast,
filled fraction), both results' error against an FP64 run of the same algorithm (oracle/fp64.py) and
each one's RMSE against the analytic cell.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "256³ TV recons/s + p50/p99 latency, served vs plain GPU path, ≤1e-4 rel err"
UNIT = "recons/s"

# Optics of the workload.
WAVELENGTH, N_MEDIUM, NA = 0.532, 1.337, 1.2
HOLO_PIXEL, FIELD_PIXEL = 0.055, 0.11
COUNT, HOLO_N, FIELD_N = 49, 512, 256
CARRIER_PX, RADIUS = 141, 65.0
ITERATIONS, TV_INNER, TV_WEIGHT = 20, 10, 1e-2
NOISE = 0.02

# Synthetic cell, painter's order; each shape lies entirely inside or outside every earlier one.
# (kind, centre z y x, semi-axes z y x, index)
CELL = [
    ("ellipsoid", (0.0, 0.0, 0.0), (4.0, 5.0, 6.0), 1.360),
    ("ellipsoid", (0.0, 0.0, -1.5), (3.0, 3.0, 3.0), 1.375),
    ("ellipsoid", (0.0, 1.5, 3.0), (1.0, 1.0, 1.0), 1.390),
    ("ellipsoid", (-1.0, -2.0, 2.5), (1.0, 1.0, 1.0), 1.390),
]

WORKLOAD = (f"{COUNT}x{HOLO_N}^2 holograms -> {FIELD_N}^2 fields -> {FIELD_N}^3 FISTA-TV "
            f"{ITERATIONS}x{TV_INNER}, synthetic cell")


def _inside(shape, z, y, x):
    _, c, a, _ = shape
    return ((z - c[0]) / a[0]) ** 2 + ((y - c[1]) / a[1]) ** 2 + ((x - c[2]) / a[2]) ** 2 <= 1.0


def _parent_index(shapes, i):
    n = N_MEDIUM
    c = shapes[i][1]
    for s in shapes[:i]:
        if _inside(s, *c):
            n = s[3]
    return n


def phantom_fields(shapes, illum, n, pixel, device=None, keep_on_device=False):
    """Rytov field ratios (count, n, n) at z = 0 of nested ellipsoids `shapes` (painter's order)
    for each illumination: the analytic first Born spectrum of each shape placed on the Ewald caps
    (an ellipsoid is an affinely scaled ball), taken as a Rytov phase -- the construction of the
    reference's forward_fields for spheres (src/phantom.cpp:102-191), extended to ellipsoids.
    Computed in float64 (fixture generation, not the measured path): with numpy when `device` is
    None, else with torch on that device (the serving streams' many large stacks)."""
    if device is None:
        xp, fft2 = np, np.fft.ifft2
        ar = np.arange(n)
        sb = np.fft.fftfreq(n, d=1.0 / n)
    else:
        import torch

        xp, fft2 = torch, torch.fft.ifft2
        ar = torch.arange(n, device=device)
        sb = torch.fft.fftfreq(n, d=1.0 / n, dtype=torch.float64, device=device)
    k0 = 2 * math.pi / WAVELENGTH
    fm2 = (N_MEDIUM / WAVELENGTH) ** 2
    fna2 = (NA / WAVELENGTH) ** 2
    df = 1.0 / (n * pixel)
    my = (sb * df)[:, None]
    mx = (sb * df)[None, :]
    par = 1.0 - 2.0 * ((ar[:, None] + ar[None, :]) % 2)
    steps = []
    for i, (_, c, a, nn) in enumerate(shapes):
        vol = 4.0 / 3.0 * math.pi * a[0] * a[1] * a[2]
        steps.append(k0 * k0 * (nn * nn - _parent_index(shapes, i) ** 2) * vol)
    out = []
    for fiy, fix in np.asarray(illum, np.float64).reshape(-1, 2):
        fiz = math.sqrt(fm2 - fiy * fiy - fix * fix)
        fy, fx = my + fiy, mx + fix
        rho2 = fy * fy + fx * fx
        ok = (rho2 <= fna2) & (rho2 < fm2)
        nuz = xp.sqrt(xp.where(ok, fm2 - rho2, 1.0 + 0.0 * rho2))
        qz = nuz - fiz
        o = 0.0
        for (_, c, a, _), st in zip(shapes, steps):
            arg = 2 * math.pi * xp.sqrt((a[0] * qz) ** 2 + (a[1] * my) ** 2 + (a[2] * mx) ** 2)
            safe = xp.where(arg < 1e-3, 1e-3 + 0.0 * arg, arg)
            ball = xp.where(arg < 1e-3, 1.0 - arg * arg / 10.0, 3.0 * (xp.sin(safe) - safe * xp.cos(safe)) / safe ** 3)
            ph = -2 * math.pi * (qz * c[0] + my * c[1] + mx * c[2])
            o = o + st * ball * xp.exp(1j * ph)
        u = 1j / (4 * math.pi * nuz) * o * par / (pixel * pixel)
        u = xp.where(ok, u, 0.0 * u)
        out.append(xp.exp(fft2(u)))
    if device is None:
        return np.stack(out).astype(np.complex64)
    res = torch.stack(out).to(torch.complex64)
    return res if keep_on_device else res.cpu().numpy()


def device_holograms(capi, ratio, illum, pixel, carrier, seed):
    """Holograms (count, n, n) float32 on the host from device field ratios, synthesised on the device
    (qhk_synthesize_holograms_device, noise sigma = NOISE)."""
    import torch

    count, n = ratio.shape[0], ratio.shape[1]
    out = torch.empty((count, n, n), dtype=torch.float32, device=ratio.device)
    capi.synthesize_holograms_device(ratio.data_ptr(), count, n, illum, pixel, carrier=carrier, noise=NOISE, seed=seed,
                                     d_out=out.data_ptr())
    return out.cpu().numpy()


def circular_scan(count, na_illumination):
    """Illumination frequencies (fy, fx), cycles/um: the first view on axis, the others evenly on a
    circle of numerical aperture na_illumination -- the reference's circular_scan (src/api.cpp:203-216),
    in float32 arithmetic as there. Fixture code shared by both arms."""
    out = np.zeros((count, 2), np.float32)
    f = np.float32(na_illumination) / np.float32(WAVELENGTH)
    for i in range(1, count):
        phi = np.float32(2.0) * np.float32(math.pi) * np.float32(i - 1) / np.float32(count - 1)
        out[i] = (f * np.float32(math.sin(float(phi))), f * np.float32(math.cos(float(phi))))
    return out


def holograms(ratio, illum, pixel, carrier_px, seed):
    """Off-axis holograms |R + u|^2 + N(0, NOISE^2) of field ratios u (count, n, n), reference wave of
    unit amplitude at the carrier (carrier_px, carrier_px) pixels of the spectrum -- the reference's
    synthesize_holograms formula (src/phantom.cpp:193-221) in float64 with numpy's seeded generator.
    Fixture code shared by both arms, so that both reconstruct exactly the same inputs."""
    count, n, _ = ratio.shape
    c = carrier_px / (n * pixel)
    r = ((np.arange(n) - n // 2) * pixel)
    ref = np.exp(-2j * math.pi * c * (r[:, None] + r[None, :]))
    rng = np.random.default_rng(seed)
    out = np.empty((count, n, n), np.float32)
    for a, (fiy, fix) in enumerate(np.asarray(illum, np.float64)):
        u = np.exp(2j * math.pi * (fiy * r[:, None] + fix * r[None, :])) * ratio[a].astype(np.complex128)
        out[a] = (np.abs(ref + u) ** 2 + rng.normal(0.0, NOISE, size=(n, n))).astype(np.float32)
    return out


def make_inputs():
    """The C2 workload's illuminations, sample holograms (seed 1) and background holograms (seed 2),
    built with numpy only, so that neither arm's library makes the other's inputs."""
    illum = circular_scan(COUNT, 0.9)
    ratio = phantom_fields(CELL, illum, HOLO_N, HOLO_PIXEL)
    holo = holograms(ratio, illum, HOLO_PIXEL, CARRIER_PX, seed=1)
    bg = holograms(np.ones_like(ratio), illum, HOLO_PIXEL, CARRIER_PX, seed=2)
    return illum, holo, bg


def cell_volume():
    """The cell's index on the 256^3 reconstruction grid (analytic phantom for the RMSE)."""
    from oracle import fp64

    return fp64.render_ellipsoids([(c, a, n) for _, c, a, n in CELL], N_MEDIUM, FIELD_PIXEL, FIELD_N, FIELD_N)


def geom_tuple():
    return (WAVELENGTH, N_MEDIUM, NA, FIELD_PIXEL)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running (read only)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if parts and parts[0] == self.gpu:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def physical_gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one middle launch of the two-step FGP
# kernel at 256^3 with 8-row tiles, from one ncu capture of `python bench.py --kernel-case fgp`
# (profiles/k_fgp2_256cubed.txt, which gives the command). A constant, not a live measurement: no
# DRAM counter is readable from inside an unprofiled run. Update it with the profile.
FGP2_TRAFFIC_BYTES = 1037607168.0
FGP_TRAFFIC_BYTES = None  # the one-step kernel (not the tuned form at 256^3) has no capture here


def fgp_form(capi, n):
    """The FGP form the autotuner chose for an n^3 volume: (two_step, rows per CTA)."""
    for line in capi.autotune_report().splitlines():
        m = re.match(rf"fgp_rows device \d+ shape {n} {n} {n} 4 0 0 -> (\d+)", line.strip())
        if m:
            choice = int(m.group(1))
            return choice // 16 == 2, choice % 16
    return False, 0


def fgp_roofline(torch, capi, stream, live):
    """Roofline of the FGP kernel the TV proximal step runs at 256^3. Its average launch duration is
    `live` = (milliseconds, launches) of the proximal steps inside the timed reconstructions (CUDA events
    the pipeline records on its stream around each step, Pipeline.time_prox); the same kernel timed alone
    on random data (a 12-volume workspace, so that the tuned form runs) is reported beside it. Algorithmic
    bytes: a launch reads b, r (3), p (3) and writes p (3), r (3) (13 volumes); the first reads p as r and
    the last writes no r (10 volumes each). The one-step form (k_fgp) does one FGP step per launch, the
    two-step form (k_fgp2) two, so a prox of TV_INNER steps takes TV_INNER or TV_INNER / 2 launches."""
    n = FIELD_N
    vol = n * n * n
    b = torch.rand((n, n, n), device="cuda")
    x = torch.empty_like(b)
    work = torch.zeros((12, n, n, n), device="cuda")
    lam = TV_WEIGHT * (2 * math.pi / WAVELENGTH) ** 2

    def timed(inner, reps=5):
        capi.tv_prox_workspace(b.data_ptr(), x.data_ptr(), work.data_ptr(), 12, n, n, n, lam, inner, stream)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            capi.tv_prox_workspace(b.data_ptr(), x.data_ptr(), work.data_ptr(), 12, n, n, n, lam, inner, stream)
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    t10, t0 = timed(TV_INNER), timed(0)
    two_step, rows = fgp_form(capi, n)
    launches = TV_INNER // 2 if two_step else TV_INNER
    t_alone = (t10 - t0) / launches
    live_ms, live_launches = live
    if live_launches % launches:
        raise RuntimeError(f"proximal-step timing saw {live_launches} launches, not a multiple of {launches}")
    t_launch = live_ms / live_launches
    volumes = (10 + 13 * (launches - 2) + 10) / launches
    alg = volumes * vol * 4
    peak, which = measured_peaks()
    achieved = alg / (t_launch * 1e-3) / 1e9
    del b, x, work
    kernel = (f"k_fgp2 (two FGP steps per launch, {rows} rows per CTA, 256^3)" if two_step else
              "k_fgp (one FGP step of the TV proximal operator, 256^3)")
    return {"kernel": kernel, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_source": f"{which} hbm_gbs (burst copy)", "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": FGP2_TRAFFIC_BYTES if two_step else FGP_TRAFFIC_BYTES,
            "traffic_source": "ncu capture of one middle launch (constant in bench.py)",
            "algorithmic_bytes_per_launch": alg, "avg_launch_ms": round(t_launch, 5),
            "timing": f"CUDA events around the {live_launches} FGP launches of the timed reconstructions",
            "fgp_steps_per_launch": 2 if two_step else 1,
            "ms_per_fgp_step": round(t_launch / (2 if two_step else 1), 5),
            "alone_avg_launch_ms": round(t_alone, 5),
            "alone": "the same kernel timed alone on random data (b uniform in [0, 1)), L2 warm"}


def reference_run(holo, bg, illum):
    """One full run of the reference CPU Pipeline (oracle/_ref, the reference's own CPU sources) on the
    workload: all ITERATIONS x TV_INNER iterations. Returns (index volume, filled, milliseconds of the
    run as the reference's own Pipeline timing reports it)."""
    from oracle import refimpl

    ri, filled, ms = refimpl.pipeline(holo, bg, (CARRIER_PX, CARRIER_PX), RADIUS, FIELD_N, illum, geom_tuple(),
                                      iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER)
    return ri, filled, ms["run"]


def reference_threads():
    from oracle import refimpl

    return refimpl.threads()


def cpu_baseline(holo, bg, illum, runs=2):
    """Reference CPU rate from `runs` full reconstructions of the workload (no extrapolation); the last
    run's volume and filled fraction are returned for the parity check."""
    from oracle import refimpl

    if not refimpl.available():
        return None, None, None
    ms, ri, filled = [], None, None
    for _ in range(runs):
        ri, filled, t = reference_run(holo, bg, illum)
        ms.append(t)
    base = {"value": round(1000.0 * runs / sum(ms), 5), "unit": UNIT, "cores": reference_threads(),
            "kind": "reference",
            "sample": (f"{runs} full runs of the reference Pipeline (oracle/_ref, the reference's CPU sources, "
                       f"OpenMP) on the same {COUNT}x{HOLO_N}^2 holograms -> {FIELD_N}^3 FISTA-TV "
                       f"{ITERATIONS}x{TV_INNER}: {', '.join(f'{t:.0f}' for t in ms)} ms")}
    return base, ri, filled


def reference_cuda_leg(holo, bg, illum, ref_cpu, runs=3):
    """The reference's own CUDA backend (oracle/_ref/libqhref_cuda.so: its src/cuda/*.cu built
    unmodified for sm_100a with cuFFT) on the same workload through its public Pipeline::run on this
    B200: milliseconds of the last of `runs` runs (the earlier ones warm cuFFT plans), and its
    error against the reference CPU result. The per-kernel comparison with ours comes from a launch
    list of `--kernel-case refcuda`."""
    from oracle import fp64, refimpl

    if not refimpl.cuda_available():
        return {"unavailable": "oracle/_ref/libqhref_cuda.so is not built"}
    try:
        refimpl.select(cuda=True)
        ri, filled, ms = refimpl.pipeline(holo, bg, (CARRIER_PX, CARRIER_PX), RADIUS, FIELD_N, illum, geom_tuple(),
                                          iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT,
                                          tv_inner=TV_INNER, runs=runs)
    finally:
        refimpl.select(cuda=False)
    out = {"ms_per_recon": round(ms["run"], 2), "recons_per_s": round(1000.0 / ms["run"], 3),
           "stage_ms": {k: round(float(ms[k]), 2) for k in ("fields", "rytov", "fft2", "mapping", "normalize",
                                                             "solve", "finish")},
           "filled": filled,
           "path": "reference Pipeline::run (host holograms in, host volume out) with its CUDA backend, "
                   f"last of {runs} runs, its own host-clock timing"}
    if ref_cpu is not None:
        out["rel_err_vs_reference_cpu"] = fp64.rel_contrast_err(ri, ref_cpu, N_MEDIUM)
    return out


def parity_report(ours, ours_filled, ref, ref_filled, holo, bg, illum):
    """Our volume against the reference CPU volume of the same inputs (index-contrast error, the
    measure of the reference's tests/test_cuda.cpp:92-97, and the filled fraction), both against an
    FP64 run of the same algorithm (oracle/fp64.py), and each one's RMSE against the analytic cell."""
    from oracle import fp64

    out = {}
    if ref is not None:
        out["rel_err_vs_reference_cpu"] = fp64.rel_contrast_err(ours, ref, N_MEDIUM)
        out["filled_equal_reference_cpu"] = bool(abs(ours_filled - ref_filled) < 0.5 / FIELD_N ** 3)
    t0 = time.perf_counter()
    ri64, filled64 = fp64.pipeline(holo, bg, (CARRIER_PX, CARRIER_PX), RADIUS, FIELD_N, illum, geom_tuple(),
                                   iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER)
    out["rel_err_vs_fp64"] = fp64.rel_contrast_err(ours, ri64, N_MEDIUM)
    if ref is not None:
        out["reference_rel_err_vs_fp64"] = fp64.rel_contrast_err(ref, ri64, N_MEDIUM)
    phantom = cell_volume()
    out["rmse_vs_phantom"] = {"ours": fp64.rmse(ours, phantom), "fp64": fp64.rmse(ri64, phantom)}
    if ref is not None:
        out["rmse_vs_phantom"]["reference_cpu"] = fp64.rmse(ref, phantom)
    out["fp64_run"] = (f"oracle/fp64.py: the same pipeline in float64 ({fp64.threads()} threads, "
                       f"{time.perf_counter() - t0:.0f} s); filled {filled64:.6f}")
    return out


def combine_ranks(local_ms, steps, world, dist=None, device="cpu"):
    """Max over ranks of the local timed milliseconds, and the whole-job rate: every rank ran
    `steps` reconstructions, so value = world * steps / max time."""
    import torch

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if dist is not None and world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    return max_ms, world * steps * 1000.0 / max_ms


def percentile(sorted_values, q):
    """Nearest-rank percentile of a sorted list."""
    return sorted_values[min(len(sorted_values) - 1, max(0, math.ceil(q * len(sorted_values)) - 1))]


def bench_config(world):
    """The `config` object of both arms' lines (the same keys and values)."""
    return {"workload": WORKLOAD, "holograms": [COUNT, HOLO_N, HOLO_N], "fields": [FIELD_N, FIELD_N],
            "volume": [FIELD_N] * 3, "solver": "tv", "iterations": ITERATIONS, "tv_inner": TV_INNER,
            "tv_weight": TV_WEIGHT, "parallelism": f"replicas{world}",
            "l2": "GPU arm: flushed (256 MiB write) before every timed step"}


def run_reference_arm(args):
    """The reference's own CPU implementation (oracle/_ref: its src/ and src/cpu/ sources compiled
    unmodified, OpenMP on all host threads) through its public Pipeline API (set_background once, then
    Pipeline::run per step, host holograms in and host volume out), every step a full reconstruction of
    the workload. Inputs are the same numpy-made holograms the GPU arm reconstructs; nothing of
    qoraholo_b200 is loaded. Under torchrun rank 0 alone runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        from oracle import refimpl

        if not refimpl.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) is missing"}))
            return 0
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed to load: {e}"}))
        return 0
    illum, holo, bg = make_inputs()
    for _ in range(args.warmup):
        reference_run(holo, bg, illum)
    steps = []
    for _ in range(args.steps):
        _, _, t = reference_run(holo, bg, illum)
        steps.append(t)
    total_ms = sum(steps)
    value = 1000.0 * len(steps) / total_ms
    cores = reference_threads()
    lat = sorted(steps)
    sample = (f"each step: one full reconstruction by the reference Pipeline::run (oracle/_ref) of the "
              f"{COUNT}x{HOLO_N}^2 holograms -> {FIELD_N}^3 FISTA-TV {ITERATIONS}x{TV_INNER}, host clock")
    line = {"metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / len(steps), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args.gpus), "impl": "reference",
            "latency_ms": {"p50": round(statistics.median(lat), 3), "p99": round(percentile(lat, 0.99), 3),
                           "path": "reference Pipeline::run"},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# Serving mix (three geometries with resident state, Poisson arrivals):
# (name, share, count, N, hologram pixel, field side, carrier px, crop radius, solver options)
SERVE_MIX = [
    ("49x256^2 -> 128^3 GP-20", 0.4, 49, 256, 0.1, 128, 70, 59.0, dict(iterations=20, solver="gp")),
    ("49x512^2 -> 256^3 FISTA-TV 20x10", 0.4, 49, 512, 0.055, 256, 141, 65.0,
     dict(iterations=20, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER)),
    ("97x1024^2 -> 384^3 GP-20", 0.2, 97, 1024, 0.04125, 384, 212, 98.0, dict(iterations=20, solver="gp")),
]
SERVE_BUDGET = 40 << 30
SERVE_INFLIGHT = 4


def serve_sample(rng, kind):
    """A seeded phantom with a random position and index step dn ~ U[0.01, 0.04]: a bead of radius
    2.5 um for the small geometry, the nested cell (body, nucleus, vesicles) otherwise."""
    dn = rng.uniform(0.01, 0.04)
    dy, dx = rng.uniform(-2.0, 2.0, 2)
    if kind == 0:
        return [("ellipsoid", (0.0, dy, dx), (2.5, 2.5, 2.5), N_MEDIUM + dn)]
    out = []
    for i, (k, c, a, n) in enumerate(CELL):
        step = (n - CELL[0][3]) if i else 0.0
        out.append((k, (c[0], c[1] + dy, c[2] + dx), a, N_MEDIUM + dn + step))
    return out


def serving_setup(qh, stacks_per_geometry=2, seed=2024):
    """Per mix entry: illuminations, geometry, background holograms and distinct request stacks
    (field ratios and holograms computed on the device)."""
    import torch

    from qoraholo_b200 import capi

    rng = np.random.default_rng(seed)
    geos = []
    for idx, (name, share, count, n, hpix, out, carrier, radius, opts) in enumerate(SERVE_MIX):
        fpix = hpix * n / out
        geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=fpix)
        illum = qh.circular_scan(count, 0.9, geom)
        c = carrier / (n * hpix)
        stacks = []
        for k in range(stacks_per_geometry):
            ratio = phantom_fields(serve_sample(rng, idx), illum, n, hpix, "cuda", keep_on_device=True)
            stacks.append(device_holograms(capi, ratio, illum, hpix, (c, c), seed=100 * idx + k + 1))
        ones = torch.ones((count, n, n), dtype=torch.complex64, device="cuda")
        bg = device_holograms(capi, ones, illum, hpix, (c, c), seed=100 * idx + 99)
        del ones
        geos.append(dict(name=name, share=share, count=count, n=n, out=out, carrier=carrier, radius=radius,
                         opts=opts, geom=geom, illum=illum, stacks=stacks, bg=bg))
    return geos


def serving_stream(geos, requests, rate, seed=7):
    """(arrival seconds, geometry index, stack index) for `requests` Poisson arrivals at `rate`/s
    with the mix's shares."""
    rng = np.random.default_rng(seed)
    shares = np.array([g["share"] for g in geos])
    kinds = rng.choice(len(geos), size=requests, p=shares / shares.sum())
    gaps = rng.exponential(1.0 / rate, size=requests)
    t = np.cumsum(gaps) - gaps[0]
    return [(float(t[i]), int(kinds[i]), int(rng.integers(len(geos[kinds[i]]["stacks"])))) for i in range(requests)]


def plain_request(qh, g, bg_fields, holo):
    """The per-call API, one call per stage, host arrays in and out (the reference's per-call
    chain: extract_fields, field_ratio, rytov, reconstruct)."""
    crop = dict(center=(g["carrier"], g["carrier"]), radius=g["radius"], output_size=g["out"])
    f = qh.extract_fields(holo, **crop)
    u = qh.rytov(qh.field_ratio(f, bg_fields))
    return qh.reconstruct(u, g["illum"], g["geom"], **g["opts"])


def served_run(sv, ids, geos, stream, plain_out=None):
    """Submits `stream` (arrival s, geometry, stack) from one thread at its arrival times and waits
    for every result in order from this one. Returns latencies (ms, completion - arrival), the span
    from the first arrival to the last completion (s), per-geometry (service, gpu) ms, and the largest
    relative difference from the plain results given."""
    lat, per_geo, worst = [], {}, 0.0
    tickets = [None] * len(stream)
    t0 = time.perf_counter()

    def submitter():
        for j, (arr, gi, si) in enumerate(stream):
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            start = time.perf_counter() - t0
            tickets[j] = (sv.submit(ids[gi], geos[gi]["stacks"][si]), start)

    th = threading.Thread(target=submitter)
    th.start()
    done_at = 0.0
    for j, (arr, gi, si) in enumerate(stream):
        while tickets[j] is None:
            time.sleep(0.0002)
        ri, _, times = sv.wait(tickets[j][0])
        done_at = max(done_at, tickets[j][1] + times["total"] / 1000.0)
        lat.append(1000.0 * (tickets[j][1] - arr) + times["total"])
        per_geo.setdefault(gi, []).append((times["service"], times["gpu"]))
        ref = (plain_out or {}).get((gi, si))
        if ref is not None:
            worst = max(worst, float(np.linalg.norm(ri.astype(np.float64) - ref) /
                                     np.linalg.norm(ref.astype(np.float64) - N_MEDIUM)))
    th.join()
    return sorted(lat), done_at, per_geo, worst


SERVE_SATURATE = 200.0  # arrivals per second well above any capacity: the queue builds, completions/s = capacity


def serving_leg(qh, capi, requests, rate, inflight=SERVE_INFLIGHT, plain=True):
    """Served stream vs the plain per-call path. Capacity: both take the same saturating Poisson
    stream (SERVE_SATURATE arrivals/s, so requests queue and completions/s measure what each path
    sustains); throughput = requests / (last completion - first arrival). Latency: the served path
    again at `rate` arrivals/s, a load it sustains, completion - arrival on the host clock."""
    geos = serving_setup(qh)
    saturated = serving_stream(geos, requests, SERVE_SATURATE)
    loaded = serving_stream(geos, requests, rate, seed=8)
    # Plain path: serial per-call API; background fields computed once per geometry (a per-call
    # user would cache them too).
    bgf = [qh.extract_fields(g["bg"], center=(g["carrier"], g["carrier"]), radius=g["radius"], output_size=g["out"])
           for g in geos]
    for i, g in enumerate(geos):
        plain_request(qh, g, bgf[i], g["stacks"][0])
    plain_out = {}
    plain_lat = []
    plain_ms = {}
    t0 = time.perf_counter()
    for j, (arr, gi, si) in enumerate(saturated if plain else []):
        now = time.perf_counter() - t0
        if now < arr:
            time.sleep(arr - now)
        t_req = time.perf_counter()
        ri = plain_request(qh, geos[gi], bgf[gi], geos[gi]["stacks"][si])
        plain_ms.setdefault(gi, []).append(1000.0 * (time.perf_counter() - t_req))
        plain_lat.append(1000.0 * (time.perf_counter() - t0 - arr))
        plain_out.setdefault((gi, si), ri)
    plain_span = time.perf_counter() - t0

    # Resident path: one qoraholo_b200.Pipeline per geometry, built once with its background (plans,
    # background fields and Ewald constants resident), requests run back to back through Pipeline.run
    # (numpy in, numpy out) on the same saturating arrivals -- the best a caller without the server
    # does with the public API.
    res_span = float("nan")
    res_lat = []
    if plain:
        pipes = []
        for g in geos:
            pp = qh.Pipeline(g["count"], g["n"], (g["carrier"], g["carrier"]), g["illum"], g["geom"], radius=g["radius"],
                             output_size=g["out"], **g["opts"])
            pp.set_background(g["bg"])
            pp.run(g["stacks"][0])
            pipes.append(pp)
        t0 = time.perf_counter()
        for arr, gi, si in saturated:
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            pipes[gi].run(geos[gi]["stacks"][si])
            res_lat.append(1000.0 * (time.perf_counter() - t0 - arr))
        res_span = time.perf_counter() - t0
        del pipes

    with capi.Server(hbm_budget=SERVE_BUDGET, max_inflight=inflight) as sv:
        ids = []
        for g in geos:
            ids.append(sv.add_geometry(g["count"], g["n"], (g["carrier"], g["carrier"]), g["illum"], g["geom"],
                                       g["bg"], radius=g["radius"], output_size=g["out"], **g["opts"]))
        for _ in range(2):  # every workspace runs once eagerly, then is captured as a graph
            warm = [sv.submit(ids[gi], geos[gi]["stacks"][0]) for gi in range(len(geos)) for _ in range(inflight)]
            for t in warm:
                sv.wait(t)
        alone_ms = []
        for gi in range(len(geos)):  # each geometry alone on an idle device: its service time
            alone_ms.append(sv.wait(sv.submit(ids[gi], geos[gi]["stacks"][0]))[2]["gpu"])
        sat_lat, sat_span, per_geo, worst = served_run(sv, ids, geos, saturated, plain_out)
        load_lat, load_span, _, _ = served_run(sv, ids, geos, loaded)
        stats = sv.stats()
    pl = sorted(plain_lat) or [float("nan")]
    rl = sorted(res_lat) or [float("nan")]
    served_v = requests / sat_span
    plain_v = requests / plain_span if plain else float("nan")
    res_v = requests / res_span if plain else float("nan")
    counts = {g["name"]: sum(1 for _, gi, _ in saturated if gi == i) for i, g in enumerate(geos)}
    serial_bound = 1000.0 / sum(g["share"] * alone_ms[i] for i, g in enumerate(geos))
    # Details first, the headline figures last (they then survive a truncated line).
    return {
        "path": "qoraholo_b200.capi.Server (submit/wait from Python, numpy in/out), host clock",
        "requests": requests, "saturating_arrivals_per_s": SERVE_SATURATE, "mix": counts,
        "hbm_budget_bytes": SERVE_BUDGET, "max_inflight": inflight,
        "server": {k: stats[k] for k in ("workspaces_created", "workspaces_evicted", "graph_launches",
                                          "passed_over", "peak_used", "peak_inflight")},
        "alone_gpu_ms": {g["name"]: round(alone_ms[i], 3) for i, g in enumerate(geos)},
        "median_service_gpu_ms": {g["name"]: [round(statistics.median(v[0] for v in per_geo[i]), 2),
                                              round(statistics.median(v[1] for v in per_geo[i]), 2)]
                                  for i, g in enumerate(geos) if i in per_geo},
        "plain": {"value": round(plain_v, 3), "unit": UNIT, "p50_ms": round(statistics.median(pl), 2),
                  "p99_ms": round(percentile(pl, 0.99), 2),
                  "median_request_ms": {g["name"]: round(statistics.median(plain_ms[i]), 1)
                                        for i, g in enumerate(geos) if i in plain_ms},
                  "path": "per-call API (extract_fields, field_ratio, rytov, reconstruct) serially, numpy in/out, "
                          "same saturating arrivals (latency is queueing)"},
        "resident_pipelines": {"value": round(res_v, 3), "unit": UNIT, "p50_ms": round(statistics.median(rl), 2),
                               "p99_ms": round(percentile(rl, 0.99), 2),
                               "path": "one resident qoraholo_b200.Pipeline per geometry, Pipeline.run back to back, "
                                       "numpy in/out, same saturating arrivals"},
        "serial_gpu_bound": round(serial_bound, 3),
        "latency_at": f"{rate:g} Poisson arrivals/s ({requests} requests, {requests / load_span:.1f} recons/s done)",
        "saturated_p50_p99_ms": [round(statistics.median(sat_lat), 2), round(percentile(sat_lat, 0.99), 2)],
        "max_rel_err_served_vs_plain": worst,
        "speedup_vs_resident_pipelines": round(served_v / res_v, 3),
        "speedup_vs_serial_gpu_bound": round(served_v / serial_bound, 3),
        "speedup": round(served_v / plain_v, 3),
        "p50_ms": round(statistics.median(load_lat), 2), "p99_ms": round(percentile(load_lat, 0.99), 2),
        "value": round(served_v, 3), "unit": UNIT,
    }


BPM_N, BPM_NZ, BPM_VIEWS, BPM_PIXEL, BPM_ITERS, BPM_EVERY, BPM_REF_VIEWS = 256, 128, 49, 0.2, 50, 16, 4


def bpm_leg(qh, torch, iterations=BPM_ITERS, reference=True):
    """Gradient inversion with the BPM model behind torch.autograd: 256^2 x 128 slices (dz = pixel =
    0.2 um), 49 views at NA 0.9, 20 overlapping spheres (radii 1-3 um, dn <= 0.05) rendered on the
    grid, data = the model's fields of that volume; `iterations` steps of gradient descent on
    1/2 |y - data|^2 / views with step 1 / Lipschitz, checkpoint every 16 slices. Times one
    iteration (forward + backward) with CUDA events; the reference CPU gradient (bpm_forward +
    bpm_vjp of oracle/_ref) is timed once at the starting point and compared."""
    from qoraholo_b200.autograd import BpmModel

    rng = np.random.default_rng(17)
    geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=BPM_PIXEL)
    illum = qh.circular_scan(BPM_VIEWS, 0.9, geom)
    spheres = [qh.Sphere(z=float(rng.uniform(-5, 5)), y=float(rng.uniform(-8, 8)), x=float(rng.uniform(-8, 8)),
                         radius=float(rng.uniform(1, 3)), n=float(N_MEDIUM + rng.uniform(0.005, 0.05)))
               for _ in range(20)]
    truth = qh.render_phantom(spheres, geom, BPM_NZ, BPM_N)
    model = BpmModel(BPM_NZ, BPM_N, illum, geom, checkpoint_every=BPM_EVERY)
    with torch.no_grad():
        data = model(torch.from_numpy(np.ascontiguousarray(truth, np.float32)).cuda())
    x = torch.full((BPM_NZ, BPM_N, BPM_N), N_MEDIUM, device="cuda", requires_grad=True)
    phase = 2 * math.pi / WAVELENGTH * BPM_PIXEL
    opt = torch.optim.SGD([x], lr=1.0 / (BPM_NZ * phase * phase))

    def step():
        opt.zero_grad(set_to_none=False)
        loss = 0.5 * (model(x) - data).abs().pow(2).sum() / BPM_VIEWS
        loss.backward()
        opt.step()
        return loss

    first = float(step().detach())  # warm-up (allocations, twiddles)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(iterations - 1):
        last = step()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / max(iterations - 1, 1)
    flops = BPM_VIEWS * BPM_NZ * 6 * 5.0 * BPM_N * BPM_N * math.log2(BPM_N * BPM_N)
    out = {"workload": f"BPM gradient inversion {BPM_N}^2 x {BPM_NZ}, {BPM_VIEWS} views, 20 spheres, "
                       f"{iterations} iterations, checkpoint every {BPM_EVERY} slices",
           "ms_per_iteration": round(ms, 3), "iterations_per_s": round(1000.0 / ms, 3),
           "fft_gflops": round(flops / (ms * 1e-3) / 1e9, 1),
           "fft_flop_model": "6 2D FFTs (2 forward, 2 recompute, 2 adjoint) per slice per view x 5 N log2 N",
           "plan_device_bytes": model.plan.device_bytes, "loss_first": first, "loss_last": float(last.detach())}
    if reference:
        # Bounded sample of the reference CPU gradient: the first BPM_REF_VIEWS illuminations (the
        # gradient is a sum over views, its cost linear in them), scaled to all views; our gradient of
        # the same views is compared with it.
        try:
            from oracle import refimpl

            if refimpl.available():
                k = BPM_REF_VIEWS
                il_k = np.ascontiguousarray(np.reshape(illum, (-1, 2))[:k])
                x0n = np.full((BPM_NZ, BPM_N, BPM_N), N_MEDIUM, np.float32)
                t0 = time.perf_counter()
                y = refimpl.bpm_forward(x0n, il_k, geom_bpm_tuple())
                r = (y - data[:k].cpu().numpy()).astype(np.complex64)
                want = refimpl.bpm_vjp(x0n - N_MEDIUM, r, il_k, geom_bpm_tuple())
                ref_ms = 1000.0 * (time.perf_counter() - t0) * BPM_VIEWS / k
                model_k = BpmModel(BPM_NZ, BPM_N, il_k, geom, checkpoint_every=BPM_EVERY)
                xk = torch.full_like(x, N_MEDIUM).requires_grad_(True)
                model_k(xk).backward(torch.from_numpy(r).cuda())
                ours = xk.grad.cpu().numpy()
                model_k.plan.close()
                out["reference_cpu_ms_per_gradient"] = round(ref_ms, 1)
                out["reference_cpu_sample"] = f"first {k} of {BPM_VIEWS} views, scaled by views"
                out["reference_cpu_cores"] = refimpl.threads()
                out["rel_err_gradient_vs_reference_cpu"] = float(np.linalg.norm(ours - want) / np.linalg.norm(want))
        except Exception as ex:  # noqa: BLE001
            out["reference_cpu_error"] = f"{type(ex).__name__}: {ex}"
    model.plan.close()
    return out


def geom_bpm_tuple():
    return (WAVELENGTH, N_MEDIUM, NA, BPM_PIXEL)


C4_UNWRAP, C4_SIDES, C4_ODT = 512, (128, 192, 256, 384, 512), 64


def phase_maps(torch, shapes, seed=31):
    """Wrapped phase maps of smooth random surfaces: 3-6 Gaussians plus a tilt, peak-to-peak
    ~U[10, 60] rad, plus N(0, 0.1 rad) noise (computed with torch on the GPU; fixture data)."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    rng = np.random.default_rng(seed)
    out = []
    for ny, nx in shapes:
        y = torch.arange(ny, device="cuda", dtype=torch.float32)[:, None] / ny
        x = torch.arange(nx, device="cuda", dtype=torch.float32)[None, :] / nx
        surf = float(rng.uniform(-1, 1)) * y + float(rng.uniform(-1, 1)) * x
        for _ in range(int(rng.integers(3, 7))):
            cy, cx, sy, sx = rng.uniform(0, 1), rng.uniform(0, 1), rng.uniform(0.05, 0.3), rng.uniform(0.05, 0.3)
            surf = surf + float(rng.uniform(-1, 1)) * torch.exp(-((y - cy) / sy) ** 2 - ((x - cx) / sx) ** 2)
        surf = (surf - surf.min()) / (surf.max() - surf.min()).clamp_min(1e-9) * float(rng.uniform(10, 60))
        surf = surf + 0.1 * torch.randn((ny, nx), device="cuda", generator=g)
        out.append(torch.remainder(surf + math.pi, 2 * math.pi) - math.pi)
    return out


def c4_leg(qh, capi, torch, reps=5):
    """C4 batching: (1) 512 least-squares unwrap instances of sizes drawn from {128..512}^2 in single
    persistent launches (one per pass, graph-replayed) vs a per-image launch loop and the reference
    CPU; (2) 64 reconstructions 49 x 128^2 -> 64^2 -> 64^3 GP-10 in one batched, graph-replayed
    pipeline vs one pipeline run per request and the reference CPU."""
    out = {}
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    sides = [int(v) for v in rng.choice(C4_SIDES, C4_UNWRAP)]
    shapes = [(s_, s_) for s_ in sides]
    maps = phase_maps(torch, shapes)
    plan = capi.UnwrapBatch(shapes)
    d_in = torch.cat([m.reshape(-1) for m in maps])
    d_out = torch.empty_like(d_in)
    pixels = plan.total

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(n):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / n

    launches0 = capi.kernel_launches()
    plan.run(d_in.data_ptr(), d_out.data_ptr(), stream, graph=True)  # direct first call
    launches_batch = capi.kernel_launches() - launches0
    t_graph = timed(lambda: plan.run(d_in.data_ptr(), d_out.data_ptr(), stream, graph=True), reps)
    t_direct = timed(lambda: plan.run(d_in.data_ptr(), d_out.data_ptr(), stream, graph=False), reps)
    batch_result = d_out.clone()
    loop_out = torch.empty_like(d_in)

    def per_image():
        for off, (ny, nx) in zip(plan.offsets, shapes):
            capi.unwrap_noalloc(d_in.data_ptr() + 4 * off, loop_out.data_ptr() + 4 * off, 1, ny, nx, stream)

    t_loop = timed(per_image, 2)
    diff = float((batch_result - loop_out).abs().max())
    peak, which = measured_peaks()
    alg = 8.0 * pixels
    out["unwrap"] = {
        "workload": f"{C4_UNWRAP} unwrap instances, sides drawn from {list(C4_SIDES)} (seeded), "
                    f"{pixels} pixels, {alg / 1e6:.0f} MB algorithmic (read + write one float per pixel)",
        "batched_graph_ms": round(t_graph, 3), "batched_direct_ms": round(t_direct, 3),
        "per_image_loop_ms": round(t_loop, 3), "instances_per_s": round(C4_UNWRAP / (t_graph * 1e-3), 1),
        "launches_per_batch": int(launches_batch), "launches_per_image_loop": 5 * C4_UNWRAP,
        "achieved_gbs": round(alg / (t_graph * 1e-3) / 1e9, 1), "peak_gbs": peak, "peak_source": which,
        "max_abs_diff_vs_per_image_loop": diff,
        "per_image_loop": "qhk_unwrap_noalloc per image (five launches each), device buffers"}
    try:
        from oracle import refimpl

        if refimpl.available():
            sample = list(range(0, C4_UNWRAP, C4_UNWRAP // 16))
            host = [maps[i].cpu().numpy() for i in sample]
            t0 = time.perf_counter()
            for h in host:
                refimpl.unwrap(h[None])
            ref_s = time.perf_counter() - t0
            frac = sum(shapes[i][0] * shapes[i][1] for i in sample) / pixels
            out["unwrap"]["reference_cpu_ms"] = round(1000.0 * ref_s / frac, 1)
            out["unwrap"]["reference_cpu_sample"] = (f"{len(sample)} of the {C4_UNWRAP} instances, "
                                                     f"scaled by pixel count, {refimpl.threads()} threads")
    except Exception as e:  # noqa: BLE001
        out["unwrap"]["reference_cpu_error"] = str(e)
    del d_in, d_out, batch_result, loop_out, maps

    # (2) small reconstructions
    n_holo, m, count, carrier = 128, 64, 49, 35
    geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=0.2)
    hgeom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=0.1)
    illum = qh.circular_scan(count, 0.9, geom)
    c = carrier / (n_holo * 0.1)
    stacks = []
    for k in range(C4_ODT):
        sample_ = [("ellipsoid", (0.0, float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))), (2.5, 2.5, 2.5),
                    N_MEDIUM + float(rng.uniform(0.01, 0.04)))]
        ratio = phantom_fields(sample_, illum, n_holo, 0.1, "cuda")
        stacks.append(qh.synthesize_holograms(ratio, illum, hgeom, carrier=(c, c), noise=NOISE, seed=k + 1))
    bg = qh.synthesize_holograms(np.ones((count, n_holo, n_holo), np.complex64), illum, hgeom, carrier=(c, c),
                                 noise=NOISE, seed=999)
    gt = (WAVELENGTH, N_MEDIUM, NA, 0.2)
    kw = dict(radius=30.0, output_size=m, iterations=10, solver="gp")
    batched = capi.Pipeline(count, n_holo, (carrier, carrier), illum, gt, batch=C4_ODT, **kw)
    batched.set_background(bg)
    single = capi.Pipeline(count, n_holo, (carrier, carrier), illum, gt, **kw)
    single.set_background(bg)
    d_holo = torch.from_numpy(np.concatenate(stacks)).cuda()
    d_index = torch.empty(batched.shape, dtype=torch.float32, device="cuda")
    d_one = torch.empty(single.shape, dtype=torch.float32, device="cuda")
    batched.process_device_graph(d_holo.data_ptr(), d_index.data_ptr(), stream)
    launches0 = capi.kernel_launches()
    batched.process_device_graph(d_holo.data_ptr(), d_index.data_ptr(), stream)
    launches_b = capi.kernel_launches() - launches0
    t_b = timed(lambda: batched.process_device_graph(d_holo.data_ptr(), d_index.data_ptr(), stream), reps)
    stack = count * n_holo * n_holo

    def per_request():
        for k in range(C4_ODT):
            single.process_device(d_holo.data_ptr() + 4 * k * stack, d_one.data_ptr(), stream)

    t_s = timed(per_request, 2)
    same = True
    for k in (0, C4_ODT // 2, C4_ODT - 1):
        single.process_device(d_holo.data_ptr() + 4 * k * stack, d_one.data_ptr(), stream)
        same = same and bool(torch.equal(d_one, d_index[k]))
    out["small_odt"] = {
        "workload": f"{C4_ODT} x ({count}x{n_holo}^2 holograms -> {m}^2 fields -> {m}^3 GP-10), bead phantoms",
        "batched_graph_ms": round(t_b, 3), "per_request_loop_ms": round(t_s, 3),
        "recons_per_s": round(C4_ODT / (t_b * 1e-3), 1), "launches_per_batch": int(launches_b),
        "batch_equals_single": same}
    try:
        from oracle import refimpl

        if refimpl.available():
            _, _, ms = refimpl.pipeline(stacks[0], bg, (carrier, carrier), 30.0, m, illum, gt, iterations=10,
                                        solver="gp")
            out["small_odt"]["reference_cpu_ms_per_recon"] = round(ms["run"], 1)
            out["small_odt"]["reference_cpu_cores"] = refimpl.threads()
    except Exception as e:  # noqa: BLE001
        out["small_odt"]["reference_cpu_error"] = str(e)
    batched.close()
    single.close()
    return out


def kernel_case(name, reps, tv_form=0):
    """Small standalone launches of one kernel family for profiling (no JSON line): `c2` runs the C2
    reconstruction (the bench workload, device-resident) `reps` times after a warm-up run, each inside
    the NVTX range "c2_step"; `refcuda` the reference's CUDA Pipeline::run on the same workload (`reps`
    runs); `unwrapbatch` the C4 batch of 512 uneven unwraps (`reps` runs, no graph); `bpmstep` one BPM
    gradient (forward + backward, 256^2 x 128 slices, 49 views, checkpoint every 16 slices) after a warm-up,
    inside the NVTX range "bpm_step"; `fgp` runs the
    TV proximal step at 256^3 on a 12-volume workspace (10 FGP steps in the tuned form + final primal
    per rep); `fft` a 256^3 rfft3 + irfft3
    per rep; `kspace` a 256^3 GP-4 solve from 49 random 256^2 fields per rep (the k-space step's
    row and axis passes); `pipeline` the full device pipeline on 9 x 128^2 holograms -> 64^3."""
    import torch

    from qoraholo_b200 import capi

    stream = torch.cuda.current_stream().cuda_stream
    capi.tv_form(tv_form)
    if name == "fft":
        n = FIELD_N
        x = torch.rand((n, n, n), device="cuda")
        half = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        for _ in range(reps):
            capi.rfft3(x.data_ptr(), half.data_ptr(), n, n, n, stream)
            capi.irfft3(half.data_ptr(), x.data_ptr(), n, n, n, 1.0 / n ** 3, stream)
    elif name == "kspace":
        import qoraholo_b200 as qh

        n = FIELD_N
        geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=FIELD_PIXEL)
        illum = qh.circular_scan(COUNT, 0.9, geom)
        plan = capi.OdtPlan(n, COUNT, illum, geom_tuple(), iterations=4, solver="gp")
        fields = torch.randn((COUNT, n, n), dtype=torch.complex64, device="cuda")
        index = torch.empty(plan.shape, dtype=torch.float32, device="cuda")
        for _ in range(reps):
            plan.run(fields.data_ptr(), index.data_ptr(), stream)
    elif name == "c2":
        import qoraholo_b200 as qh

        illum, holo, bg = make_inputs()
        pipe = capi.Pipeline(COUNT, HOLO_N, (CARRIER_PX, CARRIER_PX), illum, geom_tuple(), radius=RADIUS,
                             output_size=FIELD_N, iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT,
                             tv_inner=TV_INNER)
        pipe.set_background(bg)
        d_holo = torch.from_numpy(holo).cuda()
        d_index = torch.empty(pipe.shape, dtype=torch.float32, device="cuda")
        pipe.process_device(d_holo.data_ptr(), d_index.data_ptr(), stream)  # warm (plans, tuning)
        torch.cuda.synchronize()
        for _ in range(reps):  # ncu --nvtx --nvtx-include "c2_step/" captures exactly these launches
            torch.cuda.nvtx.range_push("c2_step")
            pipe.process_device(d_holo.data_ptr(), d_index.data_ptr(), stream)
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        pipe.check_waits(stream)
    elif name == "bpmstep":
        import qoraholo_b200 as qh
        from qoraholo_b200.autograd import BpmModel

        geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=BPM_PIXEL)
        illum = circular_scan(BPM_VIEWS, 0.9)
        model = BpmModel(BPM_NZ, BPM_N, illum, geom, checkpoint_every=BPM_EVERY)
        x = torch.full((BPM_NZ, BPM_N, BPM_N), N_MEDIUM + 0.01, device="cuda", requires_grad=True)
        g = torch.ones((BPM_VIEWS, BPM_N, BPM_N), dtype=torch.complex64, device="cuda")
        model(x).backward(g)  # warm (plans, checkpoints)
        torch.cuda.synchronize()
        for _ in range(reps):  # ncu --nvtx --nvtx-include "bpm_step/" captures one gradient
            torch.cuda.nvtx.range_push("bpm_step")
            x.grad = None
            model(x).backward(g)
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        model.plan.close()
    elif name == "unwrapbatch":
        rng = np.random.default_rng(5)
        shapes = [(int(v), int(v)) for v in rng.choice(C4_SIDES, C4_UNWRAP)]
        maps = phase_maps(torch, shapes)
        plan = capi.UnwrapBatch(shapes)
        d_in = torch.cat([m.reshape(-1) for m in maps])
        d_out = torch.empty_like(d_in)
        del maps
        for _ in range(reps):
            plan.run(d_in.data_ptr(), d_out.data_ptr(), stream, graph=False)
    elif name == "refcuda":
        from oracle import refimpl

        illum, holo, bg = make_inputs()
        refimpl.select(cuda=True)
        _, _, ms = refimpl.pipeline(holo, bg, (CARRIER_PX, CARRIER_PX), RADIUS, FIELD_N, illum, geom_tuple(),
                                    iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER,
                                    runs=reps)
        refimpl.select(cuda=False)
        print(f"reference CUDA Pipeline::run: {ms['run']:.1f} ms (last of {reps})")
    elif name == "fgp":
        n = FIELD_N
        b = torch.rand((n, n, n), device="cuda")
        x = torch.empty_like(b)
        work = torch.zeros((12, n, n, n), device="cuda")
        lam = TV_WEIGHT * (2 * math.pi / WAVELENGTH) ** 2
        for _ in range(reps):
            capi.tv_prox_workspace(b.data_ptr(), x.data_ptr(), work.data_ptr(), 12, n, n, n, lam, TV_INNER, stream)
    else:
        import qoraholo_b200 as qh

        geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=0.22)
        holo_geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=0.11)
        illum = qh.circular_scan(9, 0.9, geom)
        ratio = phantom_fields(CELL, illum, 128, 0.11, "cuda")
        c = 35 / (128 * 0.11)
        holo = qh.synthesize_holograms(ratio, illum, holo_geom, carrier=(c, c), noise=NOISE, seed=1)
        bg = qh.synthesize_holograms(np.ones_like(ratio), illum, holo_geom, carrier=(c, c), noise=NOISE, seed=2)
        pipe = capi.Pipeline(9, 128, (35, 35), illum, (WAVELENGTH, N_MEDIUM, NA, 0.22), radius=16.0, output_size=64,
                             iterations=4, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER)
        pipe.set_background(bg)
        d_holo = torch.from_numpy(holo).cuda()
        d_index = torch.empty(pipe.shape, dtype=torch.float32, device="cuda")
        for _ in range(reps):
            pipe.process_device(d_holo.data_ptr(), d_index.data_ptr(), stream)
    torch.cuda.synchronize()
    print(f"kernel case {name}: {reps} reps done")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel-case", choices=["fgp", "fft", "kspace", "pipeline", "c2", "refcuda", "unwrapbatch",
                                              "bpmstep", "serve", "bpm", "c4"],
                    default=None,
                    help="run only a small profiling case and exit")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tv-form", type=int, default=0, choices=[0, 1, 2, 3, 18, 20, 24],
                    help="with --kernel-case: FGP form (0 tuned/default, 1 stored r, 2 recomputed r, 3 two steps, "
                         "16 + rows two steps with that many rows per CTA)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--serve-requests", type=int, default=80, help="requests in the served / plain stream")
    ap.add_argument("--serve-no-plain", action="store_true", help="with --kernel-case serve: served stream only")
    ap.add_argument("--serve-rate", type=float, default=30.0,
                    help="Poisson arrivals per s of the served latency run (a load the server sustains)")
    ap.add_argument("--serve-inflight", type=int, default=SERVE_INFLIGHT, help="concurrent requests of the server")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving comparison")
    ap.add_argument("--no-bpm", action="store_true", help="skip the BPM gradient-inversion leg")
    ap.add_argument("--no-c4", action="store_true", help="skip the uneven-batch leg")
    args = ap.parse_args()
    if args.kernel_case == "serve":
        import qoraholo_b200 as qh
        from qoraholo_b200 import capi

        print(json.dumps(serving_leg(qh, capi, args.serve_requests, args.serve_rate, args.serve_inflight,
                                     plain=not args.serve_no_plain)))
        return 0
    if args.kernel_case == "c4":
        import torch

        import qoraholo_b200 as qh
        from qoraholo_b200 import capi

        print(json.dumps(c4_leg(qh, capi, torch)))
        return 0
    if args.kernel_case == "bpm":
        import torch

        import qoraholo_b200 as qh

        print(json.dumps(bpm_leg(qh, torch)))
        return 0
    if args.kernel_case:
        return kernel_case(args.kernel_case, args.reps, args.tv_form)
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(args.warmup, 3)

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import qoraholo_b200 as qh
    from qoraholo_b200 import capi

    illum, holo, bg = make_inputs()
    geom = qh.Geometry(wavelength=WAVELENGTH, n_medium=N_MEDIUM, na=NA, pixel=FIELD_PIXEL)
    stream = torch.cuda.current_stream().cuda_stream
    pipe = capi.Pipeline(COUNT, HOLO_N, (CARRIER_PX, CARRIER_PX), illum, geom_tuple(), radius=RADIUS,
                         output_size=FIELD_N, iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT,
                         tv_inner=TV_INNER)
    pipe.set_background(bg)
    d_holo = torch.from_numpy(holo).cuda()
    d_index = torch.empty(pipe.shape, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    for _ in range(args.warmup):
        pipe.process_device(d_holo.data_ptr(), d_index.data_ptr(), stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = capi.kernel_launches()
    pipe.time_prox(True)  # CUDA events around every TV proximal step of the timed runs (the roofline)
    with ClockSampler(physical_gpu_index(local)) as clocks:
        for s, e in events:
            flush.zero_()
            s.record()
            pipe.process_device(d_holo.data_ptr(), d_index.data_ptr(), stream)
            e.record()
        torch.cuda.synchronize()
    launches = capi.kernel_launches() - launches0
    prox_live = pipe.prox_time()  # (ms, FGP launches) of the proximal steps inside the timed runs
    pipe.time_prox(False)
    step_ms = [s.elapsed_time(e) for s, e in events]
    if dist:
        dist.barrier()
    max_ms, value = combine_ranks(sum(step_ms), args.steps, world, dist, "cuda")
    filled = pipe.filled_device(stream)  # also raises if a bounded device wait ran out
    ours = d_index.cpu().numpy() if rank == 0 else None  # the last timed step's volume

    # End to end through the public API: numpy holograms in, numpy volume out.
    api = qh.Pipeline(COUNT, HOLO_N, (CARRIER_PX, CARRIER_PX), illum, geom, radius=RADIUS, output_size=FIELD_N,
                      iterations=ITERATIONS, solver="tv", tv_weight=TV_WEIGHT, tv_inner=TV_INNER, upload_chunks=7)
    api.set_background(bg)
    for _ in range(2):
        ri = api.run(holo)
    torch.cuda.synchronize()
    e2e_steps = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ri = api.run(holo)
    _, per_call_value = combine_ranks(1000.0 * (time.perf_counter() - t0), e2e_steps, world, dist, "cuda")
    stage_ms = api.timings
    # The same steps as one stream of stacks (Pipeline.run_stream): every step's holograms still go
    # host -> device and its volume device -> host, but each transfer overlaps a neighbour's solve.
    stream_in = np.repeat(holo[None], e2e_steps, axis=0)
    api.run_stream(stream_in)  # untimed: pools the page-locked result buffer of this size
    t0 = time.perf_counter()
    rs = api.run_stream(stream_in)
    _, e2e_value = combine_ranks(1000.0 * (time.perf_counter() - t0), e2e_steps, world, dist, "cuda")
    stream_equals_run = bool(all(np.array_equal(rs[i], ri) for i in range(e2e_steps)))
    del rs, stream_in, api

    roof = fgp_roofline(torch, capi, stream, prox_live)

    bpm = None
    if rank == 0 and world == 1 and not args.no_bpm:
        try:
            bpm = bpm_leg(qh, torch)
        except Exception as e:  # noqa: BLE001
            bpm = {"error": f"{type(e).__name__}: {e}"}

    batching = None
    if rank == 0 and world == 1 and not args.no_c4:
        try:
            batching = c4_leg(qh, capi, torch)
        except Exception as e:  # noqa: BLE001
            batching = {"error": f"{type(e).__name__}: {e}"}

    served = None
    if rank == 0 and world == 1 and not args.no_serve:
        try:
            served = serving_leg(qh, capi, args.serve_requests, args.serve_rate, args.serve_inflight)
        except Exception as e:  # noqa: BLE001
            served = {"value": None, "error": f"{type(e).__name__}: {e}"}

    cpu = None
    parity = None
    ref_cuda = None
    if rank == 0 and world == 1:
        ref = None
        try:
            cpu, ref, ref_filled = cpu_baseline(holo, bg, illum)
            parity = parity_report(ours, filled, ref, ref_filled, holo, bg, illum)
        except Exception as e:  # noqa: BLE001
            cpu = cpu or {"value": None, "unit": UNIT, "cores": None, "kind": "reference", "sample": f"failed: {e}"}
            parity = {"error": f"{type(e).__name__}: {e}"}
        try:
            ref_cuda = reference_cuda_leg(holo, bg, illum, ref)
        except Exception as e:  # noqa: BLE001
            ref_cuda = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        lat = sorted(step_ms)
        p99 = percentile(lat, 0.99)
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(world),
            "latency_ms": {"p50": round(statistics.median(lat), 3), "p99": round(p99, 3), "path": "plain device pipeline"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "filled": filled,
            "stage_ms": {k: round(v, 3) for k, v in stage_ms.items()},
            "autotune": [ln for ln in capi.autotune_report().strip().splitlines() if "shape 256 " in ln],
            "bpm_gradient": bpm,
            "batching": batching,
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity": parity,
            "reference_cuda": ref_cuda,
            "rel_err_vs_reference_cpu": (parity or {}).get("rel_err_vs_reference_cpu"),
            "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(holo.nbytes),
                    "d2h_bytes_per_step": int(FIELD_N ** 3 * 4),
                    "path": (f"qoraholo_b200.Pipeline.run_stream over {e2e_steps} stacks (numpy in, numpy out; "
                             "each stack's upload and volume's download overlap a neighbour's solve), host wall clock"),
                    "per_call_value": round(per_call_value, 4),
                    "per_call_path": "qoraholo_b200.Pipeline.run per stack, synchronous, host wall clock",
                    "stream_equals_run": stream_equals_run},
            # The serving comparison comes last so that its figures survive a truncated line.
            "served": served,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
