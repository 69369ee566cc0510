"""Benchmark of the match_template search on B200.

Workload (the reference's metric configuration that fits one GPU): a
4096 x 4096 micrograph (80 Gaussian-atom particles, SNR 0.03, defocus
12,000 A, 300 kV, Cs 2.7 mm, A 0.07) searched with a 256^3 template at
1.0 A/px (120,000 atoms, 110 A radius) on the C1 grid of 2.5 deg
out-of-plane / 1.5 deg in-plane steps (1,595,420 orientations).  All inputs
are seeded synthetic data.  A step is one tm_run_plane call over a contiguous
chunk of that grid (successive steps take successive chunks).

metric: search points/s = original micrograph pixels x orientations / time.
value : device time (CUDA events on the library's stream) of K steps with
        prepared inputs resident in HBM.
e2e   : the same steps through the C ABI with host buffers: per step the
        prepared spectra and filter are copied host->device (pinned memory),
        the plane is searched, and MIP / best angles / sums / histogram are
        copied device->host and decoded; timed by the host clock.
accuracy_vs_fp64_oracle: after timing, the CPU-baseline leg searches a few
        orientations of the workload with the FP64 oracle as the checker and
        reports the MIP (relative) and z-score (absolute) errors.

--impl reference times the reference CPU algorithm (the FP32 build of the
oracle's restatement, all host threads) on a bounded sample of the same
workload; the reference itself cannot be built here (it needs wxWidgets and
FFTW).  With --gpus N > 1 every rank runs an independent replica (the search
has no data-path exchange on one micrograph) and the job value is the sum
over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "search points/s (original micrograph pixels x orientations)"
UNIT = "points/s"

WORKLOADS = {
    # the metric's configuration (default)
    "full": dict(name="4096x4096 micrograph, 256^3 template @1.0 A/px, C1 2.5/1.5 deg grid",
                 nx=4096, ny=4096, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=80,
                 snr=0.03, defocus=12000.0, angular_step=2.5, psi_step=1.5),
    # the CPU-runnable configuration
    "cpu1024": dict(name="1024x1024 micrograph, 64^3 template @1.5 A/px, C1 15/15 deg grid",
                    nx=1024, ny=1024, T=64, pixel_size=1.5, n_atoms=3000, radius_A=40.0, particles=10,
                    snr=0.05, defocus=12000.0, angular_step=15.0, psi_step=15.0),
    # the coarse search of the learned-proposal configuration
    "coarse": dict(name="4096x4096 micrograph, 256^3 template @1.0 A/px, C1 7.5/5.0 deg grid (coarse)",
                   nx=4096, ny=4096, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=80,
                   snr=0.03, defocus=12000.0, angular_step=7.5, psi_step=5.0),
    # the uneven micrograph sizes of the batched configuration, one at a time
    "uneven3710": dict(name="3838x3710 micrograph (padded 4096x3888), 256^3 template @1.0 A/px, C1 3.0/2.0 deg grid",
                       nx=3838, ny=3710, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=70,
                       snr=0.03, defocus=14000.0, angular_step=3.0, psi_step=2.0),
    "uneven5760": dict(name="5760x4092 micrograph (padded 5832x4096, rotated), 256^3 template @1.0 A/px, C1 3.0/2.0 deg grid",
                       nx=5760, ny=4092, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=110,
                       snr=0.03, defocus=10000.0, angular_step=3.0, psi_step=2.0),
    # the stress configuration's geometry (one micrograph, one plane)
    "stress384": dict(name="5760x4092 micrograph (padded 5832x4096, rotated), 384^3 template @0.8 A/px, C1 2.5/1.5 deg grid",
                      nx=5760, ny=4092, T=384, pixel_size=0.8, n_atoms=250000, radius_A=150.0, particles=40,
                      snr=0.03, defocus=12000.0, angular_step=2.5, psi_step=1.5),
    # a binned camera format: K3 at 2x (2880 x 2046, padded 2916 x 2048 and rotated)
    "binned2880": dict(name="2880x2046 micrograph (padded 2916x2048, rotated), 256^3 template @1.0 A/px, C1 3.0/2.0 deg grid",
                       nx=2880, ny=2046, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=30,
                       snr=0.03, defocus=12000.0, angular_step=3.0, psi_step=2.0),
    # a size without compiled kernels (2700 = 2^2 3^3 5^2, kept by the factorisation): the
    # run-time-length kernels
    "generic2700": dict(name="2700x2700 micrograph (run-time-length kernels), 256^3 template @1.0 A/px, C1 3.0/2.0 deg grid",
                        nx=2700, ny=2700, T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, particles=35,
                        snr=0.03, defocus=12000.0, angular_step=3.0, psi_step=2.0),
}
WORKLOAD = WORKLOADS["full"]


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def tensor_peaks():
    """Dense FP16/BF16 tensor throughput (TFLOP/s): burst (a kernel timed alone) and sustained."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops_sustained"]), float(p["bf16_tflops"])
    except Exception:
        return 1400.0, 1590.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(seed=20261204):
    """Synthetic micrograph and template, prepared as the reference's
    DoCalculation prepares them: size factorisation with edge-mean padding and
    the 90-degree rotation (match_template.cpp:520-596, C++ host library),
    whitening, template spectrum, CTF filter."""
    from cistem_downstream_bah_b200 import hostprep, prep, synthetic
    w = WORKLOAD
    vol = synthetic.template_volume(w["T"], w["pixel_size"], w["n_atoms"], w["radius_A"], seed=seed)
    mic, _ = synthetic.micrograph(w["ny"], w["nx"], w["pixel_size"], w["n_atoms"], w["radius_A"], w["particles"],
                                  w["snr"], w["defocus"], seed=seed + 1, atom_seed=seed)
    X = hostprep.factorize_dimension(w["nx"], w["T"])
    Y = hostprep.factorize_dimension(w["ny"], w["T"])
    if (X, Y) != (w["nx"], w["ny"]):
        mic = hostprep.clip_into(mic, X, Y, hostprep.edge_mean(mic))
    if not hostprep.lib().tmh_is_power_of_two(X) and hostprep.lib().tmh_is_power_of_two(Y):
        mic = hostprep.rotate90(mic, True)
        X, Y = Y, X
    ispec, curve = prep.whiten(mic)
    tspec = prep.template_spectrum(vol)
    filt = prep.projection_filter(w["T"], curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07,
                                  defocus1=w["defocus"], defocus2=w["defocus"], pixel_size=w["pixel_size"])
    grid = prep.search_grid(w["angular_step"])
    from cistem_downstream_bah_b200.core import orientation_list
    angles = orientation_list(grid, 0.0, w["psi_step"], 360.0)
    hmin, hstep = prep.histogram_scaled(X, Y)
    return dict(X=X, Y=Y, T=w["T"], ispec=ispec, tspec=tspec, filt=filt, angles=angles, hmin=hmin, hstep=hstep,
                mic=mic, vol=vol)


def preparation_ms(inp, device):
    """Wall time of the per-micrograph and per-pixel-plane preparation on the
    device (whitening of the padded micrograph; template spectrum at a
    pixel-size factor of 1 and 1.02), host buffers in and out."""
    from cistem_downstream_bah_b200 import core
    out = {}
    core.whiten_micrograph(inp["mic"], device=device)   # first call pays for module loading
    t = time.perf_counter()
    core.whiten_micrograph(inp["mic"], device=device)
    out["whiten"] = (time.perf_counter() - t) * 1e3
    for f in (1.0, 1.02):
        t = time.perf_counter()
        core.template_spectrum_device(inp["vol"], f, device=device)
        out["template_factor_%g" % f] = (time.perf_counter() - t) * 1e3
    return out


_PINNED = []


def pinned_copy(a):
    """numpy array in page-locked host memory (torch is used only as the allocator)."""
    import torch
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    _PINNED.append(t)
    out = t.numpy().view(a.dtype).reshape(a.shape)
    out[...] = a
    return out


def dist_init(args):
    from cistem_downstream_bah_b200 import distributed as D
    return D.init_from_env("nccl")


def barrier(world):
    from cistem_downstream_bah_b200 import distributed as D
    D.barrier(world)


def max_over_ranks(world, v):
    from cistem_downstream_bah_b200 import distributed as D
    return D.max_over_ranks(world, v)


BATCHED = dict(name="batched: 8 micrographs (3838x3710, 4096^2 x3, 5760x4092 x2, 2048^2 x2) x 13 defocus planes, "
                    "256^3 template @1.0 A/px, C1 3.0/2.0 deg grid",
               sizes=[(3838, 3710), (4096, 4096), (4096, 4096), (4096, 4096), (5760, 4092), (5760, 4092),
                      (2048, 2048), (2048, 2048)],
               T=256, pixel_size=1.0, n_atoms=120000, radius_A=110.0, snr=0.03, angular_step=3.0, psi_step=2.0,
               defocus_range=1200.0, defocus_step=200.0)


def run_batched(args, seed=20261210):
    """The batched configuration: every micrograph is prepared as the reference
    prepares it and searched over the 13 defocus planes; a step is one chunk of
    orientations on every plane of every micrograph (one context at a time)."""
    from cistem_downstream_bah_b200 import core, hostprep, prep, synthetic
    from cistem_downstream_bah_b200.core import orientation_list
    b = BATCHED
    world, rank, local = dist_init(args)
    rng = np.random.default_rng(seed)
    vol = synthetic.template_volume(b["T"], b["pixel_size"], b["n_atoms"], b["radius_A"], seed=seed)
    tspec = prep.template_spectrum(vol)
    angles = orientation_list(prep.search_grid(b["angular_step"]), 0.0, b["psi_step"], 360.0)
    per_plane = args.orientations_per_step // 8 or 32
    n_planes = 2 * int(round(b["defocus_range"] / b["defocus_step"])) + 1
    # host preparation of every micrograph (outside the timed regions)
    mics = []
    for k, (nx, ny) in enumerate(b["sizes"]):
        defocus = float(rng.uniform(8000.0, 20000.0))
        mic, _ = synthetic.micrograph(ny, nx, b["pixel_size"], b["n_atoms"], b["radius_A"], max(4, nx * ny // 200000),
                                      b["snr"], defocus, seed=seed + 1 + k, atom_seed=seed)
        X, Y = hostprep.factorize_dimension(nx, b["T"]), hostprep.factorize_dimension(ny, b["T"])
        if (X, Y) != (nx, ny):
            mic = hostprep.clip_into(mic, X, Y, hostprep.edge_mean(mic))
        if not hostprep.lib().tmh_is_power_of_two(X) and hostprep.lib().tmh_is_power_of_two(Y):
            mic = hostprep.rotate90(mic, True)
            X, Y = Y, X
        ispec, curve = hostprep.whiten(mic)
        filts = [prep.projection_filter(b["T"], curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=defocus,
                                        defocus2=defocus, pixel_size=b["pixel_size"],
                                        defocus_offset=(i - n_planes // 2) * b["defocus_step"]) for i in range(n_planes)]
        mics.append(dict(nx=nx, ny=ny, X=X, Y=Y, ispec=pinned_copy(ispec), filts=filts))
    # one search context per padded geometry, set up as a long-running service keeps it: template
    # uploaded, orientation batch autotuned, kernels warmed
    contexts = {}
    precisions = {}
    for m in mics:
        key = (m["X"], m["Y"])
        if key in contexts:
            continue
        hmin, hstep = prep.histogram_scaled(*key)
        sc = core.SearchCore(key[0], key[1], b["T"], histogram_min_scaled=hmin, histogram_step_scaled=hstep,
                             orientation_batch=args.batch, device=local)
        if args.precision == "fp16":
            try:
                sc.set_precision(core.PRECISION_FP16_TENSOR)
            except core.TmError:
                pass   # geometries without the FP16 kernels (5832-high) stay FP32
        precisions[key] = "f16" if sc.precision() == core.PRECISION_FP16_TENSOR else "f32"
        sc.set_template(tspec)
        sc.set_image(m["ispec"])
        if args.batch == 0:
            sc.autotune(m["filts"][n_planes // 2], angles[:256])
        for i in range(max(args.warmup, 1)):
            sc.run_plane(m["filts"][0], angles[:per_plane])
        contexts[key] = sc
    barrier(world)
    dev_ms, e2e_s, points, n_launch_batches = 0.0, 0.0, 0.0, 0
    with ClockSampler(local) as clk:
        for m in mics:
            sc = contexts[(m["X"], m["Y"])]
            t0 = time.perf_counter()
            sc.set_image(m["ispec"])
            sc.reset()
            for step in range(args.steps):
                chunk = angles[(step * per_plane) % len(angles):][:per_plane]
                for i in range(n_planes):
                    sc.run_plane(m["filts"][i], chunk, defocus_offset=(i - n_planes // 2) * b["defocus_step"])
                    dev_ms += sc.last_timing()["total_ms"]
                    points += m["nx"] * m["ny"] * len(chunk)
                    n_launch_batches += -(-len(chunk) // sc.orientation_batch())
            sc.results()
            e2e_s += time.perf_counter() - t0
    for sc in contexts.values():
        sc.close()
    dev_ms = max_over_ranks(world, dev_ms)
    e2e_s = max_over_ranks(world, e2e_s)
    if rank == 0:
        line = {"metric": METRIC, "value": world * points / (dev_ms * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "mixed",
                "data": "synthetic",
                "config": {"workload": b["name"], "orientations_per_plane_per_step": per_plane,
                           "precision_by_padded_geometry": {f"{k[0]}x{k[1]}": v for k, v in precisions.items()},
                           "defocus_planes": n_planes, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2"},
                "e2e": {"value": world * points / e2e_s, "unit": UNIT,
                        "note": "per micrograph: spectrum upload (pinned), every plane, results download and decode; "
                                "one context per padded geometry, set up before timing"},
                "gpu_launches": 6 * n_launch_batches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def _device_leg(sc, inp, args, world, local, chunk):
    """Device-resident timing of K steps (CUDA events on the library's stream)."""
    for i in range(args.warmup):
        sc.run_plane(inp["filt"], chunk(i))
    barrier(world)
    dev_ms = b_ms = c_ms = prep_ms = 0.0
    n_done = 0
    with ClockSampler(local) as clk:
        t_wall0 = time.perf_counter()
        for i in range(args.steps):
            ang = chunk(args.warmup + i)
            sc.run_plane(inp["filt"], ang)
            t = sc.last_timing()
            dev_ms += t["total_ms"]
            b_ms += t["pass_b_ms"]
            c_ms += t["pass_c_ms"]
            prep_ms += t["prep_ms"]
            n_done += len(ang)
        barrier(world)
        wall_ms = (time.perf_counter() - t_wall0) * 1e3   # the sampler's start and stop excluded
    return dict(dev_ms=max_over_ranks(world, dev_ms), b_ms=b_ms, c_ms=c_ms, prep_ms=prep_ms, n_done=n_done,
                clocks=clk.summary(), wall_ms=wall_ms)


def _e2e_leg(sc, inp, args, world, local, chunk, precision):
    """End to end through the C ABI with pinned host buffers.  As the reference
    drives one GPU from several host threads, each with its own
    TemplateMatchingCore, the steps go round-robin to --e2e-contexts host
    threads, each with its own context (stream): one thread's copies and result
    decoding overlap another's search."""
    from cistem_downstream_bah_b200 import core
    X, Y, T = inp["X"], inp["Y"], inp["T"]
    ispec_h, tspec_h, filt_h = pinned_copy(inp["ispec"]), pinned_copy(inp["tspec"]), pinned_copy(inp["filt"])
    n = X * Y
    L = sc.L
    ptr = core._ptr
    n_ctx = max(1, min(args.e2e_contexts, args.steps))
    # every host thread runs the same number of steps (the step count rounded up to a
    # multiple of the threads), so that no thread's last step runs without overlap
    n_steps = -(-args.steps // n_ctx) * n_ctx
    ctxs = [sc] + [core.SearchCore(X, Y, T, histogram_min_scaled=inp["hmin"], histogram_step_scaled=inp["hstep"],
                                   orientation_batch=sc.orientation_batch(), device=local) for _ in range(n_ctx - 1)]
    for c in ctxs[1:]:
        c.set_precision(precision)
    bufs = []
    for _ in ctxs:
        outs = {k: pinned_copy(np.zeros(n, np.float32)) for k in ("mip", "psi", "theta", "phi", "defocus", "pixel")}
        outs["sum"], outs["sumsq"] = pinned_copy(np.zeros(n, np.float64)), pinned_copy(np.zeros(n, np.float64))
        outs["hist"] = np.zeros(512, np.int64)
        bufs.append(outs)
    errors = []
    n_done = [0] * n_ctx

    def e2e_worker(k):
        try:
            c, outs = ctxs[k], bufs[k]
            for i in range(k, n_steps, n_ctx):
                ang = chunk(args.warmup + i)
                c._check(L.tm_set_image(c.h, ptr(ispec_h), X, Y))
                c._check(L.tm_set_template(c.h, ptr(tspec_h), T))
                c.reset()
                c.run_plane(filt_h, ang)
                c._check(L.tm_get_results(c.h, ptr(outs["mip"]), ptr(outs["psi"]), ptr(outs["theta"]),
                                          ptr(outs["phi"]), ptr(outs["defocus"]), ptr(outs["pixel"]),
                                          ptr(outs["sum"]), ptr(outs["sumsq"]), ptr(outs["hist"])))
                n_done[k] += len(ang)
        except Exception as e:   # re-raised below, after every thread has stopped
            errors.append(e)

    barrier(world)
    t0 = time.perf_counter()
    workers = [threading.Thread(target=e2e_worker, args=(k,)) for k in range(n_ctx)]
    for w_ in workers:
        w_.start()
    for w_ in workers:
        w_.join()
    barrier(world)
    e2e_s = max_over_ranks(world, time.perf_counter() - t0)
    if errors:
        raise errors[0]
    for c in ctxs[1:]:
        c.close()
    h2d = ispec_h.nbytes + tspec_h.nbytes + filt_h.nbytes + args.orientations_per_step * 12
    d2h = n * 4 + n * 4 + 2 * n * 8 + 512 * 8   # mip, best index, sum, sum of squares, histogram
    return dict(e2e_s=e2e_s, n_done=sum(n_done), h2d=h2d, d2h=d2h, host_threads=n_ctx)


# Issued tensor-core FLOPs of the FP16 form per launch (one orientation batch of nb):
# column pass, per item of 4 columns: stage H 2*128*256*16, stages F, 1, 2 three times
# two 128 x 128 x 128 MMAs; row pass, per block of R rows: stage 1 2*128*128*64 and
# R stage-2 MMAs 2*128*(2 N1)*max(16, N1), N1 = X / 128.
def tensor_flops_per_launch(X, Y, XP, nb):
    col = (XP // 4) * nb * (2 * 128 * 256 * 16 + 3 * 2 * 2 * 128 ** 3) if Y == 4096 else 0.0
    N1 = X // 128
    R = 64 // N1
    row = (Y // R) * nb * (2 * 128 * 128 * 64 + R * 2 * 128 * 2 * N1 * max(16, N1))
    return col, row


STRESS = dict(name="stress: 5760x4092 micrograph (padded 5832x4096, rotated), 384^3 template @0.8 A/px, "
                   "9 pixel-size planes (+-2 %, 0.5 % steps) x 21 defocus planes (+-1000 A, 100 A steps)",
              nx=5760, ny=4092, T=384, pixel_size=0.8, n_atoms=250000, radius_A=150.0, particles=40, snr=0.03,
              defocus=12000.0, angular_step=2.5, psi_step=1.5, pixel_range=0.02, pixel_step=0.005,
              defocus_range=1000.0, defocus_step=100.0)


def run_stress5(args, seed=20261220):
    """The stress configuration's plane loops on one micrograph: for each of the
    9 pixel-size planes the template spectrum is prepared on the device at that
    pixel size (ChangePixelSize, tm_set_template_volume), then the 21 defocus
    planes are searched over a chunk of the orientation grid; a step is one
    chunk over all 189 planes.  Timed end to end on the host clock (template
    preparation included); points = original pixels x orientations x planes."""
    from cistem_downstream_bah_b200 import core, hostprep, prep, synthetic
    from cistem_downstream_bah_b200.core import orientation_list
    w = STRESS
    world, rank, local = dist_init(args)
    vol = synthetic.template_volume(w["T"], w["pixel_size"], w["n_atoms"], w["radius_A"], seed=seed)
    mic, _ = synthetic.micrograph(w["ny"], w["nx"], w["pixel_size"], w["n_atoms"], w["radius_A"], w["particles"],
                                  w["snr"], w["defocus"], seed=seed + 1, atom_seed=seed)
    X, Y = hostprep.factorize_dimension(w["nx"], w["T"]), hostprep.factorize_dimension(w["ny"], w["T"])
    mic = hostprep.clip_into(mic, X, Y, hostprep.edge_mean(mic))
    if not hostprep.lib().tmh_is_power_of_two(X) and hostprep.lib().tmh_is_power_of_two(Y):
        mic = hostprep.rotate90(mic, True)
        X, Y = Y, X
    hmin, hstep = prep.histogram_scaled(X, Y)
    angles = orientation_list(prep.search_grid(w["angular_step"]), 0.0, w["psi_step"], 360.0)
    n_pix = 2 * int(round(w["pixel_range"] / w["pixel_step"])) + 1
    n_def = 2 * int(round(w["defocus_range"] / w["defocus_step"])) + 1
    per_plane = args.orientations_per_step // 16 or 32
    sc = core.SearchCore(X, Y, w["T"], histogram_min_scaled=hmin, histogram_step_scaled=hstep,
                         orientation_batch=args.batch, device=local)
    precision = "f32"
    if args.precision == "fp16":
        try:
            sc.set_precision(core.PRECISION_FP16_TENSOR)
            precision = "f16"
        except core.TmError:
            pass   # the 5832-high geometry has no FP16 kernels
    curve = sc.set_micrograph(mic)
    # the projection filters of the defocus planes (CTF x whitening curve)
    filts = [prep.projection_filter(w["T"], curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07,
                                    defocus1=w["defocus"], defocus2=w["defocus"], pixel_size=w["pixel_size"],
                                    defocus_offset=(i - n_def // 2) * w["defocus_step"]) for i in range(n_def)]
    factors = [1.0 + (j - n_pix // 2) * w["pixel_step"] for j in range(n_pix)]
    sc.set_template_volume(vol, 1.0)
    for _ in range(max(args.warmup, 1)):
        sc.run_plane(filts[0], angles[:per_plane])
    barrier(world)
    points = 0.0
    dev_ms = 0.0
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for step in range(args.steps):
            chunk = angles[(step * per_plane) % len(angles):][:per_plane]
            sc.reset()
            for j, f in enumerate(factors):
                sc.set_template_volume(vol, f)
                for i in range(n_def):
                    sc.run_plane(filts[i], chunk, defocus_offset=(i - n_def // 2) * w["defocus_step"],
                                 pixel_size_offset=(j - n_pix // 2) * w["pixel_step"] * w["pixel_size"])
                    dev_ms += sc.last_timing()["total_ms"]
                    points += w["nx"] * w["ny"] * len(chunk)
            sc.results()
        el = time.perf_counter() - t0
    sc.close()
    el = max_over_ranks(world, el)
    dev_ms = max_over_ranks(world, dev_ms)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": world * points / el, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": precision, "data": "synthetic",
            "config": {"workload": w["name"], "padded": [X, Y], "orientations_per_plane_per_step": per_plane,
                       "pixel_size_planes": n_pix, "defocus_planes": n_def, "l2": "inputs larger than L2"},
            "search_points_per_s_device": world * points / (dev_ms * 1e-3),
            "e2e": {"value": world * points / el, "unit": UNIT, "h2d_bytes_per_step": int(vol.nbytes * n_pix),
                    "d2h_bytes_per_step": int(24 * X * Y),
                    "note": "host clock: per pixel plane the template volume upload and preparation, every plane's "
                            "search, the results download"},
            "gpu_launches": None, "clocks": clk.summary()}), flush=True)


def run_ours(args):
    world, rank, local = dist_init(args)
    from cistem_downstream_bah_b200 import core
    inp = make_inputs()
    X, Y, T = inp["X"], inp["Y"], inp["T"]
    per_step = args.orientations_per_step
    n_orient_total = len(inp["angles"])
    npix_orig = WORKLOAD["nx"] * WORKLOAD["ny"]
    N = X * Y

    def chunk(i):
        a = (i * per_step) % n_orient_total
        return inp["angles"][a:a + per_step]

    def make_context(precision):
        sc = core.SearchCore(X, Y, T, histogram_min_scaled=inp["hmin"], histogram_step_scaled=inp["hstep"],
                             orientation_batch=args.batch, device=local)
        sc.set_precision(precision)
        sc.set_template(inp["tspec"])
        sc.set_image(inp["ispec"])
        if args.batch == 0:
            # the library's autotuner picks the orientations per device pass
            sc.autotune(inp["filt"], inp["angles"][:256])
        return sc

    # ---- the FP32 parity path: device-resident timing, then end to end
    precision = core.PRECISION_FP16_TENSOR if args.precision == "fp16" else core.PRECISION_FP32
    sc = make_context(precision)
    nb = sc.orientation_batch()
    dev = _device_leg(sc, inp, args, world, local, chunk)
    value = world * npix_orig * dev["n_done"] / (dev["dev_ms"] * 1e-3)
    e2e = _e2e_leg(sc, inp, args, world, local, chunk, precision)

    # ---- roofline for the dominant kernel (per launch = one orientation batch)
    hbm_peak, peak_kind = peaks()
    n_launch = dev["n_done"] / nb
    b_launch_ms = dev["b_ms"] / max(n_launch, 1)
    c_launch_ms = dev["c_ms"] / max(n_launch, 1)
    # algorithmic bytes per point: pass B reads the half spectrum (4 B) and
    # writes the intermediate (4 B); pass C reads the intermediate (4 B)
    # the column pass of 4096-high micrographs with 256^3 templates is the residue-grouped kernel
    b_name = "k_pass_b_rg" if (Y, T) == (4096, 256) else "k_pass_b"
    dominant = b_name if dev["b_ms"] >= dev["c_ms"] else "k_pass_c"
    alg_b = 8.0 * N * nb
    alg_c = 4.0 * N * nb
    # DRAM bytes per launch measured by ncu on this workload (dram__bytes_read.sum +
    # dram__bytes_write.sum); they apply to the default workload and its batches only
    prof = PROFILED_TRAFFIC.get(nb) if (X, Y, T) == (4096, 4096, 256) and precision == core.PRECISION_FP32 else None
    if dominant == b_name:
        ach = alg_b / (b_launch_ms * 1e-3) / 1e9
        traffic = args.traffic_b if args.traffic_b is not None else (prof["k_pass_b"] if prof else None)
    else:
        ach = alg_c / (c_launch_ms * 1e-3) / 1e9
        traffic = args.traffic_c if args.traffic_c is not None else (prof["k_pass_c"] if prof else None)
    # both search passes against the same HBM peak (the row pass is bound by its FP32
    # issue rather than by HBM, so its fraction is low at any speed)
    by_kernel = {}
    for name, alg, ms, tr in ((b_name, alg_b, b_launch_ms, args.traffic_b if args.traffic_b is not None else
                               (prof["k_pass_b"] if prof else None)),
                              ("k_pass_c", alg_c, c_launch_ms, args.traffic_c if args.traffic_c is not None else
                               (prof["k_pass_c"] if prof else None))):
        gbs = alg / (max(ms, 1e-9) * 1e-3) / 1e9
        by_kernel[name] = {"achieved": gbs, "frac": gbs / hbm_peak, "ms_per_launch": ms,
                           "algorithmic_bytes_per_launch": alg, "traffic": tr}

    # ---- the FP16 tensor-core form on the same workload and orientation chunks
    fp16 = None
    if precision == core.PRECISION_FP32 and not args.no_fp16_leg:
        try:
            sc16 = make_context(core.PRECISION_FP16_TENSOR)
        except core.TmError as e:
            sc16 = None
            fp16 = {"unavailable": str(e)}
        if sc16 is not None:
            nb16 = sc16.orientation_batch()
            d16 = _device_leg(sc16, inp, args, world, local, chunk)
            v16 = world * npix_orig * d16["n_done"] / (d16["dev_ms"] * 1e-3)
            e16 = _e2e_leg(sc16, inp, args, world, local, chunk, core.PRECISION_FP16_TENSOR)
            nl16 = d16["n_done"] / nb16
            b16 = d16["b_ms"] / max(nl16, 1)
            c16 = d16["c_ms"] / max(nl16, 1)
            XP = -(-(X // 2 + 1) // 4) * 4      # row pitch: 4-column chunks of the column pass
            fl_b, fl_c = tensor_flops_per_launch(X, Y, XP, nb16)
            _, tflops_peak = tensor_peaks()
            fp16 = {
                "value": v16, "unit": UNIT, "ratio_to_fp32_value": v16 / value,
                "ms_per_step": d16["dev_ms"] / args.steps, "orientation_batch": nb16,
                "e2e": {"value": world * npix_orig * e16["n_done"] / e16["e2e_s"], "unit": UNIT,
                        "h2d_bytes_per_step": int(e16["h2d"]), "d2h_bytes_per_step": int(e16["d2h"]),
                        "host_threads": e16["host_threads"]},
                "ms_per_launch": {"k_pass_b_tc": b16, "k_pass_c_tc": c16,
                                  "prep_kernels": d16["prep_ms"] / max(nl16, 1)},
                # algorithmic bytes per point in FP16 storage: pass B 4 B (half spectrum read
                # and intermediate write), pass C 2 B (intermediate read)
                "roofline": {"bound": "tensor", "kernel": "k_pass_b_tc" if b16 >= c16 else "k_pass_c_tc",
                             "achieved": (fl_b / (b16 * 1e-3) if b16 >= c16 else fl_c / (c16 * 1e-3)) / 1e12,
                             "peak": tflops_peak, "unit": "TFLOP/s",
                             "frac": (fl_b / (b16 * 1e-3) if b16 >= c16 else fl_c / (c16 * 1e-3)) / 1e12 / tflops_peak,
                             "traffic": None, "peak_source": peak_kind,
                             "hbm_achieved_gbs": {"k_pass_b_tc": 4.0 * N * nb16 / (b16 * 1e-3) / 1e9,
                                                  "k_pass_c_tc": 2.0 * N * nb16 / (c16 * 1e-3) / 1e9},
                             "note": "issued DFT-matrix MMA FLOPs per launch (FP16 operands, FP32 accumulate)"},
                "clocks": d16["clocks"],
            }
            if rank == 0 and world == 1 and args.accuracy > 0:
                fp16["accuracy_vs_fp64_oracle"] = accuracy_vs_fp64(sc16, inp, args.accuracy)
            sc16.close()

    # ---- the fast form on the same workload: coarse search (FP16 where it has kernels), network,
    # window search of the proposed tiles; the FP32 exhaustive search of the whole fine grid is the
    # judge of its recall (about three minutes)
    fast = None
    if args.workload == "full" and not args.no_fast_form and world == 1:
        pl = proposal_leg(args, inp, world, rank, local,
                          coarse_fp16=fp16 is not None and "unavailable" not in fp16)
        pr = pl["proposal"]
        rc = pr["recall"]
        fast = {"value": pl["value"], "unit": UNIT, "dtype": pl["dtype"],
                "speedup_vs_exhaustive_fp32": pr["speedup_vs_exhaustive"],
                "ratio_to_fp32_value": pl["value"] / value,
                "seconds": pl["ms_per_step"] / 1e3, "exhaustive_fp32_seconds": pr["exhaustive_s"],
                "recall_all_z7_peaks": rc["min_radius_T8"]["network_recall_z"],
                "recall_all_z7_peaks_mip": rc["min_radius_T8"]["network_recall_mip"],
                "recall_above_expected_threshold": rc["min_radius_T8"]["network_recall_above_expected_threshold"],
                "expected_threshold": rc["expected_threshold"], "z7_peaks": rc["min_radius_T8"]["z7_peaks"],
                "mip_max_rel_err_same_orientation": pr["mip_max_rel_err_same_orientation"],
                "without_network_same_tiles": pr["without_network_same_tiles"],
                "stages_s": {"coarse": pr["coarse_s"], "network": pr["network_s"], "windows": pr["windows_s"]},
                "note": "effective rate = points of the exhaustive fine search / time of the proposal path "
                        "(host buffers, synchronous calls); recall judged on the FP32 exhaustive search"}

    # the CPU-baseline leg (rank 0, N=1): the oracle timed on the host cores,
    # then the FP64 oracle as the checker of a few orientations after timing
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    cpu = cpu_baseline(inp, sample=args.cpu_sample) if cpu_leg else None
    acc = accuracy_vs_fp64(sc, inp, args.accuracy) if (rank == 0 and world == 1 and args.accuracy > 0) else None
    prep_dev = preparation_ms(inp, local) if rank == 0 else None
    sc.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev["dev_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if precision == core.PRECISION_FP32 else "f16",
            "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "micrograph": [WORKLOAD["nx"], WORKLOAD["ny"]],
                       "padded": [X, Y], "template": T, "orientations_per_step": per_step,
                       "grid_orientations": n_orient_total, "orientation_batch": nb,
                       "orientation_batch_autotuned": args.batch == 0,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2: each batch writes a %.1f GB intermediate" % (nb * Y * (X // 2 + 4) * 8 / 1e9)},
            "e2e": {"value": world * npix_orig * e2e["n_done"] / e2e["e2e_s"], "unit": UNIT,
                    "h2d_bytes_per_step": int(e2e["h2d"]), "d2h_bytes_per_step": int(e2e["d2h"]),
                    "host_threads": e2e["host_threads"]},
            "gpu_launches": int(6 * np.ceil(per_step / nb) * args.steps),
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                         "frac": ach / hbm_peak, "traffic": traffic, "peak_source": peak_kind,
                         "ms_per_launch": {b_name: b_launch_ms, "k_pass_c": c_launch_ms,
                                           "prep_kernels": dev["prep_ms"] / max(n_launch, 1)},
                         "by_kernel": by_kernel},
            "clocks": dev["clocks"],
            "wall_ms_timed_region": dev["wall_ms"],
        }
        if fp16 is not None:
            line["fp16"] = fp16
        if fast is not None:
            line["fast_form"] = fast
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if acc is not None:
            line["accuracy_vs_fp64_oracle"] = acc
        if prep_dev is not None:
            line["preparation_ms_on_device"] = prep_dev
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ncu dram__bytes_read.sum + dram__bytes_write.sum per launch at 4096^2 / 256^3, by orientation
# batch, of the column pass (k_pass_b_rg) and the row pass (k_pass_c)
PROFILED_TRAFFIC = {
    32: {"k_pass_b": 0.207e9 + 2.101e9, "k_pass_c": 2.555e9 + 0.382e9},
    128: {"k_pass_b": 0.620e9 + 8.556e9, "k_pass_c": 9.012e9 + 0.392e9},
}


def accuracy_vs_fp64(sc, inp, k):
    """MIP and z-score error of the search against the FP64 oracle on k
    orientations spread over the grid (same prepared inputs on both sides)."""
    from oracle import oracle as O
    n = len(inp["angles"])
    ang = inp["angles"][np.linspace(0, n - 1, k).astype(np.int64)]
    sc.reset()
    sc.run_plane(inp["filt"], ang)
    r = sc.results()
    st = O.SearchState(inp["X"], inp["Y"])
    O.search(st, inp["tspec"].astype(np.complex128), inp["ispec"].astype(np.complex128), inp["filt"], ang,
             hist_min_scaled=inp["hmin"], hist_step_scaled=inp["hstep"], bits=64)
    sq = float(np.sqrt(float(inp["X"] * inp["Y"])))
    mip_ref, z_ref, _, _ = O.finalize(st, k, sq)
    gpu = O.SearchState(inp["X"], inp["Y"])
    gpu.mip[:], gpu.sum[:], gpu.sumsq[:] = r["mip"], r["sum"], r["sumsq"]
    mip_got, z_got, _, _ = O.finalize(gpu, k, sq)
    scale = float(np.abs(mip_ref).max())
    from cistem_downstream_bah_b200 import core
    form = "FP16 tensor-core" if sc.precision() == core.PRECISION_FP16_TENSOR else "FP32"
    return {"orientations": int(k),
            "mip_max_rel_err": float(np.abs(mip_got - mip_ref).max() / scale),
            "z_max_abs_err": float(np.abs(z_got - z_ref).max()),
            "note": f"{form} search vs FP64 oracle, MIP error relative to the MIP scale; z over these "
                    f"{int(k)} orientations only"}


def _oracle_sample(inp, n_orient, threads):
    """Seconds of the timed CPU baseline (oracle/cpu_port.py: the reference's CPU
    loop in FP32 with pocketfft transforms) over the first n_orient orientations
    on `threads` host threads."""
    from oracle import cpu_port
    t0 = time.perf_counter()
    cpu_port.search(inp["tspec"], inp["ispec"], inp["filt"], inp["angles"][:n_orient], inp["X"], inp["Y"],
                    hist_min_scaled=inp["hmin"], hist_step_scaled=inp["hstep"], threads=threads)
    return time.perf_counter() - t0


def run_refine(args, seed=20261215):
    """refine_template's TemplateScore on the GPU: batches of candidates (one
    per refined peak, as the program's workers hand them over) on a 256^3
    template, a quarter of them with a pixel-size change.  metric: scored
    candidates per second of tm_refine_score calls (synchronous: candidate
    upload, scoring and the scores back on the host)."""
    world, rank, local = dist_init(args)
    from cistem_downstream_bah_b200 import core, hostprep, synthetic
    T, nb, n_part = 256, args.refine_batch, 64
    vol = synthetic.template_volume(T, 1.0, 120000, 110.0, seed=seed)
    mic, truth = synthetic.micrograph(1024, 1024, 1.0, 120000, 110.0, 4, 0.05, 12000.0, seed=seed + 1, atom_seed=seed)
    white = hostprep.refine_whiten(mic)
    tspec = hostprep.padded_template_spectrum(vol, T)
    rng = np.random.default_rng(seed)
    rc = core.RefineCore(tspec, T, max_batch=nb, max_particles=n_part, max_filters=8, max_operators=4, device=local)
    for k in range(n_part):
        w = hostprep.window_particle(white, int(rng.integers(-300, 300)), int(rng.integers(-300, 300)), T)
        sp = np.fft.rfft2(w.astype(np.float64)) / (T * T)
        sp *= np.where((np.arange(T)[:, None] + np.arange(T // 2 + 1)[None, :]) % 2 == 0, 1.0, -1.0)
        rc.set_particle(k, sp)
    from cistem_downstream_bah_b200 import prep
    _, curve = prep.whiten(mic)
    for k in range(8):
        rc.set_filter(k, prep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07,
                                                defocus1=11800.0 + 50.0 * k, defocus2=11800.0 + 50.0 * k,
                                                pixel_size=1.0))
    for k, f in enumerate((0.98, 0.99, 1.01, 1.02)):
        info, ar, ai, brt, bit = hostprep.pixel_size_operator(T, T, f)
        rc.set_operator(k, ar, ai, brt, bit, info["has_pad_value"])

    def batch(i):
        r = np.random.default_rng(seed + i)
        e = np.stack([r.uniform(0, 360, nb), r.uniform(0, 180, nb), r.uniform(0, 360, nb)], 1).astype(np.float32)
        op = np.where(r.uniform(size=nb) < 0.25, r.integers(0, 4, nb), -1)
        return e, r.integers(0, n_part, nb), r.integers(0, 8, nb), op

    batches = [batch(i) for i in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        rc.score(*batches[i])
    barrier(world)
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            rc.score(*batches[args.warmup + i])
        el = time.perf_counter() - t0
    el = max_over_ranks(world, el)
    rc.close()
    if rank == 0:
        rate = nb * args.steps * world / el
        print(json.dumps({
            "metric": "refine_template TemplateScore candidates/s", "value": rate, "unit": "candidates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"refine: {nb} candidates per batch (one per peak), 256^3 template, 256x256 "
                                   "windows of a 1024^2 micrograph, 1/4 with a pixel-size change",
                       "flush_l2": "inputs > L2 not needed: each batch reads its own candidates"},
            "e2e": {"value": rate, "unit": "candidates/s", "h2d_bytes_per_step": nb * 6 * 4,
                    "d2h_bytes_per_step": nb * 3 * 4},
            "gpu_launches": args.steps * 11, "clocks": clk.summary()}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


PROPOSAL_WEIGHTS = os.path.join(ROOT, "cistem_downstream_bah_b200", "data", "proposal_net.npz")


def proposal_leg(args, inp, world, rank, local, coarse_fp16=False):
    """The learned proposal on the metric's configuration (4096^2, 256^3,
    fine grid 2.5 / 1.5 deg): coarse search (7.5 / 5 deg) -> network over the
    64 x 64 tiles -> window search of the proposed tiles over the fine
    orientations of their 16 angular bins.  The exhaustive fine search runs
    after it; recall is measured on its z >= 7 peaks.  value = the exhaustive
    search's points / the proposal path's time (host buffers in and out,
    synchronous calls); the same for the method without the network
    (thresholded coarse z, bins around the coarse best direction)."""
    from cistem_downstream_bah_b200 import core, hostprep
    from cistem_downstream_bah_b200 import proposal as PR
    w = np.load(args.proposal_weights)
    params = w["params"]
    net_thr = float(w["network_logit_threshold"])
    heur_thr = float(w["heuristic_z_threshold"])
    X, Y, T = inp["X"], inp["Y"], inp["T"]
    angular = PR.AngularBins(7.5, WORKLOAD["angular_step"], WORKLOAD["psi_step"])
    coarse_angles = core.orientation_list(hostprep.search_grid(7.5), 0.0, 5.0, 360.0)
    sc = core.SearchCore(X, Y, T, histogram_min_scaled=inp["hmin"], histogram_step_scaled=inp["hstep"], device=local)
    sc.set_image(inp["ispec"])
    sc.set_template(inp["tspec"])
    # the exhaustive judge runs on this context in FP32; the coarse search optionally in FP16
    sc16 = None
    if coarse_fp16:
        sc16 = core.SearchCore(X, Y, T, histogram_min_scaled=inp["hmin"], histogram_step_scaled=inp["hstep"],
                               device=local)
        sc16.set_precision(core.PRECISION_FP16_TENSOR)
        sc16.set_image(inp["ispec"])
        sc16.set_template(inp["tspec"])
    sc_coarse = sc16 if sc16 is not None else sc
    net = PR.ProposalNet(PR.FEATURES, PR.TILE, max_batch=256, device=local)
    net.set_params(params)
    ws = PR.WindowSearch(inp["ispec"], X, Y, T, inp["tspec"], inp["filt"], angular, inp["hmin"], inp["hstep"],
                         device=local)
    # warm-up: kernels of both geometries, the network
    for _ in range(max(args.warmup, 1)):
        PR.search_maps(sc_coarse, inp["filt"], coarse_angles[:256], X, Y)
        ws.run(PR.Proposal([0], [angular.nearest([0.0, 0.0, 1.0], 1)], None))
        net.forward(np.zeros((4, PR.FEATURES, PR.TILE, PR.TILE), np.float32))
    barrier(world)
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        coarse = PR.search_maps(sc_coarse, inp["filt"], coarse_angles, X, Y)
        t1 = time.perf_counter()
        frames = PR.tile_frames(coarse["z"], coarse["theta"], coarse["phi"])
        feats = PR.tile_features(coarse["z"], coarse["theta"], coarse["phi"], frames=frames)
        out = net.forward(feats)
        prop = PR.propose_network(net, feats, frames, net_thr, angular, out=out)
        if len(prop.tiles) > args.proposal_max_tiles:   # bound the run: keep the best-scored tiles
            keep = np.sort(np.argsort(-out[prop.tiles, 0], kind="stable")[:args.proposal_max_tiles])
            prop = PR.Proposal(prop.tiles[keep], [prop.bins[i] for i in keep], prop.scores)
        t2 = time.perf_counter()
        res = ws.run(prop)
        t3 = time.perf_counter()
    t_prop = t3 - t0
    # this library's kernels in the timed path: 6 per orientation batch of the coarse search (its
    # results reset: 1), 9 per network forward call, and the window search's own count
    n_launch_coarse = 1 + 6 * -(-len(coarse_angles) // sc.orientation_batch())
    n_launch_net = 9 * -(-len(feats) // 256)
    # the method without the network at the network's tile budget (timed the same way)
    t4 = time.perf_counter()
    top = PR.propose_top_tiles(coarse, len(prop.tiles), angular)
    res_t = ws.run(top)
    t_top = (t1 - t0) + (time.perf_counter() - t4)
    # ... and with its own threshold (recall from the proposed bins; not searched)
    heur = PR.propose_heuristic(coarse, heur_thr, angular)
    exh = PR.search_maps(sc, inp["filt"], angular.fine_angles, X, Y)
    peak_sets = {"min_radius_T8": PR.find_peaks(exh, 7.0, T, WORKLOAD["pixel_size"]),
                 "min_radius_particle": PR.find_peaks(exh, 7.0, T, WORKLOAD["pixel_size"],
                                                      min_peak_radius=int(WORKLOAD["radius_A"] / WORKLOAD["pixel_size"]))}
    # the reference's expected threshold for this search (one false positive: sqrt(2) erfcinv(2 / N),
    # match_template.cpp:1282): z >= 7 peaks below it are chance maxima of the exhaustive search
    thr_ref = float(np.sqrt(2.0) * hostprep.lib().tmh_erfcinv(2.0 / (float(X) * Y * len(angular.fine_angles))))
    recalls, diags = {"expected_threshold": thr_ref}, {}
    for key, pk in peak_sets.items():
        rn = PR.recall(pk, exh, res, PR.proposal_z(res, coarse, X, Y), 7.0)
        rt = PR.recall(pk, exh, res_t, PR.proposal_z(res_t, coarse, X, Y), 7.0)
        allnet = PR.propose_network(net, feats, frames, -np.inf, angular, out=out)
        alltop = PR.propose_heuristic(coarse, -np.inf, angular)
        dg = PR.peak_diagnostics(pk, exh, coarse, {"network": prop, "top_tiles": top, "threshold": heur,
                                                   "network_all": allnet, "coarse_all": alltop}, angular)
        diags[key] = dg
        ptiles = [(int(p[1]) // PR.TILE) * PR.tile_grid(X, Y)[1] + int(p[0]) // PR.TILE for p in pk]
        curves = {"network": PR.tiles_for_recall(ptiles, dg["network_all_recovered"],
                                                 np.argsort(-out[:, 0], kind="stable")),
                  "coarse_z": PR.tiles_for_recall(ptiles, dg["coarse_all_recovered"],
                                                  np.argsort(-PR.tile_max(coarse["z"])[0], kind="stable"))}
        recalls[key] = {"z7_peaks": int(len(pk)), "network_recall_mip": rn[0], "network_recall_z": rn[1],
                        "top_tiles_recall_mip": rt[0], "top_tiles_recall_z": rt[1],
                        "threshold_recall_mip_from_bins": float(np.mean(dg["threshold_recovered"])) if len(pk) else 1.0,
                        "network_missed_tile_not_selected": int(np.sum(~dg["network_selected"])),
                        "network_missed_bin_not_proposed": int(np.sum(dg["network_selected"] & (dg["network_bin_rank"] < 0))),
                        "bin_outside_16_nearest_at_peak": int(np.sum(dg["bin_rank_at_peak_coarse_direction"] >= 16)),
                        "peaks_above_expected_threshold": int(np.sum(dg["z"] >= thr_ref)) if len(pk) else 0,
                        "network_recall_above_expected_threshold":
                            float(np.mean(dg["network_recovered"][dg["z"] >= thr_ref])) if np.any(dg["z"] >= thr_ref) else 1.0,
                        "top_tiles_recall_above_expected_threshold":
                            float(np.mean(dg["top_tiles_recovered"][dg["z"] >= thr_ref])) if np.any(dg["z"] >= thr_ref) else 1.0,
                        "tiles_for_recall": curves}
    # MIP error where the window search found the exhaustive search's best orientation
    same = np.isfinite(res["mip"]) & (res["psi"] == exh["psi"]) & (res["theta"] == exh["theta"]) & (res["phi"] == exh["phi"])
    mip_err = float(np.max(np.abs(res["mip"][same] - exh["mip"][same]) / np.maximum(np.abs(exh["mip"][same]), 1e-30))) \
        if same.any() else None
    if args.proposal_diag:
        flat = {f"{k}:{n}": v for k, d in diags.items() for n, v in d.items()}
        np.savez(args.proposal_diag, **flat)
    ws.close()
    net.close()
    sc.close()
    if sc16 is not None:
        sc16.close()
    pts_exh = exh["points"]
    line = {
            "metric": METRIC, "value": pts_exh / t_prop, "unit": UNIT, "n_gpus": world, "steps": 1,
            "warmup": args.warmup, "ms_per_step": t_prop * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("f16 tensor-core coarse search, " if sc16 is not None else "f32 coarse search, ") +
                     "f32 window search and exhaustive judge, bf16 network weights", "data": "synthetic",
            "config": {"workload": "learned proposal: " + WORKLOAD["name"] + ", coarse 7.5/5.0 deg, 16 bins per tile",
                       "flush_l2": "inputs > L2"},
            "e2e": {"value": pts_exh / t_prop, "unit": UNIT, "h2d_bytes_per_step": int(inp["ispec"].nbytes),
                    "d2h_bytes_per_step": int(6 * 4 * X * Y)},
            "proposal": {
                "exhaustive_points_per_s": pts_exh / exh["seconds"], "exhaustive_s": exh["seconds"],
                "speedup_vs_exhaustive": exh["seconds"] / t_prop,
                "coarse_s": t1 - t0, "network_s": t2 - t1, "windows_s": t3 - t2, "windows": res["windows"],
                "tiles": int(len(prop.tiles)), "tiles_total": int(len(feats)),
                "fine_points": res["points"], "exhaustive_points": pts_exh, "recall": recalls,
                "mip_max_rel_err_same_orientation": mip_err,
                "without_network_same_tiles": {"tiles": int(len(top.tiles)), "windows": res_t["windows"], "s": t_top,
                                               "speedup_vs_exhaustive": exh["seconds"] / t_top},
                "without_network_threshold": {"tiles": int(len(heur.tiles)), "z_threshold": heur_thr},
                "network_logit_threshold": net_thr},
            "gpu_launches": n_launch_coarse + n_launch_net + res["launches"], "clocks": clk.summary()}
    return line



def run_recall16(args):
    """The FP16 tensor-core form as the fast exhaustive search: the metric's
    configuration searched over the whole 2.5 / 1.5 deg grid (1,595,420
    orientations) once in FP32 (the parity path, the judge) and once in FP16.
    Reported: both rates, their ratio, the MIP error of the FP16 search against
    the FP32 one, and the recall of the FP32 search's z >= 7 peaks (the
    reference's result-aggregation loop): a peak is recovered when the FP16 z
    map reaches 7 within 1 px, or (strict) when the FP16 peak list has a peak
    within 2 px."""
    from cistem_downstream_bah_b200 import core
    from cistem_downstream_bah_b200 import proposal as PR
    world, rank, local = dist_init(args)
    inp = make_inputs()
    X, Y, T = inp["X"], inp["Y"], inp["T"]
    angles = inp["angles"] if args.recall_orientations <= 0 else inp["angles"][:args.recall_orientations]
    out = {}
    for name, prec in (("fp32", core.PRECISION_FP32), ("fp16", core.PRECISION_FP16_TENSOR)):
        sc = core.SearchCore(X, Y, T, histogram_min_scaled=inp["hmin"], histogram_step_scaled=inp["hstep"], device=local)
        sc.set_precision(prec)
        sc.set_template(inp["tspec"])
        sc.set_image(inp["ispec"])
        sc.autotune(inp["filt"], inp["angles"][:256])
        PR.search_maps(sc, inp["filt"], angles[:512], X, Y)    # warm-up
        with ClockSampler(local) as clk:
            out[name] = PR.search_maps(sc, inp["filt"], angles, X, Y)
        out[name]["clocks"] = clk.summary()
        out[name]["batch"] = sc.orientation_batch()
        sc.close()
    e, f = out["fp32"], out["fp16"]
    pk32 = PR.find_peaks(e, 7.0, T, WORKLOAD["pixel_size"])
    pk16 = PR.find_peaks(f, 7.0, T, WORKLOAD["pixel_size"])
    hit_z = hit_list = 0
    dz = []
    for x, y, z, *_ in pk32:
        x, y = int(x), int(y)
        win = f["z"][max(0, y - 1):y + 2, max(0, x - 1):x + 2]
        hit_z += float(win.max()) >= 7.0
        dz.append(float(f["z"][y, x]) - float(z))
        if len(pk16):
            hit_list += float(np.min(np.hypot(pk16[:, 0] - x, pk16[:, 1] - y))) <= 2.0
    n = max(len(pk32), 1)
    npix_orig = WORKLOAD["nx"] * WORKLOAD["ny"]
    v32 = npix_orig * len(angles) / e["seconds"]
    v16 = npix_orig * len(angles) / f["seconds"]
    scale = float(np.abs(e["mip"]).max())
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": v16, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": f["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16 tensor-core transforms, f32 MIP, f64 sums", "data": "synthetic",
            "config": {"workload": "exhaustive search, FP16 tensor-core form against the FP32 path: " + WORKLOAD["name"],
                       "orientations": int(len(angles)), "orientation_batch": {"fp32": e["batch"], "fp16": f["batch"]}},
            "e2e": {"value": v16, "unit": UNIT, "h2d_bytes_per_step": int(inp["ispec"].nbytes + inp["tspec"].nbytes),
                    "d2h_bytes_per_step": int(24 * X * Y),
                    "note": "each search: one tm_run_plane over the whole grid and the results to the host"},
            "fp32_value": v32, "ratio_fp16_to_fp32": v16 / v32,
            "fp32_seconds": e["seconds"], "fp16_seconds": f["seconds"],
            "mip_max_rel_err_fp16_vs_fp32": float(np.abs(f["mip"] - e["mip"]).max() / scale),
            "z_peaks_fp32": int(len(pk32)), "z_peaks_fp16": int(len(pk16)),
            "recall_z7_within_1px": hit_z / n, "recall_z7_peak_list_within_2px": hit_list / n,
            "z_diff_at_fp32_peaks": {"min": float(min(dz)) if dz else None, "max": float(max(dz)) if dz else None},
            "gpu_launches": None, "clocks": {"fp32": e["clocks"], "fp16": f["clocks"]}}), flush=True)


def run_proposal(args):
    world, rank, local = dist_init(args)
    line = proposal_leg(args, make_inputs(), world, rank, local, coarse_fp16=args.precision == "fp16")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _cpu_threads():
    """Host threads for the CPU legs (each thread holds ~0.8 GB of 4096^2 buffers)."""
    threads = min(os.cpu_count() or 1, 32)
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    return int(os.environ["OMP_NUM_THREADS"])


def cpu_baseline(inp, sample=None):
    threads = _cpu_threads()
    n = sample or 2 * threads
    secs = _oracle_sample(inp, n, threads)
    pts = WORKLOAD["nx"] * WORKLOAD["ny"] * n / secs
    return {"value": pts, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {n} orientations of the grid on the full {inp['X']}x{inp['Y']} (padded) micrograph: "
                      f"the reference's CPU loop in FP32 with pocketfft transforms (oracle/cpu_port.py), "
                      f"{threads} host threads over orientation ranges, {secs:.1f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    inp = make_inputs()
    threads = _cpu_threads()
    n = args.cpu_sample or 2 * threads
    for _ in range(args.warmup):
        _oracle_sample(inp, threads, threads)
    total = 0.0
    for _ in range(args.steps):
        total += _oracle_sample(inp, n, threads)
    pts = WORKLOAD["nx"] * WORKLOAD["ny"] * n * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": pts, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "orientations_per_step": n},
            "cpu_baseline": {"value": pts, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n} orientations per step on the full micrograph: the reference's CPU loop "
                                       "in FP32 with pocketfft transforms (oracle/cpu_port.py; the reference itself "
                                       "needs wxWidgets/FFTW, absent here)"},
            "e2e": {"value": pts, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--orientations-per-step", type=int, default=1024)
    ap.add_argument("--batch", type=int, default=0, help="orientations per device pass; 0 = autotuned")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16"],
                    help="fp32 = the parity path; fp16 = FP16 correlation spectra with the tensor-core row transform")
    ap.add_argument("--cpu-sample", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fast-form", action="store_true",
                    help="skip the learned-proposal fast form (and its three-minute exhaustive judge)")
    ap.add_argument("--no-fp16-leg", action="store_true",
                    help="skip the FP16 tensor-core form that the default run times beside the FP32 path")
    ap.add_argument("--accuracy", type=int, default=4,
                    help="orientations compared with the FP64 oracle after timing, in the CPU-baseline leg (0 = skip)")
    ap.add_argument("--recall-orientations", type=int, default=0,
                    help="--workload recall16: orientations searched (0 = the whole grid)")
    ap.add_argument("--workload", default="full",
                    choices=sorted(WORKLOADS) + ["batched", "refine", "proposal", "recall16", "stress5"],
                    help="full = the metric's 4096^2 configuration; the others are the uneven and stress geometries")
    ap.add_argument("--e2e-contexts", type=int, default=2,
                    help="host threads (each with its own search context) sharing the GPU in the e2e leg")
    ap.add_argument("--refine-batch", type=int, default=256, help="candidates per TemplateScore batch (--workload refine)")
    ap.add_argument("--proposal-weights", default=PROPOSAL_WEIGHTS,
                    help="trained proposal network (--workload proposal)")
    ap.add_argument("--proposal-max-tiles", type=int, default=512,
                    help="most tiles the proposal's window search takes (--workload proposal)")
    ap.add_argument("--proposal-diag", default=None, help="npz of per-peak diagnostics (--workload proposal)")
    ap.add_argument("--traffic-b", type=float, default=None, help="ncu DRAM bytes per pass-B launch")
    ap.add_argument("--traffic-c", type=float, default=None, help="ncu DRAM bytes per pass-C launch")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS.get(args.workload, WORKLOADS["full"])
    if args.warmup < 3 and args.impl == "ours":
        print("note: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "refine":
        run_refine(args)
    elif args.workload == "proposal":
        run_proposal(args)
    elif args.workload == "recall16":
        run_recall16(args)
    elif args.workload == "stress5":
        run_stress5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
