#!/usr/bin/env python
"""Training iterations per second of the tile-based differentiable Gaussian
rasterizer on B200, on the workload the headline metric is quoted on: 1M
Gaussians, SH degree 3, 1237x822 views (the Mip-NeRF 360 "bicycle" images_4
size), 64 cameras on a hemisphere of radius 5. The photos themselves are not
available here, so the scene and the targets are seeded synthetic data of
those shapes (means in [-2, 2]^3, log-scales N(-4, 0.5), opacity logits
N(-1, 1.5), unit quaternions from N(0,1)^4, DC colour U(0,1), higher SH
N(0, 0.05), 60 degree horizontal field of view).

One step = one training iteration (forward, SSIM + L1 loss, backward, Adam)
on one view, views in turn. Reported:
  value  iterations/s with the targets resident in HBM (device-timed, CUDA
         events on the trainer's stream, max over ranks, times the ranks);
  e2e    the same through the public step() call with host (numpy) targets:
         the host->device copy of each target and the stats read-back are
         inside the timed region;
  plain  the plain FP32 form (FP32 SH and Adam state, the reference's
         two-sort order, host read-back of the entry count, no CUDA graph,
         deterministic exp/log) on the same views, for the 2x target;
  roofline, clocks, gpu_launches;
  cpu_baseline  the reference's FP64 CPU twin on whole views, one view per
         host thread on every thread, with an FP64 Adam step: views/s, and
         one thread's seconds for one whole view;
  precision.vs_fp64  the chosen and the plain form's render, loss and
         gradients on the first view against the FP64 oracle (oracle/fp64.py);
  fd_config2  both backward variants against FP64 central differences on
         256 parameters at the full training step's shape (100k Gaussians,
         800x800);
  batched, memory_adjoint  the other measured shapes, compact: 8 uneven
         views per step at 3M Gaussians, and recompute against store-everything
         at 6M Gaussians and 3840x2160;
  score_view_ms, densify (densification rounds on the GPU, first and later,
         beside the reference's densify_cloud on the same statistics;
         relocation rounds), prune: the cloud edits after the timed steps.
The checkers (the FP64 oracle, central differences, the CPU twin) run outside
every timed region.
--workload memory-adjoint, batched and session run the other measured
shapes at full length (each prints its own JSON line).
With --gpus N > 1 every rank trains its own replica (the path does not shard:
replicas only), and value is the sum over ranks.
--impl reference times the reference's own FP64 CPU twin (src/train/
reference.cpp, compiled from the reference's sources into oracle/_ref) on the
host cores instead: whole views, one per thread, in full rounds covering the
K steps, each with an FP64 Adam step.
"""
from __future__ import annotations

import argparse
import copy
import importlib
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT = 1237, 822
GAUSSIANS = 1_000_000
DEGREE = 3
VIEWS = 64
METRIC = "train iters/s @1M Gaussians 1237x822"
WORKLOAD = ("1M Gaussians, SH degree 3, 1237x822, 64 cameras on a radius-5 hemisphere, 60 deg horizontal fov "
            "(synthetic shapes of the bicycle scene)")
SEED = 3
SH_C0 = 0.28209479177387814


def make_scene(n: int = GAUSSIANS, degree: int = DEGREE, seed: int = SEED, log_scale=(-4.0, 0.5)):
    """The seeded synthetic scene: GaussianCloud arrays (float32)."""
    rng = np.random.default_rng(seed)
    coeffs = (degree + 1) ** 2
    positions = rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32)
    scales = rng.normal(log_scale[0], log_scale[1], (n, 3)).astype(np.float32)
    q = rng.normal(0.0, 1.0, (n, 4))
    rotations = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    opacities = rng.normal(-1.0, 1.5, n).astype(np.float32)
    sh = np.zeros((n, coeffs, 3), np.float32)
    sh[:, 0, :] = (rng.uniform(0.0, 1.0, (n, 3)) - 0.5) / SH_C0
    if coeffs > 1:
        sh[:, 1:, :] = rng.normal(0.0, 0.05, (n, coeffs - 1, 3))
    return positions.ravel(), scales.ravel(), rotations.ravel(), opacities, sh.ravel()


def hemisphere_views(count: int = VIEWS, radius: float = 5.0, width: int = WIDTH, height: int = HEIGHT):
    """Cameras on the upper hemisphere (z >= 0.15 r) looking at the origin:
    (view 4x4 world->camera, centre, fx, fy, cx, cy, W, H)."""
    fx = (width / 2) / math.tan(math.radians(30.0))
    golden = math.pi * (3.0 - math.sqrt(5.0))
    out = []
    for k in range(count):
        z = 0.15 + 0.85 * (k + 0.5) / count
        r = math.sqrt(1.0 - z * z)
        eye = radius * np.array([r * math.cos(golden * k), r * math.sin(golden * k), z])
        forward = -eye / np.linalg.norm(eye)
        right = np.cross(forward, np.array([0.0, 0.0, 1.0]))
        right /= np.linalg.norm(right)
        down = np.cross(forward, right)
        rot = np.stack([right, down, forward])
        view = np.eye(4)
        view[:3, :3] = rot
        view[:3, 3] = -rot @ eye
        out.append((view.astype(np.float32), eye.astype(np.float32), fx, fx, width / 2, height / 2, width, height))
    return out


def ring_views(count: int = 16, radius: float = 6.0, width: int = 800, height: int = 800, lift: float = 0.5):
    """Cameras on a horizontal ring of the given radius (at height `lift`)
    looking at the origin, 60 degree horizontal field of view: the full
    training step's 16 cameras. Same tuple layout as hemisphere_views."""
    fx = (width / 2) / math.tan(math.radians(30.0))
    out = []
    for k in range(count):
        a = 2.0 * math.pi * k / count
        eye = np.array([radius * math.cos(a), radius * math.sin(a), lift])
        forward = -eye / np.linalg.norm(eye)
        right = np.cross(forward, np.array([0.0, 0.0, 1.0]))
        right /= np.linalg.norm(right)
        down = np.cross(forward, right)
        rot = np.stack([right, down, forward])
        view = np.eye(4)
        view[:3, :3] = rot
        view[:3, 3] = -rot @ eye
        out.append((view.astype(np.float32), eye.astype(np.float32), fx, fx, width / 2, height / 2, width, height))
    return out


def config2_scene(n: int = 100_000, seed: int = 2):
    """The full training step's scene: n Gaussians of SH degree 3, means
    uniform in [-2, 2]^3, log-scales N(-3, 0.3), unit quaternions from
    N(0, 1)^4, opacity logits N(0, 1), DC colour U(0, 1), higher SH
    N(0, 0.05). GaussianCloud arrays (float32)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32).ravel()
    scales = rng.normal(-3.0, 0.3, (n, 3)).astype(np.float32).ravel()
    q = rng.normal(size=(n, 4))
    rot = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32).ravel()
    opac = rng.normal(0.0, 1.0, n).astype(np.float32)
    sh = np.zeros((n, 16, 3), np.float32)
    sh[:, 0, :] = (rng.uniform(0.0, 1.0, (n, 3)) - 0.5) / SH_C0
    sh[:, 1:, :] = rng.normal(0.0, 0.05, (n, 15, 3))
    return pos, scales, rot, opac, sh.ravel()


def fd_picks(rng, visible: np.ndarray, degree: int = DEGREE) -> list:
    """256 parameters of Gaussians a view sees: 64 position, 48 log-scale, 48
    rotation, 32 opacity and 64 SH coordinates, each of a random Gaussian."""
    coeffs = (degree + 1) ** 2
    picks = []
    for group, count, per in (("positions", 64, 3), ("scales", 48, 3), ("rotations", 48, 4), ("opacities", 32, 1),
                              ("sh", 64, 3 * coeffs)):
        for g in rng.choice(visible, count, replace=False):
            picks.append((group, int(g) * per + int(rng.integers(0, per))))
    return picks


def agreement(a, b) -> dict:
    """The reference's gradient comparison (tests/test_train.cpp:38-54): cosine
    and length ratio of a against b."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    aa, bb = float(a @ a), float(b @ b)
    if aa == 0.0 or bb == 0.0:
        return {"cosine": 0.0, "length_ratio": 0.0}
    return {"cosine": float(a @ b) / math.sqrt(aa * bb), "length_ratio": math.sqrt(aa / bb)}


def fd_config2(splat, torch, step: float = 1e-4, lam: float = 0.2) -> dict:
    """The full training step's adjoint against central differences of the
    FP64 oracle's loss (oracle/fp64.py, 0.8 L1 + 0.2 (1 - SSIM)) on 256
    parameters, h = 1e-4, for both backward variants (fixed-point and float
    sums), FP32 parameters, camera 0 of the ring, a seeded U(0, 1) target. A
    checker run outside every timed region; the criteria are the reference
    tests' (float: cosine > 0.999, length within 1 %, tests/test_train.cpp:99-112;
    fixed point: cosine > 0.97, within 10 %, :286-291)."""
    from oracle import fp64
    from oracle import oracle as O

    arrays = config2_scene()
    cam = ring_views()[0]
    view = O.View(*cam)
    rng = np.random.default_rng(5)
    target = rng.integers(0, 256, (800 * 800, 4), dtype=np.uint8)
    target[:, 3] = 255
    target = target.ravel()
    dc = fp64.DeviceCloud(O.Cloud(DEGREE, *arrays))
    out = {"workload": "100k Gaussians, SH degree 3, 800x800, camera 0 of 16 on a radius-6 ring, 256 parameters, h = 1e-4",
           "differences": "central, of the FP64 loss with the base render's blended (splat, pixel) pairs held fixed"}
    picks = None
    fd = None
    for fixed in (False, True):
        opts = splat.TrainerOptions(force_fixed_point=fixed, sh_storage=splat.SH_F32, state_storage=splat.STATE_F32)
        trainer = splat.Trainer(splat.GaussianCloud(DEGREE, *arrays), opts)
        stats = trainer.compute_gradients(splat.Camera(*cam), target)
        g = trainer.gradients()
        del trainer
        if picks is None:
            visible = np.nonzero(np.abs(g.opacities) > 0)[0]
            picks = fd_picks(np.random.default_rng(17), visible)
            t0 = time.perf_counter()
            fd = fp64.finite_differences(dc, view, target, lam, picks, step=step)
            out["fd_seconds"] = time.perf_counter() - t0
            base = fp64.render_full(dc, view)
            loss64, _, _, adjoint = fp64.loss(base.rgb, target, view.width, view.height, lam)
            out["loss_fp64"] = loss64
            g64 = fp64.gradients(dc, view, base, adjoint)
            out["fp64_adjoint"] = agreement([g64[gr][ix] for gr, ix in picks], fd)
            del base, adjoint
        analytic = np.array([getattr(g, group)[index] for group, index in picks], np.float64)
        agree = agreement(analytic, fd)
        agree["loss"] = stats.loss
        agree["groups"] = {name: agreement(analytic[[k for k, (gr, _) in enumerate(picks) if gr == name]],
                                           fd[[k for k, (gr, _) in enumerate(picks) if gr == name]])
                           for name in ("positions", "scales", "rotations", "opacities", "sh")}
        if fixed:
            # Fixed-point sums resolve 1 / (3 W H 64) per warp total (the
            # reference's scale, about 8e-9 at 800x800). A warp's dL/dcov
            # total, behind the scales and rotations, is mostly smaller and
            # rounds away; the criterion applies to the groups it resolves.
            resolved = np.isin(np.array([gr for gr, _ in picks]), ("positions", "opacities", "sh"))
            agree["resolved_groups"] = dict(agreement(analytic[resolved], fd[resolved]), count=int(resolved.sum()),
                                            groups=["positions", "opacities", "sh"])
            agree["note"] = ("scales and rotations come from dL/dcov sums that mostly fall below the fixed scale "
                             "1/(3 W H 64) per warp at 800x800 and round away (the reference's design); "
                             "tests/test_configs.py checks splat by splat that this rounding is the whole difference")
            judged = agree["resolved_groups"]
            cos, ratio = 0.97, 0.1
        else:
            judged, cos, ratio = agree, 0.999, 0.01
        agree["passes"] = judged["cosine"] > cos and abs(judged["length_ratio"] - 1.0) < ratio
        out["fixed_point" if fixed else "float"] = agree
    torch.cuda.empty_cache()
    return out


def make_targets(count: int = VIEWS, width: int = WIDTH, height: int = HEIGHT, seed: int = SEED):
    rng = np.random.default_rng(seed + 1)
    t = rng.integers(0, 256, (count, height * width * 4), dtype=np.uint8)
    t[:, 3::4] = 255
    return t


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ----------------------------------------------------------------- clocks


class ClockSampler:
    """SM clock and throttle reasons while running: NVML every 5 ms when it
    loads (read-only queries), else nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    # NVML clock event reason bits.
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.samples = []
        self.stop = threading.Event()
        self.nvml = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            prop = torch.cuda.get_device_properties(self.device)
            bus = f"{prop.pci_domain_id:08X}:{prop.pci_bus_id:02X}:{prop.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self):
        nv, h = self.nvml
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM), int(reasons(h))))
            except Exception:
                break
            self.stop.wait(0.005)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        if self.samples:
            for clock, top, bits in self.samples:
                sm.append(float(clock))
                mx = max(mx, float(top))
                reasons.update(name for name, bit in self.REASONS.items() if bits & bit)
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                    "source": "nvml, 5 ms"}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 200 ms"}


# ----------------------------------------------------------------- CPU reference


def adam_step_fp64(params: dict, grads, rates: dict, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-15) -> None:
    """One Adam step in FP64 from a zero state (a run's first iteration),
    selective as the reference's (a parameter without a gradient stays), in
    place on the float32 parameter arrays: the reference's step
    (shaders/train_step.glsl, constants src/train/trainer.cpp:23) restated in
    numpy, since the reference has it only as a shader. rates: per group; SH
    above DC at rates['sh_rest']."""
    c1, c2 = 1.0 - beta1, 1.0 - beta2
    for group in ("positions", "scales", "rotations", "opacities", "sh"):
        g = np.asarray(getattr(grads, group), np.float64)
        m = (1.0 - beta1) * g
        v = (1.0 - beta2) * g * g
        lr = np.full(g.shape, rates[group])
        if group == "sh":
            coeffs = g.size // (params["opacities"].size * 3)
            lr = lr.reshape(-1, coeffs, 3)
            lr[:, 1:, :] = rates["sh_rest"]
            lr = lr.ravel()
        step = lr * (m / c1) / (np.sqrt(v / c2) + eps)
        step[g == 0.0] = 0.0
        params[group] -= step.astype(np.float32)


def twin_views_per_core(oracle, arrays, views, targets, threads: int, adam: bool = True) -> dict:
    """The reference's FP64 CPU twin (src/train/reference.cpp, compiled from its
    sources into oracle/_ref) on whole views, one view per host thread, as many
    views at once as there are threads: per view reference_render,
    reference_loss and reference_gradients (which renders again), then, with
    adam, an FP64 Adam step on a copy of the parameters. Returns the wall time,
    the views done, and each view's own seconds (one thread's time for one
    whole view)."""
    import concurrent.futures

    pos, sc, rot, op, sh = arrays
    rates = {"positions": 1.6e-4, "scales": 0.005, "rotations": 0.001, "opacities": 0.05, "sh": 0.025,
             "sh_rest": 0.025 * 0.05}

    def one(job):
        view, target = job
        t0 = time.perf_counter()
        cloud = oracle.Cloud(DEGREE, pos, sc, rot, op, sh)
        rgb, _, _ = oracle.ref_render(cloud, view)
        _, _, _, adjoint = oracle.ref_loss(rgb, view.width, view.height, target, 0.2)
        grads = oracle.ref_gradients(cloud, view, adjoint)
        if adam:
            params = {"positions": pos.copy(), "scales": sc.copy(), "rotations": rot.copy(), "opacities": op.copy(),
                      "sh": sh.copy()}
            adam_step_fp64(params, grads, rates)
        return time.perf_counter() - t0

    jobs = list(zip(views, targets))
    start = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as pool:
        per_view = list(pool.map(one, jobs))
    return {"seconds": time.perf_counter() - start, "views": len(jobs), "per_view_seconds": per_view}


def reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    if not O.have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsplatref.so was not built "
                          "(the reference's src/train/reference.cpp compiles only where its tree is present)"}))
        return
    arrays = make_scene()
    threads = cpu_count()
    # K steps, each one whole view (render, loss, gradients, Adam) on one host
    # thread, run as full rounds of one view per thread: K rounded up to a
    # multiple of the thread count, so that no round leaves cores idle.
    count = threads * math.ceil(max(args.steps, 1) / threads)
    views = [O.View(*hemisphere_views()[i % VIEWS]) for i in range(count)]
    targets = make_targets(8)
    run = twin_views_per_core(O, arrays, views, [targets[i % 8] for i in range(count)], threads)
    value = run["views"] / run["seconds"]
    per_view = float(np.mean(run["per_view_seconds"]))
    sample = (f"{run['views']} whole views (1M Gaussians, SH degree 3, 1237x822), one per host thread on {threads} threads "
              f"({run['seconds']:.0f} s): reference_render + reference_loss + reference_gradients of the reference's FP64 "
              f"twin and an FP64 Adam step; {per_view:.0f} s per view on one thread")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iters/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * run["seconds"] / run["views"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(),
        "form": "the reference's FP64 CPU twin (src/train/reference.cpp) per whole view, one view per core, with an "
                "FP64 Adam step restated from its shader",
        "cpu_baseline": {"value": value, "unit": "iters/s", "cores": threads, "kind": "reference", "sample": sample,
                         "single_thread_seconds_per_view": per_view},
        "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def bench_config() -> dict:
    """The workload both arms report as their config."""
    return {"workload": WORKLOAD, "views": VIEWS, "loss": "0.8 L1 + 0.2 (1 - SSIM)", "optimiser": "Adam, one step per view",
            "l2": "inputs larger than L2 (1M-Gaussian parameters and state, 64 x 4 MB targets)"}


# ----------------------------------------------------------------- our arm


def stage_bytes(n: int, visible: int, entries: int, pixels: int, depth_passes: int, reached: float | None = None) -> dict:
    """Algorithmic HBM bytes per step of each timed stage, for the chosen form
    (BF16 SH above DC, BF16-pair Adam state): what each stage must read and
    write at least once, not what it happens to move. `reached`: the Gaussians
    the one-view selective step moves (a non-zero backward sum), measured; the
    visible count when it was not."""
    sh_bytes = 12 + 45 * 2  # DC in FP32, 45 higher coefficients in BF16
    moved = visible if reached is None else reached
    return {
        # positions, scales, rotations, opacity (44 B) and SH in; splat (48),
        # reach, depth key and index (12) out.
        "project": n * (44 + sh_bytes + 60),
        # keys and values read and written per pass, plus the histogram's read.
        "depth sort": n * (16 * depth_passes + 4),
        # per item: key, index, splat centre and conic, reach in; offset and mask out.
        "count tiles": n * 8 + visible * (32 + 4 + 8),
        # emission (offset, mask, rectangle in; tile and index out), two sort
        # passes and a histogram over the entries, ranges.
        "tile lists": visible * 24 + entries * (8 + 2 * 16 + 4 + 4),
        # per entry its index and 48-byte splat; per pixel colour, log T and stop out.
        "composite": entries * 52 + pixels * 20,
        # image and target in for SSIM, 9 field planes out and in, adjoint out.
        "loss": pixels * (16 + 4 + 36 + 36 + 16 + 16 + 4),
        # per entry index and splat; per pixel image, adjoint, stop; sums out.
        "backward": entries * 52 + pixels * 36 + visible * 56,
        # the 64-byte row of backward sums of every Gaussian (the reached test);
        # colour in, and densification statistics (8 words), parameters, SH
        # and Adam state (59 words) read and written, for the reached ones.
        "chain rule and step": n * 64 + moved * (16 + 2 * (32 + 44 + sh_bytes + 59 * 4)),
    }


def reached_count(splat, trainer, cams, targets, rates, views: int = 4) -> float:
    """Mean count of the Gaussians a view reaches: those with a backward sum
    that is not zero (a float sum of -0 counts as zero), the test the
    one-view selective step makes. Each view's gradients are applied
    afterwards, so the trainer ends a whole step further on."""
    n = trainer.gaussian_count()
    counts = []
    for i in range(views):
        trainer.compute_gradients(cams[i % len(cams)], targets[i % len(cams)])
        raw = trainer.debug_download(splat.DEBUG_RAW, np.uint32).reshape(-1, 16)[:n, :14]
        if not trainer.uses_fixed_point():
            raw = raw & np.uint32(0x7FFFFFFF)
        counts.append(int(np.count_nonzero(raw.any(axis=1))))
        trainer.apply_gradients(rates)
    return float(np.mean(counts))


def form_key(opts) -> str:
    """The rasterizer form a profile line must name for its figure to be used:
    tile edge, batch depth, launch shape, backward sums and pixels per thread
    decide which kernels the composite and backward stages launch."""
    return (f"tile{opts.tile_size} batch{opts.batch_depth} {'persistent' if opts.persistent_raster else 'grid'} "
            f"{'grouped' if opts.grouped_backward else 'atomic'} px{opts.forward_pixels_per_thread}/"
            f"{opts.backward_pixels_per_thread}")


def profile_figure(kind: str, stage: str, form: str):
    """A per-launch figure of the stage's kernel from the committed ncu summary
    of the bench workload (profiles/*.md, a line '<kind> <stage> [<form>]: N'):
    kind 'traffic' for DRAM bytes, 'instructions' for warp-instructions. A line
    taken on another rasterizer form (another kernel) is not used. Or None."""
    head = f"{kind} {stage} [{form}]:"
    for path in sorted((ROOT / "profiles").glob("*.md")):
        for line in path.read_text().splitlines():
            if line.startswith(head):
                try:
                    return int(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def measured_traffic(stage: str, form: str):
    return profile_figure("traffic", stage, form)


def chosen_options(splat):
    return splat.TrainerOptions(sh_storage=splat.SH_BF16, state_storage=splat.STATE_BF16_PAIR,
                                sort_form=splat.SORT_TILE_DEPTH_64, exact_math=False, use_graph=True, digit_bits=8,
                                forward_pixels_per_thread=2, backward_pixels_per_thread=2)


def plain_options(splat):
    return splat.TrainerOptions(sh_storage=splat.SH_F32, state_storage=splat.STATE_F32,
                                sort_form=splat.SORT_DEPTH_THEN_TILE, exact_math=True, use_graph=False, digit_bits=8,
                                forward_pixels_per_thread=1, backward_pixels_per_thread=1)


def time_steps(torch, trainer, step_fn, steps: int, stream_handle: int) -> float:
    """Device milliseconds for `steps` calls of step_fn, by CUDA events on the trainer's stream."""
    stream = torch.cuda.ExternalStream(stream_handle)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for i in range(steps):
        step_fn(i)
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def psnr(image: np.ndarray, reference: np.ndarray) -> float:
    mse = float(np.mean((np.asarray(image, np.float64) - np.asarray(reference, np.float64)) ** 2))
    return 10.0 * math.log10(1.0 / max(mse, 1e-30))


def tuned_options(chosen, tuned: dict):
    """The chosen form's options with the autotuner's picks applied."""
    opts = copy.copy(chosen)
    if tuned:
        opts.sort_form = tuned.get("sort_form", chosen.sort_form)
        opts.digit_bits = tuned.get("digit_bits", chosen.digit_bits)
        opts.forward_pixels_per_thread = tuned.get("forward_pixels_per_thread", chosen.forward_pixels_per_thread)
        opts.backward_pixels_per_thread = tuned.get("backward_pixels_per_thread", chosen.backward_pixels_per_thread)
        opts.tile_size = tuned.get("tile_size", chosen.tile_size)
        opts.batch_depth = tuned.get("batch_depth", chosen.batch_depth)
        opts.persistent_raster = bool(tuned.get("persistent_raster", chosen.persistent_raster))
        opts.grouped_backward = bool(tuned.get("grouped_backward", chosen.grouped_backward))
    return opts


def precision_check(splat, torch, cloud, cams, host_targets, rates, chosen, tuned, steps: int = 20) -> dict:
    """The chosen form against the plain FP32 form from the same cloud: PSNR of
    one's render against the other's, then, after `steps` identical training
    steps (views in turn), each render's PSNR against the target and the
    difference."""
    forms = {"chosen": tuned_options(chosen, tuned), "plain": plain_options(splat)}
    renders, after = {}, {}
    target0 = host_targets[0].reshape(-1, 4)[:, :3].astype(np.float64) / 255.0
    for name, opts in forms.items():
        trainer = splat.Trainer(cloud, opts)
        renders[name] = trainer.render(cams[0]).reshape(-1, 4)[:, :3]
        for i in range(steps):
            trainer.step(cams[i % len(cams)], host_targets[i % len(cams)], rates)
        after[name] = psnr(trainer.render(cams[0]).reshape(-1, 4)[:, :3], target0)
        del trainer
        torch.cuda.empty_cache()
    return {"render_psnr_chosen_vs_plain_db": psnr(renders["chosen"], renders["plain"]),
            "steps": steps, "psnr_vs_target_db": after,
            "psnr_difference_db": abs(after["chosen"] - after["plain"])}


def precision_vs_fp64(splat, torch, arrays, camera, view, target, forms: dict, lam: float = 0.2) -> dict:
    """Each form's render, loss and gradients on one view against the FP64
    oracle (oracle/fp64.py: the reference twin's render, loss and gradients
    restated in double precision on the GPU, pinned against the twin by
    tests/test_configs.py) on the same cloud, with the SH coefficients the
    form stores (BF16-rounded for the BF16 form): per-group relative error
    ||g - g64|| / ||g64||, the render's PSNR against the FP64 render, and both
    losses. A checker run outside every timed region."""
    from oracle import fp64
    from oracle import oracle as O

    pos, sc, rot, op, sh = arrays
    out = {}
    for name, opts in forms.items():
        trainer = splat.Trainer(splat.GaussianCloud(DEGREE, pos, sc, rot, op, sh), opts)
        image = trainer.render(camera).reshape(-1, 4)[:, :3].astype(np.float64)
        stats = trainer.compute_gradients(camera, target)
        g = trainer.gradients()
        del trainer
        torch.cuda.empty_cache()
        storage = {splat.SH_BF16: "bf16", splat.SH_F16: "f16"}.get(opts.sh_storage, "f32")
        held = sh if storage == "f32" else O.round_sh_like_device(sh, DEGREE, storage)
        dc = fp64.DeviceCloud(O.Cloud(DEGREE, pos, sc, rot, op, held))
        rendered = fp64.render_full(dc, view)
        loss64, _, _, adjoint = fp64.loss(rendered.rgb, target, view.width, view.height, lam)
        g64 = fp64.gradients(dc, view, rendered, adjoint)
        rgb64 = rendered.rgb.cpu().numpy()
        rel = {}
        for group in ("positions", "scales", "rotations", "opacities", "sh"):
            ref = g64[group]
            rel[group] = float(np.linalg.norm(np.asarray(getattr(g, group), np.float64) - ref) / max(np.linalg.norm(ref), 1e-300))
        out[name] = {"loss": stats.loss, "loss_fp64": loss64, "render_psnr_vs_fp64_db": psnr(image, rgb64),
                     "gradient_rel_error": rel, "max_gradient_rel_error": max(rel.values()),
                     "fp64_entries": rendered.entry_count}
        del dc, rendered, adjoint
        torch.cuda.empty_cache()
    return out


def memory_adjoint_summary(gaussians: int, steps: int, warmup: int) -> dict:
    """The memory-bound adjoint: 6M Gaussians of SH degree 3 (BF16 above DC),
    3840x2160 views, log-scales N(-4.5, 0.6) for heavy per-tile overlap. The
    reverse-sweep recompute (8 bytes of per-pixel state) against the
    store-everything variant (every blended (entry, alpha) pair kept per pixel):
    iterations/s, device memory held, per-pixel state."""
    import torch

    splat = importlib.import_module("vibe-splat_b200")
    n = gaussians
    width, height, views = 3840, 2160, 4
    pos, sc, rot, op, sh = make_scene(n, log_scale=(-4.5, 0.6))
    cloud = splat.GaussianCloud(DEGREE, pos, sc, rot, op, sh)
    cams = [splat.Camera(v, p, fx, fy, cx, cy, w, h)
            for (v, p, fx, fy, cx, cy, w, h) in hemisphere_views(views, width=width, height=height)]
    targets = torch.from_numpy(make_targets(views, width, height)).cuda()
    rates = splat.LearningRates()
    pixels = width * height
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    out = {"metric": "memory-bound adjoint: recompute vs store-everything", "unit": "iters/s",
           "config": {"workload": f"{n} Gaussians, SH degree 3 (BF16 above DC), {width}x{height}, log-scales N(-4.5, 0.6), "
                                  f"{views} cameras on a radius-5 hemisphere, 60 deg horizontal fov (synthetic)"},
           "steps": steps, "warmup": warmup}
    for name, lists in (("recompute", False), ("store_everything", True)):
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        free0, _ = torch.cuda.mem_get_info()
        opts = chosen_options(splat)
        opts.sort_form = splat.SORT_DEPTH_THEN_TILE
        opts.blend_lists = lists
        opts.use_graph = not lists
        if lists:
            opts.backward_pixels_per_thread = 1
        trainer = splat.Trainer(cloud, opts)
        # Every view once at least, so that the entry and list buffers have
        # grown to the largest view's before the timed steps.
        for i in range(max(warmup, views)):
            stats = trainer.step_device_target(cams[i % views], targets[i % views].data_ptr(), rates)
        ms = time_steps(torch, trainer, lambda i: trainer.step_device_target(cams[i % views], targets[i % views].data_ptr(),
                                                                              rates), steps, trainer.stream())
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        entry = {"iters_per_s": 1000.0 * steps / ms, "ms_per_step": ms / steps,
                 "device_bytes_held": free0 - free1, "tile_entries": stats.tile_entries,
                 "mean_entries_per_tile": stats.tile_entries / tiles, "per_pixel_state_bytes": 8.0}
        if lists:
            counts = trainer.debug_download(splat.DEBUG_BLEND_COUNTS, np.uint32)[:pixels]
            blended = int(counts.astype(np.uint64).sum())
            entry["blended_pairs"] = blended
            entry["mean_blended_per_pixel"] = blended / pixels
            entry["per_pixel_state_bytes"] = 8.0 + 8.0 + 8.0 * blended / pixels
        out[name] = entry
        del trainer
    r, s = out["recompute"], out["store_everything"]
    out["memory_saved_bytes"] = s["device_bytes_held"] - r["device_bytes_held"]
    out["speed_ratio_recompute_over_store"] = r["iters_per_s"] / s["iters_per_s"]
    return out


def memory_adjoint_workload(args) -> None:
    n = 6_000_000 if args.gaussians == GAUSSIANS else args.gaussians
    print(json.dumps(memory_adjoint_summary(n, args.steps, args.warmup)))


BATCHED_SIZES = [(640, 480), (800, 600), (1024, 768), (1237, 822), (1280, 720), (1600, 1200), (960, 540), (1920, 1080)]


def batched_views():
    """The batched form's 8 views of uneven sizes, cameras at random points of
    a sphere of radius 4 to 8 looking at the origin (60 degree horizontal
    field of view), and a seeded RGBA8 target each: (view tuples as
    hemisphere_views gives them, targets)."""
    rng = np.random.default_rng(SEED + 7)
    views, targets = [], []
    for (w, h) in BATCHED_SIZES:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        eye = d * rng.uniform(4.0, 8.0)
        forward = -eye / np.linalg.norm(eye)
        up = np.array([0.0, 0.0, 1.0]) if abs(forward[2]) < 0.99 else np.array([0.0, 1.0, 0.0])
        right = np.cross(forward, up)
        right /= np.linalg.norm(right)
        down = np.cross(forward, right)
        rot = np.stack([right, down, forward])
        view = np.eye(4)
        view[:3, :3] = rot
        view[:3, 3] = -rot @ eye
        fx = (w / 2) / math.tan(math.radians(30.0))
        views.append((view.astype(np.float32), eye.astype(np.float32), fx, fx, w / 2, h / 2, w, h))
        t = rng.integers(0, 256, h * w * 4, dtype=np.uint8)
        t[3::4] = 255
        targets.append(t)
    return views, targets


def batched_summary(gaussians: int, steps: int, warmup: int) -> dict:
    """The batched form: 3M Gaussians of SH degree 3 (BF16 above DC), 8 views of
    uneven sizes per step (one launch per stage for all of them, the
    rasterizer's two persistent, 64-bit tile|depth keys, CUDA graph), cameras
    at random points of a sphere of radius
    4 to 8 looking at the origin. Against the same views one per step: views/s."""
    import torch

    splat = importlib.import_module("vibe-splat_b200")
    n = gaussians
    views, targets = batched_views()
    sizes = [(v[6], v[7]) for v in views]
    cams = [splat.Camera(*v) for v in views]
    pos, sc, rot_, op, sh = make_scene(n)
    cloud = splat.GaussianCloud(DEGREE, pos, sc, rot_, op, sh)
    rates = splat.LearningRates()
    out = {"metric": "train views/s, 8 uneven views per step", "unit": "views/s",
           "config": {"workload": f"{n} Gaussians, SH degree 3 (BF16 above DC), 8 views "
                                  + ", ".join(f"{w}x{h}" for w, h in sizes)
                                  + ", random poses on a sphere of radius 4-8, 60 deg horizontal fov (synthetic)"},
           "steps": steps, "warmup": warmup}
    # Every view's tiles in one persistent launch per rasterizer stage.
    opts = chosen_options(splat)
    opts.sort_form = splat.SORT_TILE_DEPTH_64
    opts.forward_pixels_per_thread = opts.backward_pixels_per_thread = 2
    opts.persistent_raster = True
    trainer = splat.Trainer(cloud, opts)
    for _ in range(warmup):
        stats = trainer.step_batch(cams, targets, rates)
    ms = time_steps(torch, trainer, lambda i: trainer.step_batch(cams, targets, rates), steps, trainer.stream())
    out["batched"] = {"views_per_s": 1000.0 * steps * len(cams) / ms, "ms_per_step": ms / steps,
                      "tile_entries": stats[0].tile_entries}  # every view's stats carry the batch's total
    del trainer
    torch.cuda.empty_cache()
    one = chosen_options(splat)
    one.sort_form = splat.SORT_DEPTH_THEN_TILE
    one.forward_pixels_per_thread = one.backward_pixels_per_thread = 2
    single = splat.Trainer(cloud, one)
    for i in range(warmup * len(cams)):
        single.step(cams[i % len(cams)], targets[i % len(cams)], rates)
    k = len(cams)
    ms1 = time_steps(torch, single, lambda i: single.step(cams[i % k], targets[i % k], rates,
                                                          next_target=targets[(i + 1) % k]),
                     steps * k, single.stream())
    out["one_view_per_step"] = {"views_per_s": 1000.0 * steps * k / ms1, "ms_per_view": ms1 / (steps * k)}
    out["value"] = out["batched"]["views_per_s"]
    return out


def batched_workload(args) -> None:
    n = 3_000_000 if args.gaussians == GAUSSIANS else args.gaussians
    print(json.dumps(batched_summary(n, args.steps, args.warmup)))


def slowest_over_ranks(ms: float, dist, device: str) -> float:
    """The max over ranks of one rank's device time; every rank calls this at
    the same point (a collective). Without a process group, the time itself."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_rank: float, slowest_ms: float) -> float:
    """Replicas: every rank did the same units; the job's rate is all of them
    over the slowest rank's time."""
    return world * units_per_rank * 1000.0 / slowest_ms


def our_arm(args) -> None:
    import torch

    splat = importlib.import_module("vibe-splat_b200")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    # The SM pipes' measured throughput: the roofline of the issue-bound kernels.
    try:
        sm_peaks = splat.measure_sm_peaks()
    except Exception:
        sm_peaks = {}
    pos, sc, rot, op, sh = make_scene(args.gaussians)
    cloud = splat.GaussianCloud(DEGREE, pos, sc, rot, op, sh)
    cams = [splat.Camera(v, p, fx, fy, cx, cy, w, h) for (v, p, fx, fy, cx, cy, w, h) in hemisphere_views()][: args.views]
    host_targets = make_targets(args.views)
    device_targets = torch.from_numpy(host_targets).cuda()
    rates = splat.LearningRates()
    nbytes = WIDTH * HEIGHT * 4

    tuned = {}

    def run_form(options, label: str, tune: bool = False):
        trainer = splat.Trainer(cloud, options)
        stream = trainer.stream()

        # The targets' device addresses, looked up once: the loop does no
        # tensor indexing between the (synchronous) steps.
        target_ptrs = [device_targets[k].data_ptr() for k in range(len(cams))]

        def resident(i):
            k = i % len(cams)
            return trainer.step_device_target(cams[k], target_ptrs[k], rates)

        if tune:
            # The autotuner picks the sort form and digit width (gradient passes, no parameter change).
            tuned.update(trainer.autotune(cams[0], host_targets[0], repeats=3))
        for i in range(args.warmup):
            resident(i)
        if dist is not None:
            dist.barrier()
        with ClockSampler(local) as clocks:
            ms = time_steps(torch, trainer, lambda i: resident(args.warmup + i), args.steps, stream)
        stats = resident(0)
        return trainer, ms, clocks.summary(), stats

    chosen = chosen_options(splat)
    if args.sort_form is not None:
        chosen.sort_form = args.sort_form
    if args.form:
        pixels, tile, batch, persistent, grouped = (int(v) for v in args.form.split(","))
        chosen.sort_form = splat.SORT_DEPTH_THEN_TILE if args.sort_form is None else args.sort_form
        chosen.forward_pixels_per_thread = chosen.backward_pixels_per_thread = pixels
        chosen.tile_size, chosen.batch_depth = tile, batch
        chosen.persistent_raster, chosen.grouped_backward = bool(persistent), bool(grouped)
    trainer, ms, clocks, stats = run_form(chosen, "chosen",
                                          tune=args.sort_form is None and not args.no_autotune and not args.form)
    ms = slowest_over_ranks(ms, dist, "cuda")
    ms_per_step = ms / args.steps
    value = whole_job_rate(world, args.steps, ms)

    # e2e: the public step() with host targets (H2D of the target and the stats
    # read-back in the timed region). Each call names the next view's target,
    # which the library copies to pinned memory while the step runs.
    stream = trainer.stream()
    k = len(cams)

    def host_step(i):
        return trainer.step(cams[i % k], host_targets[i % k], rates, next_target=host_targets[(i + 1) % k])

    # Warm-up through the same call: the first ones allocate the pinned and
    # device prefetch buffers and have no prefetched target yet.
    for i in range(args.warmup):
        host_step(i)
    e2e_ms = time_steps(torch, trainer, lambda i: host_step(args.warmup + i), args.steps, stream)
    e2e_ms = slowest_over_ranks(e2e_ms, dist, "cuda")
    e2e = whole_job_rate(world, args.steps, e2e_ms)

    # The FastGS scoring pass (score_view: a statistics pass with the
    # high-error pixels marked, plus the score kernel), host target, plain form.
    for i in range(2):
        trainer.score_view(cams[i % k], host_targets[i % k], 0.5)
    score_ms = time_steps(torch, trainer, lambda i: trainer.score_view(cams[i % k], host_targets[i % k], 0.5),
                          max(3, min(args.steps, 10)), stream) / max(3, min(args.steps, 10))
    trainer.reset_densify_stats()

    # Per-stage device times (serialising events, plain launches) for the roofline.
    trainer.set_timing(True)
    for i in range(max(3, min(args.steps, 10))):
        trainer.step_device_target(cams[i % len(cams)], device_targets[i % len(cams)].data_ptr(), rates)
    stages = dict(trainer.timings())
    trainer.set_timing(False)
    entries, visible = stats.tile_entries, stats.visible_splats
    pixels = WIDTH * HEIGHT
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    dominant = max(stages, key=stages.get) if stages else None
    n = args.gaussians
    digits_used = tuned.get("digit_bits", chosen.digit_bits)
    depth_passes = math.ceil(32 / digits_used)
    reached = reached_count(splat, trainer, cams, host_targets, rates)
    algorithmic = stage_bytes(n, visible, entries, pixels, depth_passes, reached)
    form = form_key(tuned_options(chosen, tuned))
    # The SM issue rate: measured by the library's FMA microbenchmark on this
    # GPU when it ran, else 148 SMs x 4 warp-instructions per clock at the SM
    # clock sampled during the timed steps (the maximum if none was sampled).
    sm_mhz = (clocks.get("sm_mhz") if isinstance(clocks, dict) else None) or 1965.0
    issue_peak = sm_peaks.get("warp_instructions") or 148 * 4 * sm_mhz * 1e6
    issue_source = "measured (splat_measure_sm_peaks)" if sm_peaks.get("warp_instructions") else "148 SMs x 4 per clock"
    stage_roof = {}
    for name, ms_stage in stages.items():
        b = algorithmic.get(name)
        if b is None or ms_stage <= 0:
            continue
        gbs = b / (ms_stage * 1e-3) / 1e9
        stage_roof[name] = {"bytes": b, "ms": ms_stage, "GB/s": gbs, "frac": gbs / hbm_peak}
        inst = profile_figure("instructions", name, form)
        if inst:
            rate = inst / (ms_stage * 1e-3)
            stage_roof[name]["issue"] = {"warp_inst_per_s": rate, "peak": issue_peak, "frac": rate / issue_peak,
                                         "instructions": inst, "peak_source": issue_source}
    roof = None
    if dominant is not None and dominant in stage_roof:
        r = stage_roof[dominant]
        traffic = measured_traffic(dominant, form)
        roof = {"kernel": dominant, "bound": "hbm", "achieved": r["GB/s"], "peak": hbm_peak, "unit": "GB/s",
                "frac": r["frac"], "traffic": traffic, "ms": r["ms"], "form": form,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"}
        if dominant in ("backward", "composite"):
            roof["note"] = ("issue-bound, not HBM-bound: the SM instruction issue rate is the limit; 'issue' gives "
                            "the kernel's warp-instructions (ncu, profiles/) over its live time against the measured "
                            "issue rate (the FMA microbenchmark's); the HBM fraction is given for the record")
            if "issue" in r:
                roof["issue"] = r["issue"]

    # Densification on the GPU with the statistics the timed steps collected:
    # the session's dense scale (1 % of the scene extent) and a count cap of
    # 5 % growth. The reference's own densify_cloud on the same cloud and
    # statistics is timed beside it on the host (its download of the cloud
    # and upload of the result not included).
    densify = None
    if not args.no_densify:
        held = trainer.cloud()
        raw = trainer.densify_stats_raw()
        centre = held.positions.reshape(-1, 3).mean(axis=0)
        extent = float(np.linalg.norm(held.positions.reshape(-1, 3) - centre, axis=1).max())
        d_opts = splat.DensifyOptions(dense_scale=0.01 * extent, max_gaussians=int(n * 1.05))
        rng = splat.Rng(1)

        def more_steps(count):
            for i in range(count):
                trainer.step_device_target(cams[i % len(cams)], device_targets[i % len(cams)].data_ptr(), rates)

        def timed(edit):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = edit()
            return r, (time.perf_counter() - t0) * 1000.0

        r, d_ms = timed(lambda: trainer.densify(d_opts, rng))
        densify = {"ms_first": d_ms, "of": n, "count": r.count, "cloned": r.cloned, "split": r.split, "pruned": r.pruned,
                   "held_back": r.held_back}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            from oracle import oracle as O

            if O.have_reference():
                c = O.Cloud(DEGREE, held.positions, held.scales, held.rotations, held.opacities, held.sh)
                t0 = time.perf_counter()
                ref = O.ref_densify(c, raw, d_opts._c(), O.RefRng(1))
                densify["reference_cpu_ms"] = (time.perf_counter() - t0) * 1000.0
                densify["reference_same_result"] = bool(np.array_equal(ref.source, r.source))
        del held, raw
        # A later round, once the edit's buffers exist: statistics of a few
        # more steps, then densify again on the same generator.
        more_steps(5)
        r, d_ms = timed(lambda: trainer.densify(d_opts, rng))
        densify["ms"] = d_ms
        densify["count_second"] = r.count
        # 3DGS-MCMC relocation (dead onto live, 5 % growth): the dead/alive
        # split and the gathers on the GPU, the draws on the host; first and
        # a later round.
        r, m_first = timed(lambda: trainer.relocate(splat.RelocateOptions(), rng))
        more_steps(5)
        r2, m_ms = timed(lambda: trainer.relocate(splat.RelocateOptions(), rng))
        densify["relocate"] = {"ms_first": m_first, "ms": m_ms, "count": r2.count, "relocated": r2.cloned,
                               "grown": r2.seeded}

    # Pruning on the GPU (remove_largest_gaussians, 1 % of the Gaussians):
    # keys, sort, scan and the gathers of parameters and optimiser state.
    t0 = time.perf_counter()
    pruned = trainer.remove_largest_gaussians(0.01)
    prune = {"removed": pruned, "ms": (time.perf_counter() - t0) * 1000.0, "of": n}

    plain = None
    if not args.no_plain:
        del trainer
        torch.cuda.empty_cache()
        p_trainer, p_ms, p_clocks, _ = run_form(plain_options(splat), "plain")
        plain = {"iters_per_s": 1000.0 * args.steps / p_ms, "ms_per_step": p_ms / args.steps,
                 "form": "FP32 SH and Adam state, depth-then-tile sort, host read-back, no graph, exact exp/log"}
        del p_trainer

    precision = None
    if not args.no_plain:
        precision = precision_check(splat, torch, cloud, cams, host_targets, rates, chosen, tuned)

    # Checkers, outside every timed region: the forms against the FP64
    # oracle on the headline view, and the full training step's adjoint
    # against FP64 central differences.
    if precision is not None and not args.no_checks:
        (v0, p0, fx0, fy0, cx0, cy0, w0, h0) = hemisphere_views()[0]
        from oracle import oracle as O

        precision["vs_fp64"] = precision_vs_fp64(splat, torch, (pos, sc, rot, op, sh), cams[0],
                                                 O.View(v0, p0, fx0, fy0, cx0, cy0, w0, h0), host_targets[0],
                                                 {"chosen": tuned_options(chosen, tuned), "plain": plain_options(splat)})
    fd2 = fd_config2(splat, torch) if not args.no_checks else None

    # The other measured shapes, compact: 8 uneven views per step (3M
    # Gaussians) and the memory-bound adjoint (6M Gaussians at 3840x2160).
    batched = batched_summary(3_000_000, 5, 2) if not args.no_checks else None
    torch.cuda.empty_cache()
    memory_adjoint = memory_adjoint_summary(6_000_000, 3, 1) if not args.no_checks else None
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        if O.have_reference():
            threads = cpu_count()
            run = twin_views_per_core(O, (pos, sc, rot, op, sh), [O.View(*hemisphere_views()[i % VIEWS]) for i in range(threads)],
                                      [host_targets[i % len(host_targets)] for i in range(threads)], threads)
            per_view = float(np.mean(run["per_view_seconds"]))
            cpu = {"value": run["views"] / run["seconds"], "unit": "iters/s", "cores": threads, "kind": "reference",
                   "single_thread_seconds_per_view": per_view,
                   "sample": f"{run['views']} whole views of the same workload, one per host thread on {threads} threads "
                             f"({run['seconds']:.0f} s): the reference's FP64 twin (render, loss, gradients) and an FP64 "
                             f"Adam step; {per_view:.0f} s per view on one thread"}

    h2d = nbytes + 1240 + 128
    d2h = 160
    form = tuned.get("sort_form", chosen.sort_form)
    digits = tuned.get("digit_bits", chosen.digit_bits)
    tile_bits = max(1, math.ceil(math.log2(((WIDTH + 15) // 16) * ((HEIGHT + 15) // 16))))
    # Kernels of one step: preprocess, [histogram + passes of the depth sort],
    # count+scan, emit, histogram + passes of the entry sort, ranges, forward,
    # SSIM, loss, loss totals, backward, the fused chain rule + Adam + SH step.
    depth_launches = (1 + math.ceil(32 / digits)) if form == 0 else 0
    entry_launches = 1 + math.ceil((tile_bits + (32 if form == 1 else 0)) / digits)
    launches_per_step = 10 + depth_launches + entry_launches
    form_name = "depth then tile sort" if form == 0 else "64-bit tile|depth keys"
    out = {
        "metric": METRIC,
        "value": value, "unit": "iters/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "fwd_bwd_ms": sum(stages.get(k, 0.0) for k in ("composite", "loss", "backward")),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; the bicycle photos are not available)",
        "config": dict(bench_config(), parallelism=f"replicas x{world}"),
        "form": f"chosen: BF16 SH + BF16-pair Adam state, {form_name} with {digits}-bit digits, "
                f"{tuned.get('forward_pixels_per_thread', chosen.forward_pixels_per_thread)}-pixel compositing, "
                f"{tuned.get('backward_pixels_per_thread', chosen.backward_pixels_per_thread)}-pixel float "
                f"backward, {tuned.get('tile_size', chosen.tile_size)}x{tuned.get('tile_size', chosen.tile_size)} tiles, "
                f"batches of {tuned.get('batch_depth', chosen.batch_depth)}, "
                f"{'persistent' if tuned.get('persistent_raster', chosen.persistent_raster) else 'one block per tile'}, "
                f"{'grouped' if tuned.get('grouped_backward', chosen.grouped_backward) else 'per-splat'} backward sums "
                f"({'autotuned' if tuned else 'fixed'}), fused one-view chain rule + Adam + SH "
                "step, CUDA graph, SFU exp/log",
        "autotune": {"ms": tuned.get("ms"), "layout_ms": tuned.get("layout_ms"), "tile_ms": tuned.get("tile_ms"),
                     "grouped_ms": tuned.get("grouped_ms")},
        "workload_counts": {"tile_entries": entries, "visible_splats": visible, "reached_gaussians": reached},
        "e2e": {"value": e2e, "unit": "iters/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "sm_peaks": sm_peaks,
        "score_view_ms": score_ms,
        "densify": densify,
        "prune": prune,
        "roofline": roof,
        "stage_roofline": stage_roof,
        "stages_ms": stages,
        "plain_fp32": plain,
        "precision": precision,
        "fd_config2": fd2,
        "batched": batched,
        "memory_adjoint": memory_adjoint,
        "speedup_vs_plain": (value / world) / plain["iters_per_s"] if plain else None,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
    }
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def session_workload(args) -> None:
    """The whole training session (coarse to fine, densification rounds with
    scored views, the growth cap, the SH ramp) on the headline views: 200k
    starting points (the bench scene's means with its DC colours), 64 views at
    1237x822 kept in HBM at full, half and quarter size, 3000 iterations with
    the reference's default schedule (quarter size until 15 %, half until 35 %,
    densification every 100 iterations from 151 to 1500, 10 scored views a
    round). Against the same session at full size throughout, and with four
    views per batched step (a quarter of the iterations, the same views).
    Session iterations/s and views/s by the wall clock around the loop, one
    JSON line."""
    import torch

    splat = importlib.import_module("vibe-splat_b200")
    n = 200_000 if args.gaussians == GAUSSIANS else args.gaussians
    iterations = 3000
    pos, sc, rot, op, sh = make_scene(n)
    colors = np.clip((sh.reshape(n, -1)[:, :3] * 0.28209479177387814 + 0.5) * 255.0, 0, 255).astype(np.uint8)
    cams = [splat.Camera(v, p, fx, fy, cx, cy, w, h) for (v, p, fx, fy, cx, cy, w, h) in hemisphere_views()]
    images = list(make_targets(len(cams)))
    out = {"metric": "session iters/s, coarse to fine", "unit": "iters/s", "higher_is_better": True,
           "config": {"workload": f"{n} starting points, {len(cams)} views 1237x822 on a radius-5 hemisphere (synthetic), "
                                  f"{iterations} iterations, SH degree 2, default schedule"}}
    for name, full, batch in (("coarse_to_fine", False, 1), ("full_resolution", True, 1), ("coarse_to_fine_4_views", False, 4)):
        options = splat.SessionOptions(iterations=iterations if batch == 1 else iterations // batch, full_resolution=full,
                                       report_every=0, seed=1, views_per_step=batch)
        trainer_options = chosen_options(splat)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        session = splat.Session(pos.reshape(-1, 3).astype(np.float64), colors, cams, images, extent=5.5, typical_depth=5.0,
                                options=options, trainer_options=trainer_options)
        setup = time.perf_counter() - t0
        levels = [0, 0, 0]
        t0 = time.perf_counter()
        while not session.finished():
            session.step()
            levels[session.state().level] += 1
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
        st = session.state()
        steps = options.iterations
        out[name] = {"iters_per_s": steps / seconds, "views_per_s": steps * batch / seconds, "seconds": seconds,
                     "setup_seconds": setup,
                     "final_gaussians": st.gaussians, "densify_rounds": st.densify_rounds,
                     "densify_seconds": st.densify_seconds, "iterations_by_level": {"half": levels[0], "quarter": levels[1],
                                                                                   "full": levels[2]},
                     "last_loss": st.last_loss}
        session.close()
        torch.cuda.empty_cache()
    out["value"] = out["coarse_to_fine"]["iters_per_s"]
    out["coarse_to_fine_speedup"] = out["coarse_to_fine"]["iters_per_s"] / out["full_resolution"]["iters_per_s"]
    print(json.dumps(out))


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=30)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--workload", choices=["step", "memory-adjoint", "batched", "session"], default="step",
                        help="step: the headline one-view training step; memory-adjoint: 6M Gaussians at 3840x2160, "
                             "recompute vs store-everything backward; batched: 3M Gaussians, 8 uneven views per step; "
                             "session: a 3000-iteration coarse-to-fine training session from 200k points")
    parser.add_argument("--no-plain", action="store_true", help="skip the plain FP32 form")
    parser.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference sample")
    parser.add_argument("--no-densify", action="store_true", help="skip the densification timing")
    parser.add_argument("--no-checks", action="store_true",
                        help="skip the FP64 checks and the batched and memory-bound summaries")
    parser.add_argument("--reference-warmup", action="store_true", help="run warm-up steps in the reference arm too")
    parser.add_argument("--no-autotune", action="store_true", help="keep the chosen form's sort settings")
    parser.add_argument("--sort-form", type=int, choices=[0, 1], default=None,
                        help="override the chosen form's tile sort (0: depth then tile, 1: 64-bit tile|depth keys)")
    parser.add_argument("--form", default=None,
                        help="the chosen form's rasterizer settings instead of the autotuner's, as "
                             "pixels,tile,batch,persistent,grouped (for example 2,32,128,1,1; for profiling runs)")
    parser.add_argument("--views", type=int, default=VIEWS,
                        help="cameras cycled through (default 64; fewer keep ncu captures small)")
    parser.add_argument("--gaussians", type=int, default=GAUSSIANS,
                        help="scene size (default 1M, the headline workload; smaller cases are for ncu captures)")
    args = parser.parse_args()
    if args.workload == "memory-adjoint":
        memory_adjoint_workload(args)
    elif args.workload == "batched":
        batched_workload(args)
    elif args.workload == "session":
        session_workload(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
