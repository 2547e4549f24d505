"""Benchmark of the cone-beam operators on the FDK workload (256^3, 360 x 384^2).

One step = forward projection of a 256^3 twelve-ellipsoid phantom onto 360
views of a 384x384 detector (sid 1000, sod 600, pixel 1, step 0.5, voxel 1)
followed by ``reconstruct_fdk`` of those projections into 256^3 -- the
"plain FDK at medium size" workload.  ``value`` is rays per second through the
whole step (Grays/s) with inputs resident in HBM; the forward projector alone
(Grays/s) and the backprojection alone (Gvoxel-views/s) are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed (one process per GPU, NCCL): every rank
reconstructs its own phantom (independent objects, weak scaling, no data-path
collective); time = max over ranks.  ``--impl reference`` times the
reference's CPU path (the FP64 oracle port of its CPU checks) on the host
cores over a bounded sample of the same workload and prints the same line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (str(ROOT / "diff-geocali_b200"), str(ROOT)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOAD = dict(name="fdk256: project 256^3 -> 360x384^2, then reconstruct_fdk 256^3",
                D=256, H=256, W=256, A=360, U=384, V=384, sid=1000.0, sod=600.0, pixel=1.0,
                step=0.5, voxel=1.0, ellipsoids=12, alpha=0.8)
METRIC = "fwd Grays/s, backproj Gvoxel-views/s; calib time to 0.1 px reproj, NN vs plain"
UNIT = "Grays/s"
# DRAM bytes (read + write) of one 360-view fp_forward_kernel launch: an ncu
# capture of the 24-view case (bench.py --workload tour --views 24) measured
# 351.7 + 17.9 MB, scaled by the view count (x15).
FWD_DRAM_BYTES_PER_LAUNCH = (351.7e6 + 17.9e6) * 15
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--views", type=int, default=None,
                    help="override the view count (smaller cases for profiler captures)")
    ap.add_argument("--volume", type=int, default=None, help="override the cubic volume size")
    ap.add_argument("--detector", type=int, default=None, help="override the square detector size")
    ap.add_argument("--workload", choices=["fdk256", "batch64", "calib", "tour", "gemm"],
                    default="fdk256",
                    help="fdk256: the FDK step (default); batch64: 64 uneven project+backward "
                         "instances, batched vs sequential; calib: calibration wall time to "
                         "0.1 px, learned warm start vs plain; tour: every kernel once on the "
                         "fdk256 instance (profiler captures); gemm: the tcgen05 GEMM at "
                         "8192^3 and at the network's largest layer shapes")
    ap.add_argument("--acq", choices=["half", "eval"], default="half",
                    help="calib: 256^3/360/384^2 (half) or 512^3/720/768^2 (eval)")
    ap.add_argument("--max-iterations", type=int, default=300, help="calib: iteration cap")
    ap.add_argument("--instances", type=int, default=64, help="batch64: number of instances")
    ap.add_argument("--batch-set", choices=["config4", "small"], default="config4",
                    help="batch64 shape sets: config4 (128^3..384x384x256, 90-720 views, "
                         "256-512 detectors) or small (48^3..64x96x96, 30-90 views, 96-160)")
    ap.add_argument("--tune-cache", default=None, help="batch64: autotuner JSON cache path")
    args = ap.parse_args(argv)
    if args.views:
        WORKLOAD["A"] = args.views
    if args.volume:
        WORKLOAD["D"] = WORKLOAD["H"] = WORKLOAD["W"] = args.volume
    if args.detector:
        WORKLOAD["U"] = WORKLOAD["V"] = args.detector
    if args.views or args.volume or args.detector:
        w = WORKLOAD
        w["name"] = (f"project {w['D']}^3 -> {w['A']}x{w['U']}^2, then reconstruct_fdk "
                     f"{w['D']}^3 (profiling size)")
    return args


# ----------------------------------------------------------------- distributed


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    import datetime

    import torch.distributed as dist

    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist if world > 1 else None


def max_over_ranks(value: float, dist, device) -> float:
    """Maximum of a per-rank float over all ranks (identity for one rank)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def instance_seed(rank: int) -> int:
    """Each rank reconstructs its own phantom (independent objects)."""
    return 1000 + rank


# ---------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.file = None
        self.device_index = device_index

    def __enter__(self):
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.device_index).uuid)
            target = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            target = str(self.device_index)
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", target], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if self.proc is None or self.file is None:
            return None
        self.file.flush()
        rows = []
        with open(self.file.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ------------------------------------------------------------------- workload


def make_instance(device, seed):
    import torch

    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    w = WORKLOAD
    vol = ellipsoid_phantom((w["D"], w["H"], w["W"]), n=w["ellipsoids"], seed=seed,
                            voxel_size=w["voxel"], device=device)
    geom = circular_geometry(w["A"], w["U"], w["V"], w["sid"], w["sod"], w["pixel"], device=device)
    torch.cuda.synchronize(device)
    return vol, geom


def step(vol, geom):
    import cbct_backprojector as cb

    w = WORKLOAD
    proj = cb.project(vol, *geom, w["pixel"], w["U"], w["V"], step_size=w["step"],
                      voxel_size=w["voxel"])
    recon = cb.reconstruct_fdk(proj, *geom, w["pixel"], (w["D"], w["H"], w["W"]), w["voxel"],
                               alpha=w["alpha"])
    return proj, recon


def measured_peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------- CPU baseline


def cpu_baseline_sample(vol_np, geom_np, threads=None, fwd_rays=None, filt_views=1, slab=4,
                        bp_views=None):
    """Time the FP64 oracle (a port of the reference's CPU checks) on a bounded sample.

    Sample: the forward projection of the first ``fwd_rays`` rays of view 0
    (default one full view), the FDK filter of ``filt_views`` views, and the
    backprojection of a ``slab``-slice z-slab over the first ``bp_views``
    views (default all).  Each part is scaled to the full step by its share of
    the work.  Returns (seconds per full step, threads used, description).
    """
    import numpy as np

    from oracle import oracle

    if threads:
        oracle.set_num_threads(threads)
    w = WORKLOAD
    A, U, V = w["A"], w["U"], w["V"]
    fwd_rays = U * V if fwd_rays is None else int(fwd_rays)
    bp_views = A if bp_views is None else int(bp_views)
    t0 = time.perf_counter()
    rays = np.arange(0, fwd_rays, dtype=np.int64)
    oracle.project_rays(vol_np, geom_np, w["pixel"], U, V, w["step"], w["voxel"], rays, mode=1)
    t_fwd = (time.perf_counter() - t0) * (A * U * V / fwd_rays)
    proj_part = np.ones((filt_views, U, V), np.float32)
    t0 = time.perf_counter()
    filt = oracle.fdk_filter(proj_part, w["pixel"], geom_np[2][:filt_views],
                             geom_np[1][:filt_views], w["alpha"])
    t_filt = (time.perf_counter() - t0) * (A / filt_views)
    proj_all = np.broadcast_to(filt[:1], (bp_views, U, V))
    t0 = time.perf_counter()
    # the central slab: slab voxel z' sits where full-volume voxel D/2 - slab/2 + z' does
    oracle.backproject(proj_all, [g[:bp_views] for g in geom_np], w["pixel"],
                       (slab, w["H"], w["W"]), w["voxel"], offset=(0.0, 0.0, 0.0))
    t_bp = (time.perf_counter() - t0) * (w["D"] / slab) * (A / bp_views)
    desc = (f"FP64 oracle on {oracle.num_threads()} threads: forward of {fwd_rays} rays of one "
            f"view, filter of {filt_views} view(s), backprojection of a {slab}-slice slab over "
            f"{bp_views} views; each scaled to the full step")
    return t_fwd + t_filt + t_bp, oracle.num_threads(), desc


# ------------------------------------------------------------------------ arms


def run_reference(args):
    """The reference's CPU path (oracle port) on the host cores; rank 0 only."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    import torch

    w = WORKLOAD
    # the same phantom as the GPU arm, generated on the CPU
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    vol = ellipsoid_phantom((w["D"], w["H"], w["W"]), n=w["ellipsoids"], seed=instance_seed(0),
                            voxel_size=w["voxel"], device="cpu").numpy()
    geom = [g.numpy().astype(np.float64) for g in
            circular_geometry(w["A"], w["U"], w["V"], w["sid"], w["sod"], w["pixel"], device="cpu")]
    # a small sample per step (a few seconds of host work), so that the
    # driver's --steps/--warmup run ends within minutes
    sample = dict(fwd_rays=w["U"] * w["V"] // 2, filt_views=1, slab=2, bp_views=w["A"] // 2)
    for _ in range(args.warmup):
        cpu_baseline_sample(vol, geom, **sample)
    times = []
    threads, desc = 1, ""
    for _ in range(args.steps):
        t, threads, desc = cpu_baseline_sample(vol, geom, **sample)
        times.append(t)
    t_step = sum(times) / len(times)
    rays = w["A"] * w["U"] * w["V"]
    value = rays / t_step / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": w["name"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    del torch
    return 0


def run_ours(args):
    import numpy as np
    import torch

    from dgc_b200 import _native, _ops

    world, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs CUDA devices")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    w = WORKLOAD
    vol, geom = make_instance(device, instance_seed(rank))
    R = w["A"] * w["U"] * w["V"]
    N = w["D"] * w["H"] * w["W"] * w["A"]
    counts = _ops.project_sample_counts((w["D"], w["H"], w["W"]), geom, w["pixel"], w["U"], w["V"],
                                        w["step"], w["voxel"])
    S = int(counts.sum().item())
    del counts
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    for _ in range(max(args.warmup, 1)):
        step(vol, geom)
    torch.cuda.synchronize(device)

    # ---- device-resident timed region
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clocks, _native.trace() as tr:
        for i in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            starts[i].record()
            step(vol, geom)
            stops[i].record()
        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    total_ms = max_over_ranks(sum(step_ms), dist, device)
    ms_per_step = total_ms / args.steps
    value = world * R * args.steps / (total_ms * 1e-3) / 1e9
    kern = {}
    for name, ms in tr.records:
        kern.setdefault(name, []).append(ms)
    launches = len(tr.records)
    fwd_ms = statistics.mean(kern["fp_forward_kernel"])
    bp_ms = statistics.mean(kern["bp_forward_kernel<fdk>"])
    fwd_ms = max_over_ranks(fwd_ms, dist, device)
    bp_ms = max_over_ranks(bp_ms, dist, device)

    # ---- end to end through the public API with host buffers
    vol_host = vol.cpu().pin_memory()
    out_host = torch.empty_like(vol_host).pin_memory()
    e_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_stop = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    vol_dev = torch.empty_like(vol)
    for _ in range(max(1, min(args.warmup, 2))):
        vol_dev.copy_(vol_host, non_blocking=True)
        _, r = step(vol_dev, geom)
        out_host.copy_(r, non_blocking=True)
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    for i in range(args.steps):
        flush.zero_()
        e_start[i].record()
        vol_dev.copy_(vol_host, non_blocking=True)
        _, r = step(vol_dev, geom)
        out_host.copy_(r, non_blocking=True)
        e_stop[i].record()
    torch.cuda.synchronize(device)
    serial_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_start, e_stop)), dist,
                               device)
    serial_value = world * R * args.steps / (serial_ms * 1e-3) / 1e9

    # ---- the same K steps as a stream of jobs: step i+1's volume upload and
    # step i-1's reconstruction download run on a copy stream while step i
    # computes (two device input buffers, two pinned host outputs); timed from
    # the first upload to the last download
    copy = torch.cuda.Stream(device)
    cur = torch.cuda.current_stream(device)
    bufs = [torch.empty_like(vol), torch.empty_like(vol)]
    outs = [out_host, torch.empty_like(vol_host).pin_memory()]
    uploaded = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]

    def pipelined(nsteps, t0=None, t1=None):
        copy.wait_stream(cur)
        with torch.cuda.stream(copy):
            if t0 is not None:
                t0.record(copy)
            bufs[0].copy_(vol_host, non_blocking=True)
            uploaded[0].record(copy)
        for i in range(nsteps):
            b = i % 2
            if i + 1 < nsteps:
                nb = (i + 1) % 2
                with torch.cuda.stream(copy):
                    if i >= 1:
                        copy.wait_event(consumed[nb])  # step i-1 has read buffer nb
                    bufs[nb].copy_(vol_host, non_blocking=True)
                    uploaded[nb].record(copy)
            flush.zero_()
            cur.wait_event(uploaded[b])
            _, r = step(bufs[b], geom)
            consumed[b].record(cur)
            with torch.cuda.stream(copy):
                copy.wait_event(consumed[b])
                outs[b].copy_(r, non_blocking=True)
                r.record_stream(copy)
        cur.wait_stream(copy)
        if t1 is not None:
            t1.record(cur)

    pipelined(max(2, min(args.warmup, 3)))
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    p_start, p_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pipelined(args.steps, p_start, p_stop)
    torch.cuda.synchronize(device)
    e2e_ms = max_over_ranks(p_start.elapsed_time(p_stop), dist, device)
    e2e_value = world * R * args.steps / (e2e_ms * 1e-3) / 1e9
    nbytes = vol.numel() * 4

    # ---- roofline of the dominant kernel (forward projector)
    peak, peak_kind = measured_peak_hbm()
    alg_bytes = 32 * S + 4 * R  # trilinear gathers + projection writes per launch
    achieved = alg_bytes / (fwd_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "fp_forward_kernel", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                "traffic": FWD_DRAM_BYTES_PER_LAUNCH, "algorithmic_bytes": alg_bytes,
                "samples": S, "ms": fwd_ms}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["name"], "volume": [w["D"], w["H"], w["W"]],
                   "views": w["A"], "detector": [w["U"], w["V"]], "sid": w["sid"], "sod": w["sod"],
                   "step": w["step"], "ellipsoids": w["ellipsoids"],
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"independent objects x{world}"},
        "fwd_grays_per_s": world * R / (fwd_ms * 1e-3) / 1e9,
        "backproj_gvoxel_views_per_s": world * N / (bp_ms * 1e-3) / 1e9,
        "kernel_ms": {k: statistics.mean(v) for k, v in kern.items()},
        "gpu_launches": launches,
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "ms_per_step": e2e_ms / args.steps,
                "transfers": "volume upload and reconstruction download of every step, on a "
                             "copy stream overlapping the neighbouring steps' compute",
                "serial": {"value": serial_value, "ms_per_step": serial_ms / args.steps}},
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vol_np = vol.cpu().numpy()
        geom_np = [g.cpu().numpy().astype(np.float64) for g in geom]
        t_cpu, threads, desc = cpu_baseline_sample(vol_np, geom_np)
        line["cpu_baseline"] = {"value": R / t_cpu / 1e9, "unit": UNIT, "cores": threads,
                                "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ batch64

BATCH64 = dict(name="batch64: uneven instances, project + backward (volume and geometry "
                    "gradients) each, one persistent launch per pass, CUDA graph",
               volumes=[(128, 128, 128), (128, 192, 192), (256, 256, 256), (256, 384, 384)],
               views=[90, 180, 360, 720], detectors=[256, 384, 512], sid=1000.0, sod=600.0,
               voxel=1.0, step=0.5, seed=4)
BATCH_SMALL = dict(BATCH64, name="batch64 small: many small uneven instances (hypotheses on "
                                 "downsampled data), project + backward each",
                   volumes=[(48, 48, 48), (64, 64, 64), (64, 96, 96)], views=[30, 60, 90],
                   detectors=[96, 128, 160])


def make_batch64(device, n, seed, c=None):
    """``n`` problems drawn from the seed: volume shape, views and detector U, V
    independently from the shape set ``c`` (default BATCH64); config-3
    perturbations of the nominal circular geometry; the pixel size makes the
    detector cover the magnified volume."""
    import numpy as np

    from dgc_b200.batch import Problem
    from dgc_b200.calibration import perturb_geometry
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    c = BATCH64 if c is None else c
    rng = np.random.default_rng(seed)
    problems = []
    for i in range(n):
        D, H, W = c["volumes"][rng.integers(len(c["volumes"]))]
        A = int(c["views"][rng.integers(len(c["views"]))])
        U = int(c["detectors"][rng.integers(len(c["detectors"]))])
        V = int(c["detectors"][rng.integers(len(c["detectors"]))])
        px = 1.2 * max(D, H, W) * c["voxel"] * (c["sid"] / c["sod"]) / min(U, V)
        vol = ellipsoid_phantom((D, H, W), n=12, seed=seed * 1000 + i, voxel_size=c["voxel"],
                                device=device)
        nominal = circular_geometry(A, U, V, c["sid"], c["sod"], px, device=device)
        true = perturb_geometry(nominal, seed * 1000 + i)
        problems.append(Problem(vol, true, px, U, V, c["step"], c["voxel"]))
    return problems


def plain_step(problems):
    """The baseline: one ``project`` call and its autograd backward per instance."""
    import torch

    import cbct_backprojector as cb

    for pr in problems:
        vol = pr.volume.detach().requires_grad_()
        geom = [g.detach().requires_grad_() for g in pr.geometry]
        p = cb.project(vol, *geom, pr.pixel_size, pr.U, pr.V, step_size=pr.step_size,
                       voxel_size=pr.voxel_size)
        torch.autograd.grad(p, [vol, *geom], grad_outputs=p.detach())


def run_batch64(args):
    import torch

    from dgc_b200 import _native, _ops
    from dgc_b200.autotune import Autotuner
    from dgc_b200.batch import ProjectionBatch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    shapes = BATCH64 if args.batch_set == "config4" else BATCH_SMALL
    problems = make_batch64(device, args.instances, shapes["seed"] + 1000 * rank, shapes)
    R = sum(pr.rays for pr in problems)
    S = 0
    for pr in problems:
        S += int(_ops.project_sample_counts(tuple(pr.volume.shape), pr.geometry, pr.pixel_size,
                                            pr.U, pr.V, pr.step_size, pr.voxel_size).sum().item())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    torch.cuda.synchronize(device)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()
        ms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return max_over_ranks(sum(ms), dist, device) / steps

    t0 = time.perf_counter()
    tuner = Autotuner(cache_path=args.tune_cache)
    tuner.choose(problems)
    tune_s = time.perf_counter() - t0
    batch = ProjectionBatch(problems)
    seq_ms = timed(lambda: plain_step(problems), args.steps, max(1, args.warmup // 2))
    eager_ms = timed(batch.step, args.steps, 1)
    batch.capture()
    with ClockSampler(local) as clocks:
        graph_ms = timed(batch.replay, args.steps, args.warmup)
    with _native.trace() as tr:
        batch.step()
        torch.cuda.synchronize(device)
    kern = {}
    for name, ms in tr.records:
        kern[name] = kern.get(name, 0.0) + ms

    # end to end: volumes from pinned host memory, geometry gradients back
    host_vols = [pr.volume.cpu().pin_memory() for pr in problems]
    host_gg = [torch.empty(g.shape, dtype=torch.float32).pin_memory() for g in batch.grad_geometry]

    def e2e_step():
        for hv, pr in zip(host_vols, problems):
            pr.volume.copy_(hv, non_blocking=True)
        batch.replay()
        for hg, g in zip(host_gg, batch.grad_geometry):
            hg.copy_(g, non_blocking=True)

    e2e_ms = timed(e2e_step, args.steps, 1)
    h2d = sum(v.numel() * 4 for v in host_vols)
    d2h = sum(g.numel() * 4 for g in host_gg)
    peak, peak_kind = measured_peak_hbm()
    bwd_ms = kern.get("batch_backward_kernel", float("nan"))
    alg = 64 * S + 4 * R  # adjoint: 8 gathers + 8 scatters per sample
    achieved = alg / (bwd_ms * 1e-3) / 1e9
    value = world * R / (graph_ms * 1e-3) / 1e9
    line = {
        "metric": "total Grays/s (forward + backward over all instances)", "value": value,
        "unit": "Grays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": graph_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": shapes["name"], "instances": len(problems),
                   "rays": R, "samples": S, "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"independent batches x{world}"},
        "sequential_plain_calls": {"ms_per_step": seq_ms,
                                   "value": world * R / (seq_ms * 1e-3) / 1e9},
        "batched_eager": {"ms_per_step": eager_ms, "value": world * R / (eager_ms * 1e-3) / 1e9},
        "speedup_vs_sequential": seq_ms / graph_ms,
        "autotune": {"seconds": tune_s, "buckets_measured": len(tuner.measured),
                     "tiles": sorted({f"{a},{b}" for a, b in (pr.tiles for pr in problems)})},
        "kernel_ms": kern, "gpu_launches": len(tr.records),
        "roofline": {"bound": "hbm", "kernel": "batch_backward_kernel", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} hbm_gbs", "traffic": None,
                     "algorithmic_bytes": alg, "ms": bwd_ms},
        "e2e": {"value": world * R / (e2e_ms * 1e-3) / 1e9, "unit": "Grays/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "memory_gb": torch.cuda.max_memory_allocated(device) / 1e9,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line))
    del batch
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# -------------------------------------------------------------------- calib


def run_calib(args):
    """Wall time to 0.1 px RMS reprojection error, and to 0.1 px together with
    0.05 deg RMS angle error: calibration from the network's warm start vs
    from nominal, same GPU, same projector, each arm with its own settings;
    every iteration timed on the host, the warm-start arm's time includes
    the nominal reprojection and the network inference."""
    import torch

    from dgc_b200 import warmstart as WS

    torch.cuda.set_device(0)
    acq = WS.HALF if args.acq == "half" else WS.EVAL
    net, meta = WS.load(WS.default_checkpoint())
    res = WS.evaluate(net, acq, seed=7, iterations=args.max_iterations, target_mm=0.1 * acq.pixel,
                      target_angle_deg=0.05, stop_at_target=True)
    p, n = res["plain"], res["warm_start"]
    line = {
        "metric": "calibration wall time to 0.1 px RMS reprojection error", "unit": "s",
        "value": n["time_to_px_target_s"], "higher_is_better": False, "n_gpus": 1,
        "steps": 1, "warmup": 0, "dtype": "f32 (network bf16/fp32)", "data": "synthetic",
        "vs_baseline": None,
        "config": {"workload": f"calibration {acq.volume}^3 x {acq.voxel} mm, {acq.views} views, "
                               f"{acq.detector}^2 x {acq.pixel} mm detector, config-3 "
                               "perturbations, Poisson I0=1e5",
                   "max_iterations": args.max_iterations, "target_px": 0.1,
                   "target_angle_deg": 0.05, "network_training_steps": meta.get("steps")},
        "plain": p, "warm_start": n,
        "speedup_to_0.1px": res["speedup_px_target"],
        "speedup_to_0.1px_and_0.05deg": res["speedup"],
        "stages": res["stages"], "warm_calibration": res["warm_calibration"],
        "warm_start_accepted": res["warm_start_accepted"], "inference_s": res["inference_s"],
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------- tour


def run_tour(args):
    """Every kernel of the library on the fdk256 instance (honouring --views /
    --volume / --detector), ``--steps`` times: project, its backward with the
    volume gradient, the fused calibration step, backproject and its backward,
    reconstruct_fdk, the filter's backward, a two-instance batched step and one warm-start network
    forward/backward (tensor-core GEMMs).  Prints the per-kernel device times
    of the last pass; meant for profiler captures of small cases."""
    import torch

    import cbct_backprojector as cb
    from dgc_b200 import _native, _ops
    from dgc_b200 import warmstart as WS
    from dgc_b200.batch import Problem, ProjectionBatch

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    w = WORKLOAD
    vol, geom = make_instance(device, instance_seed(0))
    shape = (w["D"], w["H"], w["W"])
    meas = cb.project(vol, *geom, w["pixel"], w["U"], w["V"], step_size=w["step"],
                      voxel_size=w["voxel"]) * 1.01
    net = WS.WarmStartNet().to(device)
    x = torch.randn(12, WS.INPUT_SIZE, WS.INPUT_SIZE, 2, device=device).to(torch.bfloat16)
    problems = [Problem(vol, geom, w["pixel"], w["U"], w["V"], w["step"], w["voxel"]),
                Problem(vol[: w["D"] // 2].contiguous(), [g[: max(1, w["A"] // 2)] for g in geom],
                        w["pixel"], w["U"], w["V"], w["step"], w["voxel"])]
    batch = ProjectionBatch(problems)

    def one_pass():
        v = vol.detach().requires_grad_()
        g = [t.detach().requires_grad_() for t in geom]
        p = cb.project(v, *g, w["pixel"], w["U"], w["V"], step_size=w["step"],
                       voxel_size=w["voxel"])
        torch.autograd.grad(p, [v, *g], grad_outputs=p.detach())
        _ops.fp_mse_grad(vol, geom, w["pixel"], w["U"], w["V"], w["step"], w["voxel"], meas,
                         None, 1.0 / meas.numel())
        pr = p.detach().requires_grad_()
        g2 = [t.detach().requires_grad_() for t in geom]
        b = cb.backproject(pr, *g2, w["pixel"], shape, w["voxel"])
        torch.autograd.grad(b, [pr, *g2], grad_outputs=torch.ones_like(b))
        cb.reconstruct_fdk(p.detach(), *geom, w["pixel"], shape, w["voxel"], alpha=w["alpha"])
        pf = p.detach().requires_grad_()
        sid = geom[1].detach().requires_grad_()
        f = cb.fdk_filter(pf, w["pixel"], geom[2], sid, w["alpha"])
        torch.autograd.grad(f, [pf, sid], grad_outputs=torch.ones_like(f))
        batch.step()
        out = net(x)
        out.square().sum().backward()

    for _ in range(max(0, args.warmup)):
        one_pass()
    torch.cuda.synchronize()
    kern = {}
    for _ in range(max(1, args.steps)):
        with _native.trace() as tr:
            one_pass()
            torch.cuda.synchronize()
        kern = {}
        for name, ms in tr.records:
            kern[name] = round(kern.get(name, 0.0) + ms, 4)
    print(json.dumps({"workload": "tour: " + w["name"], "kernel_ms": kern}))
    return 0


# --------------------------------------------------------------------- gemm


def run_gemm(args):
    """TFLOP/s of the tcgen05 BF16 GEMM (fp32 out) against the measured cuBLAS
    bf16 peak: 8192^3, and the forward / weight-gradient products of the
    network's widest layer on 360 views (M = 360*6*6, N = 256, K = 9*256;
    M = 256, N = 2304, K = 360*6*6)."""
    import torch

    from dgc_b200 import _native
    from dgc_b200.warmstart import gemm

    torch.cuda.set_device(0)
    try:
        peak = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"])
        peak_source = "measured bf16_tflops"
    except Exception:
        peak, peak_source = FALLBACK_BF16_TFLOPS, "fallback"
    shapes = [(8192, 8192, 8192), (360 * 36, 256, 2304), (256, 2304, 360 * 36)]
    out = {}
    g = torch.Generator(device="cuda").manual_seed(0)
    for M, N, K in shapes:
        A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
        C = torch.empty(M, N, device="cuda")
        for _ in range(max(1, args.warmup)):
            gemm(A, B, out=C)
        torch.cuda.synchronize()
        times = []
        for _ in range(max(1, args.steps)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            gemm(A, B, out=C)
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
        ms = sorted(times)[len(times) // 2]
        with _native.trace() as tr:
            gemm(A, B, out=C)
            torch.cuda.synchronize()
        tf = 2.0 * M * N * K / (ms * 1e-3) / 1e12
        err = float(((C - A.float() @ B.float().t()).abs().max()).item())
        out[f"{M}x{N}x{K}"] = {"ms": ms, "tflops": tf, "kernels": sorted({n for n, _ in tr.records}),
                               "frac_of_measured_peak":
                               None if peak is None else tf / peak, "max_abs_err": err}
    print(json.dumps({"workload": "tcgen05 bf16 GEMM", "peak_bf16_tflops": peak,
                      "peak_source": peak_source, "shapes": out}))
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.workload == "gemm":
        return run_gemm(args)
    if args.workload == "tour":
        return run_tour(args)
    if args.workload == "calib":
        return run_calib(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch64":
        return run_batch64(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
