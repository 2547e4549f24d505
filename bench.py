"""Benchmark of the cone-beam operators at the target size (512^3, 720 x 768^2).

One step = forward projection of a 512^3 twelve-ellipsoid phantom onto 720
views of a 768x768 detector (sid 1000, sod 600, pixel 1, step 0.5, voxel 1)
followed by ``reconstruct_fdk`` of those projections into 512^3.  ``value``
is rays per second through the whole step (Grays/s) with inputs resident in
HBM; the forward projector alone (Grays/s) and the backprojection alone
(Gvoxel-views/s) are reported beside it, each kernel's algorithmic gather
bytes against the L1 / L2 ceilings measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload target512|fdk256|fdk-sharded|batch64|calib|tour|gemm]

N > 1 runs under torch.distributed (one process per GPU, NCCL).  The default
workloads give every rank its own phantom (independent objects, weak scaling,
no data-path collective); ``fdk-sharded`` splits one object's views over the
ranks (``project_sharded`` + ``reconstruct_fdk_sharded``: one all-reduce of
the volume per step, strong scaling).  Time = max over ranks.
``--impl reference`` times the reference's CPU path (the FP64 oracle port of
its CPU checks) on the host cores over a bounded, stated fraction of the same
step and prints the same line.
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

WORKLOADS = {
    "target512": dict(name="target512: project 512^3 -> 720x768^2, then reconstruct_fdk 512^3",
                      D=512, H=512, W=512, A=720, U=768, V=768, sid=1000.0, sod=600.0, pixel=1.0,
                      step=0.5, voxel=1.0, ellipsoids=12, alpha=0.8),
    "fdk256": dict(name="fdk256: project 256^3 -> 360x384^2, then reconstruct_fdk 256^3",
                   D=256, H=256, W=256, A=360, U=384, V=384, sid=1000.0, sod=600.0, pixel=1.0,
                   step=0.5, voxel=1.0, ellipsoids=12, alpha=0.8),
}
WORKLOADS["fdk-sharded"] = dict(
    WORKLOADS["target512"],
    name="fdk-sharded: one 512^3 object, its 720 views of 768^2 split over the ranks: "
         "project_sharded, then reconstruct_fdk_sharded (one volume all-reduce)")
WORKLOAD = dict(WORKLOADS["target512"])
METRIC = "fwd Grays/s, backproj Gvoxel-views/s; calib time to 0.1 px reproj, NN vs plain"
UNIT = "Grays/s"
# DRAM bytes (read + write) of one fp_forward_kernel launch of a workload at
# its nominal view count: an ncu capture of a few of its views, scaled by the
# view count (the profile summaries under profiles/ give the commands and the
# captured figures; target512: 48 views = 3 view blocks of 16).
FWD_DRAM_BYTES = {"fdk256": (351.7e6 + 17.9e6) * 15, "target512": (24.812e9 + 0.120e9) * 15}
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
    ap.add_argument("--workload", default="target512",
                    choices=["target512", "fdk256", "fdk-sharded", "batch64", "calib", "tour",
                             "gemm", "arms", "refcuda"],
                    help="target512: the FDK step at 512^3 / 720 x 768^2 (default); fdk256: the "
                         "same step at 256^3 / 360 x 384^2; fdk-sharded: one target512 object "
                         "split by views over the ranks; batch64: 64 uneven project+backward "
                         "instances, batched vs sequential; calib: calibration wall time to "
                         "0.1 px, learned warm start vs plain; tour: every kernel once on the "
                         "fdk256 instance (profiler captures); gemm: the tcgen05 GEMM at "
                         "8192^3 and at the network's largest layer shapes; arms: the forward "
                         "projector's L1 and TMA arms timed at 256^3 and 512^3; refcuda: the "
                         "reference's own CUDA operators (baseline/_ref) against this library's")
    ap.add_argument("--acq", choices=["half", "eval", "config3"], default="half",
                    help="calib: 256^3 x 2 mm / 360 / 384^2 x 2 mm (half), 512^3 / 720 / 768^2 "
                         "(eval) or 256^3 x 1 mm / 360 / 384^2 x 1 mm (config3)")
    ap.add_argument("--max-iterations", type=int, default=300, help="calib: iteration cap")
    ap.add_argument("--instances", type=int, default=64, help="batch64: number of instances")
    ap.add_argument("--batch-set", choices=["config4", "small"], default="config4",
                    help="batch64 shape sets: config4 (128^3..384x384x256, 90-720 views, "
                         "256-512 detectors) or small (48^3..64x96x96, 30-90 views, 96-160)")
    ap.add_argument("--tune-cache", default=None, help="batch64: autotuner JSON cache path")
    ap.add_argument("--seeds", type=int, default=1, help="calib: held-out seeds per arm")
    args = ap.parse_args(argv)
    base = "fdk256" if args.workload == "tour" else args.workload
    if base in WORKLOADS:
        WORKLOAD.clear()
        WORKLOAD.update(WORKLOADS[base])
        WORKLOAD["key"] = base
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


def axis_range(w):
    """Ellipsoid semi-axes of the config-2 family (10-80 voxels at 256^3),
    scaled with the volume so that a larger volume holds the same phantom."""
    f = w["D"] / 256.0
    return (10.0 * f, 80.0 * f)


def make_instance(device, seed):
    import torch

    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    w = WORKLOAD
    vol = ellipsoid_phantom((w["D"], w["H"], w["W"]), n=w["ellipsoids"], seed=seed,
                            voxel_size=w["voxel"], device=device, axis_range=axis_range(w))
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


def sharded_step(vol, geom):
    """fdk-sharded: this rank's views of one object (``geom`` holds only
    them): ``project_sharded``, then ``reconstruct_fdk_sharded`` (the volume
    all-reduce over the ranks)."""
    from dgc_b200.sharded import project_sharded, reconstruct_fdk_sharded

    w = WORKLOAD
    proj = project_sharded(vol, *geom, w["pixel"], w["U"], w["V"], step_size=w["step"],
                           voxel_size=w["voxel"])
    recon = reconstruct_fdk_sharded(proj, *geom, w["pixel"], (w["D"], w["H"], w["W"]), w["voxel"],
                                    alpha=w["alpha"], views_total=w["A"])
    return proj, recon


def measured_peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def backprojection_valid_count(geom, shape, pixel, voxel, U, V):
    """Voxel-views that pass the backprojector's mask (bp.cu:43-75: q > 1e-6,
    sid + ds_n > 1e-6, 0 <= u_idx < U-1, 0 <= v_idx < V-1): per view and
    (y, x) column the mask's u part is fixed and v_idx is linear in z, so the
    valid z form an interval, counted in closed form (FP32 on the device;
    voxels exactly on an edge of the detector may be counted either way)."""
    import torch

    D, H, W = shape
    dev = geom[0].device
    xs = (torch.arange(W, device=dev, dtype=torch.float64) - W * 0.5) * voxel
    ys = (torch.arange(H, device=dev, dtype=torch.float64) - H * 0.5) * voxel
    total = 0
    for a0 in range(0, geom[0].numel(), 32):
        g = [x[a0:a0 + 32].double().view(-1, 1, 1) for x in geom]
        beta, sid, sod, u0, v0, sx, sy, sz = g
        c, s = torch.cos(beta), torch.sin(beta)
        px = xs.view(1, 1, -1) * c + ys.view(1, -1, 1) * s
        py = -xs.view(1, 1, -1) * s + ys.view(1, -1, 1) * c
        ds_u, ds_n = sx * c + sy * s, -sx * s + sy * c
        q = sod + ds_n - py
        ll = sid + ds_n
        t = ll / q
        ui = (ds_u + t * (px - ds_u)) / pixel + u0
        ok = (q > 1e-6) & (ll > 1e-6) & (ui >= 0) & (ui < U - 1)
        # 0 <= (sz + t (vz - sz)) / pixel + v0 < V - 1, vz = (z - D/2) voxel
        lo = sz + (-v0 * pixel - sz) / t
        hi = sz + ((V - 1 - v0) * pixel - sz) / t
        zlo = torch.ceil(lo / voxel + D * 0.5).clamp(0, D)
        zhi = torch.ceil(hi / voxel + D * 0.5).clamp(0, D)
        total += int(((zhi - zlo).clamp_min(0) * ok).sum().item())
    return total


def measure_ceilings(device, repeats=5):
    """Ceilings of this GPU for the gather-bound kernels (csrc/ceilings.cu),
    best of ``repeats`` launches each, CUDA events on the launching stream:
    16-byte warp loads served by L1 and by L2 (GB/s), and FFMA warp
    instructions per second."""
    import ctypes

    import torch

    from dgc_b200 import _native

    lib = _native.lib()
    buf = torch.zeros(64 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    sink = torch.zeros(4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)
    out = {}

    def best(launch):
        rate = 0.0
        for _ in range(repeats + 1):
            amount = ctypes.c_double()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _native.check(launch(ctypes.byref(amount)))
            b.record(stream)
            b.synchronize()
            rate = max(rate, amount.value / (a.elapsed_time(b) * 1e-3))
        return rate

    for level, key, iters, stride in ((1, "l1_gather_gbs", 16384, 16),
                                      (2, "l2_gather_gbs", 4096, 16),
                                      (1, "l1_gather_bp_pattern_gbs", 16384, 27)):
        out[key] = best(lambda ref, lv=level, it=iters, st=stride: lib.dgc_ceiling_gather(
            buf.data_ptr(), buf.numel() * 4, lv, it, 4, st, sink.data_ptr(), ref,
            stream.cuda_stream)) / 1e9
    out["issue_warp_inst_per_s"] = best(lambda ref: lib.dgc_ceiling_issue(
        2048, 4, sink.data_ptr(), ref, stream.cuda_stream))
    out["source"] = ("csrc/ceilings.cu, measured in this run: 16-byte warp loads of 512 "
                     "contiguous bytes from a 32 KiB (L1) or 64 MiB (L2) buffer in random "
                     "order; the same from L1 with lanes 1.69 quads apart (the "
                     "backprojector's spread at magnification 1.67); independent FFMA chains")
    del buf
    return out


# ------------------------------------------------------------- CPU baseline


def cpu_baseline_sample(vol_np, geom_np, threads=None, fwd_views=(0,), ray_stride=1, filt_views=1,
                        slab=4, bp_views=None):
    """Time the FP64 oracle (a port of the reference's CPU checks) on a bounded sample.

    Sample: the forward projection of every ``ray_stride``-th ray of views
    ``fwd_views``, the FDK filter of ``filt_views`` views, and the
    backprojection of a ``slab``-slice z-slab over the first ``bp_views``
    views (default all).  Each part is scaled to the full step by its share
    of the work.  Returns (seconds per full step, threads used, description,
    fraction of the step's work computed).
    """
    import numpy as np

    from oracle import oracle

    if threads:
        oracle.set_num_threads(threads)
    w = WORKLOAD
    A, U, V = w["A"], w["U"], w["V"]
    bp_views = A if bp_views is None else int(bp_views)
    rays = np.concatenate([np.arange(a * U * V, (a + 1) * U * V, ray_stride, dtype=np.int64)
                           for a in fwd_views])
    t0 = time.perf_counter()
    oracle.project_rays(vol_np, geom_np, w["pixel"], U, V, w["step"], w["voxel"], rays, mode=1)
    fwd_share = rays.size / (A * U * V)
    t_fwd = (time.perf_counter() - t0) / fwd_share
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
    bp_share = (slab / w["D"]) * (bp_views / A)
    t_bp = (time.perf_counter() - t0) / bp_share
    t_step = t_fwd + t_filt + t_bp
    # fraction of the step computed, weighting each part by its share of the
    # full step's CPU time
    fraction = (t_fwd * fwd_share + t_filt * filt_views / A + t_bp * bp_share) / t_step
    desc = (f"FP64 oracle on {oracle.num_threads()} threads: forward of every {ray_stride}-th ray "
            f"of {len(fwd_views)} view(s) ({rays.size} rays), filter of {filt_views} view(s), "
            f"backprojection of a {slab}-slice slab over {bp_views} views; each part timed and "
            f"scaled by its share of the full step")
    return t_step, oracle.num_threads(), desc, fraction


def host_threads():
    import torch

    return {"os_cpu_count": os.cpu_count(), "torch_num_threads": torch.get_num_threads()}


# ------------------------------------------------------------------------ arms


def run_reference(args):
    """The reference's CPU path (oracle port) on the host cores; rank 0 only."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np

    w = WORKLOAD
    # the same phantom as the GPU arm, generated on the CPU
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    vol = ellipsoid_phantom((w["D"], w["H"], w["W"]), n=w["ellipsoids"], seed=instance_seed(0),
                            voxel_size=w["voxel"], device="cpu", axis_range=axis_range(w)).numpy()
    geom = [g.numpy().astype(np.float64) for g in
            circular_geometry(w["A"], w["U"], w["V"], w["sid"], w["sod"], w["pixel"], device="cpu")]
    # a bounded sample per step (about two seconds of host work), so that the
    # driver's --steps/--warmup run ends within minutes; each step samples a
    # different view
    big = w["D"] >= 512
    sample = dict(ray_stride=4 if big else 2, filt_views=1, slab=2, bp_views=w["A"] // 2)
    for i in range(args.warmup):
        cpu_baseline_sample(vol, geom, fwd_views=(i % w["A"],), **sample)
    times, fractions = [], []
    threads, desc = 1, ""
    for i in range(args.steps):
        view = (37 * (i + 1)) % w["A"]
        t, threads, desc, frac = cpu_baseline_sample(vol, geom, fwd_views=(view,), **sample)
        times.append(t)
        fractions.append(frac)
    t_step = sum(times) / len(times)
    rays = w["A"] * w["U"] * w["V"]
    value = rays / t_step / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": w["name"], "volume": [w["D"], w["H"], w["W"]],
                                        "views": w["A"], "detector": [w["U"], w["V"]]},
        "sample_fraction": statistics.mean(fractions),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": desc + "; one such sample per step, its time scaled to the "
                                          "full step (sample_fraction = share computed)",
                         **host_threads()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def forward_traffic(w, views):
    """Measured DRAM bytes of one forward launch over ``views`` views of
    workload ``w`` (FWD_DRAM_BYTES scaled by the view count), or None when
    none was measured for its volume and detector sizes."""
    traffic = FWD_DRAM_BYTES.get(w.get("key", ""))
    nominal = WORKLOADS.get(w.get("key", ""), {})
    if traffic is None or any(w[k] != nominal[k] for k in ("D", "H", "W", "U", "V")):
        return None
    return traffic * views / nominal["A"]


def run_ours(args):
    import numpy as np
    import torch

    from dgc_b200 import _native, _ops
    from dgc_b200.sharded import view_shard

    world, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs CUDA devices")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    w = WORKLOAD
    sharded = args.workload == "fdk-sharded"
    # fdk-sharded: one object (same seed on every rank), this rank's views;
    # otherwise an object per rank with all views
    vol, geom = make_instance(device, instance_seed(0 if sharded else rank))
    run_step = step
    if sharded:
        views = view_shard(w["A"], world, rank)
        geom = [g[views.start:views.stop].contiguous() for g in geom]
        run_step = sharded_step
    A_local = geom[0].numel()
    R_local = A_local * w["U"] * w["V"]
    R_job = w["A"] * w["U"] * w["V"] * (1 if sharded else world)
    N_local = w["D"] * w["H"] * w["W"] * A_local
    counts = _ops.project_sample_counts((w["D"], w["H"], w["W"]), geom, w["pixel"], w["U"], w["V"],
                                        w["step"], w["voxel"])
    S = int(counts.sum().item())
    del counts
    n_valid = backprojection_valid_count(geom, (w["D"], w["H"], w["W"]), w["pixel"], w["voxel"],
                                         w["U"], w["V"])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    ceilings = measure_ceilings(device)

    for _ in range(max(args.warmup, 1)):
        run_step(vol, geom)
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
            run_step(vol, geom)
            stops[i].record()
        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    total_ms = max_over_ranks(sum(step_ms), dist, device)
    ms_per_step = total_ms / args.steps
    value = R_job * args.steps / (total_ms * 1e-3) / 1e9
    kern = {}
    for name, ms in tr.records:
        kern.setdefault(name, []).append(ms)
    launches = len(tr.records)
    fwd_ms = max_over_ranks(statistics.mean(kern["fp_forward_kernel"]), dist, device)
    bp_key = "bp_forward_kernel<fdk>" if "bp_forward_kernel<fdk>" in kern else \
        "bp_forward_kernel<fdk-partial>"
    bp_ms = max_over_ranks(statistics.mean(kern[bp_key]), dist, device) if bp_key in kern else None

    # ---- end to end through the public API with host buffers
    vol_host = vol.cpu().pin_memory()
    out_host = torch.empty_like(vol_host).pin_memory()
    e_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_stop = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    vol_dev = torch.empty_like(vol)
    for _ in range(max(1, min(args.warmup, 2))):
        vol_dev.copy_(vol_host, non_blocking=True)
        _, r = run_step(vol_dev, geom)
        out_host.copy_(r, non_blocking=True)
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    for i in range(args.steps):
        flush.zero_()
        e_start[i].record()
        vol_dev.copy_(vol_host, non_blocking=True)
        _, r = run_step(vol_dev, geom)
        out_host.copy_(r, non_blocking=True)
        e_stop[i].record()
    torch.cuda.synchronize(device)
    serial_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_start, e_stop)), dist,
                               device)
    serial_value = R_job * args.steps / (serial_ms * 1e-3) / 1e9

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
            _, r = run_step(bufs[b], geom)
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
    e2e_value = R_job * args.steps / (e2e_ms * 1e-3) / 1e9
    nbytes = vol.numel() * 4

    # ---- rooflines: algorithmic bytes per launch over the kernel's average
    # duration, against the L1 ceiling of 16-byte gathers measured above
    hbm_peak, hbm_kind = measured_peak_hbm()
    l1 = ceilings["l1_gather_gbs"]
    fwd_bytes = 32 * S + 4 * R_local  # two 16-byte quads per sample + projection writes
    fwd_gbs = fwd_bytes / (fwd_ms * 1e-3) / 1e9
    traffic = forward_traffic(w, A_local)
    roofline = {"bound": "l1", "kernel": "fp_forward_kernel", "achieved": fwd_gbs, "peak": l1,
                "unit": "GB/s", "frac": fwd_gbs / l1,
                "peak_source": "l1_gather_gbs of this run's ceilings (csrc/ceilings.cu)",
                "traffic": traffic, "algorithmic_bytes": fwd_bytes, "samples": S, "ms": fwd_ms,
                "l2_frac": fwd_gbs / ceilings["l2_gather_gbs"],
                "dram_gbs": None if traffic is None else traffic / (fwd_ms * 1e-3) / 1e9,
                "hbm_peak_gbs": hbm_peak, "hbm_peak_source": f"{hbm_kind} hbm_gbs"}
    rooflines = {"fp_forward_kernel": {k: roofline[k] for k in ("achieved", "frac", "ms")}}
    bp_bytes = 16 * n_valid + 4 * w["D"] * w["H"] * w["W"] + 4 * R_local
    if bp_ms is not None:
        bp_gbs = bp_bytes / (bp_ms * 1e-3) / 1e9
        rooflines[bp_key] = {"bound": "l1", "achieved": bp_gbs, "frac": bp_gbs / l1, "ms": bp_ms,
                             "frac_of_bp_pattern": bp_gbs / ceilings["l1_gather_bp_pattern_gbs"],
                             "algorithmic_bytes": bp_bytes, "valid_voxel_views": n_valid}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": w["name"], "volume": [w["D"], w["H"], w["W"]],
                   "views": w["A"], "detector": [w["U"], w["V"]], "sid": w["sid"], "sod": w["sod"],
                   "step": w["step"], "pixel": w["pixel"], "voxel": w["voxel"],
                   "ellipsoids": w["ellipsoids"], "semi_axes_voxels": list(axis_range(w)),
                   "l2": "flushed between timed steps (256 MiB write); inputs exceed L2",
                   "parallelism": (f"views split over {world} ranks, one all-reduce of the "
                                   f"volume per step" if sharded else
                                   f"independent objects x{world}")},
        "fwd_grays_per_s": world * R_local / (fwd_ms * 1e-3) / 1e9,
        "backproj_gvoxel_views_per_s": None if bp_ms is None else
        world * N_local / (bp_ms * 1e-3) / 1e9,
        "kernel_ms": {k: statistics.mean(v) for k, v in kern.items()},
        "gpu_launches": launches,
        "roofline": roofline,
        "rooflines": rooflines,
        "ceilings": ceilings,
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
        t_cpu, threads, desc, frac = cpu_baseline_sample(
            vol_np, geom_np, fwd_views=(0, w["A"] // 3), ray_stride=1, filt_views=2, slab=4)
        line["cpu_baseline"] = {"value": w["A"] * w["U"] * w["V"] / t_cpu / 1e9, "unit": UNIT,
                                "cores": threads, "kind": "port", "sample": desc,
                                "sample_fraction": frac, **host_threads()}
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
    the nominal reprojection and the network inference.  ``--seeds`` held-out
    stacks (seeds 7, 8, ...; the network was trained on seeds >= 10^6), each
    with its own clock record; the line gives the median and the range."""
    import torch

    from dgc_b200 import warmstart as WS

    torch.cuda.set_device(0)
    acq = {"half": WS.HALF, "eval": WS.EVAL, "config3": WS.CONFIG3}[args.acq]
    net, meta = WS.load(WS.default_checkpoint())
    runs = []
    for k in range(max(1, args.seeds)):
        seed = 7 + k
        with ClockSampler(0) as clocks:
            res = WS.evaluate(net, acq, seed=seed, iterations=args.max_iterations,
                              target_mm=0.1 * acq.pixel, target_angle_deg=0.05,
                              stop_at_target=True)
        res["seed"] = seed
        res["clocks"] = clocks.summary()
        runs.append(res)

    def spread(values):
        vals = [v for v in values if v is not None]
        if not vals:
            return None
        return {"median": statistics.median(vals), "min": min(vals), "max": max(vals),
                "n": len(vals), "of": len(values)}

    def arm(name, key):
        return spread([r[name][key] for r in runs])

    summary = {
        "plain_time_to_0.1px_s": arm("plain", "time_to_px_target_s"),
        "warm_time_to_0.1px_s": arm("warm_start", "time_to_px_target_s"),
        "plain_time_to_0.1px_and_0.05deg_s": arm("plain", "time_to_target_s"),
        "warm_time_to_0.1px_and_0.05deg_s": arm("warm_start", "time_to_target_s"),
        "speedup_to_0.1px": spread([r["speedup_px_target"] for r in runs]),
        "speedup_to_0.1px_and_0.05deg": spread([r["speedup"] for r in runs]),
    }
    warm = summary["warm_time_to_0.1px_s"]
    line = {
        "metric": "calibration wall time to 0.1 px RMS reprojection error", "unit": "s",
        "value": None if warm is None else warm["median"], "higher_is_better": False,
        "n_gpus": 1, "steps": len(runs), "warmup": 0, "dtype": "f32 (network bf16/fp32)",
        "data": "synthetic", "vs_baseline": None,
        "config": {"workload": f"calibration {acq.volume}^3 x {acq.voxel} mm, {acq.views} views, "
                               f"{acq.detector}^2 x {acq.pixel} mm detector, config-3 "
                               "perturbations, Poisson I0=1e5",
                   "acquisition": args.acq, "seeds": [r["seed"] for r in runs],
                   "max_iterations": args.max_iterations, "target_px": 0.1,
                   "target_angle_deg": 0.05, "network_training_steps": meta.get("steps")},
        "summary": summary,
        "runs": [{k: r[k] for k in ("seed", "plain", "warm_start", "speedup_px_target", "speedup",
                                    "warm_start_accepted", "inference_s", "clocks")}
                 for r in runs],
        "stages": runs[0]["stages"], "warm_calibration": runs[0]["warm_calibration"],
        "clocks": runs[-1]["clocks"],
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------- tour


def run_tour(args):
    """Every kernel of the library on the fdk256 instance (honouring --views /
    --volume / --detector), ``--steps`` times: project, its backward with the
    volume gradient, the fused calibration step, backproject and its backward
    (all nine gradients, then the geometry's alone), reconstruct_fdk, the
    filter's backward, a two-instance batched step and one warm-start network
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
        g3 = [t.detach().requires_grad_() for t in geom]  # geometry only (self-calibration)
        b = cb.backproject(p.detach(), *g3, w["pixel"], shape, w["voxel"])
        torch.autograd.grad(b, g3, grad_outputs=torch.ones_like(b))
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
    with ClockSampler(0) as clocks:
        for _ in range(max(1, args.steps)):
            with _native.trace() as tr:
                one_pass()
                torch.cuda.synchronize()
            kern = {}
            for name, ms in tr.records:
                kern[name] = round(kern.get(name, 0.0) + ms, 4)
    print(json.dumps({"workload": "tour: " + w["name"], "kernel_ms": kern,
                      "clocks": clocks.summary()}))
    return 0


# --------------------------------------------------------------------- arms


def run_arms(args):
    """The forward projector's arms -- quads through L1 (march unrolled once
    or twice, CTAs in view blocks of 0, 16 or 64), volume bricks staged by TMA
    (slabs of 2 or 4 cells), z pairs through L1 -- on the fdk256 and target512
    phantoms and scans, each timed on ``--views`` views (default 48) with CUDA
    events (median of ``--steps``), checked bitwise equal, with the autotuner's
    choice per volume bucket."""
    import torch

    from dgc_b200 import _native, _ops
    from dgc_b200.autotune import FORWARD_ARMS, arm_name

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    lib = _native.lib()
    out = {}
    with ClockSampler(0) as clocks:
        for key in ("fdk256", "target512"):
            WORKLOAD.clear()
            WORKLOAD.update(WORKLOADS[key])
            w = WORKLOAD
            views = args.views or 48
            WORKLOAD["A"] = views
            vol, geom = make_instance(device, instance_seed(0))
            res, ref = {}, None
            for arm, slab, unroll, vb in FORWARD_ARMS:
                _native.check(lib.dgc_fp_clear_arm_rules())
                _native.check(lib.dgc_fp_add_arm_rule(1 << 62, arm, slab, unroll, vb))

                def run():
                    return _ops.fp_forward(vol, *geom, w["pixel"], w["U"], w["V"], w["step"],
                                           w["voxel"])
                for _ in range(max(1, args.warmup)):
                    p = run()
                times = []
                for _ in range(max(3, args.steps)):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record()
                    p = run()
                    b.record()
                    b.synchronize()
                    times.append(a.elapsed_time(b))
                ms = statistics.median(times)
                spread = [min(times), max(times)]
                same = None if ref is None else bool(torch.equal(p, ref))
                if ref is None:
                    ref = p
                res[arm_name(arm, slab, unroll, vb)] = {
                    "ms": ms, "ms_range": spread,
                    "grays_per_s": views * w["U"] * w["V"] / (ms * 1e-3) / 1e9,
                    "bitwise_equal_to_l1": same}
            _native.check(lib.dgc_fp_clear_arm_rules())
            out[key] = {"views": views, "volume": w["D"], "detector": w["U"], "arms": res}
            del vol, geom, ref, p
            torch.cuda.empty_cache()
    print(json.dumps({"workload": "forward projector arms", "results": out,
                      "clocks": clocks.summary()}))
    return 0


# --------------------------------------------------------------------- gemm


def load_reference_cuda():
    """The reference's own native operators, from its pip installation under
    ``baseline/_ref`` (built for sm_100 from its sources), loaded by file path
    under their module names without entering ``sys.modules`` (the names are
    this package's shims too).  None when the installation is absent."""
    import importlib.machinery
    import importlib.util

    root = ROOT / "baseline" / "_ref"
    mods = []
    for name in ("src_cbct_forwardprojector_cuda", "src_cbct_backprojector_cuda"):
        found = sorted(root.glob(name + ".*.so"))
        if not found:
            return None
        loader = importlib.machinery.ExtensionFileLoader(name, str(found[0]))
        spec = importlib.util.spec_from_file_location(name, str(found[0]), loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        mods.append(mod)
    return mods


def run_refcuda(args):
    """The GPU bar: the reference's own CUDA operators (``load_reference_cuda``)
    against this library's on the same instance, stream and GPU -- forward
    projection, its backward with all nine gradients, backprojection, its
    backward with all nine -- on the fdk256 instance (honouring --views), and
    the forward projection and backprojection of the target512 instance
    (one timed call each).  CUDA events, median of ``--steps`` after
    ``--warmup`` calls, clocks sampled; every operator's output is compared
    with the reference's (max relative L2 over its outputs)."""
    import statistics

    import torch

    from dgc_b200 import _ops

    ref = load_reference_cuda()
    if ref is None:
        print(json.dumps({"workload": "refcuda", "unavailable": "baseline/_ref is not installed"}))
        return 0
    ref_fp, ref_bp = ref
    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)

    def timed(fn, warmup, steps):
        out = None
        for _ in range(max(1, warmup)):
            out = fn()
        torch.cuda.synchronize(device)
        ts = []
        for _ in range(max(1, steps)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts), out

    def rel(x, y):
        xs = x if isinstance(x, (list, tuple)) else [x]
        ys = y if isinstance(y, (list, tuple)) else [y]
        worst = 0.0
        for a, b in zip(xs, ys):
            if a is None or b is None or b.numel() == 0:
                continue
            n = float(b.double().norm())
            worst = max(worst, float((a.double() - b.double()).norm()) / n if n > 0 else 0.0)
        return worst

    out = {}
    with ClockSampler(0) as clocks:
        for key in ("fdk256", "target512"):
            WORKLOAD.clear()
            WORKLOAD.update(WORKLOADS[key])
            if key == "fdk256" and args.views:
                WORKLOAD["A"] = args.views
            w = WORKLOAD
            vol, geom = make_instance(device, instance_seed(0))
            px, U, V, st, vx = w["pixel"], w["U"], w["V"], w["step"], w["voxel"]
            D, H, W = w["D"], w["H"], w["W"]
            full = key == "fdk256"
            warm, steps = (args.warmup, args.steps) if full else (1, 1)
            ops = {
                "project": (lambda: _ops.fp_forward(vol, *geom, px, U, V, st, vx),
                            lambda: ref_fp.forward(vol, *geom, px, U, V, st, vx, 0.0, 0.0, 0.0)),
            }
            proj = _ops.fp_forward(vol, *geom, px, U, V, st, vx)
            ops["backproject"] = (lambda: _ops.bp_forward(proj, *geom, px, D, H, W, vx),
                                  lambda: ref_bp.forward(proj, *geom, px, D, H, W, vx, 0.0, 0.0,
                                                         0.0))
            if full:
                ops["project_backward"] = (
                    lambda: _ops.fp_backward(proj, vol, *geom, px, st, vx, True),
                    lambda: ref_fp.backward(proj, vol, *geom, px, st, vx, True, 0.0, 0.0, 0.0))
                ops["backproject_backward"] = (
                    lambda: _ops.bp_backward(vol, proj, *geom, px, vx),
                    lambda: ref_bp.backward(vol, proj, *geom, px, vx, 0.0, 0.0, 0.0))
            res = {}
            for name, (mine, theirs) in ops.items():
                t_ours, o_ours = timed(mine, warm, steps)
                t_ref, o_ref = timed(theirs, warm, steps)
                res[name] = {"ours_ms": t_ours, "reference_ms": t_ref, "speedup": t_ref / t_ours,
                             "max_rel_l2_vs_reference": rel(o_ours, o_ref)}
                del o_ours, o_ref
            out[w["name"]] = res
            del vol, geom, proj, ops
            torch.cuda.empty_cache()
    print(json.dumps({"workload": "refcuda: the reference's own CUDA operators (baseline/_ref) "
                                  "vs this library, same GPU and stream", "results": out,
                      "clocks": clocks.summary()}))
    return 0


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
    clocks = ClockSampler(0).__enter__()
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
    clocks.__exit__(None, None, None)
    print(json.dumps({"workload": "tcgen05 bf16 GEMM", "peak_bf16_tflops": peak,
                      "peak_source": peak_source, "shapes": out, "clocks": clocks.summary()}))
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.workload == "gemm":
        return run_gemm(args)
    if args.workload == "arms":
        return run_arms(args)
    if args.workload == "tour":
        return run_tour(args)
    if args.workload == "refcuda":
        return run_refcuda(args)
    if args.workload == "calib":
        return run_calib(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch64":
        return run_batch64(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
