"""Learned warm start for per-view geometry calibration.

A small network predicts per-view geometry offsets from the measured
projections and the reprojection of the known volume through the nominal
geometry; gradient calibration (``calibration.calibrate``) then starts from
the prediction -- or from nominal if the prediction raises the projection
loss.  No counterpart in the reference (its calibration pipeline is not
shipped); the design follows the task's description:

* input per view: two channels on a 96 x 96 grid (area-downsampled detector):
  the nominal reprojection and the masked residual ``measured - nominal``;
* 2-D encoder, 4 stages (32, 64, 128, 256 channels), each a stride-2 3x3
  convolution and a 3x3 convolution with ReLU, then a global average;
* a circular 1-D convolution across the view axis (the scan is a full turn)
  and a linear 1-D convolution to 8 offsets per view (the reference's eight
  geometry tensors; its "9 gradients" include the data tensor);
* ~1.5 M parameters, fp32 master weights, bf16 weights and activations in the
  products, fp32 accumulation: every convolution product -- forward,
  data gradient and weight gradient -- runs on the hand-written tcgen05 GEMM
  (``dgc_gemm_bf16``), with im2col/col2im kernels around it;
* trained on stacks the forward projector generates on the fly from random
  ellipsoid phantoms under random per-view perturbations, with the RMS
  reprojection distance between predicted and true geometry (mm on the
  detector) as the loss -- the calibration's own success metric, blind to the
  degenerate parameter directions.  The committed weights: 20,000 stacks from
  nominal, then 12,000 more of which half start from a partly corrected
  reference geometry (``train(residual_fraction=0.5)``), so that the network
  also refines its own estimate (``predict(stages=3)``).

Scales: training runs at 128^3 voxels and 256^2 pixels but with the physical
extent of the evaluation geometry (512 mm volume, 768 mm detector), so the
96 x 96 network input has the same millimetres per cell at training and at
evaluation (512^3, 720 views, 768^2).  Perturbations are physical:
angle 0.3 deg, source 1 mm, detector centre 2 mm, sid/sod 0.5 %.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, replace

import torch
import torch.nn.functional as F

from . import _native
from .calibration import (GEOMETRY_NAMES, ScanSetup, detector_coordinates, lattice_points,
                          simulate_measurement)
from .phantoms import circular_geometry, ellipsoid_phantom
from .source_only_forward_projector import project

INPUT_SIZE = 96


# ------------------------------------------------------------------ acquisitions


@dataclass(frozen=True)
class Acquisition:
    """A circular scan and its phantom family, in physical units (mm)."""

    volume: int          # cubic volume size [voxels]
    voxel: float         # mm
    views: int
    detector: int        # square detector [pixels]
    pixel: float         # mm
    sid: float = 1000.0
    sod: float = 600.0
    ellipsoid_mm: tuple = (10.0, 80.0)

    @property
    def scan(self) -> ScanSetup:
        return ScanSetup(U=self.detector, V=self.detector, pixel_size=self.pixel,
                         step_size=0.5 * self.voxel, voxel_size=self.voxel)

    def phantom(self, seed, device="cuda"):
        lo, hi = self.ellipsoid_mm
        return ellipsoid_phantom((self.volume,) * 3, seed=seed, voxel_size=self.voxel,
                                 device=device, axis_range=(lo / self.voxel, hi / self.voxel))

    def nominal(self, device="cuda"):
        return circular_geometry(self.views, self.detector, self.detector, self.sid, self.sod,
                                 self.pixel, device=device)


# the learned warm start is trained here ...
TRAIN = Acquisition(volume=128, voxel=4.0, views=180, detector=256, pixel=3.0)
# ... and evaluated here (the large calibration configuration)
EVAL = Acquisition(volume=512, voxel=1.0, views=720, detector=768, pixel=1.0)
# the same physical scan at half resolution (benchmark-sized)
HALF = Acquisition(volume=256, voxel=2.0, views=360, detector=384, pixel=2.0)
# config 3 as written: 256^3 of 1 mm voxels, 360 views of 384^2 1 mm pixels (a
# scan of half the physical extent the network was trained on)
CONFIG3 = Acquisition(volume=256, voxel=1.0, views=360, detector=384, pixel=1.0)

# physical perturbation model (1 sigma)
PERTURB = dict(angle_deg=0.3, src_mm=1.0, det_mm=2.0, dist_rel=0.005)

# How calibration continues from the network's start, chosen on held-out stacks
# of the training acquisition: three network stages (start 0.11-0.15 px
# there), then Adam with smaller steps than from nominal, ramped up over ten
# iterations -- Adam's first steps are lr-sized whatever the gradient and
# would throw a good start away.  0.1 px in 7-12 iterations, against 46-52
# for calibration from nominal with its own best settings.
WARM_STAGES = 3
WARM_CALIBRATION = dict(lr={"angles": 2e-3, "sid": 2.0, "sod": 2.0, "det_u0": 0.2,
                            "det_v0": 0.2, "src_x": 0.2, "src_y": 0.2, "src_z": 0.2},
                        warmup_iterations=10)


def perturb(nominal, acq: Acquisition, seed):
    """True geometry: nominal + N(0, sigma) per view (detector offsets in mm)."""
    from .calibration import perturb_geometry

    return perturb_geometry(nominal, seed, angle_deg=PERTURB["angle_deg"],
                            src_mm=PERTURB["src_mm"], det_px=PERTURB["det_mm"] / acq.pixel,
                            dist_rel=PERTURB["dist_rel"])


def output_scales(acq: Acquisition, device="cuda"):
    """Units of the eight network outputs (one sigma of the perturbation)."""
    return torch.tensor([math.radians(PERTURB["angle_deg"]), PERTURB["dist_rel"] * acq.sid,
                         PERTURB["dist_rel"] * acq.sod, PERTURB["det_mm"] / acq.pixel,
                         PERTURB["det_mm"] / acq.pixel, PERTURB["src_mm"], PERTURB["src_mm"],
                         PERTURB["src_mm"]], device=device, dtype=torch.float32)


# ------------------------------------------------------------ tensor-core ops


class _Scratch:
    error = {}

    @classmethod
    def flag(cls, device):
        key = torch.device(device).index
        if key not in cls.error:
            cls.error[key] = torch.zeros(1, dtype=torch.int32, device=device)
        return cls.error[key]


def _round8(n):
    return (n + 7) // 8 * 8


def gemm(A, B, bias=None, relu=False, out_bf16=False, out=None, accumulate=False, alpha=1.0):
    """out[m, n] = alpha * A[m] . B[n] (+ bias) (ReLU) on the tcgen05 tensor cores."""
    M, K = A.shape
    N = B.shape[0]
    if out is None:
        out = torch.empty((M, N), device=A.device,
                          dtype=torch.bfloat16 if out_bf16 else torch.float32)
    lib = _native.lib()
    _native.check(lib.dgc_gemm_bf16(
        A.data_ptr(), B.data_ptr(), out.data_ptr(), None if bias is None else bias.data_ptr(),
        M, N, K, A.stride(0), B.stride(0), out.stride(0), int(out.dtype == torch.bfloat16),
        int(relu), int(accumulate), float(alpha), _Scratch.flag(A.device).data_ptr(),
        torch.cuda.current_stream(A.device).cuda_stream))
    return out


def _padded_t(x, cols):
    """x.T as a contiguous bf16 [x.shape[1], cols] with zero columns beyond x.shape[0]."""
    out = torch.zeros((x.shape[1], cols), dtype=torch.bfloat16, device=x.device)
    out[:, : x.shape[0]] = x.t()
    return out


def _im2col(x, k, stride, pad, Kp):
    B, H, W, C = x.shape
    Ho, Wo = (H + 2 * pad - k) // stride + 1, (W + 2 * pad - k) // stride + 1
    col = torch.empty((B * Ho * Wo, Kp), dtype=torch.bfloat16, device=x.device)
    _native.check(_native.lib().dgc_im2col_nhwc_bf16(
        x.data_ptr(), B, H, W, C, k, k, stride, pad, col.data_ptr(), Kp,
        torch.cuda.current_stream(x.device).cuda_stream))
    return col, Ho, Wo


def _col2im(dcol, shape, k, stride, pad, Kp):
    B, H, W, C = shape
    dx = torch.empty(shape, dtype=torch.float32, device=dcol.device)
    _native.check(_native.lib().dgc_col2im_nhwc_f32(
        dcol.data_ptr(), B, H, W, C, k, k, stride, pad, Kp, dx.data_ptr(),
        torch.cuda.current_stream(dcol.device).cuda_stream))
    return dx


class _Conv2d(torch.autograd.Function):
    """NHWC bf16 convolution; forward, data and weight gradients on the tensor cores."""

    @staticmethod
    def forward(ctx, x, weight, bias, k, stride, pad, relu):
        Kp = weight.shape[1]
        col, Ho, Wo = _im2col(x, k, stride, pad, Kp)
        wb = weight.to(torch.bfloat16).contiguous()
        y = gemm(col, wb, bias=bias, relu=relu, out_bf16=True)
        ctx.save_for_backward(col, wb, y)
        ctx.cfg = (x.shape, k, stride, pad, relu, x.requires_grad)
        return y.view(x.shape[0], Ho, Wo, weight.shape[0])

    @staticmethod
    def backward(ctx, gy):
        col, wb, y = ctx.saved_tensors
        xshape, k, stride, pad, relu, need_dx = ctx.cfg
        g = gy.reshape(y.shape)
        if relu:
            g = g * (y > 0)
        g = g.to(torch.bfloat16).contiguous()
        M = g.shape[0]
        Mp = _round8(M)
        dw = gemm(_padded_t(g, Mp), _padded_t(col, Mp))          # [Cout, Kp] fp32
        db = g.float().sum(0)
        dx = None
        if need_dx:
            Cout = g.shape[1]
            wt = torch.zeros((wb.shape[1], _round8(Cout)), dtype=torch.bfloat16, device=g.device)
            wt[:, :Cout] = wb.t()
            if Cout % 8:
                gp = torch.zeros((M, _round8(Cout)), dtype=torch.bfloat16, device=g.device)
                gp[:, :Cout] = g
            else:
                gp = g
            dcol = gemm(gp, wt)                                    # [M, Kp] fp32
            dx = _col2im(dcol, xshape, k, stride, pad, wb.shape[1]).to(torch.bfloat16)
        return dx, dw, db, None, None, None, None


class _ViewConv(torch.autograd.Function):
    """Circular 1-D convolution across views: [A, Cin] -> [A, Cout] (bf16 in, fp32 out)."""

    @staticmethod
    def forward(ctx, f, weight, bias, k, relu):
        A, Cin = f.shape
        pad = k // 2
        col = torch.cat([torch.roll(f, shifts=pad - j, dims=0) for j in range(k)], 1)
        wb = weight.to(torch.bfloat16).contiguous()
        y = gemm(col.contiguous(), wb, bias=bias, relu=relu)
        ctx.save_for_backward(col, wb, y)
        ctx.cfg = (k, relu, Cin)
        return y

    @staticmethod
    def backward(ctx, gy):
        col, wb, y = ctx.saved_tensors
        k, relu, Cin = ctx.cfg
        g = gy * (y > 0) if relu else gy
        g = g.to(torch.bfloat16).contiguous()
        A, Cout = g.shape
        Ap = _round8(A)
        dw = gemm(_padded_t(g, Ap), _padded_t(col, Ap))
        db = g.float().sum(0)
        wt = torch.zeros((wb.shape[1], _round8(Cout)), dtype=torch.bfloat16, device=g.device)
        wt[:, :Cout] = wb.t()
        gp = g if Cout % 8 == 0 else torch.cat(
            [g, torch.zeros((A, _round8(Cout) - Cout), dtype=torch.bfloat16, device=g.device)], 1)
        dcol = gemm(gp.contiguous(), wt)                           # [A, k*Cin]
        pad = k // 2
        df = sum(torch.roll(dcol[:, j * Cin:(j + 1) * Cin], shifts=-(pad - j), dims=0)
                 for j in range(k))
        return df.to(torch.bfloat16), dw, db, None, None


class WarmStartNet(torch.nn.Module):
    """2-D encoder per view + circular 1-D convolutions across views -> 8 offsets per view."""

    CHANNELS = (32, 64, 128, 256)

    def __init__(self, in_channels=2, head_channels=256, head_kernel=5, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.convs = []
        params = []
        cin = in_channels
        for cout in self.CHANNELS:
            for stride, ci in ((2, cin), (1, cout)):
                K = 9 * ci
                w = torch.randn(cout, _round8(K), generator=g) * math.sqrt(2.0 / K)
                w[:, K:] = 0.0
                params.append(torch.nn.Parameter(w))
                params.append(torch.nn.Parameter(torch.zeros(cout)))
                self.convs.append((stride, ci, cout))
            cin = cout
        self.conv_params = torch.nn.ParameterList(params)
        hk = head_kernel
        self.w1 = torch.nn.Parameter(torch.randn(head_channels, hk * cin, generator=g) *
                                     math.sqrt(2.0 / (hk * cin)))
        self.b1 = torch.nn.Parameter(torch.zeros(head_channels))
        self.w2 = torch.nn.Parameter(torch.randn(8, 3 * head_channels, generator=g) *
                                     (0.1 / math.sqrt(3 * head_channels)))
        self.b2 = torch.nn.Parameter(torch.zeros(8))
        self.head_kernel = hk

    def forward(self, x):
        """x: [A, 96, 96, 2] bf16 -> [A, 8] fp32 (offsets in units of one sigma)."""
        h = x
        for i, (stride, _, _) in enumerate(self.convs):
            h = _Conv2d.apply(h, self.conv_params[2 * i], self.conv_params[2 * i + 1], 3, stride, 1,
                              True)
        f = h.float().mean(dim=(1, 2)).to(torch.bfloat16)
        f = _ViewConv.apply(f, self.w1, self.b1, self.head_kernel, True)
        return _ViewConv.apply(f.to(torch.bfloat16), self.w2, self.b2, 3, False)


# ----------------------------------------------------------------- data


def canvas_padding(acq) -> int:
    """Detector pixels of zero padding on each side that put a scan on the
    network's physical canvas: the training detector's extent (256 x 3 mm =
    768 mm), which the 96^2 input grid covers at 8 mm per cell.  Zero for
    scans of that extent (HALF, EVAL) and for ``acq`` None; a smaller
    detector (CONFIG3: 384 mm) is centred on the canvas, so that the network
    sees objects at the scale it was trained on (line integrals are in
    physical units already)."""
    if acq is None:
        return 0
    extent = TRAIN.detector * TRAIN.pixel
    return max(0, int(round((extent / acq.pixel - acq.detector) / 2)))


def network_input(measured, nominal_projection, mask, acq=None):
    """[A, 96, 96, 2] bf16: nominal reprojection and masked residual on the
    96^2 grid, the detector placed on the network's canvas (``canvas_padding``)."""
    pad = canvas_padding(acq)
    resid = (measured - nominal_projection) * mask
    if pad:
        nominal_projection = F.pad(nominal_projection, (pad, pad, pad, pad))
        resid = F.pad(resid, (pad, pad, pad, pad))
    p = F.interpolate(nominal_projection[:, None], size=(INPUT_SIZE, INPUT_SIZE), mode="area")
    r = F.interpolate(resid[:, None], size=(INPUT_SIZE, INPUT_SIZE), mode="area")
    x = torch.cat([p * 0.1, r], 1)                      # [A, 2, 96, 96]
    return x.permute(0, 2, 3, 1).contiguous().to(torch.bfloat16)


def make_stack(acq: Acquisition, seed, I0=1e5, device="cuda"):
    """One training/evaluation stack generated by the forward projector."""
    vol = acq.phantom(seed, device)
    nominal = acq.nominal(device)
    true = perturb(nominal, acq, seed + 1_000_003)
    scan = acq.scan
    measured, mask = simulate_measurement(vol, true, scan, I0=I0, seed=seed)
    with torch.no_grad():
        p_nom = project(vol, *nominal, scan.pixel_size, scan.U, scan.V,
                        step_size=scan.step_size, voxel_size=scan.voxel_size)
    return dict(volume=vol, nominal=nominal, true=true, measured=measured, mask=mask,
                nominal_projection=p_nom)


def predicted_geometry(net_out, nominal, acq: Acquisition):
    scales = output_scales(acq, net_out.device)
    delta = net_out * scales
    return [n + delta[:, k] for k, n in enumerate(nominal)], [delta[:, k] for k in range(8)]


def reprojection_loss(pred_geometry, true_geometry, points, pixel_size):
    """Mean squared detector distance [mm^2] over views and lattice points."""
    da = detector_coordinates(points, pred_geometry, pixel_size)
    db = detector_coordinates(points, true_geometry, pixel_size)
    return ((da - db) * pixel_size).square().sum(-1).mean()


# -------------------------------------------------------------- train / predict


def train(steps=20000, lr=1e-3, seed=0, device="cuda", log_every=500, time_budget_s=None,
          acq: Acquisition = TRAIN, checkpoint=None, init=None, residual_fraction=0.0,
          min_lr_fraction=0.05):
    """Train on ``steps`` projector-generated stacks (one stack per step).

    Stack seeds are ``1_000_000 * (seed + 1) + step``.  ``init`` continues
    from a network (and its ``meta``) instead of a fresh one.  With
    probability ``residual_fraction`` a step starts from a partly corrected
    reference geometry ``nominal + a * (true - nominal)``, a ~ U(0.5, 1): the
    input is the reprojection through that reference and its residual, the
    target the remaining offset -- what the network sees in its second and
    later stages (``predict(stages > 1)``).
    """
    prior_steps = 0
    if init is not None:
        net, prior_meta = init
        prior_steps = int(prior_meta.get("steps", 0))
    else:
        net = WarmStartNet(seed=seed).to(device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.LambdaLR(
        opt, lambda it: min_lr_fraction + (1 - min_lr_fraction) * 0.5 *
        (1 + math.cos(math.pi * min(it, steps) / steps)))
    pts = lattice_points((acq.volume,) * 3, acq.voxel, n=4, device=device)
    gen = torch.Generator().manual_seed(seed)
    scan = acq.scan
    history = []
    t0 = time.perf_counter()
    for step in range(steps):
        st = make_stack(acq, seed=1_000_000 * (seed + 1) + step, device=device)
        ref, p_ref = st["nominal"], st["nominal_projection"]
        if residual_fraction > 0 and float(torch.rand((), generator=gen)) < residual_fraction:
            a = 0.5 + 0.5 * float(torch.rand((), generator=gen))
            ref = [n + a * (t - n) for n, t in zip(st["nominal"], st["true"])]
            with torch.no_grad():
                p_ref = project(st["volume"], *ref, scan.pixel_size, scan.U, scan.V,
                                step_size=scan.step_size, voxel_size=scan.voxel_size)
        x = network_input(st["measured"], p_ref, st["mask"], acq)
        out = net(x)
        pred, _ = predicted_geometry(out, ref, acq)
        loss = reprojection_loss(pred, st["true"], pts, acq.pixel) + 1e-4 * out.square().mean()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        if log_every and (step % log_every == 0 or step == steps - 1):
            with torch.no_grad():
                base = reprojection_loss(ref, st["true"], pts, acq.pixel)
            history.append({"step": prior_steps + step, "loss_mm2": float(loss.detach()),
                            "reference_mm2": float(base), "time_s": time.perf_counter() - t0})
            print(history[-1], flush=True)
        if time_budget_s is not None and time.perf_counter() - t0 > time_budget_s:
            break
    if checkpoint:
        save(net, checkpoint, meta={"steps": prior_steps + step + 1, "history": history,
                                    "residual_fraction": residual_fraction})
    return net, history


def save(net, path, meta=None):
    torch.save({"state": {k: v.detach().cpu() for k, v in net.state_dict().items()},
                "meta": meta or {}}, path)


def load(path, device="cuda"):
    ck = torch.load(path, map_location="cpu", weights_only=False)
    net = WarmStartNet()
    net.load_state_dict(ck["state"])
    return net.to(device), ck.get("meta", {})


@torch.no_grad()
@torch.no_grad()
def predict(net, measured, nominal_projection, mask, nominal, acq: Acquisition, volume=None,
            stages=1):
    """Warm-start offsets (8 tensors [A]) for ``calibration.calibrate``.

    ``stages`` > 1 applies the network again to its own estimate: the volume
    is reprojected through the geometry predicted so far and the network
    predicts the remaining offsets from that reprojection and the new
    residual (it was trained to map (reference reprojection, residual) to
    true - reference geometry).  Needs ``volume`` for stages > 1.
    """
    out = net(network_input(measured, nominal_projection, mask, acq))
    geometry, delta = predicted_geometry(out, nominal, acq)
    scan = acq.scan
    for _ in range(1, int(stages)):
        if volume is None:
            raise ValueError("stages > 1 needs the volume")
        p = project(volume, *geometry, scan.pixel_size, scan.U, scan.V, step_size=scan.step_size,
                    voxel_size=scan.voxel_size)
        out = net(network_input(measured, p, mask, acq))
        geometry, _ = predicted_geometry(out, geometry, acq)
    return [g - n for g, n in zip(geometry, nominal)]


def evaluate(net, acq: Acquisition = HALF, seed=7, iterations=200, target_mm=0.1,
             target_angle_deg=None, stop_at_target=False, log_every=0, calibrate_kw=None,
             warm_calibrate_kw=None, stages=None):
    """Calibrate one generated stack twice: from nominal, and from the network.

    Times include everything each arm computes after the measurement exists:
    the warm-start arm adds the nominal reprojection, network input and
    inference before its calibration.  The target is ``target_mm`` RMS
    reprojection distance on the detector (0.1 mm = 0.1 px of the 768^2
    evaluation detector) and optionally ``target_angle_deg``.
    ``calibrate_kw`` applies to both arms, ``warm_calibrate_kw`` (default
    ``WARM_CALIBRATION``) to the warm-started arm on top of it; ``stages``
    (default ``WARM_STAGES``) is passed to ``predict``.
    """
    from .calibration import calibrate, lattice_points

    stages = WARM_STAGES if stages is None else stages
    warm_calibrate_kw = WARM_CALIBRATION if warm_calibrate_kw is None else warm_calibrate_kw
    st = make_stack(acq, seed=seed)
    scan = acq.scan
    pts = lattice_points(st["volume"].shape, acq.voxel, device=st["volume"].device)
    target_px = target_mm / acq.pixel
    kw = dict(iterations=iterations, true_geometry=st["true"], points=pts, target_px=target_px,
              target_angle_deg=target_angle_deg, stop_at_target=stop_at_target,
              log_every=log_every, mask=st["mask"], **(calibrate_kw or {}))
    torch.cuda.synchronize()
    plain = calibrate(st["volume"], st["measured"], st["nominal"], scan, **kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.no_grad():
        p_nom = project(st["volume"], *st["nominal"], scan.pixel_size, scan.U, scan.V,
                        step_size=scan.step_size, voxel_size=scan.voxel_size)
        warm = predict(net, st["measured"], p_nom, st["mask"], st["nominal"], acq,
                       volume=st["volume"], stages=stages)
    torch.cuda.synchronize()
    t_infer = time.perf_counter() - t0
    nn = calibrate(st["volume"], st["measured"], st["nominal"], scan, warm_start=warm,
                   **dict(kw, **(warm_calibrate_kw or {})))

    def first(h, angle):
        return next((e for e in h if e["reproj_px"] <= target_px and
                     (angle is None or e["angle_err_deg"] <= angle)), None)

    def summary(res, extra=0.0):
        h = res.history
        px = first(h, None)
        both = first(h, target_angle_deg) if target_angle_deg is not None else px
        return {"time_to_target_s": None if both is None else both["time_s"] + extra,
                "iterations_to_target": None if both is None else both["iteration"],
                "time_to_px_target_s": None if px is None else px["time_s"] + extra,
                "iterations_to_px_target": None if px is None else px["iteration"],
                "start_reproj_mm": h[0]["reproj_px"] * acq.pixel,
                "final_reproj_mm": h[-1]["reproj_px"] * acq.pixel,
                "start_angle_err_deg": h[0]["angle_err_deg"],
                "final_angle_err_deg": h[-1]["angle_err_deg"],
                "iterations": h[-1]["iteration"],
                "ms_per_iteration": 1e3 * h[-1]["time_s"] / max(h[-1]["iteration"], 1)}

    out = {"plain": summary(plain), "warm_start": summary(nn, t_infer), "stages": stages,
           "warm_calibration": {k: v for k, v in warm_calibrate_kw.items()},
           "warm_start_accepted": nn.warm_start_accepted, "inference_s": t_infer,
           "acquisition": {"volume": acq.volume, "voxel_mm": acq.voxel, "views": acq.views,
                           "detector": acq.detector, "pixel_mm": acq.pixel},
           "target_mm": target_mm, "target_angle_deg": target_angle_deg}
    tp, tn = out["plain"]["time_to_target_s"], out["warm_start"]["time_to_target_s"]
    out["speedup"] = (tp / tn) if (tp and tn) else None
    tp, tn = out["plain"]["time_to_px_target_s"], out["warm_start"]["time_to_px_target_s"]
    out["speedup_px_target"] = (tp / tn) if (tp and tn) else None
    return out


def default_checkpoint():
    from pathlib import Path

    return Path(__file__).resolve().parent / "warmstart_weights.pt"


__all__ = ["Acquisition", "TRAIN", "EVAL", "HALF", "CONFIG3", "WarmStartNet", "gemm", "make_stack",
           "network_input", "predict", "train", "save", "load", "reprojection_loss", "evaluate",
           "GEOMETRY_NAMES", "replace"]
