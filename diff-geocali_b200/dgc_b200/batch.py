"""Batched forward projection + backward over many uneven problems.

A ``ProjectionBatch`` holds N independent ``project`` problems -- each with its
own volume size, views, detector and per-view geometry -- and runs all of them
as a handful of launches of ``libdgc.so``:

* one launch re-lays out every volume into its quad-packed copy;
* one persistent launch marches every ray of every problem, its CTAs taking
  (problem, view, ray tile) items from a work queue;
* for the backward, one persistent launch of the adjoint / geometry-gradient
  kernel over the same queue, one launch of the per-view FP64 reductions and
  one of the volume-gradient folds.

Results equal those of ``project`` and its autograd backward problem by
problem (forward and geometry gradients bitwise for the same tile shape; the
volume gradient up to the order of its float atomics).  Because nothing on
the host runs between the launches, a forward+backward step can be captured
into a CUDA graph once (``capture``) and replayed.  No counterpart in the
reference, which runs one problem per call.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _native
from ._ops import _GEOM_NAMES


@dataclass
class Problem:
    """One ``project`` problem: the arguments of ``project`` for one volume."""

    volume: torch.Tensor                  # [D, H, W] float32, CUDA
    geometry: list                        # eight [A] float32 CUDA tensors (reference order)
    pixel_size: float
    U: int
    V: int
    step_size: float = 0.2
    voxel_size: float = 1.0
    offset: tuple = (0.0, 0.0, 0.0)
    grad_projections: torch.Tensor | None = None  # None: the forward output (grad of 0.5*|p|^2)
    tiles: tuple = field(default=(0, 0))  # (forward, backward) columns per CTA tile; 0 = 8

    @property
    def rays(self) -> int:
        return int(self.geometry[0].numel()) * int(self.U) * int(self.V)


def _check_problem(i, pr: Problem):
    def req(cond, msg):
        if not cond:
            raise RuntimeError(f"problem {i}: {msg}")

    req(isinstance(pr.volume, torch.Tensor) and pr.volume.dim() == 3,
        "volume must be a [D,H,W] tensor")
    req(pr.volume.is_cuda and pr.volume.dtype == torch.float32, "volume must be float32 CUDA")
    req(len(pr.geometry) == 8, "geometry must hold eight per-view tensors")
    A = pr.geometry[0].numel()
    for name, t in zip(_GEOM_NAMES, pr.geometry):
        req(t.is_cuda and t.dtype == torch.float32 and t.device == pr.volume.device,
            f"{name} must be float32 on the volume's device")
        req(t.numel() == A, f"{name} must contain A elements")
    if pr.grad_projections is not None:
        g = pr.grad_projections
        req(g.is_cuda and g.dtype == torch.float32 and g.device == pr.volume.device and
            tuple(g.shape) == (A, int(pr.U), int(pr.V)),
            "grad_projections must be float32 [A,U,V] on the volume's device")


class ProjectionBatch:
    """N ``project`` problems run together (forward and backward).

    Outputs, allocated once and overwritten by every run:
    ``projections[i]`` [A,U,V], ``grad_volumes[i]`` [D,H,W] (if
    ``grad_volume``) and ``grad_geometry[i]`` [8, A] (reference order).
    """

    def __init__(self, problems, grad_volume=True):
        problems = list(problems)
        if not problems:
            raise RuntimeError("a batch needs at least one problem")
        for i, pr in enumerate(problems):
            _check_problem(i, pr)
        self.problems = problems
        self.device = problems[0].volume.device
        if any(pr.volume.device != self.device for pr in problems):
            raise RuntimeError("all problems of a batch must be on one device")
        self._keep = []
        self.projections, self.grad_volumes, self.grad_geometry = [], [], []
        arr = (_native.FpInstance * len(problems))()
        for i, pr in enumerate(problems):
            vol = pr.volume.contiguous()
            geom = [t.contiguous() for t in pr.geometry]
            A, U, V = geom[0].numel(), int(pr.U), int(pr.V)
            proj = torch.zeros((A, U, V), dtype=torch.float32, device=self.device)
            gproj = proj if pr.grad_projections is None else pr.grad_projections.contiguous()
            gvol = torch.zeros(vol.shape, dtype=torch.float32, device=self.device) \
                if grad_volume else None
            ggeo = torch.zeros((8, A), dtype=torch.float32, device=self.device)
            self._keep += [vol, gproj, *geom]
            self.projections.append(proj)
            self.grad_volumes.append(gvol)
            self.grad_geometry.append(ggeo)
            D, H, W = vol.shape
            inst = arr[i]
            inst.volume = vol.data_ptr()
            inst.D, inst.H, inst.W = int(D), int(H), int(W)
            for name, t in zip(_GEOM_NAMES, geom):
                setattr(inst, name, t.data_ptr())
            inst.A, inst.U, inst.V = int(A), U, V
            inst.pixel_size = float(pr.pixel_size)
            inst.step_size = float(pr.step_size)
            inst.voxel_size = float(pr.voxel_size)
            inst.off_x, inst.off_y, inst.off_z = (float(x) for x in pr.offset)
            inst.projections = proj.data_ptr()
            inst.grad_projections = gproj.data_ptr()
            inst.grad_volume = None if gvol is None else gvol.data_ptr()
            inst.grad_geometry = ggeo.data_ptr()
            inst.tile_forward, inst.tile_backward = (int(x) for x in pr.tiles)
        self._instances = arr
        lib = _native.lib()
        nbytes = lib.dgc_batch_workspace_bytes(arr, len(problems))
        if nbytes == 0:
            raise RuntimeError("invalid batch shapes")
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        self.plan = _native.BatchPlan()
        with torch.cuda.device(self.device):
            _native.check(lib.dgc_batch_prepare(arr, len(problems), self.workspace.data_ptr(),
                                                int(nbytes), ctypes.byref(self.plan),
                                                torch.cuda.current_stream().cuda_stream))
        self.rays = int(self.plan.rays)
        self._graph = None

    def __len__(self):
        return len(self.problems)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def forward(self):
        """Projections of every problem into ``projections``."""
        with torch.cuda.device(self.device):
            _native.check(_native.lib().dgc_batch_project(ctypes.byref(self.plan), self._stream()))
        return self.projections

    def backward(self, rebuild_quads=False):
        """Volume and geometry gradients of every problem.

        ``rebuild_quads=False`` reuses the packed volumes of the last
        ``forward`` (valid while the volumes are unchanged).
        """
        with torch.cuda.device(self.device):
            _native.check(_native.lib().dgc_batch_project_backward(
                ctypes.byref(self.plan), int(bool(rebuild_quads)), self._stream()))
        return self.grad_volumes, self.grad_geometry

    def step(self):
        """Forward then backward (quads built once)."""
        self.forward()
        self.backward(rebuild_quads=False)

    def capture(self):
        """Capture one ``step`` into a CUDA graph (after one eager warm-up step)."""
        self.step()
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.device(self.device), torch.cuda.graph(graph):
            self.step()
        self._graph = graph
        return graph

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()


__all__ = ["Problem", "ProjectionBatch"]
