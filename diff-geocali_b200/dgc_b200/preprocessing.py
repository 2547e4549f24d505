"""Raw detector frames to the line integrals the operators take.

The reference requires dark/flat-field correction and the negative log
upstream of its operators (README.md:108) and transposes frames stored
[A,V,U] with ``permute(0,2,1)`` (docs/USAGE.md:247-251); it ships no code for
either.  ``preprocess`` does both in one kernel pass (``dgc_preprocess``).
"""

from __future__ import annotations

import torch

from . import _native


def preprocess(raw, dark=None, flat=None, layout="AVU", min_ratio=1e-6):
    """``-log(max((raw - dark) / (flat - dark), min_ratio))`` as float32 [A,U,V].

    ``raw``: CUDA float32 frames, ``layout`` "AVU" ([A,V,U], U fastest) or
    "AUV"; ``dark`` / ``flat``: one frame in the same layout ([V,U] or [U,V])
    or None (0 / 1).  Ratios below ``min_ratio`` (and 0/0) are clamped to it.
    """
    if layout not in ("AVU", "AUV"):
        raise ValueError("layout must be 'AVU' or 'AUV'")
    if not (isinstance(raw, torch.Tensor) and raw.is_cuda and raw.dtype == torch.float32
            and raw.dim() == 3):
        raise ValueError("raw must be a 3-D float32 CUDA tensor")
    if not min_ratio > 0:
        raise ValueError("min_ratio must be positive")
    raw = raw.contiguous()
    A = raw.shape[0]
    if layout == "AVU":
        V, U = raw.shape[1], raw.shape[2]
    else:
        U, V = raw.shape[1], raw.shape[2]
    frames = []
    for name, f in (("dark", dark), ("flat", flat)):
        if f is None:
            frames.append(None)
            continue
        if not (isinstance(f, torch.Tensor) and f.is_cuda and f.dtype == torch.float32 and
                tuple(f.shape) == tuple(raw.shape[1:]) and f.device == raw.device):
            raise ValueError(f"{name} must be one float32 CUDA frame shaped like raw[0]")
        frames.append(f.contiguous())
    out = torch.empty((A, U, V), dtype=torch.float32, device=raw.device)
    with torch.cuda.device(raw.device):
        _native.check(_native.lib().dgc_preprocess(
            raw.data_ptr(), None if frames[0] is None else frames[0].data_ptr(),
            None if frames[1] is None else frames[1].data_ptr(), A, U, V,
            int(layout == "AVU"), float(min_ratio), out.data_ptr(),
            torch.cuda.current_stream(raw.device).cuda_stream))
    return out


__all__ = ["preprocess"]
