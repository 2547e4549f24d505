"""Synthetic ellipsoid phantoms and circular-orbit geometry.

Workload definitions of the benchmark configurations (no real data is
needed): a volume is the sum of ``n`` ellipsoids with uniform attenuation,
centres uniform in the inner 70 % of the field, semi-axes uniform in
``axis_range`` voxels, uniform Euler angles and attenuation uniform in
``mu_range`` per unit length.  Generated on the target device with torch.
"""

from __future__ import annotations

import math

import torch


def _rotation(alpha, beta, gamma):
    ca, sa = math.cos(alpha), math.sin(alpha)
    cb, sb = math.cos(beta), math.sin(beta)
    cg, sg = math.cos(gamma), math.sin(gamma)
    rz1 = torch.tensor([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]], dtype=torch.float64)
    ry = torch.tensor([[cb, 0.0, sb], [0.0, 1.0, 0.0], [-sb, 0.0, cb]], dtype=torch.float64)
    rz2 = torch.tensor([[cg, -sg, 0.0], [sg, cg, 0.0], [0.0, 0.0, 1.0]], dtype=torch.float64)
    return rz1 @ ry @ rz2


def ellipsoid_parameters(shape, n=12, seed=0, voxel_size=1.0, axis_range=(10.0, 80.0),
                         mu_range=(0.05, 0.5)):
    """List of (centre_xyz, semi_axes_xyz, rotation 3x3, mu) in world units."""
    g = torch.Generator().manual_seed(int(seed))
    D, H, W = shape
    extent = torch.tensor([W, H, D], dtype=torch.float64) * voxel_size
    out = []
    for _ in range(n):
        u = torch.rand(3, generator=g, dtype=torch.float64)
        centre = (u - 0.5) * 0.7 * extent
        axes = (axis_range[0] + (axis_range[1] - axis_range[0]) *
                torch.rand(3, generator=g, dtype=torch.float64)) * voxel_size
        eul = torch.rand(3, generator=g, dtype=torch.float64) * 2 * math.pi
        mu = mu_range[0] + (mu_range[1] - mu_range[0]) * torch.rand(1, generator=g).item()
        out.append((centre, axes, _rotation(*eul.tolist()), mu))
    return out


def ellipsoid_phantom(shape, n=12, seed=0, voxel_size=1.0, offset=(0.0, 0.0, 0.0),
                      device="cuda", axis_range=(10.0, 80.0), mu_range=(0.05, 0.5)):
    """float32 [D,H,W] phantom; voxel (z,y,x) at ((x-W/2)*vs+off_x, ...) as the operators use."""
    D, H, W = shape
    params = ellipsoid_parameters(shape, n, seed, voxel_size, axis_range, mu_range)
    dev = torch.device(device)
    xs = (torch.arange(W, device=dev, dtype=torch.float32) - W * 0.5) * voxel_size + offset[0]
    ys = (torch.arange(H, device=dev, dtype=torch.float32) - H * 0.5) * voxel_size + offset[1]
    zs = (torch.arange(D, device=dev, dtype=torch.float32) - D * 0.5) * voxel_size + offset[2]
    vol = torch.zeros((D, H, W), dtype=torch.float32, device=dev)
    chunk = 32
    for z0 in range(0, D, chunk):
        zc = zs[z0:z0 + chunk, None, None]
        block = vol[z0:z0 + chunk]
        for centre, axes, rot, mu in params:
            r = rot.tolist()
            c = centre.tolist()
            a = axes.tolist()
            px = xs[None, None, :] - c[0]
            py = ys[None, :, None] - c[1]
            pz = zc - c[2]
            # body coordinates q = R^T p, scaled by the semi-axes
            q0 = (r[0][0] * px + r[1][0] * py + r[2][0] * pz) / a[0]
            q1 = (r[0][1] * px + r[1][1] * py + r[2][1] * pz) / a[1]
            q2 = (r[0][2] * px + r[1][2] * py + r[2][2] * pz) / a[2]
            block += (q0.square() + q1.square() + q2.square() <= 1.0).float() * mu
    return vol


def circular_geometry(A, U, V, sid, sod, pixel_size=1.0, device="cuda", full_turn=True):
    """Eight float32 [A] tensors for a nominal circular scan (detector centred)."""
    dev = torch.device(device)
    span = 2 * math.pi if full_turn else math.pi
    angles = torch.arange(A, dtype=torch.float32, device=dev) * (span / A)
    full = lambda x: torch.full((A,), float(x), dtype=torch.float32, device=dev)  # noqa: E731
    return [angles, full(sid), full(sod), full((U - 1) / 2.0), full((V - 1) / 2.0),
            full(0.0), full(0.0), full(0.0)]
