"""Seeded synthetic single-axis tilt series for tests and benchmarks.

A phantom is a set of ellipsoids (semi-axes, density, random orientation) and
Gaussian blobs (sigma, amplitude) on a constant background inside a volume of
nx (x) by ny (y, the tilt axis) by nz (z, thickness) voxels.  Projections are
exact line integrals, computed slice by slice: with the tilt axis along y, the
ray of detector pixel (u, y) stays in the plane y = const, where every
ellipsoid cuts an ellipse and every blob a 2-D Gaussian, whose chords have
closed forms.  Noise is additive Gaussian with variance var(clean)/SNR over the
whole stack (that is the SNR definition used throughout).

Works with torch on the CPU or on a GPU (the maths is the same); object
parameters always come from a CPU generator so the phantom does not depend on
the device.  This module only makes input data; it is not part of the
reconstruction path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class Phantom:
    shape: tuple            # (nx, ny, nz)
    centers: torch.Tensor   # (E, 3) ellipsoid centres, voxel units, origin at the volume centre
    amat: torch.Tensor      # (E, 3, 3) quadratic form R diag(1/a^2) R^T
    dens: torch.Tensor      # (E,)
    bcent: torch.Tensor     # (G, 3) blob centres
    bsig: torch.Tensor      # (G,)
    bamp: torch.Tensor      # (G,)
    background: float


def _random_rotations(g: torch.Generator, n: int) -> torch.Tensor:
    q = torch.randn(n, 4, generator=g, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    R = torch.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], dim=1)
    return R.view(n, 3, 3)


def make_phantom(shape, n_ellipsoids, n_blobs=0, seed=0, semi=(2.0, 20.0), density=(0.2, 1.0),
                 sigma=(1.0, 4.0), amplitude=(0.5, 2.0), background=0.0) -> Phantom:
    nx, ny, nz = shape
    g = torch.Generator().manual_seed(int(seed))
    ext = torch.tensor([nx, ny, nz], dtype=torch.float64)
    E = int(n_ellipsoids)
    cen = (torch.rand(E, 3, generator=g, dtype=torch.float64) - 0.5) * ext
    ax = semi[0] + (semi[1] - semi[0]) * torch.rand(E, 3, generator=g, dtype=torch.float64)
    dens = density[0] + (density[1] - density[0]) * torch.rand(E, generator=g, dtype=torch.float64)
    R = _random_rotations(g, E)
    amat = R @ torch.diag_embed(1.0 / ax ** 2) @ R.transpose(1, 2)
    G = int(n_blobs)
    bcent = (torch.rand(G, 3, generator=g, dtype=torch.float64) - 0.5) * ext
    bsig = sigma[0] + (sigma[1] - sigma[0]) * torch.rand(G, generator=g, dtype=torch.float64)
    bamp = amplitude[0] + (amplitude[1] - amplitude[0]) * torch.rand(G, generator=g, dtype=torch.float64)
    return Phantom(tuple(shape), cen, amat, dens, bcent, bsig, bamp, float(background))


def tilt_angles(lo=-60.0, hi=60.0, step=2.0) -> np.ndarray:
    n = int(round((hi - lo) / step)) + 1
    return (lo + step * np.arange(n)).astype(np.float32)


def project(ph: Phantom, tilts_deg, ys=None, device="cpu", chunk=16) -> torch.Tensor:
    """Clean projections rows[s, i, k] = line integral at tilt i, detector
    pixel k, of volume slice ys[s].  Returns float32 (S, ntilt, nx)."""
    nx, ny, nz = ph.shape
    if ys is None:
        ys = range(ny)
    ys = list(ys)
    dev = torch.device(device)
    th = torch.tensor(np.asarray(tilts_deg, dtype=np.float64) * math.pi / 180.0, device=dev)
    ct, st = torch.cos(th), torch.sin(th)                          # (T,)
    u = torch.arange(nx, dtype=torch.float64, device=dev) + 0.5 - nx / 2.0   # detector pixel centres
    # Ray: p(t) = u*(cos, sin) + t*(-sin, cos) in the (x, z) plane.
    p0x = u[None, :] * ct[:, None]
    p0z = u[None, :] * st[:, None]
    dx = (-st)[:, None].expand_as(p0x)
    dz = ct[:, None].expand_as(p0x)
    cen = ph.centers.to(dev)
    A = ph.amat.to(dev)
    dens = ph.dens.to(dev)
    bc = ph.bcent.to(dev)
    bs = ph.bsig.to(dev)
    ba = ph.bamp.to(dev)
    out = torch.zeros(len(ys), len(tilts_deg), nx, dtype=torch.float64, device=dev)
    # Background: a constant slab of thickness nz contributes its chord length.
    if ph.background != 0.0:
        half = nz / 2.0
        cz = ct.abs().clamp_min(1e-12)
        chord = (2 * half / cz)[:, None].expand(len(tilts_deg), nx)
        # Also clip by the x extent of the volume.
        out += ph.background * chord[None]
    yc = torch.tensor(ys, dtype=torch.float64, device=dev) + 0.5 - ny / 2.0
    for s0 in range(0, len(ys), chunk):
        yy = yc[s0:s0 + chunk]                                     # (S,)
        # Ellipsoids: cross-section at y = yy.
        dy = yy[:, None] - cen[None, :, 1]                          # (S, E)
        Axx, Axz, Azz = A[:, 0, 0], A[:, 0, 2], A[:, 2, 2]
        Axy, Azy, Ayy = A[:, 0, 1], A[:, 2, 1], A[:, 1, 1]
        det = Axx * Azz - Axz * Axz
        # q0 = -dy * Axz2^{-1} [Axy, Azy]
        inv_xx, inv_xz, inv_zz = Azz / det, -Axz / det, Axx / det
        q0x = -dy * (inv_xx * Axy + inv_xz * Azy)[None]
        q0z = -dy * (inv_xz * Axy + inv_zz * Azy)[None]
        kap = 1 - Ayy[None] * dy * dy + dy * dy * (Axy * (inv_xx * Axy + inv_xz * Azy) + Azy * (inv_xz * Axy + inv_zz * Azy))[None]
        hit = kap > 0
        if bool(hit.any()):
            sidx, eidx = hit.nonzero(as_tuple=True)
            k = kap[sidx, eidx]
            bxx, bxz, bzz = Axx[eidx] / k, Axz[eidx] / k, Azz[eidx] / k
            ex = cen[eidx, 0] + q0x[sidx, eidx]
            ez = cen[eidx, 2] + q0z[sidx, eidx]
            rx = p0x[None] - ex[:, None, None]                    # (H, T, nx)
            rz = p0z[None] - ez[:, None, None]
            a = bxx[:, None, None] * dx * dx + 2 * bxz[:, None, None] * dx * dz + bzz[:, None, None] * dz * dz
            b = bxx[:, None, None] * dx * rx + bxz[:, None, None] * (dx * rz + dz * rx) + bzz[:, None, None] * dz * rz
            c = bxx[:, None, None] * rx * rx + 2 * bxz[:, None, None] * rx * rz + bzz[:, None, None] * rz * rz - 1
            disc = (b * b - a * c).clamp_min(0)
            chord = 2 * torch.sqrt(disc) / a * dens[eidx][:, None, None]
            out[s0:s0 + chunk].index_add_(0, sidx, chord)
        # Gaussian blobs.
        if bc.shape[0]:
            dyb = yy[:, None] - bc[None, :, 1]                      # (S, G)
            near = dyb.abs() < 5 * bs[None]
            if bool(near.any()):
                sidx, gidx = near.nonzero(as_tuple=True)
                sg = bs[gidx]
                wgt = ba[gidx] * torch.exp(-dyb[sidx, gidx] ** 2 / (2 * sg * sg)) * math.sqrt(2 * math.pi) * sg
                uc = bc[gidx, 0][:, None] * ct[None] + bc[gidx, 2][:, None] * st[None]   # (H, T)
                d = u[None, None, :] - uc[:, :, None]
                val = wgt[:, None, None] * torch.exp(-d * d / (2 * sg * sg)[:, None, None])
                out[s0:s0 + chunk].index_add_(0, sidx, val)
    return out.to(torch.float32)


def add_noise(rows: torch.Tensor, snr: float, seed: int) -> torch.Tensor:
    """Additive Gaussian noise with variance var(rows)/snr."""
    if snr is None or snr <= 0:
        return rows
    var = float(rows.double().var())
    g = torch.Generator(device=rows.device).manual_seed(int(seed) + 7919)
    noise = torch.randn(rows.shape, generator=g, device=rows.device, dtype=torch.float32)
    return rows + noise * math.sqrt(var / snr)


def cfg2_kind(nx, ny, thickness, seed, ys=None, device="cpu"):
    """A tilt series of the 1024x1024x300 kind at another size: ellipsoids
    and Gaussian blobs at the production phantom's density per voxel (300 and
    3000 per 1024 x 1024 x 300 voxels), background 0.1, 61 tilts -60..60 step
    2, SNR 0.1.  Returns (rows (S, 61, nx), tilts)."""
    vol = nx * ny * thickness / (1024.0 * 1024.0 * 300.0)
    tilts = tilt_angles(-60, 60, 2)
    ph = make_phantom((nx, ny, thickness), max(1, round(300 * vol)), max(1, round(3000 * vol)), seed=seed,
                      background=0.1)
    rows = project(ph, tilts, ys=ys, device=device)
    return add_noise(rows, 0.1, seed), tilts


def series(config: str, device="cpu", ys=None, seed=None):
    """Named workloads.  Returns (rows (S, ntilt, nx) float32 tensor, tilts,
    thickness, description).

    cfg1: 256x32x128 volume of 200 ellipsoids, 61 tilts -60..60 step 2,
          SNR 0.5, thickness 128.
    cfg2: 1024x1024x300 volume of 300 ellipsoids plus 3000 Gaussian blobs on
          a 0.1 background, 61 tilts stored sorted by angle, SNR 0.1,
          thickness 300.
    small: 64x4x48 volume of 30 ellipsoids, 31 tilts step 4, SNR 0.5.
    """
    if config == "cfg1":
        shape, E, G, bg, snr, tilts = (256, 32, 128), 200, 0, 0.0, 0.5, tilt_angles(-60, 60, 2)
        sd = 1001 if seed is None else seed
    elif config == "cfg2":
        shape, E, G, bg, snr, tilts = (1024, 1024, 300), 300, 3000, 0.1, 0.1, tilt_angles(-60, 60, 2)
        sd = 2002 if seed is None else seed
    elif config == "small":
        shape, E, G, bg, snr, tilts = (64, 4, 48), 30, 0, 0.0, 0.5, tilt_angles(-60, 60, 4)
        sd = 3003 if seed is None else seed
    else:
        raise ValueError(config)
    ph = make_phantom(shape, E, G, seed=sd, background=bg)
    rows = project(ph, tilts, ys=ys, device=device)
    rows = add_noise(rows, snr, sd)
    return rows, tilts, shape[2], dict(shape=shape, ellipsoids=E, blobs=G, background=bg, snr=snr, seed=sd)


def uneven_batch(n_series=24, seed=3003, slice_scale=1.0, device="cpu"):
    """The uneven multi-series workload: n_series seeded tilt series with
    width drawn from {256, 512, 768, 1024, 2048}, slice count uniform in
    [64, 512] (times slice_scale, at least 1), thickness uniform in
    [100, 400], tilt range +-U[45, 70] deg with step U[1.5, 3] deg and 10% of
    the tilts dropped at random, phantoms of ellipsoids and Gaussian blobs
    (counts scaled from the 1024x1024x300 production phantom's 300 and 3000 by
    volume, at least 20 and 100) on a 0.1 background, Gaussian noise at SNR
    U[0.1, 0.5].  Returns a list of dicts with nx, thickness, tilts, slices,
    rows (slices, ntilt, nx) float32 and snr."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_series):
        nx = int(rng.choice([256, 512, 768, 1024, 2048]))
        slices = max(1, int(round(int(rng.integers(64, 513)) * slice_scale)))
        thick = int(rng.integers(100, 401))
        rng_deg = float(rng.uniform(45.0, 70.0))
        step = float(rng.uniform(1.5, 3.0))
        n = int(math.floor(2 * rng_deg / step)) + 1
        tilts = (-rng_deg + step * np.arange(n)).astype(np.float32)
        keep = np.sort(rng.choice(n, size=n - int(round(0.1 * n)), replace=False))
        tilts = tilts[keep]
        snr = float(rng.uniform(0.1, 0.5))
        vol = nx * slices * thick / (1024.0 * 1024.0 * 300.0)
        E, G = max(20, int(round(300 * vol))), max(100, int(round(3000 * vol)))
        sd = int(seed) * 1000 + k
        ph = make_phantom((nx, slices, thick), E, G, seed=sd, background=0.1)
        rows = add_noise(project(ph, tilts, device=device), snr, sd)
        out.append(dict(nx=nx, thickness=thick, tilts=tilts, slices=slices, rows=rows, snr=snr))
    return out
