"""Seeded synthetic scalar volumes for the extraction workloads.

meshtrex loads raw scan volumes (``src/volume.h:14-43``); none ships with it,
so every workload here is synthetic. Arrays are indexed ``[z, y, x]`` with x
fastest in memory, matching meshtrex's ``z*X*Y + y*X + x`` layout. Coordinates
are ``x_i = i / (N - 1)`` in [0, 1].

The generators are written once in torch so that the same code runs on the
CPU (tests, CPU baseline) and on the GPU (full-size bench volumes). Parity
checks always compare the CUDA path and the oracle on the same bytes.

Workloads:
  blobs    256^3 uint8: 8 Gaussian blobs + N(0, 4) noise (std 4), seed 0
  fbm_ball 1024^3 uint16: radial ramp + 0.08 fBm(5 octaves, base freq 4), seed 1
  gyroid   2048^3 float32: gyroid k = 2*pi*12 + N(0, 0.02), seed 2
  batch    64 volumes, anisotropic, mixed dtypes, 1-16 isovalues each, seed 3
  torus    512^3 float32 torus SDF (R=0.3, r=0.1) + 0.05 fBm(4 octaves), seed 4
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

_M32 = 0xFFFFFFFF


def _coords(n: int, device, dtype=torch.float32) -> torch.Tensor:
    if n == 1:
        return torch.zeros(1, device=device, dtype=dtype)
    return torch.arange(n, device=device, dtype=dtype) / (n - 1)


def _hash(ix: torch.Tensor, iy: torch.Tensor, iz: torch.Tensor, seed: int) -> torch.Tensor:
    """32-bit integer hash of lattice points (int64 arithmetic, masked to 32 bits)."""
    h = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ ((seed * 2654435761) & _M32)
    h = h & _M32
    h = ((h ^ (h >> 16)) * 0x45D9F3B) & _M32
    h = ((h ^ (h >> 16)) * 0x45D9F3B) & _M32
    return h ^ (h >> 16)


# the 12 edge directions of the cube used by gradient noise
_GRAD = torch.tensor([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1],
                      [1, 0, -1], [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]],
                     dtype=torch.float32)


def _fade(t):
    return t * t * t * (t * (t * 6 - 15) + 10)


def gradient_noise(px, py, pz, seed: int) -> torch.Tensor:
    """Gradient (Perlin-style) noise at broadcastable float coordinates, ~[-1, 1]."""
    x0, y0, z0 = torch.floor(px), torch.floor(py), torch.floor(pz)
    fx, fy, fz = px - x0, py - y0, pz - z0
    ix, iy, iz = x0.long(), y0.long(), z0.long()
    u, v, w = _fade(fx), _fade(fy), _fade(fz)
    g = _GRAD.to(px.device)
    out = None
    for c in range(8):
        dx, dy, dz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        h = _hash(ix + dx, iy + dy, iz + dz, seed) % 12
        gv = g[h]
        dot = gv[..., 0] * (fx - dx) + gv[..., 1] * (fy - dy) + gv[..., 2] * (fz - dz)
        wgt = (u if dx else 1 - u) * (v if dy else 1 - v) * (w if dz else 1 - w)
        out = dot * wgt if out is None else out + dot * wgt
    return out


def fbm(px, py, pz, octaves: int, base_freq: float, seed: int, lacunarity=2.0, gain=0.5):
    acc, amp, f = None, 1.0, base_freq
    for o in range(octaves):
        n = gradient_noise(px * f, py * f, pz * f, seed * 131 + o) * amp
        acc = n if acc is None else acc + n
        amp *= gain
        f *= lacunarity
    return acc


def _slabs(Z: int, Y: int, X: int, budget_voxels: int = 1 << 24):
    step = max(1, budget_voxels // max(1, X * Y))
    for z0 in range(0, Z, step):
        yield z0, min(Z, z0 + step)


def _grids(z0, z1, Z, Y, X, device):
    """Coordinate grids of slices z0..z1 of a [Z, Y, X] volume."""
    z = _coords(Z, device)[z0:z1].view(-1, 1, 1)
    y = _coords(Y, device).view(1, -1, 1)
    x = _coords(X, device).view(1, 1, -1)
    return x, y, z


# ------------------------------------------------------------------- blobs
@dataclass
class BlobParams:
    centres: np.ndarray
    sigmas: np.ndarray
    amps: np.ndarray


def blob_params(seed: int, n: int = 8) -> BlobParams:
    r = np.random.default_rng(seed)
    return BlobParams(r.uniform(0.2, 0.8, (n, 3)), r.uniform(0.05, 0.15, n), r.uniform(0.3, 0.7, n))


def blob_field(shape_zyx, seed: int, device="cpu", out_dtype=torch.uint8, noise_std=4.0,
               scale=255.0, n_blobs=8) -> torch.Tensor:
    """clamp(round(scale * sum_k A_k exp(-|x-c_k|^2 / (2 s_k^2)) + N(0, noise_std)), dtype range)."""
    Z, Y, X = shape_zyx
    p = blob_params(seed, n_blobs)
    gen = torch.Generator(device=device).manual_seed(seed)
    out = torch.empty(shape_zyx, dtype=out_dtype, device=device)
    for z0, z1 in _slabs(Z, Y, X):
        x, y, z = _grids(z0, z1, Z, Y, X, device)
        acc = torch.zeros((z1 - z0, Y, X), device=device)
        for k in range(n_blobs):
            c = p.centres[k]
            d2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
            acc += float(p.amps[k]) * torch.exp(-d2 / (2.0 * float(p.sigmas[k]) ** 2))
        acc = acc * scale
        if noise_std:
            acc += torch.randn(acc.shape, generator=gen, device=device) * noise_std
        out[z0:z1] = _to_dtype(acc, out_dtype)
    return out


def _to_dtype(f: torch.Tensor, dt) -> torch.Tensor:
    if dt == torch.uint8:
        return torch.clamp(torch.round(f), 0, 255).to(dt)
    if dt == torch.uint16:
        return torch.clamp(torch.round(f), 0, 65535).to(torch.int32).to(dt)
    return f.to(dt)


def blobs(n: int = 256, seed: int = 0, device="cpu") -> torch.Tensor:
    return blob_field((n, n, n), seed, device)


# ---------------------------------------------------------------- fbm_ball
def fbm_ball(n: int = 1024, seed: int = 1, device="cpu", shape_zyx=None, zslab=None) -> torch.Tensor:
    """65535 * clamp(0.5 + 0.5 (0.35 - |x - 0.5|) / 0.35 + 0.08 fBm(5 oct, freq 4), 0, 1).

    zslab=(za, zb) generates only slices za..zb of the full volume."""
    Z, Y, X = shape_zyx or (n, n, n)
    za, zb = zslab or (0, Z)
    out = torch.empty((zb - za, Y, X), dtype=torch.uint16, device=device)
    for s0, s1 in _slabs(zb - za, Y, X, 1 << 23):
        z0, z1 = za + s0, za + s1
        x, y, z = _grids(z0, z1, Z, Y, X, device)
        r = torch.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
        xb, yb, zb = torch.broadcast_tensors(x, y, z)
        f = 0.5 + 0.5 * (0.35 - r) / 0.35 + 0.08 * fbm(xb, yb, zb, 5, 4.0, seed)
        out[s0:s1] = _to_dtype(65535.0 * torch.clamp(f, 0.0, 1.0), torch.uint16)
    return out


# ------------------------------------------------------------------ gyroid
def gyroid(n: int = 2048, seed: int = 2, device="cpu", shape_zyx=None, out=None) -> torch.Tensor:
    """sin(kx)cos(ky) + sin(ky)cos(kz) + sin(kz)cos(kx), k = 2 pi 12, + N(0, 0.02)."""
    Z, Y, X = shape_zyx or (n, n, n)
    if out is None:
        out = torch.empty((Z, Y, X), dtype=torch.float32, device=device)
    k = 2.0 * math.pi * 12.0
    gen = torch.Generator(device=device).manual_seed(seed)
    for z0, z1 in _slabs(Z, Y, X):
        x, y, z = _grids(z0, z1, Z, Y, X, device)
        sx, cx = torch.sin(k * x), torch.cos(k * x)
        sy, cy = torch.sin(k * y), torch.cos(k * y)
        sz, cz = torch.sin(k * z), torch.cos(k * z)
        f = sx * cy + sy * cz + sz * cx
        f = f + torch.randn(f.shape, generator=gen, device=device) * 0.02
        out[z0:z1] = f
    return out


# ------------------------------------------------------------------- torus
def torus(n: int = 512, seed: int = 4, device="cpu", shape_zyx=None, R=0.3, r=0.1) -> torch.Tensor:
    """Signed distance to a torus (tube axis z, centre 0.5) + 0.05 fBm(4 octaves)."""
    Z, Y, X = shape_zyx or (n, n, n)
    out = torch.empty((Z, Y, X), dtype=torch.float32, device=device)
    for z0, z1 in _slabs(Z, Y, X, 1 << 23):
        x, y, z = _grids(z0, z1, Z, Y, X, device)
        q = torch.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2) - R
        d = torch.sqrt(q ** 2 + (z - 0.5) ** 2) - r
        xb, yb, zb = torch.broadcast_tensors(x, y, z)
        out[z0:z1] = d + 0.05 * fbm(xb, yb, zb, 4, 4.0, seed)
    return out


# ------------------------------------------------------------------- batch
EDGES = (64, 96, 128, 192, 256, 384, 512)
DTYPES = (torch.uint8, torch.uint16, torch.float32)


@dataclass
class BatchItem:
    volume: torch.Tensor
    isovalues: list = field(default_factory=list)


def batch_specs(seed: int = 3, n: int = 64, edges=EDGES):
    """(shape_zyx, dtype, n_iso) of every volume of the batched workload."""
    r = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        X, Y, Z = (int(e) for e in r.choice(edges, 3))
        dt = DTYPES[int(r.integers(0, 3))]
        specs.append(((Z, Y, X), dt, int(r.integers(1, 17))))
    return specs


def batch(seed: int = 3, n: int = 64, device="cpu", edges=EDGES, scale_down: int = 1):
    """64 anisotropic blob volumes of mixed dtypes, each with 1-16 isovalues
    drawn uniformly between its 10th and 90th value percentiles."""
    items = []
    r = np.random.default_rng(seed + 1000)
    for i, (shape, dt, n_iso) in enumerate(batch_specs(seed, n, edges)):
        shape = tuple(max(8, s // scale_down) for s in shape)
        scale = {torch.uint8: 255.0, torch.uint16: 65535.0, torch.float32: 1.0}[dt]
        noise = {torch.uint8: 4.0, torch.uint16: 4.0 * 257, torch.float32: 4.0 / 255}[dt]
        v = blob_field(shape, seed * 1000 + i, device, dt, noise_std=noise, scale=scale)
        sample = v.flatten()[:: max(1, v.numel() // (1 << 20))].float()
        lo, hi = torch.quantile(sample.cpu(), torch.tensor([0.1, 0.9])).tolist()
        isos = [float(x) for x in r.uniform(lo, hi, n_iso)]
        if dt != torch.float32:  # integer volumes: keep isovalues exact in float32
            isos = [float(np.float32(x)) for x in isos]
        items.append(BatchItem(v, isos))
    return items
