"""Seeded synthetic scalar volumes for the extraction workloads.

meshtrex loads raw scan volumes (``src/volume.h:14-43``); none ships with it,
so every workload here is synthetic. Arrays are indexed ``[z, y, x]`` with x
fastest in memory, matching meshtrex's ``z*X*Y + y*X + x`` layout. Coordinates
are ``x_i = i / (N - 1)`` in [0, 1].

The generators are written once in torch so that the same code runs on the
CPU (tests, CPU baseline) and on the GPU (full-size bench volumes). Parity
checks always compare the CUDA path and the oracle on the same bytes.

Randomness comes from splitmix64 (Steele, Lea and Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014): output i of a stream seeded
with s is mix(s + (i + 1) * 0x9E3779B97F4A7C15).  Being counter-based, the
same seed gives the same numbers on the CPU and on the GPU and for any slab
size.  Scalar draws (blob centres, volume shapes, isovalues) come from
``Stream``; per-voxel Gaussian noise is Box-Muller over the pair of outputs
(2i, 2i + 1) of the voxel's flat index i, in float64, then rounded to float32
(``normal_noise``).  Float32 arithmetic of the fields themselves (exp, sin)
may still differ in the last bit between the CPU and the GPU, so a check
copies the bytes it compares rather than regenerating them.

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
_M64 = (1 << 64) - 1
_GOLDEN = 0x9E3779B97F4A7C15
_MIX1 = 0xBF58476D1CE4E5B9
_MIX2 = 0x94D049BB133111EB
_NOISE_KEY = 0x6E6F697365  # xor-ed into a field's seed for its per-voxel noise stream


def splitmix64(z: int) -> int:
    """The splitmix64 output function of a 64-bit state (Python ints)."""
    z &= _M64
    z = ((z ^ (z >> 30)) * _MIX1) & _M64
    z = ((z ^ (z >> 27)) * _MIX2) & _M64
    return z ^ (z >> 31)


def _s64(c: int) -> int:
    """A 64-bit constant as the int64 with the same bits."""
    return c - (1 << 64) if c >= 1 << 63 else c


def _srl(z: torch.Tensor, s: int) -> torch.Tensor:
    """Logical right shift of int64 bits."""
    return (z >> s) & ((1 << (64 - s)) - 1)


def _splitmix64_t(z: torch.Tensor) -> torch.Tensor:
    """splitmix64's output function over an int64 tensor (products wrap mod 2^64)."""
    z = (z ^ _srl(z, 30)) * _s64(_MIX1)
    z = (z ^ _srl(z, 27)) * _s64(_MIX2)
    return z ^ _srl(z, 31)


class Stream:
    """A seeded splitmix64 stream of scalar draws."""

    def __init__(self, seed: int):
        self.state = seed & _M64

    def next64(self) -> int:
        self.state = (self.state + _GOLDEN) & _M64
        return splitmix64(self.state)

    def uniform(self, lo: float = 0.0, hi: float = 1.0, n: int | None = None):
        """U[lo, hi) from the top 53 bits of one output; a list of n when n is given."""
        if n is not None:
            return [self.uniform(lo, hi) for _ in range(n)]
        return lo + (hi - lo) * ((self.next64() >> 11) * 2.0 ** -53)

    def integer(self, n: int) -> int:
        """Uniform over 0..n-1."""
        return min(n - 1, int(self.uniform() * n))


def normal_noise(seed: int, first: int, shape, device) -> torch.Tensor:
    """N(0, 1) float32 noise of the voxels with flat indices first, first + 1, ...
    (reshaped to `shape`): Box-Muller over outputs 2i and 2i + 1 of the
    splitmix64 stream seeded with seed ^ 0x6E6F697365."""
    n = 1
    for d in shape:
        n *= int(d)
    key = _s64(((seed ^ _NOISE_KEY) & _M64))
    i = torch.arange(first, first + n, device=device, dtype=torch.int64)
    c1 = key + (2 * i + 1) * _s64(_GOLDEN)
    u1 = _srl(_splitmix64_t(c1), 11).to(torch.float64) * 2.0 ** -53
    u2 = _srl(_splitmix64_t(c1 + _s64(_GOLDEN)), 11).to(torch.float64) * 2.0 ** -53
    z = torch.sqrt(-2.0 * torch.log1p(-u1)) * torch.cos((2.0 * math.pi) * u2)
    return z.to(torch.float32).view(*shape)


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
    """n blobs: centres U[0.2, 0.8]^3, then sigmas U[0.05, 0.15], then amplitudes U[0.3, 0.7]."""
    r = Stream(seed)
    centres = np.array(r.uniform(0.2, 0.8, 3 * n)).reshape(n, 3)
    return BlobParams(centres, np.array(r.uniform(0.05, 0.15, n)), np.array(r.uniform(0.3, 0.7, n)))


def blob_field(shape_zyx, seed: int, device="cpu", out_dtype=torch.uint8, noise_std=4.0,
               scale=255.0, n_blobs=8) -> torch.Tensor:
    """clamp(round(scale * sum_k A_k exp(-|x-c_k|^2 / (2 s_k^2)) + N(0, noise_std)), dtype range)."""
    Z, Y, X = shape_zyx
    p = blob_params(seed, n_blobs)
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
            acc += normal_noise(seed, z0 * Y * X, acc.shape, device) * noise_std
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
    for z0, z1 in _slabs(Z, Y, X):
        x, y, z = _grids(z0, z1, Z, Y, X, device)
        sx, cx = torch.sin(k * x), torch.cos(k * x)
        sy, cy = torch.sin(k * y), torch.cos(k * y)
        sz, cz = torch.sin(k * z), torch.cos(k * z)
        f = sx * cy + sy * cz + sz * cx
        f = f + normal_noise(seed, z0 * Y * X, f.shape, device) * 0.02
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
    r = Stream(seed)
    specs = []
    for _ in range(n):
        X, Y, Z = (int(edges[r.integer(len(edges))]) for _ in range(3))
        dt = DTYPES[r.integer(3)]
        specs.append(((Z, Y, X), dt, 1 + r.integer(16)))
    return specs


def batch(seed: int = 3, n: int = 64, device="cpu", edges=EDGES, scale_down: int = 1):
    """64 anisotropic blob volumes of mixed dtypes, each with 1-16 isovalues
    drawn uniformly between its 10th and 90th value percentiles."""
    items = []
    r = Stream(seed + 1000)
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
