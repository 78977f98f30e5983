"""Shared test helpers: seeded volumes and host/device conversions."""
import numpy as np
import torch

from meshtrex_b200 import synth

SCALE = {np.dtype(np.uint8): 255.0, np.dtype(np.uint16): 65535.0, np.dtype(np.float32): 1.0}
TORCH = {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
         np.dtype(np.float32): torch.float32}


def blob_volume(shape_zyx, dtype, seed=0, n_blobs=8) -> np.ndarray:
    """Seeded Gaussian-blob field in the dtype's range, as a numpy [z,y,x] array."""
    dt = np.dtype(dtype)
    noise = {np.dtype(np.uint8): 4.0, np.dtype(np.uint16): 4.0 * 257, np.dtype(np.float32): 4.0 / 255}[dt]
    t = synth.blob_field(shape_zyx, seed, "cpu", TORCH[dt], noise_std=noise, scale=SCALE[dt],
                         n_blobs=n_blobs)
    return to_numpy(t)


def to_numpy(t: torch.Tensor) -> np.ndarray:
    t = t.detach().cpu().contiguous()
    if t.dtype == torch.uint16:
        return t.view(torch.int16).numpy().view(np.uint16)
    return t.numpy()


def to_cuda(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16)).cuda().view(torch.uint16)
    return torch.from_numpy(a).cuda()


def mid_iso(a: np.ndarray) -> float:
    """An isovalue between the 40th and 60th percentiles, exact in float32."""
    q = float(np.percentile(a.astype(np.float64), 50))
    if a.dtype != np.float32:
        return float(round(q)) + 0.5 if a.dtype == np.uint8 else float(round(q))
    return float(np.float32(q))


def u32(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint32)
