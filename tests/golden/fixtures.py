"""Deterministic test volumes restated from meshtrex, and the script that
pins their bytes (tests/golden/fixture_pins.json).

sphere_volume(w, h, d) restates meshtrex's synthetic fixture
generateSphereVolume (src/meshtrex.cpp:23-52), which main's comment pairs
with isovalue 128 and which main runs at block edge 3
(src/meshtrex.cpp:72-73, 78): float32 arithmetic in the same order, the
result clamped to [0, 255] and truncated to uint8.  meshtrex builds without
-march flags, so nothing is contracted into FMAs on x86-64; numpy's float32
operations round the same way.  Whether the unqualified sqrt there resolves
to the float or the double overload depends on the headers in scope; the
double reading (sqrt and the subtraction in double, rounded once to float)
gives the same 64^3 bytes, which tests/test_oracle.py checks.

    python tests/golden/fixtures.py     # rewrites fixture_pins.json
"""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def sphere_volume(width: int = 64, height: int = 64, depth: int = 64) -> np.ndarray:
    """uint8 [depth, height, width], x fastest."""
    f = np.float32
    radius = f(width) * f(0.4)
    cx, cy, cz = f(width) / f(2.0), f(height) / f(2.0), f(depth) / f(2.0)
    z, y, x = np.meshgrid(np.arange(depth, dtype=f), np.arange(height, dtype=f), np.arange(width, dtype=f),
                          indexing="ij")
    dx, dy, dz = x - cx, y - cy, z - cz
    s = dx * dx + dy * dy
    s = s + dz * dz
    distance = np.sqrt(s) - radius
    normalized = (distance / radius) * f(127.0)
    normalized = normalized + f(128.0)
    normalized = normalized + f(0.001)
    normalized = np.maximum(f(0.0), np.minimum(f(255.0), normalized))
    return normalized.astype(np.uint8)  # truncation toward zero, as static_cast<uint8_t>


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    v = sphere_volume()
    pins = {"what": "bytes of sphere_volume(64, 64, 64), the restatement of meshtrex's generateSphereVolume",
            "sphere_64_sha256": sha(v), "sphere_64_histogram_128": int((v <= 128).sum())}
    with open(os.path.join(HERE, "fixture_pins.json"), "w") as f:
        json.dump(pins, f, indent=1)
    print(json.dumps(pins, indent=1))


if __name__ == "__main__":
    main()
