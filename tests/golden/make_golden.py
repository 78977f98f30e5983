"""Regenerates tests/golden/reference_pins.json from the reference itself.

Runs meshtrex's own CPU code (compiled from the reference sources into
oracle/_ref/ref_harness by `make -C oracle ref`) on the deterministic volume
of `golden_volume()` and records what it returns:
  - sha256 of computeMinMaxFromFile's block min/max (256^3 uint8, B = 4),
  - computeActiveBlockCountCPU at a few isovalues,
  - sha256 of MarchingCubes::triTable and edgeTable.
The volume is defined with integer arithmetic only, so its bytes do not
depend on any RNG or math library version.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

ISOS = (40.0, 80.0, 128.0, 200.0)


def golden_volume(n: int = 256) -> np.ndarray:
    """256^3 uint8: two integer spheres and a slab with hashed +-4 noise."""
    z, y, x = np.meshgrid(np.arange(n, dtype=np.int64), np.arange(n, dtype=np.int64),
                          np.arange(n, dtype=np.int64), indexing="ij")
    d1 = (x - 100) ** 2 + (y - 120) ** 2 + (z - 130) ** 2
    d2 = (x - 180) ** 2 + (y - 90) ** 2 + (z - 60) ** 2
    v = np.maximum(255 - np.minimum(255, d1 >> 6), 230 - np.minimum(230, d2 >> 5))
    v = np.maximum(v, np.where(np.abs(z + x // 4 - 200) < 6, 140, 0))
    h = (x * 73856093) ^ (y * 19349663) ^ (z * 83492791)
    h = (h ^ (h >> 13)) * 0x5bd1e995 & 0xFFFFFFFF
    v = v + ((h >> 24) & 7) - 4
    return np.clip(v, 0, 255).astype(np.uint8)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    from oracle import oracle as O
    if not O.have_reference_harness():
        sys.exit("oracle/_ref/ref_harness missing: run `make -C oracle ref` where the reference sources exist")
    v = golden_volume()
    with tempfile.TemporaryDirectory() as td:
        raw = os.path.join(td, "golden_256x256x256_uint8.raw")
        v.tofile(raw)
        mm = O.ref_minmax_256_u8_b4(raw)
        counts = {repr(i): O.ref_active_count(raw, i) for i in ISOS}
    tri, edge = O.ref_tables()
    pins = {
        "what": "outputs of meshtrex's own CPU code (src/testMinMax.h, src/mc_tables.h) on golden_volume()",
        "volume_sha256": sha(v),
        "minmax_core_b4_sha256": sha(mm.astype(np.uint32)),
        "minmax_core_b4_samples": {str(i): [int(mm[i, 0]), int(mm[i, 1])] for i in (0, 1, 4095, 100000, 262143)},
        "active_counts": counts,
        "triTable_sha256": sha(tri.astype(np.int32)),
        "edgeTable_sha256": sha(edge.astype(np.int32)),
    }
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(pins, f, indent=1)
    print(json.dumps(pins, indent=1))


if __name__ == "__main__":
    main()
