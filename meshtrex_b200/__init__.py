"""meshtrex-b200: meshtrex's isosurface-extraction path (block min/max ->
active-block filtering + compaction -> PMB marching cubes) as hand-written
CUDA for NVIDIA B200 (sm_100a) behind a C ABI (include/meshtrex/mtx.h).

The compute lives in libmeshtrex_b200.so; this package holds its ctypes
binding (_lib), a Python mirror of meshtrex's stage managers (api) and the
synthetic workloads (synth).
"""
import os

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(PACKAGE_DIR, "libmeshtrex_b200.so")
