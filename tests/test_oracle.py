"""The CPU oracle: pinned against meshtrex's own code, then checked for
self-consistency (brute force, FP64, mesh invariants, finite differences)."""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from golden.make_golden import ISOS, golden_volume, sha
from helpers import blob_volume

HERE = os.path.dirname(os.path.abspath(__file__))
PINS = json.load(open(os.path.join(HERE, "golden", "reference_pins.json")))


# ------------------------------------------------------------ reference pins
def test_case_table_matches_reference(oracle):
    tri, edge = oracle.decoded_tables()
    assert sha(tri.astype(np.int32)) == PINS["triTable_sha256"]
    assert sha(edge.astype(np.int32)) == PINS["edgeTable_sha256"]
    if oracle.have_reference_harness():
        rtri, redge = oracle.ref_tables()
        np.testing.assert_array_equal(tri, rtri)
        np.testing.assert_array_equal(edge, redge)


@pytest.fixture(scope="module")
def gvol():
    v = golden_volume()
    assert sha(v) == PINS["volume_sha256"], "golden volume generator drifted"
    return v


def test_core_minmax_matches_reference(oracle, gvol):
    mm = oracle.minmax_core(gvol, 4)
    assert sha(mm) == PINS["minmax_core_b4_sha256"]
    for i, (a, b) in PINS["minmax_core_b4_samples"].items():
        assert list(mm[int(i)]) == [a, b]
    if oracle.have_reference_harness():
        with tempfile.TemporaryDirectory() as td:
            raw = os.path.join(td, "golden_256x256x256_uint8.raw")
            gvol.tofile(raw)
            np.testing.assert_array_equal(mm, oracle.ref_minmax_256_u8_b4(raw))


@pytest.mark.parametrize("iso", ISOS)
def test_active_count_matches_reference(oracle, gvol, iso):
    mm = oracle.minmax_core(gvol, 4)
    # computeActiveBlockCountCPU (testMinMax.h:220-242) and the compaction rule
    # (blockFilteringTestUtils.h:456-469) agree for integral isovalues
    assert len(oracle.compact(mm, oracle.U8, iso)) == PINS["active_counts"][repr(iso)]


# ---------------------------------------------------------- restatement
def _halo_bruteforce(a, B):
    Z, Y, X = a.shape
    g = ((X + B - 1) // B, (Y + B - 1) // B, (Z + B - 1) // B)
    out = np.zeros((g[0] * g[1] * g[2], 2), np.uint32)
    keys = a.astype(np.uint32) if a.dtype != np.float32 else np.array(
        [oracle_key(f) for f in a.ravel()], np.uint32).reshape(a.shape)
    for bz in range(g[2]):
        for by in range(g[1]):
            for bx in range(g[0]):
                s = keys[bz * B:bz * B + B + 1, by * B:by * B + B + 1, bx * B:bx * B + B + 1]
                i = (bz * g[1] + by) * g[0] + bx
                out[i] = (s.min(), s.max())
    return out


def oracle_key(f):
    b = np.float32(f).view(np.uint32)
    return int(~b & 0xFFFFFFFF) if b & 0x80000000 else int(b | 0x80000000)


@pytest.mark.parametrize("dtype,B", [(np.uint8, 3), (np.uint16, 4), (np.float32, 5)])
def test_halo_minmax_is_brute_force(oracle, dtype, B):
    a = blob_volume((11, 13, 17), dtype, seed=B)
    np.testing.assert_array_equal(oracle.minmax_halo(a, B), _halo_bruteforce(a, B))


def test_pyramid_is_brute_force(oracle):
    a = blob_volume((37, 22, 45), np.uint8, seed=4)
    leaf = oracle.minmax_halo(a, 2)
    grid = oracle.block_grid(a.shape, 2)
    pyr = oracle.pyramid(leaf, grid)
    L = oracle.mip_levels(grid)
    assert L == 1 + int(np.floor(np.log2(max(grid))))
    prev = leaf.reshape(grid[2], grid[1], grid[0], 2)
    for l in range(1, L):
        e = oracle.mip_extent(grid, l)
        off = oracle.mip_offset(grid, l)
        lev = pyr[off:off + e[0] * e[1] * e[2]].reshape(e[2], e[1], e[0], 2)
        for z in range(e[2]):
            for y in range(e[1]):
                for x in range(e[0]):
                    s = prev[2 * z:2 * z + 2, 2 * y:2 * y + 2, 2 * x:2 * x + 2]
                    assert lev[z, y, x, 0] == s[..., 0].min() and lev[z, y, x, 1] == s[..., 1].max()
        prev = lev


def test_activity_rule_edge_cases(oracle):
    U8, F32 = oracle.U8, oracle.F32
    assert oracle.block_active(U8, 100, 128, 127.5)          # round(127.5) = 128
    assert not oracle.block_active(U8, 129, 200, 128.4)      # round -> 128 < min
    assert oracle.block_active(U8, 127, 200, 127.4)
    assert not oracle.block_active(U8, 50, 50, 50.0)         # min == max excluded
    assert oracle.block_active(U8, 0, 9, -0.3)               # round(-0.3) = -0 -> 0, as the reference
    assert not oracle.block_active(U8, 0, 9, -5.0)           # negative isovalues activate nothing
    k = oracle.key_of_f32
    assert oracle.block_active(F32, k(-1.0), k(2.0), 0.0)
    assert not oracle.block_active(F32, k(0.5), k(2.0), 0.25)
    assert not oracle.block_active(F32, k(-0.0), k(0.0), 0.0)  # -0 and +0 are the same value


def _sphere(n, r, dtype=np.float32):
    z, y, x = np.meshgrid(*(np.arange(n),) * 3, indexing="ij")
    c = (n - 1) / 2
    return (np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) - r).astype(dtype)


def test_closed_surface_is_watertight(oracle):
    a = _sphere(40, 13.3)
    m = oracle.extract(a, 8, 0.0, want_xyz64=True)
    V, T = m.n_vertices, m.n_triangles
    assert V > 1000 and T > 2000
    used = np.zeros(V, bool)
    used[m.indices.ravel()] = True
    assert used.all()                                       # no orphan vertices
    e = np.sort(np.concatenate([m.indices[:, [0, 1]], m.indices[:, [1, 2]], m.indices[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert (cnt == 2).all()                                 # every edge in exactly two triangles
    assert T == 2 * V - 4                                   # Euler: a sphere
    # every vertex lies on a lattice edge: two integral coordinates
    frac = np.abs(m.xyz - np.round(m.xyz)) > 0
    assert (frac.sum(axis=1) <= 1).all()
    rel = np.abs(m.xyz.astype(np.float64) - m.xyz64) / np.maximum(np.abs(m.xyz64), 1.0)
    assert rel.max() <= 1e-6


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
def test_block_edge_does_not_change_the_surface(oracle, dtype):
    a = blob_volume((24, 21, 26), dtype, seed=9)
    iso = float(np.float32(np.median(a)))
    meshes = [oracle.extract(a, B, iso) for B in (2, 4, 5, 8)]
    sets = []
    for m in meshes:
        tris = np.sort(m.xyz[m.indices].reshape(-1, 9).view(np.uint32).reshape(-1, 3, 3), axis=1)
        sets.append({t.tobytes() for t in tris})
    assert all(s == sets[0] for s in sets[1:])


def test_threads_do_not_change_the_output(oracle):
    a = blob_volume((40, 36, 44), np.uint16, seed=2)
    iso = float(np.median(a))
    m1 = oracle.extract(a, 8, iso, nthreads=1)
    m4 = oracle.extract(a, 8, iso, nthreads=4)
    np.testing.assert_array_equal(m1.xyz, m4.xyz)
    np.testing.assert_array_equal(m1.indices, m4.indices)


def _fp64_loss(field, block, iso, ids):
    from oracle import oracle as O
    m = O.mc_extract(field, block, iso, ids, want_xyz=False, want_xyz64=True, want_indices=False)
    v = m.xyz64 / (np.array(field.shape[::-1], np.float64) - 1)
    return np.mean((np.linalg.norm(v - 0.5, axis=1) - 0.35) ** 2)


def test_adjoint_matches_finite_differences(oracle):
    f = _sphere(20, 6.1).astype(np.float64) + 0.01 * np.sin(np.arange(20 ** 3).reshape(20, 20, 20))
    f32 = f.astype(np.float32)
    f = f32.astype(np.float64)
    iso = 0.0
    ids = oracle.compact(oracle.minmax_halo(f32, 4), oracle.F32, iso)
    m = oracle.mc_extract(f32, 4, iso, ids, want_xyz64=True)
    n = np.array(f.shape[::-1], np.float64) - 1
    v = m.xyz64 / n
    d = np.linalg.norm(v - 0.5, axis=1)
    g = (2 * (d - 0.35) / len(v))[:, None] * (v - 0.5) / d[:, None] / n  # dL/dxyz (voxel frame)
    dfield, diso = oracle.mc_adjoint(f32, 4, iso, ids, g.astype(np.float32))
    rng = np.random.default_rng(0)
    cand = np.argwhere(np.abs(dfield) > 1e-6)
    h = 1e-4
    for zyx in cand[rng.choice(len(cand), 20, replace=False)]:
        if abs(f[tuple(zyx)] - iso) < 4 * h:
            continue
        fp, fm = f.copy(), f.copy()
        fp[tuple(zyx)] += h
        fm[tuple(zyx)] -= h
        fd = (_fp64_loss(fp, 4, iso, ids) - _fp64_loss(fm, 4, iso, ids)) / (2 * h)
        assert abs(fd - dfield[tuple(zyx)]) <= 1e-4 * max(abs(fd), 1e-3)
    lp, lm = _fp64_loss(f - h, 4, iso, ids), _fp64_loss(f + h, 4, iso, ids)  # iso + h <=> field - h
    assert abs((lp - lm) / (2 * h) - diso) <= 1e-4 * max(abs(diso), 1e-3)


def test_meshlet_rule_on_a_hand_mesh(oracle):
    # block 0: two triangles share an edge (4 vertices fit a 4-vertex meshlet),
    # the third needs 3 more vertices and starts a new meshlet; block 1's
    # triangles start their own meshlet and reuse vertex 0 as a new copy
    nt = np.array([3, 2], np.uint32)
    idx = np.array([[0, 1, 2], [1, 2, 3], [4, 5, 6], [7, 8, 9], [8, 9, 0]], np.uint32)
    d, mv, mi = oracle.meshlets(nt, idx, 4, 126)
    np.testing.assert_array_equal(d, [[0, 0, 4, 2], [4, 6, 3, 1], [7, 9, 4, 2]])
    np.testing.assert_array_equal(mv, [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 0])
    np.testing.assert_array_equal(mv[mi], idx)
    d2, _, _ = oracle.meshlets(nt, idx, 64, 1)  # one triangle per meshlet
    assert len(d2) == 5 and (d2[:, 3] == 1).all()


# ------------------------------------------------- meshtrex's sphere fixture
def test_sphere_fixture_bytes_are_pinned():
    """sphere_volume restates generateSphereVolume (src/meshtrex.cpp:23-52);
    its bytes are pinned, and both readings of the unqualified sqrt there
    (float overload, or double sqrt and subtraction rounded once) agree."""
    from golden.fixtures import sphere_volume
    pins = json.load(open(os.path.join(HERE, "golden", "fixture_pins.json")))
    v = sphere_volume()
    assert v.shape == (64, 64, 64) and v.dtype == np.uint8
    assert sha(v) == pins["sphere_64_sha256"]
    f = np.float32
    radius = f(64) * f(0.4)
    z, y, x = np.meshgrid(*(np.arange(64, dtype=f),) * 3, indexing="ij")
    dx, dy, dz = x - f(32), y - f(32), z - f(32)
    s = (dx * dx + dy * dy) + dz * dz
    dist = (np.sqrt(s.astype(np.float64)) - np.float64(radius)).astype(f)
    n = ((dist / radius) * f(127.0) + f(128.0)) + f(0.001)
    np.testing.assert_array_equal(np.maximum(f(0), np.minimum(f(255), n)).astype(np.uint8), v)
