"""The synthetic generators' random numbers: splitmix64 and Box-Muller noise.

splitmix64 is pinned to the published test vector of its reference
implementation (seed 1234567); the vectorised torch form must give the
scalar stream's numbers at any offset, so volumes do not depend on the slab
size or on the device they are generated on.
"""
import math

import numpy as np
import torch

from meshtrex_b200 import synth

# the first five outputs of splitmix64 seeded with 1234567
SPLITMIX64_1234567 = [6457827717110365317, 3203168211198807973, 9817491932198370423,
                      4593380528125082431, 16408922859458223821]


def test_splitmix64_known_answer():
    s = synth.Stream(1234567)
    assert [s.next64() for _ in range(5)] == SPLITMIX64_1234567


def test_vector_form_matches_scalar_stream():
    seed = 77
    s = synth.Stream(seed)
    want = [s.next64() for _ in range(64)]
    i = torch.arange(64, dtype=torch.int64)
    got = synth._splitmix64_t(synth._s64(seed) + (i + 1) * synth._s64(synth._GOLDEN))
    assert [int(v) & ((1 << 64) - 1) for v in got] == want


def test_normal_noise_is_box_muller_of_the_stream():
    seed, first = 5, 1000
    z = synth.normal_noise(seed, first, (4, 8), "cpu").reshape(-1)
    s = synth.Stream(seed ^ synth._NOISE_KEY)
    for _ in range(2 * first):
        s.next64()
    for k in range(32):
        u1, u2 = s.uniform(), s.uniform()
        want = np.float32(math.sqrt(-2.0 * math.log1p(-u1)) * math.cos(2.0 * math.pi * u2))
        assert np.float32(z[k]) == want


def test_normal_noise_does_not_depend_on_the_split():
    whole = synth.normal_noise(9, 0, (6, 50), "cpu")
    parts = torch.cat([synth.normal_noise(9, 0, (2, 50), "cpu"), synth.normal_noise(9, 100, (4, 50), "cpu")])
    assert torch.equal(whole, parts)


def test_normal_noise_moments():
    z = synth.normal_noise(3, 0, (1 << 20,), "cpu").double()
    assert abs(z.mean().item()) < 5e-3
    assert abs(z.std().item() - 1.0) < 5e-3


def test_batch_specs_cover_the_stated_ranges():
    specs = synth.batch_specs(seed=3, n=64)
    assert len(specs) == 64
    for shape, dt, n_iso in specs:
        assert all(e in synth.EDGES for e in shape)
        assert dt in synth.DTYPES and 1 <= n_iso <= 16
    assert synth.batch_specs(seed=3, n=64) == specs


def test_blob_params_ranges():
    p = synth.blob_params(0)
    assert p.centres.shape == (8, 3) and ((p.centres >= 0.2) & (p.centres < 0.8)).all()
    assert ((p.sigmas >= 0.05) & (p.sigmas < 0.15)).all() and ((p.amps >= 0.3) & (p.amps < 0.7)).all()
