"""Pins the oracle's sampler tables against fixtures produced by the reference's own generator
scripts (tests/golden/make_golden.py): Sobol direction vectors, Sobol/Owen sample values and the
500000-entry acos table must match bit for bit."""
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_direction_vectors_match_reference_generator(oracle):
    ref = np.load(os.path.join(GOLDEN, "sobol_dv.npy"))
    assert ref.shape == (256, 32)
    assert np.array_equal(oracle.sobol_table(), ref)
    assert not ref[255].any()  # row 255 stays zero (the generator fills 255 rows)


def test_sobol_samples_match_reference_generator(oracle):
    g = np.load(os.path.join(GOLDEN, "sobol_samples.npz"))
    for seed in np.unique(g["seed"]):
        m = g["seed"] == seed
        vals = oracle.sobol_samples(g["index"][m], g["dim"][m], int(seed))
        assert np.array_equal(vals.view(np.uint32), g["bits"][m]), "seed %x" % seed


def test_acos_table_matches_reference_generator(oracle):
    meta = json.load(open(os.path.join(GOLDEN, "acos_lut.json")))
    lut = oracle.acos_lut(meta["precision"])
    assert hashlib.sha256(lut.tobytes()).hexdigest() == meta["sha256"]
    for k, v in meta["samples"].items():
        assert lut[int(k)] == np.float32(v)


def test_sampler_range(oracle):
    """SamplerTest.cpp:7-31 / math_random_generatorsTest.cpp:6-13: values lie in [0, 1]."""
    idx = np.repeat(np.arange(100, dtype=np.uint32), 64)
    dim = np.tile(np.arange(64, dtype=np.uint32), 100)
    for seed in (0, 0xDEADBEEF):
        v = oracle.sobol_samples(idx, dim, seed)
        assert np.all(v >= 0.0) and np.all(v <= 1.0)
