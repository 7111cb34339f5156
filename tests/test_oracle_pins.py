"""The oracle against the reference's own outputs and tables (golden fixtures)."""
import json
import os

import numpy as np

from conftest import GOLDEN


def test_morton_encode_matches_reference(oracle_mod):
    ref = np.load(os.path.join(GOLDEN, "morton_ref.npz"))["encode"]
    assert ref.shape[0] >= 16000
    for x, y, z, code in ref.tolist():
        # the reference's encoder keeps the low 32 bits of the interleave
        assert oracle_mod.morton_encode(x, y, z) & 0xFFFFFFFF == code


def test_morton_exact_below_1024(oracle_mod):
    ref = np.load(os.path.join(GOLDEN, "morton_ref.npz"))["encode"]
    small = ref[(ref[:, :3] < 1024).all(1)]
    for x, y, z, code in small.tolist():
        assert oracle_mod.morton_encode(x, y, z) == code


def test_morton_decode_matches_reference(oracle_mod):
    ref = np.load(os.path.join(GOLDEN, "morton_ref.npz"))["decode"]
    for m, x, y, z in ref.tolist():
        assert oracle_mod.morton_decode(m) == (x, y, z)


def test_tables_match_reference(oracle_mod):
    ref = json.load(open(os.path.join(GOLDEN, "luts_ref.json")))
    mine = oracle_mod.tables()
    for k, v in ref.items():
        assert np.array_equal(mine[k], np.array(v)), k
