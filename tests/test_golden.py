"""The committed golden fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py) against the oracle run now: the seeded inputs
still digest to the fixture's value, and the oracle's answers are unchanged
bit for bit (nearest leaf / toi / normal, bounded hit lists, CSR overlaps,
the two-level scene's rays, casts and regions)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import cases  # noqa: E402
import oracle as O  # noqa: E402

CASES = cases.all_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_fixture(name):
    c = CASES[name]
    z = np.load(cases.fixture_path(name))
    assert str(z["inputs_digest"]) == cases.inputs_digest(name, c), "the seeded inputs changed"
    ans = cases.oracle_answers(O, name, c)
    assert sorted(ans) == sorted(k for k in z.files if k != "inputs_digest")
    for k, v in ans.items():
        assert np.array_equal(v, z[k]), f"{name}: {k} differs from the fixture"


def test_fixtures_have_hits():
    for name in CASES:
        z = np.load(cases.fixture_path(name))
        leaf = z["ray_leaf"] if name == "tlas_mesh" else z["leaf"]
        assert (leaf != O.NO_HIT).sum() > 100, name
