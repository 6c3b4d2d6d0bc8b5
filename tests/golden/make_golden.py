"""Writes the golden fixtures (tests/golden/<case>.npz): the oracle's answers
on the small seeded cases of cases.py, with a digest of their inputs.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), HERE]

import oracle as O  # noqa: E402
import cases  # noqa: E402


def main():
    for name, c in cases.all_cases().items():
        ans = cases.oracle_answers(O, name, c)
        np.savez_compressed(cases.fixture_path(name), inputs_digest=np.array(cases.inputs_digest(name, c)), **ans)
        print(name, {k: v.shape for k, v in ans.items()})


if __name__ == "__main__":
    main()
