"""Writes known_answers.json: the reference's own known-answer cases for LU.

Each case is transcribed from rustymath's tests (cited in `source`); the expected values
are the reference's stated answers, computed here from their formulas, not from any
implementation in this repository. Run: python tests/golden/make_golden.py"""
import json
import os

import numpy as np

TINY = float(np.finfo(np.float64).tiny)


def cases():
    p, q = TINY / 1024.0, TINY / 1048576.0
    yield {"name": "subnormal pivot", "source": "tests/linalg.rs:510-511",
           "a": [[p, 1.0], [q, 1.0]], "factors": [p, q / p, 1.0, 1.0 - q / p], "perm": [0, 1]}
    swapped = [[0., 2, 0, 0], [1, 0, 0, 0], [0, 0, 3, 0], [0, 0, 0, 4]]
    yield {"name": "odd permutation determinant", "source": "tests/linalg.rs:552-555",
           "a": swapped, "det": -24.0}
    yield {"name": "singular determinant", "source": "tests/linalg.rs:556-558",
           "a": [[1.0, 0.0], [3.0, 0.0]], "det": 0.0, "regular": False}
    yield {"name": "singular inverse", "source": "tests/linalg.rs:548-549",
           "a": [[1.0, 2.0], [2.0, 4.0]], "regular": False}


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(out, "w") as fh:
        json.dump(list(cases()), fh, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
