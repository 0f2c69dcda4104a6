"""Writes kats.json: the known-answer tests of the reference's own unit tests.

Each entry restates one deterministic test of lattice-arguments/salsaa with
its inputs and expected output, and names the file:line it comes from.  The
reference is Rust + Intel HEXL and cannot be built here, so the vectors are
taken from the test sources.  When the reference tree is available,
`--check` (which needs its path in the SALSAA_REFERENCE environment variable)
confirms that every expected literal still appears at the cited place.
"""
import json
import os
import sys

Q62 = 4546383823830515713

KATS = [
    {"name": "multiply_mod", "src": "src/hexl/bindings.rs:99-106",
     "a": 12345, "b": 67890, "q": 1000000007, "expect": 838102050, "literal": "838102050"},
    {"name": "eltwise_mult_mod", "src": "src/hexl/bindings.rs:108-118",
     "a": [1, 2, 3, 4, 5], "b": [6, 7, 8, 9, 10], "q": 100, "expect": [6, 14, 24, 36, 50],
     "literal": "vec![6, 14, 24, 36, 50]"},
    {"name": "multiply_poly", "src": "src/hexl/bindings.rs:119-148",
     "a": [1, 2, 3, 1, 0, 0, 0, 0], "b": [8, 7, 6, 1, 0, 0, 0, 0], "q": 65537,
     # expected: the test's own schoolbook loop over the first n/2 coefficients
     "expect": None, "literal": "expected_result[i + j]"},
    {"name": "ring_add", "src": "src/cyclotomic_ring.rs:201-214",
     "a": [1, 2, 3, 4], "b": [4, 3, 2, 1], "q": 17, "expect": [5, 5, 5, 5], "literal": "[5, 5, 5, 5]"},
    {"name": "ring_sub", "src": "src/cyclotomic_ring.rs:216-228",
     "a": [5, 6, 7, 8], "b": [4, 3, 2, 1], "q": 17, "expect": [1, 3, 5, 7], "literal": "[1, 3, 5, 7]"},
    {"name": "ring_mul", "src": "src/cyclotomic_ring.rs:230-242",
     "a": [1, 2, 1, 0], "b": [1, 1, 1, 0], "q": 17, "expect": [0, 3, 4, 3], "literal": "[0, 3, 4, 3]"},
    {"name": "quadratic_add", "src": "src/quadratic_extension.rs:89-99",
     "a": [3, 5], "b": [7, 9], "shift": 1, "q": 17, "expect": [10, 14], "literal": "[10, 14]"},
    {"name": "quadratic_mul", "src": "src/quadratic_extension.rs:101-111",
     "a": [3, 5], "b": [7, 9], "shift": 1, "q": 17, "expect": [15, 11], "literal": "[15, 11]"},
    {"name": "tensor", "src": "src/subroutines/fast_norm_check.rs:41-57",
     "cs": [3, 5], "q": 17, "expect": [8, 7, 5, 15], "literal": "vec![8, 7, 5, 15]"},
    {"name": "sum_sq", "src": "src/subroutines/fast_norm_check.rs:264-269",
     "a": [1, 2, 3, 4, 5, 6, 7, 8], "q": 71, "expect": 62, "literal": "62"},
    {"name": "split", "src": "src/subroutines/split.rs:109-143",
     "q": Q62, "d": 8,
     "layers": [[1, 2, 4, 8, 16, 32, 64, 128], [1, 2, 4, 8], [1, 2], [1]],
     "tensors": [[1, 16], [1, 4], [1, 2]],
     "witness": [1, 2, 3, 4, 5, 6, 7, 8],
     "expect_rhs": 1793, "expect_split_rhs": [49, 109],
     "expect_split_witness": [[1, 2, 3, 4], [5, 6, 7, 8]], "literal": "vec![49, 109]"},
]


def _schoolbook(k):
    n = len(k["a"])
    out = [0] * n
    for i in range(n // 2):
        for j in range(n // 2):
            out[i + j] = (out[i + j] + k["a"][i] * k["b"][j]) % k["q"]
    return out


for _k in KATS:
    if _k["name"] == "multiply_poly":
        _k["expect"] = _schoolbook(_k)


def check(ref_root):
    bad = []
    for k in KATS:
        path, lines = k["src"].split(":")
        lo, hi = (int(x) for x in lines.split("-"))
        with open(os.path.join(ref_root, path)) as f:
            text = "".join(f.readlines()[lo - 1:hi])
        if k["literal"] not in text:
            bad.append(k["name"])
    return bad


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "kats.json"), "w") as f:
        json.dump(KATS, f, indent=1)
    if "--check" in sys.argv:
        ref = os.environ.get("SALSAA_REFERENCE")
        if not ref:
            sys.exit("--check needs SALSAA_REFERENCE set to the reference source tree")
        bad = check(ref)
        print("mismatched literals:", bad)
        sys.exit(1 if bad else 0)


if __name__ == "__main__":
    main()
