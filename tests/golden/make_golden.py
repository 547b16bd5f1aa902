"""Writes reference_kats.json: the known-answer vectors of the reference's
iris-mpc-common example data, so the oracle tests run without the reference
tree.  Run from the repository root with the reference checked out:

    python tests/golden/make_golden.py /path/to/iris-mpc

Sources (read as data):
  iris-mpc-common/src/example-data/random_codes.txt  -- two irises (code, mask
      base64) and their fractional distances at rotation 0 and the best of the
      31 rotations (galois_engine.rs:784-867)
  iris-mpc-common/src/example-data/flipped_codes.txt -- an iris and its
      mirror (galois_engine.rs:938-996, iris.rs:742-766)
  iris-mpc-common/src/example-data/all_rotations.txt -- an iris and the bit
      strings of its rotations -15..15 (iris.rs:726-741); stored here as the
      SHA-256 of each rotation's bit string.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys


def _lines(path):
    return [ln.strip() for ln in open(path) if ln.strip()]


def main(ref_root: str) -> None:
    ex = os.path.join(ref_root, "iris-mpc-common", "src", "example-data")
    rnd = _lines(os.path.join(ex, "random_codes.txt"))
    flp = _lines(os.path.join(ex, "flipped_codes.txt"))
    rot = _lines(os.path.join(ex, "all_rotations.txt"))
    rots = {}
    for ln in rot[1:]:
        k, v = ln.split(":", 1)
        rots[int(k)] = hashlib.sha256(v.replace(" ", "").strip().encode()).hexdigest()
    out = {
        "random_codes": {"code1": rnd[0], "mask1": rnd[1], "code2": rnd[2], "mask2": rnd[3],
                         "distance_rot0": float(rnd[4]), "distance_min_rot": float(rnd[5])},
        "flipped_codes": {"code": flp[0], "mask": flp[1], "flipped_code": flp[2], "flipped_mask": flp[3]},
        "all_rotations": {"code": rot[0], "rotation_bits_sha256": {str(k): v for k, v in sorted(rots.items())}},
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IRIS_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <path to a worldcoin/iris-mpc checkout> (or set IRIS_REFERENCE)")
    main(root)
