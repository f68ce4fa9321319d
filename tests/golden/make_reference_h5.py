"""Copies a subset of the reference's own HDF5 test data into tests/golden/reference_h5/ (the reference tree is not
present where the GPU tests run) and records each file's size and sha256 in manifest.json.

* tests/svd/testmatrices/svdmatrix_<n>.h5: the complex two-site matrices the reference's SVD test decomposes
  (tests/svd/main.cpp:69-87, truncation limit 1e-8).  The subset spans the shapes in the set: the smallest (2 x 8),
  square, wide, tall, the widest (70 x 172), the tallest (138 x 90) and the one whose truncation rank sits closest to
  the 1e-8 limit (98 x 90).
* bench/svd/data/svd-failed.h5: the SVD bench's matrices on which the reference's MKL gesdd returned info = 1 or -13
  (bench/svd/main.cpp:89-108), with their rank_max and threshold attributes.
* tests/testmatrices/lapacke_matrix-{1,2}{A,B}.h5: real symmetric 8 x 8 and 64 x 64 matrices with the eigenvalues and
  eigenvectors the reference's LAPACK computed for them, a state theta and its overlaps |<v_i|theta>| with the
  eigenvectors (the dense eigenproblem of a small H_eff, solved with ?syevr when the problem is small,
  AlgorithmFinite.cpp:318).

Run from the repository root with the reference checked out at REFERENCE (default /root/reference):
    python tests/golden/make_reference_h5.py
"""
import hashlib
import json
import os
import shutil
import sys

REFERENCE = os.environ.get("REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_h5")

FILES = ([f"tests/svd/testmatrices/svdmatrix_{n}.h5" for n in (6, 96, 0, 17, 170, 101, 48)] + ["bench/svd/data/svd-failed.h5"]
         + [f"tests/testmatrices/lapacke_matrix-{n}.h5" for n in ("1A", "1B", "2A", "2B")])


def main():
    if not os.path.isdir(REFERENCE):
        sys.exit(f"reference tree not found at {REFERENCE}")
    os.makedirs(OUT, exist_ok=True)
    manifest = {}
    for rel in FILES:
        src = os.path.join(REFERENCE, rel)
        dst = os.path.join(OUT, os.path.basename(rel))
        shutil.copyfile(src, dst)
        with open(dst, "rb") as fh:
            data = fh.read()
        manifest[os.path.basename(rel)] = {"source": rel, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(OUT, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
        fh.write("\n")


if __name__ == "__main__":
    main()
