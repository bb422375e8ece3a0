"""Build recipe for the reference-side golden harnesses (test infrastructure).

Compiles, where the reference tree is present, into oracle/_ref/:
  * ref_tables: oracle/ref_tables.cpp against the reference's own table headers
    (src/MortonLUT.h and src/cuAcc/MarchingCubes/LookTable.h);
  * ref_bspline: oracle/ref_bspline.cpp against the reference's own src/BSpline.hpp, with
    oracle/ref_stub/BasicDataType.h standing in for the Eigen types it names (-I- keeps the
    reference's own BasicDataType.h, which needs Eigen, out of the search).
The rest of the reference needs Eigen, libigl and MSVC and is unbuildable here.
The reference tree is taken from $ITS_REFERENCE_DIR, else from the path the build container
mounts it at.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("ITS_REFERENCE_DIR", "/root/reference")
REF = os.path.join(REF_ROOT, "src")
OUT = os.path.join(HERE, "_ref")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def build(verbose=False):
    """Return the path of the table harness (the B-spline harness beside it), or None when the
    reference is absent."""
    if not os.path.isdir(REF):
        return None
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "ref_tables")
    _run(["g++", "-std=c++17", "-O1", "-w", "-I", os.path.join(HERE, "ref_stub"),
          "-I", REF, "-I", os.path.join(REF, "cuAcc", "MarchingCubes"),
          os.path.join(HERE, "ref_tables.cpp"), "-o", exe], verbose)
    # IEEE arithmetic as the oracle compiles it (no contraction), so values compare bit for bit
    _run(["g++", "-std=c++17", "-O1", "-w", "-ffp-contract=off", "-I-", "-I", os.path.join(HERE, "ref_stub"),
          "-I", REF, os.path.join(HERE, "ref_bspline.cpp"), "-o", os.path.join(OUT, "ref_bspline")], verbose)
    return exe


def bspline_harness():
    return os.path.join(OUT, "ref_bspline")


if __name__ == "__main__":
    print(build(verbose=True) or "reference not present", file=sys.stderr)
