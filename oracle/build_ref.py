"""Build recipe for the reference-side golden harness (test infrastructure).

Compiles oracle/ref_tables.cpp against the reference's own table headers, where they
lie under /root/reference, into oracle/_ref/ref_tables. Only the two self-contained
headers are used (src/MortonLUT.h and src/cuAcc/MarchingCubes/LookTable.h); the rest
of the reference needs Eigen, libigl and MSVC and is unbuildable here.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = "/root/reference/src"
OUT = os.path.join(HERE, "_ref")


def build(verbose=False):
    """Return the path of the built harness, or None when the reference is absent."""
    if not os.path.isdir(REF):
        return None
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "ref_tables")
    cmd = ["g++", "-std=c++17", "-O1", "-w",
           "-I", os.path.join(HERE, "ref_stub"),
           "-I", REF, "-I", os.path.join(REF, "cuAcc", "MarchingCubes"),
           os.path.join(HERE, "ref_tables.cpp"), "-o", exe]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return exe


if __name__ == "__main__":
    print(build(verbose=True) or "reference not present", file=sys.stderr)
