"""Build recipe for the CPU oracle (test infrastructure): oracle/liboracle.so.

IEEE arithmetic without FMA contraction (-ffp-contract=off) so that its results are
bit-comparable with the CUDA product, which follows the same conventions.
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False, verbose=False):
    srcs = sorted(glob.glob(os.path.join(HERE, "orc_*.cpp")))
    deps = srcs + glob.glob(os.path.join(HERE, "orc_*.hpp")) + [
        os.path.join(HERE, "..", "its_b200", "csrc", "mc_tables.inc")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v2", "-ffp-contract=off", "-fopenmp",
           "-fPIC", "-shared", "-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
