"""Generate golden vectors from the reference itself (run in the build container only).

Writes tests/golden/ref_tables.json with:
  * Morton encode/decode pairs produced by the reference's own MortonLUT.h
    (compiled by oracle/build_ref.py);
  * the marching-cubes case tables of the reference's LookTable.h;
  * the neighbour / shared-corner / shared-edge LUTs of the reference's SVO.cu,
    read as text (SVO.cu needs Eigen and Thrust and cannot be compiled here).
Writes tests/golden/ref_bspline.json: the reference's own hat values and gradients
(src/BSpline.hpp, BaseFunction4Point and de_BaseFunction4Point, compiled by
oracle/build_ref.py) at known-answer and pseudo-random points.
Also writes its_b200/csrc/mc_tables.inc: the same case table repacked as one
64-bit word per case (low nibble = vertex count, nibble k+1 = k-th edge index),
which the CUDA product and the oracle include. The standard Lorensen/Bourke case
table must be identical for triangle parity, so it is carried over, not re-derived.
"""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.build_ref import REF, bspline_harness, build  # noqa: E402

SVO_CU = os.path.join(REF, "cuAcc", "SVO.cu")


def parse_table(src, name):
    m = re.search(re.escape(name) + r"\s*(\[[^=]*)=\s*\{(.*?)\};", src, re.S)
    if not m:
        raise RuntimeError("table %s not found" % name)
    nums = [int(v) for v in re.findall(r"-?\d+", m.group(2))]
    return nums


def main():
    exe = build()
    if exe is None:
        sys.exit("reference not present; golden vectors cannot be regenerated here")
    data = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
    src = open(SVO_CU, encoding="utf-8", errors="replace").read()
    data["neighbor_LUTparent"] = parse_table(src, "neighbor_LUTparent")
    data["neighbor_LUTchild"] = parse_table(src, "neighbor_LUTchild")
    data["edgeSharedLUT"] = parse_table(src, "d_edgeSharedLUT")
    data["vertSharedLUT"] = parse_table(src, "d_vertSharedLUT")
    data["source"] = {
        "morton": "src/MortonLUT.h:292-343 (compiled)",
        "mc": "src/cuAcc/MarchingCubes/LookTable.h (compiled)",
        "luts": "src/cuAcc/SVO.cu:242-348 (parsed)",
    }
    out = os.path.join(ROOT, "tests", "golden", "ref_tables.json")
    with open(out, "w") as f:
        json.dump(data, f, separators=(",", ":"))
    # Repacked MC case table for the product and the oracle.
    words = []
    for c in range(256):
        n = data["nVertsTable"][c]
        edges = [e for e in data["triTable"][c] if e >= 0]
        if len(edges) != n:
            raise RuntimeError("case %d: table count mismatch" % c)
        w = n
        for k, e in enumerate(edges):
            w |= e << (4 * (k + 1))
        words.append(w)
    inc = os.path.join(ROOT, "its_b200", "csrc", "mc_tables.inc")
    with open(inc, "w") as f:
        f.write("// Marching-cubes case table (standard Lorensen/Bourke triangulation, as used by the\n"
                "// reference's LookTable.h), one word per case: bits 0-3 = number of triangle\n"
                "// vertices, bits 4k+4..4k+7 = edge index of the k-th vertex. Generated by\n"
                "// tests/golden/make_ref_tables.py; corner/edge numbering follows MarchingCubes.cu:233-262.\n")
        for i in range(0, 256, 4):
            f.write("  " + ", ".join("0x%016xull" % w for w in words[i:i + 4]) + ",\n")
    hats = json.loads(subprocess.run([bspline_harness()], check=True, capture_output=True, text=True).stdout)
    hats["source"] = "src/BSpline.hpp:4-57 (compiled): rows p.x p.y p.z w q.x q.y q.z value grad.x grad.y grad.z"
    out2 = os.path.join(ROOT, "tests", "golden", "ref_bspline.json")
    with open(out2, "w") as f:
        json.dump(hats, f, separators=(",", ":"))
    print("wrote", out, out2, "and", inc)


if __name__ == "__main__":
    main()
