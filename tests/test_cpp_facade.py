"""The C++ facade (include/its/ThinShells.hpp) in the reference's call order:
ctor -> creatShell() -> getShellIsoVal() -> mcVisualization(), checked against the oracle."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from its_b200 import meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compile(tmp_path):
    exe = str(tmp_path / "thin_shells_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "thin_shells_demo.cpp"), "-L", os.path.join(ROOT, "its_b200"),
                    "-lits", "-Wl,-rpath," + os.path.join(ROOT, "its_b200"), "-o", exe], check=True)
    return exe


def _write_off(path, V, F):
    with open(path, "w") as f:
        f.write("OFF\n%d %d 0\n" % (len(V), len(F)))
        for v in V:
            f.write("%.17g %.17g %.17g\n" % tuple(v))
        for t in F:
            f.write("3 %d %d %d\n" % tuple(t))


def test_facade_compiles(tmp_path):
    assert os.path.exists(_compile(tmp_path))


@pytest.mark.gpu
def test_facade_matches_oracle(tmp_path):
    exe = _compile(tmp_path)
    V, F = meshes.config_mesh("c0")
    off = str(tmp_path / "c0.off")
    _write_off(off, V, F)
    out = subprocess.run([exe, off, "32", str(tmp_path / "c0")], check=True, capture_output=True, text=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    Vr = np.loadtxt(off, skiprows=2, max_rows=len(V))  # the values the demo read
    Vn = oracle.model_to_unit_cube(Vr)
    o, e, w = oracle.uniform_bbox(Vn)
    ref = oracle.Svo(Vn, F, 32, o, w)
    assert r["depth"] == ref.depth and r["converged"] == 1
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, Vn, F)
    rp, col, val = ref.assemble()
    lam, rep = oracle.cgls(rp, col, val, b, 1e-10, 100000, 0)
    pts, _ = ref.intersections()
    f, miss = ref.eval_points(lam, np.vstack([Vn, pts]))
    lo, hi = f[miss == 0].min(), f[miss == 0].max()
    assert abs(r["inner"] - lo) <= 1e-8 * (hi - lo) and abs(r["outer"] - hi) <= 1e-8 * (hi - lo)
    for side in ("inner", "outer"):
        obj = str(tmp_path / ("c0_%s.obj" % side))
        assert os.path.getsize(obj) > 0


@pytest.mark.gpu
def test_facade_learned_start_and_obj_io(tmp_path):
    # OBJ input (readObj), the learned creatShell (an exact solution, residual at rounding
    # level) and the welded OBJ output; iso levels equal the plain fit's to 1e-9 of the range
    exe = _compile(tmp_path)
    V, F = meshes.config_mesh("c0")
    obj = str(tmp_path / "c0.obj")
    with open(obj, "w") as f:
        for v in V:
            f.write("v %.17g %.17g %.17g\n" % tuple(v))
        for t in F:
            f.write("f %d/1 %d/1 %d/1\n" % tuple(t + 1))
    plain = json.loads(subprocess.run([exe, obj, "32", str(tmp_path / "p")], check=True, capture_output=True,
                                      text=True).stdout.strip().splitlines()[-1])
    net = os.path.join(ROOT, "its_b200", "share_net.f32")
    learned = json.loads(subprocess.run([exe, obj, "32", str(tmp_path / "l"), net], check=True, capture_output=True,
                                        text=True).stdout.strip().splitlines()[-1])
    assert learned["rel_residual"] <= 1e-13 and learned["iterations"] == 0
    span = plain["outer"] - plain["inner"]
    assert abs(learned["inner"] - plain["inner"]) <= 1e-6 * span and abs(learned["outer"] - plain["outer"]) <= 1e-6 * span
    welded = [l.split() for l in open(str(tmp_path / "l_outer_welded.obj"))]
    nv = sum(1 for l in welded if l and l[0] == "v")
    faces = [l for l in welded if l and l[0] == "f"]
    assert nv > 0 and len(faces) > 0 and nv < 3 * len(faces)  # shared vertices
    assert max(int(i) for fc in faces for i in fc[1:]) == nv
