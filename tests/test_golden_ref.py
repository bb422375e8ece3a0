"""Pins the oracle's Morton codes, octree LUTs, MC table and hat basis against the reference's
own headers (tests/golden/ref_tables.json and ref_bspline.json, made by
tests/golden/make_ref_tables.py from the reference's MortonLUT.h, LookTable.h, SVO.cu and
BSpline.hpp)."""
import json
import os

import numpy as np

import oracle

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_tables.json")))
HATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_bspline.json")))


def test_morton_encode_decode_match_reference_tables():
    rows = np.array(GOLD["encode"], dtype=np.uint32)
    xyz, m, dec = rows[:, :3], rows[:, 3], rows[:, 4:]
    assert np.array_equal(oracle.morton_encode(xyz), m)
    assert np.array_equal(oracle.morton_decode(m), dec)
    assert np.array_equal(dec, xyz)


def test_neighbour_and_sharing_luts_match_reference():
    p, c, v, e = oracle.luts()
    assert np.array_equal(p.reshape(-1), np.array(GOLD["neighbor_LUTparent"]))
    assert np.array_equal(c.reshape(-1), np.array(GOLD["neighbor_LUTchild"]))
    assert np.array_equal(v, np.array(GOLD["vertSharedLUT"]))
    assert np.array_equal(e, np.array(GOLD["edgeSharedLUT"]))


def test_packed_mc_table_matches_reference():
    path = os.path.join(os.path.dirname(__file__), "..", "its_b200", "csrc", "mc_tables.inc")
    words = [int(t.rstrip("ul,"), 16) for line in open(path) if not line.startswith("//")
             for t in line.split() if t.startswith("0x")]
    assert len(words) == 256
    for c in range(256):
        n = words[c] & 15
        edges = [(words[c] >> (4 * (k + 1))) & 15 for k in range(n)]
        ref = [x for x in GOLD["triTable"][c] if x >= 0]
        assert n == GOLD["nVertsTable"][c]
        assert edges == ref


def test_share_network_oracle_gradient_finite_differences():
    # the float64 backward of the share-network oracle against central differences
    from oracle import mlp
    rng = np.random.default_rng(0)
    P = mlp.init_params(1).astype(np.float64)
    X = rng.standard_normal((16, mlp.N_IN))
    y = rng.standard_normal(16)
    g, _ = mlp.gradient(P, X, y, bf16_round=False)
    idx = rng.choice(mlp.NUM_PARAMS, 40, replace=False)
    for i in list(idx) + [mlp.NUM_PARAMS - 1]:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp = np.mean((mlp.forward(Pp, X, False) - y) ** 2)
        lm = np.mean((mlp.forward(Pm, X, False) - y) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_hat_basis_matches_reference_bspline():
    # BaseFunction4Point / de_BaseFunction4Point of the reference's own BSpline.hpp (compiled),
    # at the node, the support ends (the 1e-9 cut), half-way and arbitrary points: bit-exact
    rows = np.array(HATS["hat"], dtype=np.float64)
    assert rows.shape[0] >= 700
    val, grad = oracle.hat(rows[:, 0:3], rows[:, 3], rows[:, 4:7])
    assert np.array_equal(val, rows[:, 7])
    assert np.array_equal(grad, rows[:, 8:11])
    # the known answers of the hat: 1 at the node, 0 at the support ends, 1/2 half-way
    on_axis = rows[:144]
    w = on_axis[:, 3]
    a = (on_axis[:, 4] - on_axis[:, 0]) / w
    b = (on_axis[:, 5] - on_axis[:, 1]) / w
    want = np.where((np.abs(a) < 1) & (np.abs(b) < 1), (1 - np.abs(a)) * (1 - np.abs(b)) * 0.75, 0.0)
    ends = (np.abs(np.abs(a) - 1) < 1e-6) | (np.abs(np.abs(b) - 1) < 1e-6)
    assert np.allclose(on_axis[~ends, 7], want[~ends], atol=1e-12)
