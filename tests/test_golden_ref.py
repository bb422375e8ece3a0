"""Pins the oracle's Morton codes, octree LUTs and MC table against the reference's own
headers (tests/golden/ref_tables.json, made by tests/golden/make_ref_tables.py from the
reference's MortonLUT.h, LookTable.h and SVO.cu)."""
import json
import os

import numpy as np

import oracle

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_tables.json")))


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
