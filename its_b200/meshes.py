"""Seeded synthetic meshes for the thin-shell workloads, and a small OFF reader.

The reference ships a single model (bunny.off) and measures on no public suite, so the
workloads are closed manifold meshes generated here from a seed:

* ``sphere_mesh``   -- geodesic sphere from a pentagonal bipyramid (10 faces), split
  4-to-1 ``subdiv`` times: 10*4^k faces, 5*4^k+2 vertices (k=5: 10,240 / 5,122;
  k=9: 2,621,440 faces), radius 1 + amp*f with f a real spherical-harmonic series of
  degree <= 4 and N(0,1) coefficients.
* ``torus_knot_tube`` -- a (p,q) torus-knot tube, rings x segments quads split in two
  (3,5 knot, 4096 x 128 -> 1,048,576 faces), vertices rounded to FP32, N(0, sigma)
  jitter.
* ``torus_mesh`` / ``superquadric_mesh`` -- the other two families of the batch mix.

All generators return (V float64 (n,3), F int32 (m,3)) with outward-facing triangles.
"""
import math

import numpy as np


def _bipyramid():
    ang = np.arange(5) * (2 * np.pi / 5)
    ring = np.stack([np.cos(ang), np.sin(ang), np.zeros(5)], 1)
    V = np.vstack([ring, [[0, 0, 1], [0, 0, -1]]]).astype(np.float64)
    F = []
    for i in range(5):
        j = (i + 1) % 5
        F.append([i, j, 5])      # upper cap, counter-clockwise seen from outside
        F.append([j, i, 6])      # lower cap
    return V, np.array(F, np.int64)


def _subdivide(V, F):
    """4-to-1 split with shared edge midpoints projected to the unit sphere."""
    e = np.sort(np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]), axis=1)
    uniq, inv = np.unique(e, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    mid = V[uniq[:, 0]] + V[uniq[:, 1]]
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    base = V.shape[0]
    m = F.shape[0]
    a, b, c = F[:, 0], F[:, 1], F[:, 2]
    ab, bc, ca = base + inv[:m], base + inv[m:2 * m], base + inv[2 * m:]
    F2 = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                         np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)])
    return np.vstack([V, mid]), F2


def _geodesic(k):
    """Unit sphere from the bipyramid with every face split into k x k (frequency k): 10 k^2
    faces, 5 k^2 + 2 vertices, any k >= 1."""
    V0, F0 = _bipyramid()
    I, J = np.meshgrid(np.arange(k + 1), np.arange(k + 1), indexing="ij")
    keep = (I + J) <= k
    I, J = I[keep], J[keep]
    local = -np.ones((k + 1, k + 1), np.int64)
    local[I, J] = np.arange(I.size)
    i, j = np.meshgrid(np.arange(k), np.arange(k), indexing="ij")
    up = (i + j) <= k - 1
    dn = (i + j) <= k - 2
    tri = np.concatenate([np.stack([local[i[up], j[up]], local[i[up] + 1, j[up]], local[i[up], j[up] + 1]], 1),
                          np.stack([local[i[dn] + 1, j[dn]], local[i[dn] + 1, j[dn] + 1], local[i[dn], j[dn] + 1]], 1)])
    P, T = [], []
    for f, (a, b, c) in enumerate(F0):
        pts = V0[a] + (V0[b] - V0[a]) * (I[:, None] / k) + (V0[c] - V0[a]) * (J[:, None] / k)
        P.append(pts / np.linalg.norm(pts, axis=1, keepdims=True))
        T.append(tri + f * I.size)
    P, T = np.vstack(P), np.vstack(T)
    # weld the copies of the shared edges
    _, first, inv = np.unique(np.round(P * 2 ** 30).astype(np.int64), axis=0, return_index=True, return_inverse=True)
    return P[first], inv.reshape(-1)[T]


def _real_sh(lmax, theta, phi):
    """Real spherical harmonics up to degree lmax at (theta polar, phi azimuth)."""
    from scipy.special import lpmv
    x = np.cos(theta)
    out = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            p = lpmv(am, l, x)
            if m > 0:
                out.append(math.sqrt(2) * norm * p * np.cos(am * phi))
            elif m < 0:
                out.append(math.sqrt(2) * norm * p * np.sin(am * phi))
            else:
                out.append(norm * p)
    return np.stack(out, 1)


def sphere_mesh(subdiv, amp=0.1, seed=0, lmax=4):
    V, F = _bipyramid()
    for _ in range(subdiv):
        V, F = _subdivide(V, F)
    rng = np.random.default_rng(seed)
    theta = np.arccos(np.clip(V[:, 2], -1, 1))
    phi = np.arctan2(V[:, 1], V[:, 0])
    Y = _real_sh(lmax, theta, phi)
    coef = rng.standard_normal(Y.shape[1])
    f = Y @ coef
    r = 1.0 + amp * f
    return V * r[:, None], F.astype(np.int32)


def _sh_perturb(V, amp, seed, lmax=4):
    rng = np.random.default_rng(seed)
    theta = np.arccos(np.clip(V[:, 2], -1, 1))
    phi = np.arctan2(V[:, 1], V[:, 0])
    Y = _real_sh(lmax, theta, phi)
    return V * (1.0 + amp * (Y @ rng.standard_normal(Y.shape[1])))[:, None]


def _closed_grid_faces(rings, segs):
    i = np.arange(rings)[:, None]
    j = np.arange(segs)[None, :]
    a = i * segs + j
    b = ((i + 1) % rings) * segs + j
    c = ((i + 1) % rings) * segs + (j + 1) % segs
    d = i * segs + (j + 1) % segs
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return F.astype(np.int32)


def torus_knot_tube(p=3, q=5, rings=4096, segs=128, tube=0.08, jitter=1e-3, seed=1, fp32=True):
    t = np.arange(rings) * (2 * np.pi / rings)

    def curve(t):
        r = 2.0 + np.cos(q * t)
        return np.stack([r * np.cos(p * t), r * np.sin(p * t), -np.sin(q * t)], 1)

    C0 = curve(t)
    T = curve(t + 1e-4) - curve(t - 1e-4)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    # Rotation-minimising frame by projection, with the closing twist spread evenly.
    N = np.zeros_like(T)
    a = np.array([0.0, 0.0, 1.0])
    n0 = a - (a @ T[0]) * T[0]
    N[0] = n0 / np.linalg.norm(n0)
    for k in range(1, rings):
        v = N[k - 1] - (N[k - 1] @ T[k]) * T[k]
        N[k] = v / np.linalg.norm(v)
    v = N[-1] - (N[-1] @ T[0]) * T[0]
    v /= np.linalg.norm(v)
    B0 = np.cross(T[0], N[0])
    twist = math.atan2(v @ B0, v @ N[0])
    B = np.cross(T, N)
    ang = -twist * np.arange(rings) / rings
    N, B = np.cos(ang)[:, None] * N + np.sin(ang)[:, None] * B, -np.sin(ang)[:, None] * N + np.cos(ang)[:, None] * B
    s = np.arange(segs) * (2 * np.pi / segs)
    V = (C0[:, None, :] + tube * (np.cos(s)[None, :, None] * N[:, None, :] +
                                 np.sin(s)[None, :, None] * B[:, None, :])).reshape(-1, 3)
    if fp32:
        V = V.astype(np.float32)
    rng = np.random.default_rng(seed)
    V = V + rng.normal(0.0, jitter, V.shape).astype(V.dtype)
    V = V.astype(np.float32).astype(np.float64) if fp32 else V
    F = _closed_grid_faces(rings, segs)
    # Orientation: make triangle normals point away from the tube axis.
    n = np.cross(V[F[1, 1]] - V[F[1, 0]], V[F[1, 2]] - V[F[1, 0]])
    if n @ (V[F[1, 0]] - C0[0]) < 0:
        F = F[:, [0, 2, 1]]
    return V, F


def torus_mesh(R=0.75, r=0.2, rings=64, segs=32):
    u = np.arange(rings) * (2 * np.pi / rings)
    v = np.arange(segs) * (2 * np.pi / segs)
    cu, su, cv, sv = np.cos(u)[:, None], np.sin(u)[:, None], np.cos(v)[None, :], np.sin(v)[None, :]
    V = np.stack([(R + r * cv) * cu, (R + r * cv) * su, r * sv + 0 * cu], -1).reshape(-1, 3)
    F = _closed_grid_faces(rings, segs)
    n = np.cross(V[F[0, 1]] - V[F[0, 0]], V[F[0, 2]] - V[F[0, 0]])
    if n @ (V[F[0, 0]] - np.array([R, 0, 0])) < 0:
        F = F[:, [0, 2, 1]]
    return V, F


def superquadric_mesh(e1=1.0, e2=1.0, subdiv=3, freq=None):
    """Superellipsoid |x|^(2/e2)+|y|^(2/e2))^(e2/e1)+|z|^(2/e1)=1 over a geodesic sphere
    (4-to-1 splits ``subdiv`` times, or frequency ``freq`` when given)."""
    if freq is not None:
        V, F = _geodesic(freq)
    else:
        V, F = _bipyramid()
        for _ in range(subdiv):
            V, F = _subdivide(V, F)
    x, y, z = V[:, 0], V[:, 1], V[:, 2]
    theta = np.arcsin(np.clip(z, -1, 1))
    phi = np.arctan2(y, x)
    sp = lambda w, e: np.sign(w) * np.abs(w) ** e  # noqa: E731
    cth, sth = np.cos(theta), np.sin(theta)
    V2 = np.stack([sp(cth, e1) * sp(np.cos(phi), e2), sp(cth, e1) * sp(np.sin(phi), e2), sp(sth, e1)], 1)
    return V2, F.astype(np.int32)


def batch_meshes(count=256, seed=3, fmin=2000, fmax=200000):
    """The uneven multi-mesh workload: face counts log-uniform in [fmin, fmax]; thirds of
    perturbed geodesic spheres (radius 1 + 0.1 f, f a degree-4 real SH series), tori
    (R in [0.5, 1], r in [0.1, 0.3]) and superquadrics (exponents in [0.3, 3]); octree
    depth 7, 8 or 9 (res 64 / 128 / 256) by size, the thirds of the log range.

    Returns a list of dicts (V, F, kind, res, faces) in generation order."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = math.log(fmin), math.log(fmax)
    for i in range(count):
        target = math.exp(rng.uniform(lo, hi))
        kind = i % 3
        if kind == 0:
            k = max(2, int(round(math.sqrt(target / 10.0))))
            V, F = _geodesic(k)
            V = _sh_perturb(V, 0.1, seed * 100000 + i)
        elif kind == 1:
            R, r = rng.uniform(0.5, 1.0), rng.uniform(0.1, 0.3)
            segs = max(8, int(round(math.sqrt(target / 2.0 * r / R))))
            rings = max(8, int(round(target / (2.0 * segs))))
            V, F = torus_mesh(R, r, rings, segs)
        else:
            e1, e2 = rng.uniform(0.3, 3.0), rng.uniform(0.3, 3.0)
            k = max(2, int(round(math.sqrt(target / 10.0))))
            V, F = superquadric_mesh(e1, e2, freq=k)
        nf = F.shape[0]
        t = (math.log(nf) - lo) / (hi - lo)
        res = 64 if t < 1 / 3 else (128 if t < 2 / 3 else 256)
        out.append(dict(V=np.ascontiguousarray(V, np.float64), F=np.ascontiguousarray(F, np.int32),
                        kind=("sphere", "torus", "superquadric")[kind], res=res, faces=nf))
    return out


def read_off(path):
    """Minimal OFF reader (vertex and triangle blocks only)."""
    with open(path) as f:
        toks = [t for line in f for t in line.split("#")[0].split()]
    assert toks[0] == "OFF"
    nv, nf = int(toks[1]), int(toks[2])
    pos = 4
    V = np.array(toks[pos:pos + 3 * nv], dtype=np.float64).reshape(nv, 3)
    pos += 3 * nv
    F = []
    for _ in range(nf):
        k = int(toks[pos])
        idx = [int(t) for t in toks[pos + 1:pos + 1 + k]]
        for j in range(1, k - 1):
            F.append([idx[0], idx[j], idx[j + 1]])
        pos += 1 + k
    return V, np.array(F, np.int32)


def config_mesh(name, seed=None):
    """The synthetic mesh of a named workload: 'c0', 'c1', 'c2', or 'small' (tests)."""
    if name == "c0":
        return sphere_mesh(5, amp=0.1, seed=0 if seed is None else seed)
    if name == "c1":
        return torus_knot_tube(seed=1 if seed is None else seed)
    if name == "c2":
        return sphere_mesh(9, amp=0.15, seed=2 if seed is None else seed)
    if name == "small":
        return sphere_mesh(3, amp=0.1, seed=0 if seed is None else seed)
    raise KeyError(name)


def batch_face_counts(count=256, seed=3, **kw):
    """Face counts of batch_meshes(count, seed) in generation order (what the batch's
    sharding over ranks is decided by)."""
    return [m["faces"] for m in batch_meshes(count, seed, **kw)]
