"""CPU oracle (test infrastructure) of the share-network features (restated in numpy).

Follows the feature definition of libits' its_share_features: for every corner vertex
coincident with a coarser corner (lattice coordinates all even below the root depth), 64
values -- signed distance, zero-share surplus values of its coincident copies and lattice
neighbours, neighbour presence, depth, cell width, and the face samples (centroids, unit
normals) summed over the owner node's 27-neighbourhood. Node sums are formed the same way
(finest nodes sum their faces in face order, every coarser node its 8 children in order),
so the FP64 sums agree exactly and the FP32 features to rounding of the last step.
"""
import math

import numpy as np

NONE = 0xFFFFFFFF


def _morton(x, y, z):
    m = 0
    for i in range(10):
        m |= ((x >> i) & 1) << (3 * i) | ((y >> i) & 1) << (3 * i + 1) | ((z >> i) & 1) << (3 * i + 2)
    return m


def share_features(svo, b, V, F, lam0):
    """(features n x 64 float32, vertex ids) of an oracle.Svo."""
    res, o, w = svo.res, np.asarray(svo.origin, np.float64), np.asarray(svo.width, np.float64)
    w0 = w[0] / res
    ncount, vcount = svo.depth_counts()
    D = len(vcount)
    vstart = np.concatenate([[0], np.cumsum(vcount)])
    nstart = np.concatenate([[0], np.cumsum(ncount)])
    pos, owner = svo.vertices()
    nodes = svo.nodes()
    n = len(pos)
    vd = np.searchsorted(vstart, np.arange(n), side="right") - 1
    wd = w0 * (2.0 ** vd)
    L = np.rint((pos - o[None, :]) / wd[:, None]).astype(np.int64)
    index = {(int(vd[i]), int(L[i, 0]), int(L[i, 1]), int(L[i, 2])): i for i in range(n)}

    def vert(d, X, Y, Z):
        return index.get((d, X, Y, Z), -1)

    # face samples and node sums
    A, B, Cc = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    cent = (A + B + Cc) / 3.0
    u, v = B - A, Cc - A
    nrm = np.stack([u[:, 1] * v[:, 2] - u[:, 2] * v[:, 1], u[:, 2] * v[:, 0] - u[:, 0] * v[:, 2],
                    u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]], 1)
    ln = np.sqrt(nrm[:, 0] * nrm[:, 0] + nrm[:, 1] * nrm[:, 1] + nrm[:, 2] * nrm[:, 2])
    nrm = np.where(ln[:, None] > 0, nrm / np.where(ln > 0, ln, 1.0)[:, None], nrm)
    fine = {int(m): k for k, m in enumerate(nodes["morton"][:ncount[0]])}
    N = len(nodes["morton"])
    cnt = np.zeros(N, np.float32)
    sp, sn = np.zeros((N, 3)), np.zeros((N, 3))
    for f in range(F.shape[0]):
        dx, dy, dz = (int((cent[f, a] - o[a]) / w0) for a in range(3))
        if min(dx, dy, dz) < 0 or max(dx, dy, dz) >= res:
            continue
        t = fine.get(_morton(dx, dy, dz))
        if t is None:
            continue
        cnt[t] += np.float32(1.0)
        sp[t] += cent[f]
        sn[t] += nrm[f]
    for lev in range(1, D):
        for t in range(nstart[lev], nstart[lev + 1]):
            ch = nodes["childs"][t]
            if ch[0] == NONE:
                continue
            c, p, q = np.float32(0.0), np.zeros(3), np.zeros(3)
            for k in range(8):
                c += cnt[ch[k]]
                p += sp[ch[k]]
                q += sn[ch[k]]
            cnt[t], sp[t], sn[t] = c, p, q
    ids = [i for i in range(n) if vd[i] + 1 < D and not (L[i] & 1).any()]
    out = np.zeros((len(ids), 64), np.float32)
    ex, ey, ez = [1, -1, 0, 0, 0, 0], [0, 0, 1, -1, 0, 0], [0, 0, 0, 0, 1, -1]
    for row, i in enumerate(ids):
        d = int(vd[i])
        X, Y, Z = (int(t) for t in L[i])
        wv = w0 * float(1 << d)
        f = np.zeros(64)
        up, down, top, one_up = 0, 0, i, 0.0
        X1, Y1, Z1 = X, Y, Z
        for dd in range(d + 1, D):
            if (X1 | Y1 | Z1) & 1:
                break
            X1, Y1, Z1 = X1 >> 1, Y1 >> 1, Z1 >> 1
            uu = vert(dd, X1, Y1, Z1)
            if uu < 0:
                break
            if dd == d + 1:
                one_up = lam0[uu]
            top, up = uu, up + 1
        for dd in range(d - 1, -1, -1):
            s = d - dd
            if vert(dd, X << s, Y << s, Z << s) < 0:
                break
            down += 1
        f[0], f[1], f[2] = b[i], lam0[top], one_up
        f[3] = d / (D - 1) if D > 1 else 0.0
        f[4], f[5] = up / D, down / D
        for k in range(6):
            uu = vert(d, X + ex[k], Y + ey[k], Z + ez[k])
            if uu >= 0:
                f[6 + k], f[12 + k], f[18 + k] = 1.0, b[uu] - b[i], lam0[uu]
            if d > 0:
                q = vert(d - 1, 2 * X + ex[k], 2 * Y + ey[k], 2 * Z + ez[k])
                if q >= 0:
                    f[24 + k], f[30 + k] = 1.0, lam0[q]
        f[36], f[37] = wv, b[i] / wv
        c, p, q = 0.0, np.zeros(3), np.zeros(3)
        for t in nodes["neighbors"][owner[i]]:
            if t == NONE:
                continue
            c += float(cnt[t])
            p += sp[t]
            q += sn[t]
        f[38] = math.log1p(c)
        if c > 0:
            m = q / c
            f[39:42] = (p / c - pos[i]) / wv
            f[42:45] = m
            f[45] = 1.0 - math.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])
        out[row] = f.astype(np.float32)
    return out, np.array(ids, np.int64)
