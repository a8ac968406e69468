"""Seeded synthetic shapes for the benchmark configurations.

The reference reads meshes from disk (VTK isosurfaces of segmentations); every
figure here uses synthetic shapes generated from a seed instead:

* ``icosphere(k)``: subdivided icosahedron on the unit sphere, 10*4^k+2
  vertices / 20*4^k faces, faces oriented outward (positive volume);
* ``bumped_sphere``: target surface, vertices moved along their normal by a
  sum of Gaussian bumps of the chord distance to random sphere points;
* ``ellipse_curve`` / ``bumped_curve``: closed 2-D curves for curve matching,
  resampled by arc length;
* ``decimate``: random edge collapse down to a requested vertex count, used
  for the ragged serving mix.
"""
import numpy as np


def _icosahedron():
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, f


def _orient_outward(v, f):
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(b - a, c - a)
    flip = (n * (a + b + c)).sum(axis=1) < 0
    f = f.copy()
    f[flip] = f[flip][:, [0, 2, 1]]
    return f


def icosphere(subdiv, radius=1.0):
    """Returns (vertices (10*4^k+2, 3), faces (20*4^k, 3) int64)."""
    v, f = _icosahedron()
    f = _orient_outward(v, f)
    verts = [p for p in v]
    for _ in range(int(subdiv)):
        cache = {}

        def mid(i, j):
            key = (i, j) if i < j else (j, i)
            idx = cache.get(key)
            if idx is None:
                p = verts[i] + verts[j]
                p = p / np.linalg.norm(p)
                verts.append(p)
                idx = len(verts) - 1
                cache[key] = idx
            return idx

        nf = np.empty((4 * len(f), 3), dtype=np.int64)
        for q, (a, b, c) in enumerate(f):
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf[4 * q + 0] = (a, ab, ca)
            nf[4 * q + 1] = (b, bc, ab)
            nf[4 * q + 2] = (c, ca, bc)
            nf[4 * q + 3] = (ab, bc, ca)
        f = nf
    v = np.array(verts) * radius
    return v, f


def vertex_normals(v, f):
    """Area-weighted vertex normals (unit length)."""
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(b - a, c - a)
    vn = np.zeros_like(v)
    for j in range(3):
        np.add.at(vn, f[:, j], n)
    return vn / np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-300)


def bumped_sphere(v, f, n_bumps, width, amp, rng):
    """Each vertex moved along its normal by sum_i A_i exp(-g_i^2 / (2 width^2)),
    g_i the chord distance to a centre uniform on the sphere, A_i ~ U[-amp, amp]."""
    c = rng.standard_normal((n_bumps, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    A = rng.uniform(-amp, amp, n_bumps)
    nrm = vertex_normals(v, f)
    r = np.linalg.norm(v, axis=1, keepdims=True)
    g2 = ((v[:, None, :] / r[:, :, None] - c[None]) ** 2).sum(axis=2)
    disp = (A[None, :] * np.exp(-g2 / (2 * width ** 2))).sum(axis=1)
    return v + disp[:, None] * nrm


def resample_closed(pts, n):
    """Arc-length resampling of a closed polygon to n vertices."""
    P = np.vstack([pts, pts[:1]])
    seg = np.linalg.norm(np.diff(P, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    t = np.linspace(0.0, s[-1], n, endpoint=False)
    out = np.empty((n, pts.shape[1]))
    for j in range(pts.shape[1]):
        out[:, j] = np.interp(t, s, P[:, j])
    return out


def ellipse_curve(n=256, a=1.0, b=0.6):
    """Closed ellipse with n vertices at equal parameter spacing; edges k->k+1, last->0."""
    th = 2 * np.pi * np.arange(n) / n
    v = np.stack([a * np.cos(th), b * np.sin(th)], axis=1)
    f = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int64)
    return v, f


def bumped_curve(v, n_bumps, width, amp_std, rng, n_out=None):
    """Template displaced by sum_i A_i exp(-|x-c_i|^2/(2 width^2)), c_i ~ U[-1,1]^2,
    A_i ~ N(0, amp_std^2) per axis, then resampled by arc length."""
    c = rng.uniform(-1, 1, (n_bumps, 2))
    A = rng.normal(0.0, amp_std, (n_bumps, 2))
    d2 = ((v[:, None, :] - c[None]) ** 2).sum(axis=2)
    w = np.exp(-d2 / (2 * width ** 2))
    out = v + w @ A
    n = v.shape[0] if n_out is None else n_out
    out = resample_closed(out, n)
    f = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int64)
    return out, f


def decimate(v, f, target_vertices, rng):
    """Random edge collapse (midpoint) until ``target_vertices`` remain.

    Each round proposes one random edge per face with a random priority and
    collapses, all at once, the edges whose priority is the smallest within
    the 1-rings of both end points (so simultaneous collapses never touch the
    same triangles) and whose end points share exactly two neighbours (the
    link condition: the surface stays a closed 2-manifold).  Faces that
    degenerate are dropped and vertex indices are compacted at the end;
    orientation of the surviving faces is unchanged."""
    import scipy.sparse as sp
    v = v.copy()
    f = np.asarray(f, dtype=np.int64).copy()
    nv = len(v)
    alive = np.ones(nv, dtype=bool)
    n_alive = nv
    while n_alive > target_vertices and len(f) > 4:
        rows = np.arange(len(f))
        j = rng.integers(3, size=len(f))
        a = f[rows, j]
        b = f[rows, (j + 1) % 3]
        pr = rng.random(len(f))
        best = np.full(nv, np.inf)
        np.minimum.at(best, a, pr)
        np.minimum.at(best, b, pr)
        fb = best[f].min(axis=1)
        ring = np.full(nv, np.inf)
        for c in range(3):
            np.minimum.at(ring, f[:, c], fb)
        sel = np.flatnonzero((ring[a] == pr) & (ring[b] == pr) & (a != b))
        if sel.size:
            e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
            adj = sp.csr_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(nv, nv))
            adj = ((adj + adj.T) > 0).astype(np.float64)
            common = np.asarray(adj[a[sel]].multiply(adj[b[sel]]).sum(axis=1)).ravel()
            sel = sel[common == 2]
        cap = n_alive - target_vertices
        sel = sel[np.argsort(pr[sel], kind="stable")[:cap]]
        if sel.size == 0:
            break
        a, b = a[sel], b[sel]
        v[a] = 0.5 * (v[a] + v[b])
        alive[b] = False
        n_alive -= sel.size
        remap = np.arange(nv)
        remap[b] = a
        f = remap[f]
        keep = (f[:, 0] != f[:, 1]) & (f[:, 1] != f[:, 2]) & (f[:, 2] != f[:, 0])
        f = f[keep]
    idx = np.flatnonzero(alive)
    new = -np.ones(nv, dtype=np.int64)
    new[idx] = np.arange(len(idx))
    return v[idx], new[f]
