"""Mesh files and per-vertex geometry of triangulated surfaces (host side, numpy).

Readers and writers keep the file formats py-lddmm/surfaces.py reads and
writes, and the vertex-area / vertex-normal routines keep its arithmetic,
as whole-array numpy operations instead of per-face Python loops:

  read_byu / write_byu          surfaces.py:757-849  (Movie.BYU, 1-based, last index of a face negated)
  read_off                      surfaces.py:719-754  ('#' comment lines skipped)
  read_vtk / write_vtk          surfaces.py:851-955  (legacy ASCII POLYDATA: POINTS + triangle POLYGONS)
  read_obj                      surfaces.py:957-985  ('v' and 'f' records)
  vertex_area                   surfaces.py:77-126   (mixed Voronoi / obtuse-face areas)
  vertex_normals                surfaces.py:128-139  (sum of incident surfels, normalised)

The reference reads .vtk and .obj through the VTK library; here the legacy
ASCII polydata that its own writer produces and plain OBJ text are parsed
directly (binary VTK files are not read).  Like the reference's VTK path, a
polygon with more than three corners keeps its first three.
"""
import logging

import numpy as np


class vtkFields:
    """Point-data fields of a VTK file (surfaces.py:16-21): each list holds
    name, array, name, array, ..."""

    def __init__(self):
        self.scalars = []
        self.vectors = []
        self.normals = []
        self.tensors = []


def readskip(f, c):
    """Next line of f that does not start with c (surfaces.py:1279-1284)."""
    ln0 = f.readline()
    while len(ln0) > 0 and ln0[0] == c:
        ln0 = f.readline()
    return ln0


# -- Movie.BYU -------------------------------------------------------------------------------
def read_byu(path):
    """(vertices (n, 3) float64, faces (f, 3) int) of a .byu file: header
    `ncomponents npoints nfaces ...`, one line per component, the coordinates,
    then the 1-based face indices with the last index of each face negated."""
    with open(path) as fh:
        head = fh.readline().split()
        ncomp, npoints, nfaces = int(head[0]), int(head[1]), int(head[2])
        for _ in range(ncomp):
            fh.readline()
        tokens = fh.read().split()
    nv = 3 * npoints
    if len(tokens) < nv + 3 * nfaces:
        raise ValueError("%s: truncated .byu file" % path)
    vertices = np.array(tokens[:nv], dtype=np.float64).reshape(npoints, 3)
    faces = np.abs(np.array(tokens[nv:nv + 3 * nfaces], dtype=np.int64)).reshape(nfaces, 3) - 1
    return vertices, faces


def write_byu(path, vertices, faces):
    """The reference's .byu writer, byte for byte (surfaces.py:807-849): two
    vertices per line, 16 face indices per line."""
    V = np.asarray(vertices, dtype=np.float64)
    F = np.asarray(faces)
    npoints, nfaces = V.shape[0], F.shape[0]
    out = ['{0: d} {1: d} {2: d} {3: d} 0\n'.format(1, npoints, nfaces, 3 * nfaces), '1 {0: d}\n'.format(nfaces)]
    for k in range(0, npoints, 2):
        out.append('{0: f} {1: f} {2: f} '.format(V[k, 0], V[k, 1], V[k, 2]))
        if k + 1 < npoints:
            out.append('{0: f} {1: f} {2: f}\n'.format(V[k + 1, 0], V[k + 1, 1], V[k + 1, 2]))
        else:
            out.append('\n')
    idx = (F[:, :3].astype(np.int64) + 1)
    idx[:, 2] = -idx[:, 2]
    flat = idx.reshape(-1)
    for j in range(0, flat.size, 16):
        out.append(''.join('{0: d} '.format(int(i)) for i in flat[j:j + 16]))
        if j + 16 <= flat.size:
            out.append('\n')
    with open(path, 'w') as fh:
        fh.write(''.join(out))


# -- OFF ----------------------------------------------------------------------------------------
def read_off(path):
    """(vertices, faces) of an OFF file with triangular faces; lines starting
    with '#' are skipped as in the reference."""
    with open(path) as fh:
        def nxt():
            ln = readskip(fh, '#')
            while ln and not ln.strip():
                ln = readskip(fh, '#')
            return ln.split()
        ln = nxt()
        if not ln or ln[0].lower() != 'off':
            raise ValueError("%s: not OFF format" % path)
        ln = nxt()
        npoints, nfaces = int(ln[0]), int(ln[1])
        V = np.empty((npoints, 3))
        for k in range(npoints):
            V[k] = [float(s) for s in nxt()[:3]]
        F = np.empty((nfaces, 3), dtype=np.int64)
        for k in range(nfaces):
            ln = nxt()
            if int(ln[0]) != 3:
                raise ValueError("%s: reading only triangulated surfaces" % path)
            F[k] = [int(s) for s in ln[1:4]]
    return V, F


# -- VTK legacy ASCII polydata ------------------------------------------------------------------
def read_vtk(path):
    """(vertices, faces) of a legacy ASCII VTK POLYDATA file (POINTS and
    POLYGONS sections; other sections are skipped)."""
    with open(path) as fh:
        tokens = fh.read().split()
    V = F = None
    i = 0
    n = len(tokens)
    while i < n:
        t = tokens[i].upper()
        if t == 'BINARY':
            raise ValueError("%s: binary VTK files are not read" % path)
        if t == 'POINTS':
            npoints = int(tokens[i + 1])
            V = np.array(tokens[i + 3:i + 3 + 3 * npoints], dtype=np.float64).reshape(npoints, 3)
            i += 3 + 3 * npoints
            continue
        if t == 'POLYGONS':
            npoly, size = int(tokens[i + 1]), int(tokens[i + 2])
            rec = np.array(tokens[i + 3:i + 3 + size], dtype=np.int64)
            F = np.empty((npoly, 3), dtype=np.int64)
            j = 0
            for k in range(npoly):
                c = int(rec[j])
                if c < 3:
                    raise ValueError("%s: polygon with fewer than 3 corners" % path)
                F[k] = rec[j + 1:j + 4]
                j += c + 1
            i += 3 + size
            continue
        i += 1
    if V is None:
        raise ValueError("%s: no POINTS section" % path)
    if F is None:
        F = np.empty((0, 3), dtype=np.int64)
    return V, F


def write_vtk(path, vertices, faces, fields=None):
    """The reference's legacy ASCII POLYDATA writer (surfaces.py:869-925):
    points and triangles, then the point-data fields of a vtkFields."""
    V = np.asarray(vertices, dtype=np.float64)
    F = np.asarray(faces)
    out = ['# vtk DataFile Version 3.0\nSurface Data\nASCII\nDATASET POLYDATA\n',
           '\nPOINTS {0: d} float'.format(V.shape[0])]
    out += ['\n{0: f} {1: f} {2: f}'.format(p[0], p[1], p[2]) for p in V]
    out.append('\nPOLYGONS {0:d} {1:d}'.format(F.shape[0], 4 * F.shape[0]))
    out += ['\n3 {0: d} {1: d} {2: d}'.format(int(f[0]), int(f[1]), int(f[2])) for f in F]
    if fields is not None:
        hdr = ['\nPOINT_DATA {0: d}'.format(V.shape[0])]

        def header():
            if hdr:
                out.append(hdr.pop())
        for k in range(len(fields.scalars) // 2):
            header()
            out.append('\nSCALARS ' + fields.scalars[2 * k] + ' float 1\nLOOKUP_TABLE default')
            s = np.asarray(fields.scalars[2 * k + 1]).reshape(-1)
            out += ['\n {0: .5f}'.format(float(s[ll])) for ll in range(V.shape[0])]
        for kind, lst in (('VECTORS', fields.vectors), ('NORMALS', fields.normals)):
            for k in range(len(lst) // 2):
                header()
                out.append('\n' + kind + ' ' + lst[2 * k] + ' float')
                a = np.asarray(lst[2 * k + 1])
                out += ['\n {0: .5f} {1: .5f} {2: .5f}'.format(a[ll, 0], a[ll, 1], a[ll, 2])
                        for ll in range(V.shape[0])]
        for k in range(len(fields.tensors) // 2):
            header()
            out.append('\nTENSORS ' + fields.tensors[2 * k] + ' float')
            a = np.asarray(fields.tensors[2 * k + 1])
            for ll in range(V.shape[0]):
                for kk in range(2):
                    out.append('\n {0: .5f} {1: .5f} {2: .5f}'.format(a[ll, kk, 0], a[ll, kk, 1], a[ll, kk, 2]))
        out.append('\n')
    with open(path, 'w') as fh:
        fh.write(''.join(out))


# -- OBJ ----------------------------------------------------------------------------------------
def read_obj(path):
    """(vertices, faces) of an OBJ file: 'v x y z' and 'f i j k ...' records
    (1-based or negative relative indices, 'i/t/n' forms accepted)."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            p = line.split()
            if not p:
                continue
            if p[0] == 'v':
                verts.append([float(s) for s in p[1:4]])
            elif p[0] == 'f':
                idx = []
                for s in p[1:4]:
                    i = int(s.split('/')[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                if len(idx) < 3:
                    raise ValueError("%s: face with fewer than 3 corners" % path)
                faces.append(idx)
    return np.array(verts, dtype=np.float64).reshape(-1, 3), np.array(faces, dtype=np.int64).reshape(-1, 3)


# -- per-vertex geometry -------------------------------------------------------------------------
def vertex_area(vertices, faces):
    """(AV (nv, 1), AF (nf, 1)): face areas and the mixed vertex areas of
    surfaces.py:77-126 -- half / quarter of the area to the corners of an
    obtuse face, the cotangent (Voronoi) shares otherwise.  Contributions are
    accumulated in the reference's order (face by face, corners in order)."""
    V = np.asarray(vertices, dtype=np.float64)
    F = np.asarray(faces)
    x12 = V[F[:, 1]] - V[F[:, 0]]
    x13 = V[F[:, 2]] - V[F[:, 0]]
    x23 = V[F[:, 2]] - V[F[:, 1]]
    s12, s13, s23 = (x12 ** 2).sum(axis=1), (x13 ** 2).sum(axis=1), (x23 ** 2).sum(axis=1)
    n12, n13, n23 = np.sqrt(s12), np.sqrt(s13), np.sqrt(s23)
    c1 = (x12 * x13).sum(axis=1) / (n12 * n13)
    c2 = -(x12 * x23).sum(axis=1) / (n12 * n23)
    c3 = (x13 * x23).sum(axis=1) / (n13 * n23)
    AF = np.sqrt((np.cross(x12, x13) ** 2).sum(axis=1)) / 2
    ob1 = c1 < 0
    ob2 = ~ob1 & (c2 < 0)
    ob3 = ~ob1 & ~ob2 & (c3 < 0)
    acute = ~(ob1 | ob2 | ob3)
    contrib = np.empty((F.shape[0], 3))
    half, quarter = AF / 2, AF / 4
    for m, big in ((ob1, 0), (ob2, 1), (ob3, 2)):
        for j in range(3):
            contrib[m, j] = half[m] if j == big else quarter[m]
    with np.errstate(divide='ignore', invalid='ignore'):
        cot1 = c1 / np.sqrt(1 - c1 ** 2)
        cot2 = c2 / np.sqrt(1 - c2 ** 2)
        cot3 = c3 / np.sqrt(1 - c3 ** 2)
    a = acute
    contrib[a, 0] = (s12[a] * cot3[a] + s13[a] * cot2[a]) / 8
    contrib[a, 1] = (s12[a] * cot3[a] + s23[a] * cot1[a]) / 8
    contrib[a, 2] = (s13[a] * cot2[a] + s23[a] * cot1[a]) / 8
    AV = np.zeros(V.shape[0])
    np.add.at(AV, F[:, :3].reshape(-1), contrib.reshape(-1))
    iso = np.flatnonzero(np.fabs(AV) < 1e-10)
    if iso.size:
        logging.warning('vertices %s have no face; use removeIsolated', iso[:10].tolist())
    return AV.reshape(-1, 1), AF.reshape(-1, 1)


def vertex_normals(vertices, faces):
    """Unit vertex normals: the sum of the incident faces' surfels
    (x2 - x1) x (x3 - x1), normalised (surfaces.py:128-139)."""
    V = np.asarray(vertices, dtype=np.float64)
    F = np.asarray(faces)
    x1, x2, x3 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    surfel = np.cross(x2 - x1, x3 - x1)
    normals = np.zeros(V.shape)
    np.add.at(normals, F[:, :3].reshape(-1), np.repeat(surfel, 3, axis=0))
    af = np.sqrt((normals ** 2).sum(axis=1))
    return normals / af.reshape(-1, 1)
