"""Mesh files for headless scenes: a Gmsh MSH 4.1 ASCII tetrahedral-mesh
reader (replacing the reference's gmsh-library loader), an MSH writer, and
OBJ / PLY surface writers for frame dumps.

`read_msh` follows MeshUtils::loadTetMeshFromGmshFile
(common/mesh/MeshUtils.cpp:66-191): vertices are the nodes of every entity
in (dimension, tag) order, element node tags map to vertex index tag - 1,
4-node tetrahedra (element type 4) become elements and 3-node triangles
(type 2) become surface faces; other element types are ignored.
"""
from __future__ import annotations

import numpy as np


class MshError(ValueError):
    pass


def _sections(lines):
    """{name: [lines between $name and $Endname]} (first occurrence)."""
    out, cur, buf = {}, None, []
    for ln in lines:
        s = ln.strip()
        if s.startswith("$"):
            if cur is None:
                cur, buf = s[1:], []
            elif s == "$End" + cur:
                out.setdefault(cur, buf)
                cur = None
            continue
        if cur is not None:
            buf.append(s)
    if cur is not None:
        raise MshError(f"section ${cur} is not closed")
    return out


def read_msh(path: str):
    """Returns (vertices float64 [n, 3], tets int64 [m, 4], faces int64 [k, 3])."""
    with open(path, "r") as f:
        lines = f.read().splitlines()
    sec = _sections(lines)
    if "MeshFormat" not in sec:
        raise MshError("not a Gmsh MSH file ($MeshFormat missing)")
    ver, ftype = sec["MeshFormat"][0].split()[:2]
    if not ver.startswith("4"):
        raise MshError(f"MSH version {ver} not supported (4.1 expected)")
    if ftype != "0":
        raise MshError("binary MSH not supported (ASCII expected)")
    # nodes, per entity block
    tok = " ".join(sec["Nodes"]).split()
    it = iter(tok)
    nblocks, _nnodes = int(next(it)), int(next(it))
    next(it), next(it)
    blocks = []
    for _ in range(nblocks):
        dim, tag, param, cnt = int(next(it)), int(next(it)), int(next(it)), int(next(it))
        tags = [int(next(it)) for _ in range(cnt)]
        ncoord = 3 + (dim if param else 0)
        xyz = np.array([float(next(it)) for _ in range(cnt * ncoord)], dtype=np.float64).reshape(cnt, ncoord)[:, :3]
        blocks.append(((dim, tag), tags, xyz))
    blocks.sort(key=lambda b: b[0])
    tags = [t for b in blocks for t in b[1]]
    verts = np.concatenate([b[2] for b in blocks]) if blocks else np.zeros((0, 3))
    if tags != list(range(1, len(tags) + 1)):
        raise MshError("node tags are not 1..n in entity order (the reference indexes vertices by tag - 1)")
    # elements, per entity block
    tok = " ".join(sec.get("Elements", ["0 0 0 0"])).split()
    it = iter(tok)
    nblocks = int(next(it))
    next(it), next(it), next(it)
    eblocks = []
    nodes_per = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 11: 10, 15: 1}
    for _ in range(nblocks):
        dim, tag, etype, cnt = int(next(it)), int(next(it)), int(next(it)), int(next(it))
        if etype not in nodes_per:
            raise MshError(f"element type {etype} not supported")
        k = nodes_per[etype]
        rows = [[int(next(it)) for _ in range(k + 1)] for _ in range(cnt)]
        eblocks.append(((dim, tag), etype, rows))
    eblocks.sort(key=lambda b: b[0])
    tets = [r[1:] for b in eblocks if b[1] == 4 for r in b[2]]
    faces = [r[1:] for b in eblocks if b[1] == 2 for r in b[2]]
    tets = np.array(tets, dtype=np.int64).reshape(-1, 4) - 1
    faces = np.array(faces, dtype=np.int64).reshape(-1, 3) - 1
    n = len(verts)
    for a in (tets, faces):
        if a.size and (a.min() < 0 or a.max() >= n):
            raise MshError("element references a node that does not exist")
    return verts, tets, faces


def grid_vertices(n: int, size: float = 1.0):
    """Vertices of an n^3-cell cube grid, x fastest (the vertex order of
    scenes.hex_grid_tets)."""
    m = n + 1
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * (size / n)


def outward_surface(vertices, tets):
    """Boundary triangles of a tet mesh, each wound counter-clockwise seen
    from outside (the orientation gmsh writes, which the volume-weighted
    centre of mass of ParticleMesh::massCenter relies on)."""
    X = np.asarray(vertices, dtype=np.float64)
    T = np.asarray(tets, dtype=np.int64).reshape(-1, 4)
    faces, opp = [], []
    for a, b, c, d in ((0, 1, 2, 3), (0, 1, 3, 2), (0, 2, 3, 1), (1, 2, 3, 0)):
        faces.append(T[:, [a, b, c]])
        opp.append(T[:, d])
    F, O = np.concatenate(faces), np.concatenate(opp)
    _, inv, cnt = np.unique(np.sort(F, axis=1), axis=0, return_inverse=True, return_counts=True)
    keep = cnt[inv.ravel()] == 1
    F, O = F[keep], O[keep]
    n = np.cross(X[F[:, 1]] - X[F[:, 0]], X[F[:, 2]] - X[F[:, 0]])
    inward = np.einsum("ij,ij->i", n, X[O] - X[F[:, 0]]) > 0
    F[inward] = F[inward][:, [0, 2, 1]]
    return F


def write_msh(path: str, vertices, tets, faces=None):
    """MSH 4.1 ASCII: one volume entity holding all nodes, its tetrahedra and
    (optionally) surface triangles in one surface entity."""
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(tets, dtype=np.int64).reshape(-1, 4)
    fc = np.asarray(faces if faces is not None else np.zeros((0, 3)), dtype=np.int64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        f.write("$Nodes\n1 %d 1 %d\n3 1 0 %d\n" % (len(v), len(v), len(v)))
        f.write("".join("%d\n" % (i + 1) for i in range(len(v))))
        f.write("".join("%.17g %.17g %.17g\n" % tuple(p) for p in v))
        f.write("$EndNodes\n")
        nb = 1 + (1 if len(fc) else 0)
        f.write("$Elements\n%d %d 1 %d\n" % (nb, len(t) + len(fc), len(t) + len(fc)))
        k = 1
        if len(fc):
            f.write("2 1 2 %d\n" % len(fc))
            for r in fc:
                f.write("%d %d %d %d\n" % (k, r[0] + 1, r[1] + 1, r[2] + 1))
                k += 1
        f.write("3 1 4 %d\n" % len(t))
        for r in t:
            f.write("%d %d %d %d %d\n" % (k, r[0] + 1, r[1] + 1, r[2] + 1, r[3] + 1))
            k += 1
        f.write("$EndElements\n")


def write_obj(path: str, vertices, faces, lines=None):
    """Wavefront OBJ of triangles (and optional polylines, e.g. rods)."""
    v = np.asarray(vertices, dtype=np.float64)
    with open(path, "w") as f:
        f.write("".join("v %.9g %.9g %.9g\n" % tuple(p) for p in v))
        f.write("".join("f %d %d %d\n" % (a + 1, b + 1, c + 1) for a, b, c in np.asarray(faces).reshape(-1, 3)))
        for pl in lines or []:
            f.write("l " + " ".join(str(int(i) + 1) for i in pl) + "\n")


def write_ply(path: str, vertices, faces):
    """Binary little-endian PLY of triangles (float32 positions)."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
    fc = np.asarray(faces, dtype=np.int32).reshape(-1, 3)
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\nproperty float x\nproperty float y\n"
            "property float z\nelement face %d\nproperty list uchar int vertex_indices\nend_header\n" % (len(v), len(fc)))
    rec = np.zeros(len(fc), dtype=[("n", "u1"), ("i", "<i4", 3)])
    rec["n"] = 3
    rec["i"] = fc
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(v.astype("<f4").tobytes())
        f.write(rec.tobytes())
