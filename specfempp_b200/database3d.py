"""The reference's 3D mesh database (``database.bin`` written by its 3D
mesher) and its mapping onto the structured hexahedral lattice of the 3D
library.

``read_database3d`` follows the record order of the reference's reader
(src/io/mesh/impl/fortran/dim3/mesh.cpp:14-70): a Fortran unformatted
sequential file whose records are ``[int32 n][n bytes][int32 n]``, holding

* the earth-chunk flag (a 4-byte logical; a chunk mesh is refused, mesh.cpp:24-30);
* ``ngnod``, ``nnodes`` and one ``(index, x, y, z)`` record per control node
  (read_control_nodes.cpp:8-57);
* ``(nmaterials, nundefined)``, 17 doubles per material (rho, vp, vs, Qkappa,
  Qmu, anisotropy flag, material id, ...), ``nspec``, ``(ngllz, nglly,
  ngllx)`` and one ``(index, material, tomographic flag, ngnod node ids)``
  record per element (read_materials.cpp:12-157);
* six ``(direction, nfaces)`` records, then per face ``(element, 4 or 9
  node ids)`` (read_boundaries.cpp:181-276);
* the PML count and the MPI-interface counts, both zero
  (read_pml_boundaries.cpp, read_mpi_interfaces.cpp), and the adjacency
  list (read_adjacency_graph.cpp), which is not needed here.

``lattice_mesh`` turns the element list into the library's lattice
(``meshgen.Mesh3D``): elements are linked through shared faces (the +xi face
``(1, 2, 6, 5)`` of one element is the -xi face ``(0, 3, 7, 4)`` of its
neighbour, likewise for eta and zeta, with the reference's corner order of
read_boundaries.cpp:96-112), each element's lattice position is its
distance along the -xi, -eta and -zeta chains, and every lattice node must
receive the same control node from all elements that share it.  Meshes that
are not such a lattice (unstructured or inconsistently oriented elements,
curved 27-node elements) are refused with the reason.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

from . import meshgen

# corner order of an 8-node hexahedron: bottom (zeta = -1) 0 1 2 3, top 4 5 6 7,
# corner c at (xi, eta, zeta) signs CORNER_SIGNS[c]
CORNER_SIGNS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
# faces as corner tuples: the minus face of the next element along an axis
# repeats the plus face of this one in the same order
MINUS_FACE = {0: (0, 3, 7, 4), 1: (0, 1, 5, 4), 2: (0, 1, 2, 3)}
PLUS_FACE = {0: (1, 2, 6, 5), 1: (3, 2, 6, 7), 2: (4, 5, 6, 7)}
# directions of the boundary records: xmin, xmax, ymin, ymax, zmin, zmax
DIRECTIONS = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


@dataclass
class Database3D:
    ngnod: int
    coords: np.ndarray            # [nnodes, 3] float64, control node i at row i
    elements: np.ndarray          # [nspec, ngnod] int64, 0-based control node ids
    material_of: np.ndarray       # [nspec] int64, 0-based material index
    materials: np.ndarray         # [nmaterials, 17] float64
    ngll: tuple                   # (ngllz, nglly, ngllx)
    faces: dict                   # direction -> ([nfaces] element ids, [nfaces, 4|9] node ids), 0-based

    @property
    def nspec(self):
        return len(self.elements)


def _records(buf: bytes):
    out, o, n = [], 0, len(buf)
    while o < n:
        if o + 4 > n:
            raise ValueError("database: truncated record header")
        ln = struct.unpack_from("<i", buf, o)[0]
        if ln < 0 or o + 8 + ln > n or struct.unpack_from("<i", buf, o + 4 + ln)[0] != ln:
            raise ValueError(f"database: malformed record at byte {o}")
        out.append(buf[o + 4:o + 4 + ln])
        o += 8 + ln
    return out


def parse_database3d(buf: bytes) -> Database3D:
    """Parse the bytes of a 3D ``database.bin`` (record layout above)."""
    recs = _records(buf)
    it = iter(recs)

    def nxt(fmt=None):
        try:
            r = next(it)
        except StopIteration:
            raise ValueError("database: ends early") from None
        if fmt is None:
            return r
        if struct.calcsize(fmt) != len(r):
            raise ValueError(f"database: record of {len(r)} bytes where {fmt} was expected")
        return struct.unpack(fmt, r)

    chunk = nxt()
    if any(chunk):
        raise ValueError("Mesh of earth chunk is not supported")
    (ngnod,) = nxt("<i")
    if ngnod not in (8, 27):
        raise ValueError(f"database: {ngnod} control nodes per element (8 or 27 expected)")
    (nnodes,) = nxt("<i")
    node_recs = [nxt() for _ in range(nnodes)]
    nodes = np.frombuffer(b"".join(node_recs), dtype=np.dtype([("i", "<i4"), ("x", "<f8", 3)]))
    if len(nodes) != nnodes:
        raise ValueError("database: control node records of unexpected size")
    idx = nodes["i"].astype(np.int64) - 1
    if idx.min() < 0 or idx.max() >= nnodes or len(np.unique(idx)) != nnodes:
        raise ValueError("database: control node indices are not 1..nnodes")
    coords = np.zeros((nnodes, 3))
    coords[idx] = nodes["x"]
    nmat, nundef = nxt("<ii")
    materials = np.array([nxt("<17d") for _ in range(nmat)], dtype=np.float64).reshape(nmat, 17)
    for _ in range(nundef):
        nxt()
    (nspec,) = nxt("<i")
    ngll = nxt("<iii")
    el = np.frombuffer(b"".join(nxt() for _ in range(nspec)), dtype="<i4")
    if el.size != nspec * (3 + ngnod):
        raise ValueError("database: element records of unexpected size")
    el = el.reshape(nspec, 3 + ngnod).astype(np.int64)
    eidx = el[:, 0] - 1
    if eidx.min() < 0 or eidx.max() >= nspec or len(np.unique(eidx)) != nspec:
        raise ValueError("Error reading material indices")
    if (el[:, 1] < 1).any() or (el[:, 1] > nmat).any():
        raise ValueError("Error reading material indices (tomographic or undefined materials are not supported)")
    elements = np.zeros((nspec, ngnod), np.int64)
    elements[eidx] = el[:, 3:] - 1
    material_of = np.zeros(nspec, np.int64)
    material_of[eidx] = el[:, 1] - 1
    if elements.min() < 0 or elements.max() >= nnodes:
        raise ValueError("database: element refers to a missing control node")
    counts = []
    for d in range(6):
        num, nf = nxt("<ii")
        if num != d + 1:
            raise ValueError(f"Invalid database format: expected boundary number {d + 1}")
        counts.append(nf)
    nface_nodes = 4 if ngnod == 8 else 9
    faces = {}
    for d, nf in enumerate(counts):
        f = np.frombuffer(b"".join(nxt() for _ in range(nf)), dtype="<i4")
        if f.size != nf * (1 + nface_nodes):
            raise ValueError("database: face records of unexpected size")
        f = f.reshape(nf, 1 + nface_nodes).astype(np.int64) - 1
        faces[DIRECTIONS[d]] = (f[:, 0], f[:, 1:])
    (npml,) = nxt("<i")
    if npml != 0:
        raise ValueError("PML boundaries are not supported")
    nif, maxel = nxt("<ii")
    if nif != 0 and maxel != 0:
        raise ValueError("MPI interfaces are not supported")
    return Database3D(ngnod, coords, elements, material_of, materials, tuple(ngll), faces)


def read_database3d(path: str) -> Database3D:
    with open(path, "rb") as f:
        return parse_database3d(f.read())


def _face_neighbours(corners: np.ndarray, axis: int) -> np.ndarray:
    """[nspec] element across the +axis face of each element, or -1."""
    n = len(corners)
    minus = corners[:, MINUS_FACE[axis]]
    plus = corners[:, PLUS_FACE[axis]]
    allf = np.concatenate([minus, plus])
    _, inv = np.unique(allf, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    owner_minus = np.full(inv.max() + 1, -1, np.int64)
    if len(np.unique(inv[:n])) != n:
        raise ValueError("the mesh is not a hexahedral lattice: a face is the minus face of two elements")
    owner_minus[inv[:n]] = np.arange(n)
    return owner_minus[inv[n:]]


def _chain_length(prev: np.ndarray, limit: int) -> np.ndarray:
    """Number of steps back along ``prev`` (element before, or -1) to the chain's start."""
    pos = np.zeros(len(prev), np.int64)
    has = prev >= 0
    for _ in range(limit + 1):
        new = np.where(has, pos[np.maximum(prev, 0)] + 1, 0)
        if np.array_equal(new, pos):
            return pos
        pos = new
    raise ValueError("the mesh is not a hexahedral lattice: its element chains are cyclic")


def lattice_of(db: Database3D):
    """(nex, ney, nez, lattice position [nspec, 3], lattice node -> control
    node id [(nez+1)(ney+1)(nex+1)]) of the database's elements."""
    n = db.nspec
    corners = db.elements[:, :8]
    pos = np.zeros((n, 3), np.int64)
    for axis in range(3):
        after = _face_neighbours(corners, axis)
        before = np.full(n, -1, np.int64)
        m = after >= 0
        before[after[m]] = np.nonzero(m)[0]
        pos[:, axis] = _chain_length(before, n)
    ne = pos.max(axis=0) + 1
    nex, ney, nez = (int(v) for v in ne)
    if nex * ney * nez != n:
        raise ValueError(f"the mesh is not a hexahedral lattice ({n} elements in a "
                         f"{nex} x {ney} x {nez} bounding lattice)")
    slot = (pos[:, 2] * ney + pos[:, 1]) * nex + pos[:, 0]
    if len(np.unique(slot)) != n:
        raise ValueError("the mesh is not a hexahedral lattice: two elements share a lattice position")
    nnode = (nez + 1) * (ney + 1) * (nex + 1)
    node_id = np.full(nnode, -1, np.int64)
    for c in range(8):
        p = pos + CORNER_SIGNS[c]
        lat = (p[:, 2] * (ney + 1) + p[:, 1]) * (nex + 1) + p[:, 0]
        prev = node_id[lat]
        clash = (prev >= 0) & (prev != corners[:, c])
        if clash.any():
            raise ValueError("the mesh is not a hexahedral lattice: elements disagree on a shared corner")
        node_id[lat] = corners[:, c]
    if (node_id < 0).any():
        raise ValueError("the mesh is not a hexahedral lattice: a lattice node has no element")
    return nex, ney, nez, pos, node_id


# the 19 extra nodes of a 27-node hexahedron sit at the edge midpoints, face
# centres and centre, (xi, eta, zeta) in {0, 1/2, 1} with at least one 1/2
_HEX27_REST = np.array([[a, b, c] for c in (0, 1, 2) for b in (0, 1, 2) for a in (0, 1, 2)
                        if 1 in (a, b, c)]) / 2.0


def _check_hex27_affine(db: Database3D, tol: float = 1e-6):
    """27-node elements are accepted when each extra node sits where the
    trilinear map of the 8 corners puts one of the 19 midpoints (straight-
    sided elements; the check does not depend on the order of the extra
    nodes)."""
    P = db.coords[db.elements[:, :8]]                       # [nspec, 8, 3]
    w = np.array([[(a if s[0] else 1 - a) * (b if s[1] else 1 - b) * (c if s[2] else 1 - c)
                   for s in CORNER_SIGNS] for a, b, c in _HEX27_REST])        # [19, 8]
    want = np.einsum("kc,ncd->nkd", w, P)                   # [nspec, 19, 3]
    got = db.coords[db.elements[:, 8:]]                     # [nspec, 19, 3]
    dist = np.linalg.norm(got[:, :, None, :] - want[:, None, :, :], axis=-1).min(axis=2)
    size = np.abs(P.max(axis=1) - P.min(axis=1)).max(axis=1)
    if (dist.max(axis=1) > tol * np.maximum(size, 1.0)).any():
        raise ValueError("curved 27-node elements are not supported (the library maps each hexahedron "
                         "trilinearly from its 8 corners)")


def absorbing_sides(db: Database3D, pos: np.ndarray, ne) -> tuple:
    """Lattice sides (xmin, xmax, ymin, ymax, zmin, zmax) fully covered by the
    database's face lists; a listed face that is not on the lattice's outer
    side of its direction is refused."""
    out = []
    for d, name in enumerate(DIRECTIONS):
        elem, fnodes = db.faces[name]
        axis, upper = d // 2, d % 2
        if len(elem) == 0:
            out.append(0)
            continue
        face = PLUS_FACE[axis] if upper else MINUS_FACE[axis]
        want = np.sort(db.elements[elem][:, face], axis=1)
        got = np.sort(fnodes[:, :4], axis=1)
        side = pos[elem, axis] == (ne[axis] - 1 if upper else 0)
        if not (np.array_equal(want, got) and side.all()):
            raise ValueError(f"boundary faces of direction {name} do not lie on that side of the lattice")
        full = np.prod([ne[a] for a in range(3) if a != axis])
        out.append(int(len(np.unique(elem)) == full))
    return tuple(out)


def lattice_mesh(db: Database3D, absorbing: bool = False) -> meshgen.Mesh3D:
    """The library's lattice mesh of a database: control-node coordinates on
    the lattice, elastic isotropic material per GLL point (rho, vp, vs from
    the element's material), and, when ``absorbing``, Stacey on the sides that
    the database lists except the top (zmax, the free surface).  The
    reference's own 3D path applies no absorbing condition, so the default is
    none."""
    if db.ngll != (5, 5, 5):
        raise ValueError(f"NGLL {db.ngll} is not supported (5 x 5 x 5 expected)")
    if db.ngnod == 27:
        _check_hex27_affine(db)
    nex, ney, nez, pos, node_id = lattice_of(db)
    m = db.materials
    for k in range(len(m)):
        rho, vp, vs, mid, aniso = m[k, 0], m[k, 1], m[k, 2], int(m[k, 6]), int(m[k, 5])
        if mid == 1 or vs == 0.0:
            raise ValueError("acoustic 3D media are not supported (elastic isotropic only)")
        if mid != 2 or aniso > 0 or vs < 0.0:
            raise ValueError(f"material {k + 1} (id {mid}, anisotropy {aniso}) is not elastic isotropic")
    order = np.empty(db.nspec, np.int64)
    slot = (pos[:, 2] * ney + pos[:, 1]) * nex + pos[:, 0]
    order[slot] = np.arange(db.nspec)
    mat = db.materials[db.material_of[order]]              # lattice element order
    ones = np.ones((1, 125), np.float32)
    nodes = db.coords[node_id]
    x = nodes.reshape(nez + 1, ney + 1, nex + 1, 3)
    # right-handed lattice: d/dxi x (d/deta x) . d/dzeta x > 0 at the first element
    e0 = np.cross(x[0, 0, 1] - x[0, 0, 0], x[0, 1, 0] - x[0, 0, 0]) @ (x[1, 0, 0] - x[0, 0, 0])
    if e0 <= 0:
        raise ValueError("the lattice is left-handed (negative Jacobian); mirrored meshes are not supported")
    ab = (0, 0, 0, 0, 0, 0)
    if absorbing:
        ab = absorbing_sides(db, pos, (nex, ney, nez))
        ab = ab[:5] + (0,)
    return meshgen.Mesh3D(nex, ney, nez, nodes,
                          (mat[:, 0:1] * ones).astype(np.float32), (mat[:, 1:2] * ones).astype(np.float32),
                          (mat[:, 2:3] * ones).astype(np.float32), ab)


def database3d_bytes(mesh: meshgen.Mesh3D, materials, material_of, element_order=None, node_order=None) -> bytes:
    """A 3D ``database.bin`` (the layout ``parse_database3d`` reads) of a
    lattice mesh with 8-node elements: ``materials`` rows (rho, vp, vs),
    ``material_of`` [nspec] 0-based per lattice element; ``element_order`` /
    ``node_order`` permute the element records and the control-node ids (to
    write a database whose numbering is not the lattice's)."""
    nex, ney, nez = mesh.nex, mesh.ney, mesh.nez
    nspec = nex * ney * nez
    nnode = len(mesh.nodes)
    nid = np.arange(nnode) if node_order is None else np.asarray(node_order)    # lattice node -> id
    eo = np.arange(nspec) if element_order is None else np.asarray(element_order)
    rec = []

    def put(fmt, *v):
        b = struct.pack(fmt, *v)
        rec.append(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))

    put("<i", 0)
    put("<i", 8)
    put("<i", nnode)
    inv = np.empty(nnode, np.int64)
    inv[nid] = np.arange(nnode)
    for i in range(nnode):
        put("<iddd", i + 1, *(float(v) for v in mesh.nodes[inv[i]]))
    put("<ii", len(materials), 0)
    for rho, vp, vs in materials:
        put("<17d", rho, vp, vs, 0.0, 0.0, 0.0, 2.0, *([0.0] * 10))
    put("<i", nspec)
    put("<iii", 5, 5, 5)
    e = np.arange(nspec)
    ex, ey, ez = e % nex, (e // nex) % ney, e // (nex * ney)
    corner = np.stack([nid[((ez + s[2]) * (ney + 1) + ey + s[1]) * (nex + 1) + ex + s[0]]
                       for s in CORNER_SIGNS], -1)
    rank = np.empty(nspec, np.int64)
    rank[eo] = np.arange(nspec)                 # lattice element -> record position
    for k, le in enumerate(eo):
        put("<iii8i", k + 1, int(material_of[le]) + 1, 0, *(int(c) + 1 for c in corner[le]))
    pos = np.stack([ex, ey, ez], -1)
    ne = (nex, ney, nez)
    for d in range(6):
        axis, upper = d // 2, d % 2
        sel = np.nonzero(pos[:, axis] == (ne[axis] - 1 if upper else 0))[0]
        put("<ii", d + 1, len(sel))
    for d in range(6):
        axis, upper = d // 2, d % 2
        sel = np.nonzero(pos[:, axis] == (ne[axis] - 1 if upper else 0))[0]
        face = PLUS_FACE[axis] if upper else MINUS_FACE[axis]
        for le in sel:
            put("<i4i", int(rank[le]) + 1, *(int(corner[le, c]) + 1 for c in face))
    put("<i", 0)
    put("<ii", 0, 0)
    put("<i", 0)
    return b"".join(rec)
