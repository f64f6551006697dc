"""Oracle-side reader for SPECFEM2D ``database.bin`` mesh files.

TEST INFRASTRUCTURE ONLY: this module belongs to the CPU oracle.  Only the
test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product path never does.

The file is a sequence of Fortran unformatted records (``int32 n``, payload,
``int32 n``).  The record order restated here follows the reference reader:

* header: ``src/io/mesh/impl/fortran/dim2/read_mesh_database.cpp:12-158``
  (42 fixed records, one optional 16-byte record, then 22 records);
* control nodes: ``read_mesh_database.cpp:161-183``;
* mesh parameters: ``src/io/mesh/impl/fortran/dim2/read_parameters.cpp:8-45``;
* attenuation record: ``read_mesh_database.cpp:185-205``;
* materials and element records:
  ``src/io/mesh/impl/fortran/dim2/read_material_properties.cpp:163-170,484-532``;
* interfaces header: ``src/io/mesh/impl/fortran/dim2/mesh.cpp:97-100``;
* absorbing / acoustic free surface / forcing records:
  ``src/io/mesh/impl/fortran/dim2/read_boundaries.cpp`` (absorbing edges with
  the 4 ``codeabs`` flags; free surface ``(ispec, type, e1, e2)``);
* fluid-solid pairs: ``mesh.cpp:107-121``; tangential and axial records
  ``read_elements.cpp``; adjacency graph ``read_adjacency_graph.cpp:11-40``.

Edge types use the reference's ``mesh_entity`` naming: 0 bottom, 1 right,
2 top, 3 left (``read_boundaries.cpp`` ``codeabsread1..4``).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

BOTTOM, RIGHT, TOP, LEFT = 0, 1, 2, 3
ACOUSTIC, ELASTIC = 0, 1


@dataclass
class Mesh2D:
    nspec: int
    npgeo: int
    ngnod: int
    coorg: np.ndarray            # [npgeo, 2] float64 (x, z)
    knods: np.ndarray            # [nspec, ngnod] int32, 0-based
    kmato: np.ndarray            # [nspec] int32, 0-based material index
    mat_medium: np.ndarray       # [numat] 0 acoustic, 1 elastic
    mat_rho: np.ndarray          # [numat]
    mat_vp: np.ndarray           # [numat]
    mat_vs: np.ndarray           # [numat]
    abs_ispec: np.ndarray        # [nabs] absorbing edges (element, edge type)
    abs_type: np.ndarray
    free_ispec: np.ndarray       # [nfree] acoustic free-surface edges
    free_type: np.ndarray
    coupled_pairs: np.ndarray    # [ncoupled, 2] (element a, element b)
    title: str = ""
    extra: dict = field(default_factory=dict)
    # anisotropic elastic materials: (c11, c13, c15, c33, c35, c55) per
    # material, NaN rows for isotropic ones; None when every material is isotropic
    mat_aniso: np.ndarray | None = None
    # [numat][8] Cosserat constants (rho, kappa, mu, nu, j, lambda_c, mu_c, nu_c);
    # NaN rows for other materials
    mat_cosserat: np.ndarray | None = None
    # [numat][13] isotropic poroelastic constants (rho_s, rho_f, phi,
    # tortuosity, kxx, kxz, kzz, kappa_s, kappa_f, kappa_fr, eta_f, mu_fr,
    # Q_mu); NaN rows are other materials
    mat_poro: np.ndarray | None = None


def _records(buf: bytes):
    pos, n = 0, len(buf)
    while pos < n:
        (ln,) = struct.unpack_from("<i", buf, pos)
        if ln < 0 or pos + 8 + ln > n:
            raise ValueError(f"corrupt Fortran record at byte {pos}")
        payload = buf[pos + 4: pos + 4 + ln]
        (ln2,) = struct.unpack_from("<i", buf, pos + 4 + ln)
        if ln2 != ln:
            raise ValueError(f"record length mismatch at byte {pos}")
        yield payload
        pos += 8 + ln


def _corner_type(e1: int, e2: int, kn: np.ndarray, kind: int) -> int:
    """Edge type from control-node ids, ``read_boundaries.cpp`` get_boundary_type."""
    if kind == 1:  # a single node (corner) — the reference maps it to a corner type
        raise ValueError("acoustic free surface given by a single node is not supported")
    pairs = {(0, 1): BOTTOM, (0, 3): LEFT, (1, 2): RIGHT, (2, 3): TOP}
    for (a, b), t in pairs.items():
        if {e1, e2} == {int(kn[a]), int(kn[b])}:
            return t
    raise ValueError("could not classify acoustic free-surface edge")


def read_database(path: str, elastic_wave: str = "psv") -> Mesh2D:
    with open(path, "rb") as f:
        buf = f.read()
    recs = list(_records(buf))
    i = 0

    def take():
        nonlocal i
        r = recs[i]
        i += 1
        return r

    title = take()[:512].split(b"\x00")[0].decode("latin-1").strip()
    take()                                             # noise, pml flags
    (nspec,) = struct.unpack("<i", take())
    npgeo, _nproc = struct.unpack("<ii", take())
    for _ in range(38):                                 # records 4..41
        take()
    if len(recs[i]) == 16:                               # optional EM attenuation record
        take()
    for _ in range(22):
        take()

    coorg = np.zeros((npgeo, 2))
    for _ in range(npgeo):
        ip, x, z = struct.unpack("<idd", take())
        if ip < 1 or ip > npgeo:
            raise ValueError("Error reading coordinates")
        coorg[ip - 1] = (x, z)

    numat, ngnod, nspec2, _pointsdisp, _plot = struct.unpack("<iiiii", take())
    if nspec2 != nspec:
        raise ValueError("nspec mismatch between header and parameters")
    (nelemabs, nelem_acforcing, nelem_acoustic_surface, num_fluid_solid,
     num_fluid_poro, num_solid_poro, nnodes_tangential, nelem_on_axis) = struct.unpack("<8i", take())
    take()                                             # attenuation (n_sls, f0, flag)

    mat_medium = np.zeros(numat, np.int32)
    mat_rho = np.zeros(numat)
    mat_vp = np.zeros(numat)
    mat_vs = np.zeros(numat)
    mat_aniso = np.full((numat, 6), np.nan)
    mat_cos = np.full((numat, 8), np.nan)
    mat_poro = np.full((numat, 13), np.nan)
    for m in range(numat):
        vals = struct.unpack("<ii13d", take())
        n, indic = vals[0], vals[1]
        v = vals[2:]
        if n != m + 1:
            raise ValueError("Wrong material set number")
        if indic == 2:
            # anisotropic elastic: rho, c11, c13, c15, c33, c35, c55, c12, c23, c25
            # (src/io/mesh/impl/fortran/dim2/read_material_properties.cpp:252-291)
            mat_rho[m] = v[0]
            mat_aniso[m] = v[1:7]
            mat_vp[m] = np.sqrt(v[4] / v[0])          # sqrt(c33 / rho)
            mat_vs[m] = np.sqrt(v[6] / v[0])          # sqrt(c55 / rho)
            mat_medium[m] = ELASTIC
            continue
        if indic == 5:
            # isotropic Cosserat elastic (P-SV-T): rho, kappa, mu, nu, j,
            # lambda_c, mu_c, nu_c (read_material_properties.cpp:366-395)
            mat_cos[m] = v[0:8]
            mat_rho[m] = v[0]
            mat_vp[m] = np.sqrt((v[1] + 4.0 / 3.0 * v[2]) / v[0])
            mat_vs[m] = np.sqrt(v[2] / v[0])
            mat_medium[m] = ELASTIC
            continue
        if indic == 3:
            # isotropic poroelastic: rho_s, rho_f, phi, tortuosity, kxx, kxz,
            # kzz, kappa_s, kappa_f, kappa_fr, eta_f, mu_fr, Q_mu
            # (read_material_properties.cpp:303-332)
            mat_poro[m] = v[0:13]
            mat_rho[m] = (1.0 - v[2]) * v[0] + v[2] * v[1]      # rho_bar
            mat_vp[m] = mat_vs[m] = 0.0                        # unused: Biot constants
            mat_medium[m] = ELASTIC
            continue
        if indic != 1:
            raise ValueError(f"material type {indic} is outside this path")
        mat_rho[m], mat_vp[m], mat_vs[m] = v[0], v[1], v[2]
        mat_medium[m] = ACOUSTIC if v[2] == 0 else ELASTIC

    knods = np.zeros((nspec, ngnod), np.int32)
    kmato = np.zeros(nspec, np.int32)
    fmt = "<ii%dii" % ngnod
    for _ in range(nspec):
        vals = struct.unpack(fmt, take())
        n, km = vals[0], vals[1]
        knods[n - 1] = np.asarray(vals[2:2 + ngnod]) - 1
        kmato[n - 1] = km - 1

    take()                                             # ninterfaces, max_interface_size

    abs_ispec, abs_type = [], []
    for _ in range(max(nelemabs, 0)):
        vals = struct.unpack("<i4ii8i", take())
        flags = vals[1:5]
        if sum(1 for c in flags if c) != 1:
            raise ValueError("must have one and only one absorbing edge per line")
        abs_ispec.append(vals[0] - 1)
        abs_type.append([BOTTOM, RIGHT, TOP, LEFT][[bool(c) for c in flags].index(True)])

    free_ispec, free_type = [], []
    for _ in range(nelem_acoustic_surface):
        isp, kind, e1, e2 = struct.unpack("<4i", take())
        free_ispec.append(isp - 1)
        free_type.append(_corner_type(e1 - 1, e2 - 1, knods[isp - 1], kind))

    for _ in range(nelem_acforcing):
        take()

    pairs = []
    for count in (num_fluid_solid, num_fluid_poro, num_solid_poro):
        for _ in range(count):
            a, b = struct.unpack("<ii", take())
            pairs.append((b - 1, a - 1))

    take()                                             # tangential flags
    for _ in range(nnodes_tangential):
        take()
    for _ in range(nelem_on_axis):
        take()
    extra = {}
    if i < len(recs):
        (nadj,) = struct.unpack("<i", take())
        extra["n_adjacency"] = nadj
        adj = np.zeros((nadj, 4), np.int32)
        for k in range(nadj):
            e, nb, conn, orient = struct.unpack("<4i", take())
            if conn not in (1, 3):
                raise ValueError("Unknown connection type in adjacency graph.")
            adj[k] = (e - 1, nb - 1, conn, orient - 1)
        extra["adjacency"] = adj
    if i != len(recs):
        raise ValueError("The Database file wasn't fully read")

    return Mesh2D(nspec=nspec, npgeo=npgeo, ngnod=ngnod, coorg=coorg, knods=knods,
                  kmato=kmato, mat_medium=mat_medium, mat_rho=mat_rho, mat_vp=mat_vp,
                  mat_vs=mat_vs, abs_ispec=np.asarray(abs_ispec, np.int32),
                  abs_type=np.asarray(abs_type, np.int32),
                  free_ispec=np.asarray(free_ispec, np.int32),
                  free_type=np.asarray(free_type, np.int32),
                  coupled_pairs=np.asarray(pairs, np.int32).reshape(-1, 2),
                  title=title, extra=extra,
                  mat_aniso=mat_aniso if np.isfinite(mat_aniso).any() else None,
                  mat_cosserat=mat_cos if np.isfinite(mat_cos).any() else None,
                  mat_poro=mat_poro if np.isfinite(mat_poro).any() else None)
