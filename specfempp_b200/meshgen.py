"""Structured 2D meshes and the benchmark configurations.

The reference builds its meshes with the Fortran mesher xmeshfem2D, which
writes ``database.bin``.  This module is the stand-in for the structured
(rectangular-grid) part of that mesher: it creates the same in-memory mesh
(control nodes, 4-node elements, materials, absorbing and free-surface edge
lists) and can write it as a ``database.bin`` with the record layout that
``src/io/mesh/impl/fortran/dim2/*.cpp`` reads.

It also defines the synthetic workloads used by the tests and the benchmark
(all inputs seeded; no dataset is involved):

* ``elastic_psv_80x60``    80x60 quads over 4000x3000 m, vp 2500, vs 1445,
                           rho 2200, free top + Stacey on the other sides,
                           Ricker 10 Hz force source, 5 receivers, dt 5e-4, 1600 steps;
* ``coupled_400x200``      400x200 quads over 20x10 km: 1.5 km of water
                           (vp 1500, rho 1020) over 4 elastic layers with seeded
                           vp in [2500, 5000], vs = vp/1.73, rho = 1700 + 0.2 vp;
                           pressure Ricker 5 Hz source in the water, 200
                           receivers along the seafloor, dt 1e-3, 4000 steps;
* ``elastic_grf_1000x500`` 1000x500 quads, vp = 3000 (1 + 0.1 GRF(500 m)).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

BOTTOM, RIGHT, TOP, LEFT = 0, 1, 2, 3
ACOUSTIC, ELASTIC = 0, 1


@dataclass
class Mesh:
    nspec: int
    npgeo: int
    ngnod: int
    coorg: np.ndarray
    knods: np.ndarray
    kmato: np.ndarray
    mat_medium: np.ndarray
    mat_rho: np.ndarray
    mat_vp: np.ndarray
    mat_vs: np.ndarray
    abs_ispec: np.ndarray
    abs_type: np.ndarray
    free_ispec: np.ndarray
    free_type: np.ndarray
    coupled_pairs: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    nx: int = 0
    nz: int = 0
    # optional [numat][6] anisotropic constants (c11, c13, c15, c33, c35, c55);
    # NaN rows are isotropic materials
    mat_aniso: np.ndarray | None = None
    # optional [numat][8] Cosserat constants (rho, kappa, mu, nu, j, lambda_c,
    # mu_c, nu_c); NaN rows are other materials
    mat_cosserat: np.ndarray | None = None
    # optional [numat][13] isotropic poroelastic constants (rho_s, rho_f, phi,
    # tortuosity, kxx, kxz, kzz, kappa_s, kappa_f, kappa_fr, eta_f, mu_fr,
    # Q_mu); NaN rows are other materials
    mat_poro: np.ndarray | None = None
    # optional adjacency records [n][4]: (element, neighbour, connection 1
    # strongly conforming / 3 nonconforming, orientation of the shared entity
    # on the element: 0 bottom 1 right 2 top 3 left, 4..7 corners
    # bottom-left, bottom-right, top-right, top-left), 0-based
    adjacency: np.ndarray | None = None


def structured_mesh(nx, nz, xmin, xmax, zmin, zmax, row_material, materials,
                    absorbing=("bottom", "right", "left"), free_surface=("top",)) -> Mesh:
    """Rectangular grid of nx*nz 4-node quads, element e = iz*nx + ix (bottom row first).

    ``row_material``: [nz] material index per element row.
    ``materials``: list of (medium, rho, vp, vs) with medium 0 acoustic, 1 elastic.
    Absorbing edges are listed side by side (bottom, right, top, left), the
    acoustic free surface on the sides named in ``free_surface`` (acoustic
    elements only).
    """
    xs = np.linspace(xmin, xmax, nx + 1)
    zs = np.linspace(zmin, zmax, nz + 1)
    X, Z = np.meshgrid(xs, zs)
    coorg = np.stack([X.ravel(), Z.ravel()], axis=1)
    iz, ix = np.divmod(np.arange(nx * nz), nx)
    n0 = iz * (nx + 1) + ix
    knods = np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], axis=1).astype(np.int32)
    row_material = np.asarray(row_material, np.int32)
    kmato = row_material[iz].astype(np.int32)
    med = np.asarray([m[0] for m in materials], np.int32)
    abs_i, abs_t = [], []
    sides = {"bottom": (iz == 0, BOTTOM), "right": (ix == nx - 1, RIGHT),
             "top": (iz == nz - 1, TOP), "left": (ix == 0, LEFT)}
    for name in ("bottom", "right", "top", "left"):
        if name in absorbing:
            mask, t = sides[name]
            e = np.nonzero(mask)[0]
            abs_i.append(e)
            abs_t.append(np.full(len(e), t))
    fr_i, fr_t = [], []
    for name in free_surface:
        mask, t = sides[name]
        e = np.nonzero(mask & (med[kmato] == ACOUSTIC))[0]
        fr_i.append(e)
        fr_t.append(np.full(len(e), t))
    cat = lambda l: np.concatenate(l).astype(np.int32) if l else np.zeros(0, np.int32)
    # fluid-solid element pairs across horizontal interfaces
    pairs = []
    below = kmato.reshape(nz, nx)
    for r in range(nz - 1):
        a, b = med[below[r, 0]], med[below[r + 1, 0]]
        if a != b:
            for c in range(nx):
                e1, e2 = r * nx + c, (r + 1) * nx + c
                pairs.append((e1, e2) if a == ACOUSTIC else (e2, e1))
    return Mesh(nspec=nx * nz, npgeo=(nx + 1) * (nz + 1), ngnod=4, coorg=coorg, knods=knods,
                kmato=kmato, mat_medium=med,
                mat_rho=np.asarray([m[1] for m in materials], np.float64),
                mat_vp=np.asarray([m[2] for m in materials], np.float64),
                mat_vs=np.asarray([m[3] for m in materials], np.float64),
                abs_ispec=cat(abs_i), abs_type=cat(abs_t), free_ispec=cat(fr_i), free_type=cat(fr_t),
                coupled_pairs=np.asarray(pairs, np.int32).reshape(-1, 2), nx=nx, nz=nz)


# header record sizes of database.bin (read_mesh_database.cpp:12-158)
_HEADER = [512, 8, 4, 8, 8, 4, 4, 4, 4, 4, 8, 8, 8, 8, 8, 4, 4, 4, 12, 8, 32, 8, 4, 16, 516,
           512, 512, 512, 16, 4, 12, 4, 4, 8, 4, 4, 4, 4, 4, 4, 4, 16, 4, 4, 8, 4, 8, 4, 4, 4,
           8, 4, 8, 4, 4, 8, 4, 4, 12, 4, 4, 4, 4, 8]


def write_database(mesh: Mesh, path: str, title: str = "structured mesh") -> None:
    """Write ``mesh`` as a SPECFEM2D database.bin (Fortran unformatted records)."""
    out = bytearray()

    def rec(payload: bytes):
        out.extend(struct.pack("<i", len(payload)))
        out.extend(payload)
        out.extend(struct.pack("<i", len(payload)))

    for k, n in enumerate(_HEADER):
        if k == 0:
            rec(title.encode().ljust(512, b" ")[:512])
        elif k == 2:
            rec(struct.pack("<i", mesh.nspec))
        elif k == 3:
            rec(struct.pack("<ii", mesh.npgeo, 1))
        else:
            rec(bytes(n))
    for i in range(mesh.npgeo):
        rec(struct.pack("<idd", i + 1, float(mesh.coorg[i, 0]), float(mesh.coorg[i, 1])))
    rec(struct.pack("<iiiii", len(mesh.mat_rho), mesh.ngnod, mesh.nspec, 0, 0))
    rec(struct.pack("<8i", len(mesh.abs_ispec), 0, len(mesh.free_ispec), len(mesh.coupled_pairs),
                    0, 0, 0, 0))
    rec(struct.pack("<idi", 1, 0.0, 0))
    for m in range(len(mesh.mat_rho)):
        if mesh.mat_poro is not None and np.isfinite(mesh.mat_poro[m]).all():
            rec(struct.pack("<ii13d", m + 1, 3, *[float(x) for x in mesh.mat_poro[m]]))
            continue
        vs = 0.0 if mesh.mat_medium[m] == ACOUSTIC else float(mesh.mat_vs[m])
        rec(struct.pack("<ii13d", m + 1, 1, float(mesh.mat_rho[m]), float(mesh.mat_vp[m]), vs,
                        0.0, 0.0, 9999.0, 9999.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0))
    fmt = "<ii%dii" % mesh.ngnod
    for e in range(mesh.nspec):
        rec(struct.pack(fmt, e + 1, int(mesh.kmato[e]) + 1, *[int(k) + 1 for k in mesh.knods[e]], 0))
    rec(struct.pack("<ii", 0, 0))
    for e, t in zip(mesh.abs_ispec, mesh.abs_type):
        codes = [int(t == BOTTOM), int(t == RIGHT), int(t == TOP), int(t == LEFT)]
        rec(struct.pack("<i4ii8i", int(e) + 1, *codes, 0, *([0] * 8)))
    corners = {BOTTOM: (0, 1), RIGHT: (1, 2), TOP: (2, 3), LEFT: (0, 3)}
    for e, t in zip(mesh.free_ispec, mesh.free_type):
        a, b = corners[int(t)]
        rec(struct.pack("<4i", int(e) + 1, 2, int(mesh.knods[e, a]) + 1, int(mesh.knods[e, b]) + 1))
    for ac, el in mesh.coupled_pairs:
        rec(struct.pack("<ii", int(ac) + 1, int(el) + 1))
    rec(struct.pack("<ii", 0, 0))
    adj = np.zeros((0, 4), np.int32) if mesh.adjacency is None else np.asarray(mesh.adjacency)
    rec(struct.pack("<i", len(adj)))
    for e, nb, conn, orient in adj:
        rec(struct.pack("<4i", int(e) + 1, int(nb) + 1, int(conn), int(orient) + 1))
    with open(path, "wb") as f:
        f.write(bytes(out))


# ------------------------------------------------------------------ configs ---

@dataclass
class Workload:
    name: str
    mesh: Mesh
    sources: list
    rec_x: np.ndarray
    rec_z: np.ndarray
    dt: float
    nstep: int
    point_rho: np.ndarray | None = None
    point_vp: np.ndarray | None = None
    point_vs: np.ndarray | None = None
    description: str = ""


@dataclass
class RickerSource:
    x: float
    z: float
    f0: float
    factor: float
    tshift: float = 0.0
    angle: float = 0.0
    stf: str = "ricker"
    shot: int = 0


def elastic_psv_80x60(nstep: int = 1600) -> Workload:
    mesh = structured_mesh(80, 60, 0.0, 4000.0, 0.0, 3000.0, np.zeros(60, np.int32),
                           [(ELASTIC, 2200.0, 2500.0, 1445.0)],
                           absorbing=("bottom", "right", "left"), free_surface=())
    rng = np.random.default_rng(0)
    rx = np.sort(rng.uniform(500.0, 3500.0, 5))
    rz = np.full(5, 2800.0)
    src = [RickerSource(2000.0, 2500.0, 10.0, 1e10)]
    return Workload("elastic_psv_80x60", mesh, src, rx, rz, 5e-4, nstep,
                    description="2D elastic P-SV 80x60, NGLL=5, Stacey L/R/B, free top")


def coupled_400x200(nstep: int = 4000, nx: int = 400, nz: int = 200, seed: int = 0) -> Workload:
    """Water layer (top 1.5 km) over 4 seeded elastic layers, 20 x 10 km."""
    rng = np.random.default_rng(seed)
    vps = rng.uniform(2500.0, 5000.0, 4)
    mats = [(ACOUSTIC, 1020.0, 1500.0, 0.0)]
    for vp in vps:
        mats.append((ELASTIC, 1700.0 + 0.2 * vp, vp, vp / 1.73))
    depth = 10000.0
    h = depth / nz
    n_water = int(round(1500.0 / h))
    n_el = nz - n_water
    bounds = np.linspace(0, n_el, 5).round().astype(int)
    row_mat = np.zeros(nz, np.int32)
    for k in range(4):
        # bottom-up rows: layer 4 (deepest) first
        row_mat[bounds[k]:bounds[k + 1]] = 4 - k
    row_mat[n_el:] = 0
    mesh = structured_mesh(nx, nz, 0.0, 20000.0 * nx / 400, 0.0, depth, row_mat, mats,
                           absorbing=("bottom", "right", "left"), free_surface=("top",))
    seafloor = n_el * h
    xmax = 20000.0 * nx / 400
    rx = np.linspace(0.05 * xmax, 0.95 * xmax, 200)
    rz = np.full(200, seafloor - 0.25 * h)
    src = [RickerSource(0.5 * xmax, seafloor + 0.5 * (depth - seafloor), 5.0, 1e9)]
    return Workload("coupled_400x200", mesh, src, rx, rz, 1e-3, nstep,
                    description=f"2D coupled acoustic-elastic {nx}x{nz}, water 1.5 km, "
                                f"elastic vp={np.round(vps, 1).tolist()}")


def _grid_adjacency(nx, nz, first):
    """Strongly conforming adjacency records of an nx*nz grid of elements
    numbered first + iz*nx + ix: edge neighbours and diagonal corner neighbours."""
    recs = []
    steps = [(0, -1, BOTTOM), (1, 0, RIGHT), (0, 1, TOP), (-1, 0, LEFT),
             (-1, -1, 4), (1, -1, 5), (1, 1, 6), (-1, 1, 7)]
    for iz in range(nz):
        for ix in range(nx):
            for dx, dz, o in steps:
                jx, jz = ix + dx, iz + dz
                if 0 <= jx < nx and 0 <= jz < nz:
                    recs.append((first + iz * nx + ix, first + jz * nx + jx, 1, o))
    return recs


def nonconforming_coupled(nx_el: int = 30, nx_ac: int = 45, nz_el: int = 16, nz_ac: int = 12,
                          width: float = 3000.0, h_el: float = 1600.0, h_ac: float = 1200.0,
                          nstep: int = 1200, absorbing=("bottom", "right", "left"),
                          free_surface=("top",)) -> Workload:
    """An elastic block (nx_el x nz_el quads) under a water block (nx_ac x
    nz_ac quads) of the same width, with no shared control nodes: the
    horizontal fluid-solid interface at z = h_el is nonconforming whenever
    nx_el != nx_ac, and every overlapping pair of interface edges is listed
    as a nonconforming adjacency record (both directions), the grid
    neighbours as strongly conforming ones.  Elastic elements come first.
    Stacey on the sides named in ``absorbing`` (both blocks), an acoustic free
    surface on the top; Ricker 8 Hz pressure source in the water, 8
    receivers on both sides of the interface, dt 5e-4."""
    xs_e, zs_e = np.linspace(0.0, width, nx_el + 1), np.linspace(0.0, h_el, nz_el + 1)
    xs_a, zs_a = np.linspace(0.0, width, nx_ac + 1), np.linspace(h_el, h_el + h_ac, nz_ac + 1)
    Xe, Ze = np.meshgrid(xs_e, zs_e)
    Xa, Za = np.meshgrid(xs_a, zs_a)
    coorg = np.concatenate([np.stack([Xe.ravel(), Ze.ravel()], 1), np.stack([Xa.ravel(), Za.ravel()], 1)])
    off = (nx_el + 1) * (nz_el + 1)

    def quads(nx, nz, base):
        iz, ix = np.divmod(np.arange(nx * nz), nx)
        n0 = base + iz * (nx + 1) + ix
        return np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], axis=1)

    knods = np.concatenate([quads(nx_el, nz_el, 0), quads(nx_ac, nz_ac, off)]).astype(np.int32)
    ne = nx_el * nz_el
    nspec = ne + nx_ac * nz_ac
    kmato = np.concatenate([np.zeros(ne, np.int32), np.ones(nx_ac * nz_ac, np.int32)])
    abs_i, abs_t = [], []
    for nx, nz, base in ((nx_el, nz_el, 0), (nx_ac, nz_ac, ne)):
        iz, ix = np.divmod(np.arange(nx * nz), nx)
        top_block = base == ne
        sides = {"bottom": (iz == 0) & (not top_block), "right": ix == nx - 1,
                 "top": (iz == nz - 1) & top_block, "left": ix == 0}
        for name, t in (("bottom", BOTTOM), ("right", RIGHT), ("top", TOP), ("left", LEFT)):
            if name in absorbing:
                e = base + np.nonzero(sides[name])[0]
                abs_i.append(e)
                abs_t.append(np.full(len(e), t))
    fr = np.arange(ne + (nz_ac - 1) * nx_ac, nspec) if "top" in free_surface else np.zeros(0, int)
    adj = _grid_adjacency(nx_el, nz_el, 0) + _grid_adjacency(nx_ac, nz_ac, ne)
    tol = 1e-9 * width
    for i in range(nx_el):
        e = (nz_el - 1) * nx_el + i
        for j in range(nx_ac):
            a = ne + j
            lo, hi = max(xs_e[i], xs_a[j]), min(xs_e[i + 1], xs_a[j + 1])
            if hi - lo > tol:
                adj.append((e, a, 3, TOP))
                adj.append((a, e, 3, BOTTOM))
    mesh = Mesh(nspec=nspec, npgeo=len(coorg), ngnod=4, coorg=coorg, knods=knods, kmato=kmato,
                mat_medium=np.array([ELASTIC, ACOUSTIC], np.int32),
                mat_rho=np.array([2400.0, 1020.0]), mat_vp=np.array([3000.0, 1500.0]),
                mat_vs=np.array([1700.0, 0.0]),
                abs_ispec=np.concatenate(abs_i).astype(np.int32) if abs_i else np.zeros(0, np.int32),
                abs_type=np.concatenate(abs_t).astype(np.int32) if abs_t else np.zeros(0, np.int32),
                free_ispec=fr.astype(np.int32), free_type=np.full(len(fr), TOP, np.int32),
                adjacency=np.asarray(adj, np.int32))
    rx = np.linspace(0.3 * width, 0.6 * width, 8)
    rz = np.array([h_el - 230.0, h_el - 130.0, h_el - 70.0, h_el - 20.0,
                   h_el + 20.0, h_el + 70.0, h_el + 130.0, h_el + 230.0])
    src = [RickerSource(0.43 * width, h_el + 0.45 * h_ac, 8.0, 1e9)]
    return Workload(f"nonconforming_coupled_{nx_el}_{nx_ac}", mesh, src, rx, rz, 5e-4, nstep,
                    description=f"2D acoustic-elastic, nonconforming interface {nx_el}:{nx_ac}")


# the saturated sandstone of the reference's poroelastic fixture:
# rho_s, rho_f, phi, tortuosity, kxx, kxz, kzz, kappa_s, kappa_f, kappa_fr,
# eta_f, mu_fr, Q_mu
POROUS_SANDSTONE = (2650.0, 880.0, 0.1, 2.0, 1e-9, 0.0, 1e-9, 12.2e9, 1.985e9, 9.6e9, 0.0, 5.1e9, 9999.0)


def poroelastic_model(nx: int = 50, nz: int = 50, width: float = 1000.0, height: float = 1000.0,
                      eta_f: float = 0.0, kxz: float = 0.0, nstep: int = 1000,
                      layered: bool = False) -> Workload:
    """A block of fluid-saturated porous rock (the sandstone above, viscosity
    eta_f and off-diagonal permeability kxz as given), free edges; with
    ``layered`` the upper half has 20% porosity and a softer frame.
    Ricker 30 Hz force source (both phases) in the middle, 6 receivers,
    dt 1e-4."""
    row_mat = np.zeros(nz, np.int32)
    mats = [(ELASTIC, 0.0, 0.0, 0.0)]
    poro = [list(POROUS_SANDSTONE)]
    poro[0][10] = eta_f
    poro[0][5] = kxz
    if layered:
        row_mat[nz // 2:] = 1
        mats.append((ELASTIC, 0.0, 0.0, 0.0))
        soft = list(poro[0])
        soft[2], soft[9], soft[11] = 0.2, 6.0e9, 3.2e9
        poro.append(soft)
    mesh = structured_mesh(nx, nz, 0.0, width, 0.0, height, row_mat, mats, absorbing=(), free_surface=())
    mesh.mat_poro = np.asarray(poro, np.float64)
    mesh.mat_rho = np.asarray([(1 - p[2]) * p[0] + p[2] * p[1] for p in poro])
    rx = np.linspace(0.3 * width, 0.7 * width, 6)
    rz = np.full(6, 0.62 * height)
    src = [RickerSource(0.5 * width, 0.45 * height, 30.0, 1e10)]
    return Workload(f"poroelastic_{nx}x{nz}", mesh, src, rx, rz, 1e-4, nstep,
                    description=f"2D isotropic poroelastic {nx}x{nz}, eta_f {eta_f}")


def merge_interface_nodes(mesh: Mesh) -> Mesh:
    """The conforming twin of a nonconforming_coupled mesh whose interface
    edges coincide (nx_el == nx_ac): the water block's interface nodes are
    replaced by the elastic block's nodes at the same place, and the
    adjacency records are dropped, so the interface couples through shared
    edges."""
    import copy
    m = copy.deepcopy(mesh)
    key = {}
    for i, (x, z) in enumerate(m.coorg):
        key.setdefault((round(x, 6), round(z, 6)), i)
    remap = np.arange(m.npgeo)
    for i, (x, z) in enumerate(m.coorg):
        remap[i] = key[(round(x, 6), round(z, 6))]
    m.knods = remap[m.knods].astype(np.int32)
    m.adjacency = None
    return m


def gaussian_random_field(shape, spacing, corr_len, rng) -> np.ndarray:
    """Zero-mean unit-std field with a Gaussian covariance of correlation length corr_len."""
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n, d=spacing) * 2 * np.pi for n in shape]
    K2 = sum(np.meshgrid(*[kk ** 2 for kk in k], indexing="ij"))
    filt = np.exp(-K2 * corr_len ** 2 / 8.0)
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
    return (f - f.mean()) / f.std()


def grf_point_model(mesh: Mesh, xmax, zmax, base_vp, std, corr_len, seed, ngrid=None):
    """Per-GLL-point vp = base (1 + std * GRF) sampled bilinearly at GLL points."""
    rng = np.random.default_rng(seed)
    ngrid = ngrid or (max(64, mesh.nz * 2), max(64, mesh.nx * 2))
    dz, dx = zmax / (ngrid[0] - 1), xmax / (ngrid[1] - 1)
    field_ = gaussian_random_field(ngrid, min(dx, dz), corr_len, rng)
    gz, gx = gll_coordinates(mesh)
    fz = np.clip(gz / dz, 0, ngrid[0] - 1.000001)
    fx = np.clip(gx / dx, 0, ngrid[1] - 1.000001)
    i0, j0 = fz.astype(int), fx.astype(int)
    tz, tx = fz - i0, fx - j0
    v = (field_[i0, j0] * (1 - tz) * (1 - tx) + field_[i0 + 1, j0] * tz * (1 - tx) +
         field_[i0, j0 + 1] * (1 - tz) * tx + field_[i0 + 1, j0 + 1] * tz * tx)
    return base_vp * (1.0 + std * v)


def gll_coordinates(mesh: Mesh):
    """(z, x) of every element GLL point [nspec, 25] for the bilinear 4-node mesh."""
    r = np.sqrt(3.0 / 7.0)
    z1 = np.array([-1.0, -r, 0.0, r, 1.0])
    XI, GA = np.meshgrid(z1, z1)            # [iz, ix]
    s = np.stack([0.25 * (XI - 1) * (GA - 1), -0.25 * (XI + 1) * (GA - 1),
                  0.25 * (XI + 1) * (GA + 1), -0.25 * (XI - 1) * (GA + 1)], -1).reshape(25, 4)
    cx = mesh.coorg[mesh.knods, 0]
    cz = mesh.coorg[mesh.knods, 1]
    return cz @ s.T, cx @ s.T


GLL_NODES = np.array([-1.0, -np.sqrt(3.0 / 7.0), 0.0, np.sqrt(3.0 / 7.0), 1.0])
GLL_WEIGHTS = np.array([0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1])


def _shape2d(ngnod: int, xi, ga):
    """Shape functions and their xi / gamma derivatives [..., ngnod] of the
    4-node bilinear and 9-node biquadratic quadrilaterals (node order: corners
    counter-clockwise from (-1, -1), then the edge mid-points, then the centre)."""
    if ngnod == 4:
        s = np.stack([0.25 * (xi - 1) * (ga - 1), -0.25 * (xi + 1) * (ga - 1),
                      0.25 * (xi + 1) * (ga + 1), -0.25 * (xi - 1) * (ga + 1)], -1)
        dx = np.stack([0.25 * (ga - 1), -0.25 * (ga - 1), 0.25 * (ga + 1), -0.25 * (ga + 1)], -1)
        dg = np.stack([0.25 * (xi - 1), -0.25 * (xi + 1), 0.25 * (xi + 1), -0.25 * (xi - 1)], -1)
        return s, dx, dg
    lx = [0.5 * xi * (xi - 1), 1 - xi * xi, 0.5 * xi * (xi + 1)]
    lg = [0.5 * ga * (ga - 1), 1 - ga * ga, 0.5 * ga * (ga + 1)]
    dlx = [xi - 0.5, -2 * xi, xi + 0.5]
    dlg = [ga - 0.5, -2 * ga, ga + 0.5]
    ix = [0, 2, 2, 0, 1, 2, 1, 0, 1]
    ig = [0, 0, 2, 2, 0, 1, 2, 1, 1]
    s = np.stack([lx[a] * lg[b] for a, b in zip(ix, ig)], -1)
    dx = np.stack([dlx[a] * lg[b] for a, b in zip(ix, ig)], -1)
    dg = np.stack([lx[a] * dlg[b] for a, b in zip(ix, ig)], -1)
    return s, dx, dg


def gll_geometry(mesh):
    """(x, z, |J|) of every element GLL point [nspec, 25] (point q = iz*5 + ix)
    for 4- and 9-node meshes (FP64)."""
    GA, XI = np.meshgrid(GLL_NODES, GLL_NODES, indexing="ij")      # [iz, ix]
    s, dx, dg = (a.reshape(25, -1) for a in _shape2d(int(mesh.ngnod), XI, GA))
    kn = np.asarray(mesh.knods).reshape(int(mesh.nspec), int(mesh.ngnod))
    cx = np.asarray(mesh.coorg)[kn, 0]
    cz = np.asarray(mesh.coorg)[kn, 1]
    x, z = cx @ s.T, cz @ s.T
    jac = (cx @ dx.T) * (cz @ dg.T) - (cx @ dg.T) * (cz @ dx.T)
    return x, z, jac


def elastic_grf_1000x500(nstep: int = 3000, nshots: int = 32, nrec: int = 400,
                         nx: int = 1000, nz: int = 500, seed: int = 0) -> Workload:
    xmax, zmax = 25.0 * nx, 25.0 * nz
    mesh = structured_mesh(nx, nz, 0.0, xmax, 0.0, zmax, np.zeros(nz, np.int32),
                           [(ELASTIC, 2200.0, 3000.0, 3000.0 / np.sqrt(3.0))],
                           absorbing=("bottom", "right", "left"), free_surface=())
    vp = grf_point_model(mesh, xmax, zmax, 3000.0, 0.1, 500.0, seed)
    vs = vp / np.sqrt(3.0)
    rho = np.full_like(vp, 2200.0)
    rng = np.random.default_rng(seed + 1)
    srcs = [RickerSource(float(rng.uniform(0.1, 0.9) * xmax), float(rng.uniform(0.5, 0.9) * zmax),
                         float(rng.uniform(4.0, 12.0)), 1e10, shot=s) for s in range(nshots)]
    rx = np.linspace(0.02 * xmax, 0.98 * xmax, nrec)
    rz = np.full(nrec, 0.95 * zmax)
    return Workload("elastic_grf_1000x500", mesh, srcs, rx, rz, 5e-4, nstep, rho.astype(np.float32),
                    vp.astype(np.float32), vs.astype(np.float32),
                    description=f"2D elastic {nx}x{nz} GRF(10%, 500 m) on vp 3000, {nshots} shots")


@dataclass
class AdjointWorkload:
    """Waveform-inversion test case: an initial model (the workload's point
    model) and the true model that made the observed data."""
    workload: Workload
    true_rho: np.ndarray
    true_vp: np.ndarray
    true_vs: np.ndarray
    anomaly: tuple  # (x0, z0, radius) of the Gaussian anomaly
    interval: int   # steps between forward checkpoints


def elastic_adjoint_500x250(nstep: int = 4000, nx: int = 500, nz: int = 250, nsrc: int = 8,
                            nrec: int = 200, seed: int = 0) -> AdjointWorkload:
    """2D elastic 500x250 quads over 12.5 x 6.25 km (h = 25 m); true model
    vp 3000, vs 1730, rho 2300 times (1 + 0.05 exp(-r^2/400^2)) around a seeded
    point, initial model without the anomaly; seeded sources at depth, a
    receiver line under the free surface; Stacey left/right/bottom."""
    xmax, zmax = 25.0 * nx, 25.0 * nz
    mesh = structured_mesh(nx, nz, 0.0, xmax, 0.0, zmax, np.zeros(nz, np.int32),
                           [(ELASTIC, 2300.0, 3000.0, 1730.0)],
                           absorbing=("bottom", "right", "left"), free_surface=())
    rng = np.random.default_rng(seed)
    x0 = float(rng.uniform(0.35, 0.65) * xmax)
    z0 = float(rng.uniform(0.40, 0.70) * zmax)
    radius = 400.0
    gz, gx = gll_coordinates(mesh)
    bump = np.exp(-((gx - x0) ** 2 + (gz - z0) ** 2) / radius ** 2)
    ones = np.ones((mesh.nspec, 25))
    srcs = [RickerSource(float(rng.uniform(0.05, 0.95) * xmax), float(rng.uniform(0.10, 0.35) * zmax),
                         8.0, 1e10) for _ in range(nsrc)]
    rx = np.linspace(0.02 * xmax, 0.98 * xmax, nrec)
    rz = np.full(nrec, zmax - 50.0)
    w = Workload(f"elastic_adjoint_{nx}x{nz}", mesh, srcs, rx, rz, 5e-4, nstep,
                 (2300.0 * ones).astype(np.float32), (3000.0 * ones).astype(np.float32),
                 (1730.0 * ones).astype(np.float32),
                 description=f"2D elastic {nx}x{nz} adjoint: +5% Gaussian (r=400 m) at "
                             f"({x0:.0f}, {z0:.0f}) m, {nsrc} sources, {nrec} receivers")
    f = 1.0 + 0.05 * bump
    return AdjointWorkload(w, (2300.0 * f).astype(np.float32), (3000.0 * f).astype(np.float32),
                           (1730.0 * f).astype(np.float32), (x0, z0, radius), 200)


def smooth_perturbations(mesh: Mesh, xmax: float, zmax: float, n: int, margin: float, seed: int):
    """n seeded smooth perturbations [n, nspec, 25] (sums of 3 Gaussians of
    radius 300-800 m, centres at least ``margin`` from the sides and bottom)."""
    rng = np.random.default_rng(seed)
    gz, gx = gll_coordinates(mesh)
    out = np.zeros((n, mesh.nspec, 25))
    for i in range(n):
        for _ in range(3):
            x0 = rng.uniform(margin, xmax - margin)
            z0 = rng.uniform(margin, zmax - 0.1 * zmax)
            r = rng.uniform(300.0, 800.0)
            out[i] += rng.choice([-1.0, 1.0]) * np.exp(-((gx - x0) ** 2 + (gz - z0) ** 2) / r ** 2)
    return out


# ------------------------------------------------------------------- 3D ---

@dataclass
class Mesh3D:
    """Structured lattice of 8-node hexahedra: element e = (ez*ney + ey)*nex + ex,
    control node (i, j, k) at nodes[(k*(ney+1) + j)*(nex+1) + i] = (x, y, z);
    per-GLL-point model [nspec, 125] (point q = (iz*5 + iy)*5 + ix);
    absorbing: Stacey on faces (xmin, xmax, ymin, ymax, zmin, zmax)."""
    nex: int
    ney: int
    nez: int
    nodes: np.ndarray
    rho: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    absorbing: tuple = (0, 0, 0, 0, 0, 0)

    @property
    def nspec(self):
        return self.nex * self.ney * self.nez

    @property
    def nglob(self):
        return (4 * self.nex + 1) * (4 * self.ney + 1) * (4 * self.nez + 1)


def hex_lattice(nex, ney, nez, x0, x1, y0, y1, z0, z1) -> np.ndarray:
    xs = np.linspace(x0, x1, nex + 1)
    ys = np.linspace(y0, y1, ney + 1)
    zs = np.linspace(z0, z1, nez + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X, Y, Z], -1).reshape(-1, 3)


def gll_coordinates3d(mesh: Mesh3D):
    """(x, y, z) of every element GLL point, each [nspec, 125], for the trilinear map."""
    r = np.sqrt(3.0 / 7.0)
    z1 = np.array([-1.0, -r, 0.0, r, 1.0])
    G, E, X = np.meshgrid(z1, z1, z1, indexing="ij")     # [iz, iy, ix]
    cs = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    N = np.stack([0.125 * (1 + c[0] * X) * (1 + c[1] * E) * (1 + c[2] * G) for c in cs], -1).reshape(125, 8)
    e = np.arange(mesh.nspec)
    ex, ey, ez = e % mesh.nex, (e // mesh.nex) % mesh.ney, e // (mesh.nex * mesh.ney)
    idx = np.stack([((ez + (c[2] > 0)) * (mesh.ney + 1) + ey + (c[1] > 0)) * (mesh.nex + 1) + ex + (c[0] > 0)
                    for c in cs], -1)                    # [nspec, 8]
    P = mesh.nodes[idx]                                  # [nspec, 8, 3]
    return tuple(P[:, :, k] @ N.T for k in range(3))


def homogeneous_hex_mesh(nex, ney, nez, extent, rho, vp, vs, absorbing=(0, 0, 0, 0, 0, 0)) -> Mesh3D:
    x0, x1, y0, y1, z0, z1 = extent
    nodes = hex_lattice(nex, ney, nez, x0, x1, y0, y1, z0, z1)
    n = nex * ney * nez
    one = np.ones((n, 125))
    return Mesh3D(nex, ney, nez, nodes, rho * one, vp * one, vs * one, tuple(absorbing))


@dataclass
class Workload3D:
    name: str
    mesh: Mesh3D
    sources: list       # oracle.runner3d.Source3D-like objects (x, y, z, f0, factor, kind, comp, tshift)
    rec_xyz: np.ndarray
    dt: float
    nstep: int
    description: str = ""


@dataclass
class Source3D:
    x: float
    y: float
    z: float
    f0: float
    factor: float
    kind: str = "force"
    comp: tuple = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    tshift: float = 0.0


def elastic3d_layered_grf(nex=128, ney=128, nez=64, nstep=5000, nrec=1000, seed=0, grf=True) -> Workload3D:
    """Hexahedral mesh over 64 x 64 x 32 km (h = 500 m at 128 x 128 x 64): a 1D
    layered background (vp 4.0 to 6.5 km/s with depth, vs = vp/1.73,
    rho = 1700 + 0.2 vp) times (1 + 0.05 GRF(corr. 4 km)); free surface on top
    (z = 0), Stacey on the other five faces; a seeded moment tensor with a
    Ricker of 1 Hz at 10 km depth; nrec receivers on the surface; dt = 2 ms."""
    rng = np.random.default_rng(seed)
    X, Y, Z = 64000.0 * nex / 128, 64000.0 * ney / 128, 32000.0 * nez / 64
    nodes = hex_lattice(nex, ney, nez, 0.0, X, 0.0, Y, -Z, 0.0)
    m = Mesh3D(nex, ney, nez, nodes, None, None, None, (1, 1, 1, 1, 1, 0))
    gx, gy, gz = gll_coordinates3d(m)
    depth = -gz
    vp = np.interp(depth, [0.0, 3000.0, 12000.0, 20000.0, 32000.0], [4000.0, 4800.0, 5800.0, 6300.0, 6500.0])
    if grf:
        ng = (max(16, nez), max(16, ney), max(16, nex))
        f = gaussian_random_field(ng, max(X, Y, Z) / max(ng), 4000.0, rng)
        iz = np.clip((depth / Z * (ng[0] - 1)).round().astype(int), 0, ng[0] - 1)
        iy = np.clip((gy / Y * (ng[1] - 1)).round().astype(int), 0, ng[1] - 1)
        ix = np.clip((gx / X * (ng[2] - 1)).round().astype(int), 0, ng[2] - 1)
        vp = vp * (1.0 + 0.05 * f[iz, iy, ix])
    m.vp = vp
    m.vs = vp / 1.73
    m.rho = 1700.0 + 0.2 * vp
    M = rng.standard_normal(6)
    src = [Source3D(0.5 * X + rng.uniform(-0.1, 0.1) * X, 0.5 * Y + rng.uniform(-0.1, 0.1) * Y, -10000.0 * nez / 64,
                    1.0, 1e15, "moment_tensor", tuple(float(c) for c in M))]
    rx = rng.uniform(0.05 * X, 0.95 * X, nrec)
    ry = rng.uniform(0.05 * Y, 0.95 * Y, nrec)
    rec = np.stack([rx, ry, np.zeros(nrec)], -1)
    return Workload3D(f"elastic3d_{nex}x{ney}x{nez}", m, src, rec, 2e-3, nstep,
                      description=f"3D elastic {nex}x{ney}x{nez} hexes, layered + 5% GRF, moment tensor 1 Hz, "
                                  f"{nrec} surface receivers, free top + Stacey")
