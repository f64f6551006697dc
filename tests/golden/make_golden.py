"""Build the golden fixtures under tests/golden/ from the reference checkout.

Each ``<fixture>.npz`` holds, for one of SPECFEM++'s Newmark regression
fixtures (``tests/unit-tests/displacement_tests/Newmark/serial/dim2/<name>``):
the mesh read from its ``database.bin`` (control nodes, connectivity,
materials, absorbing / free-surface edges), its sources, its stations, dt,
nstep and the golden displacement traces (``*.semd``, produced by Fortran
SPECFEM2D), stored as float32.  The tests rebuild a Case2D from it, so they
run without the reference tree.

Usage:  python tests/golden/make_golden.py [REFERENCE_ROOT [FIXTURE ...]]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import runner  # noqa: E402

FIXTURES = {
    "HomogeneousElasticDomain": ("BXX", "BXZ"),
    "HomogeneousElasticDomainStaceyDirichletBC": ("BXX", "BXZ"),
    "HomogeneousElasticDomainStaceyBC": ("BXX", "BXZ"),
    "HomogeneousAcousticDomainDirichletBC": ("BXX", "BXZ"),
    "AcousticElasticCoupledDomainVariant2": ("BXX", "BXZ"),
    "HomogeneousElasticDomainMomentTensor": ("BXX", "BXZ"),
    "HomogeneousElasticIsotropicDomainSH": ("BXY",),
    "HomogeneousElasticAnisotropicDomain": ("BXX", "BXZ"),
    "HomogeneousAcousticDomain": ("BXX", "BXZ"),
    "HomogeneousAcousticDomainCompositeStaceyDirichletBC": ("BXX", "BXZ"),
    "HomogeneousElasticDomainMomentTensorHeaviside": ("BXX", "BXZ"),
    "HomogeneousElasticDomainWAdjacencyMap": ("BXX", "BXZ"),
    "HomogeneousIsotropicCosseratDomainNu0": ("BXX", "BXZ"),
    "HomogeneousIsotropicCosseratDomain": ("BXX", "BXZ"),
    "HomogeneousIsotropicCosseratDomainHighFrequency": ("BXX", "BXZ"),
    "AcousticElasticNonconformingCoupledDomain": ("BXX", "BXZ"),
    "PoroelasticCoupledDomainPSV": ("BXX", "BXZ"),
    "AcousticElasticCoupledDomain": ("BXX", "BXZ"),
}


def rebuilt_coupled_domain(d):
    """AcousticElasticCoupledDomain ships no database.bin (its Snakefile runs
    xmeshfem2D): the mesh is rebuilt from its provenance Par_file and
    topography.dat, the mesher's internal structured grid of 144 x 108
    elements over 6400 x 4800 m with flat interfaces at 0, 2400 and 4800 m,
    rows 1-54 elastic (rho 2500, vp 3400, vs 1963), rows 55-108 water (rho
    1020, vp 1500), no absorbing edge, the acoustic top a free surface.  Its
    NGNOD = 9 elements are rectangles, so 4-node elements carry the same
    geometry.  Stations and sources are the fixture's own."""
    from specfempp_b200 import meshgen
    row = np.zeros(108, np.int32)
    row[54:] = 1
    mesh = meshgen.structured_mesh(144, 108, 0.0, 6400.0, 0.0, 4800.0, row,
                                   [(meshgen.ELASTIC, 2500.0, 3400.0, 1963.0),
                                    (meshgen.ACOUSTIC, 1020.0, 1500.0, 0.0)],
                                   absorbing=(), free_surface=("top",))
    names, rx, rz = runner.read_stations(os.path.join(d, "STATIONS"))
    src = runner.read_sources_yaml(os.path.join(d, "sources.yaml"))
    return runner.Case2D(mesh=mesh, sources=src, rec_x=rx, rec_z=rz, dt=0.85e-3, nstep=600,
                         stations=names)


REBUILT = {"AcousticElasticCoupledDomain": rebuilt_coupled_domain}

# time-function codes stored in the fixtures' source rows
STF_CODES = ["ricker", "dirac", "gaussian", "gaussian_hdur", "dgaussian", "heaviside"]


def make(ref_root: str, name: str, comps) -> str:
    d = os.path.join(ref_root, "tests/unit-tests/displacement_tests/Newmark/serial/dim2", name)
    case = REBUILT[name](d) if name in REBUILT else runner.load_fixture(d)
    m = case.mesh
    traces = {}
    t0 = None
    for ext in ("semd", "semv", "sema"):
        if not os.path.exists(os.path.join(d, "traces", f"{case.stations[0][0]}.{case.stations[0][1]}.S2.{comps[0]}.{ext}")):
            continue
        tr = np.zeros((len(case.stations), len(comps), case.nstep), np.float32)
        for r, (net, sta) in enumerate(case.stations):
            for c, comp in enumerate(comps):
                t, v = runner.read_trace(os.path.join(d, "traces", f"{net}.{sta}.S2.{comp}.{ext}"))
                tr[r, c, : len(v)] = v[: case.nstep]
                t0 = t[0]
        traces[ext] = tr
    # scalar traces: pressure (PRE) and, for Cosserat media, rotation,
    # intrinsic rotation and curl (BXY)
    for ext, ch in (("semp", "PRE"), ("semr", "BXY"), ("semir", "BXY"), ("semc", "BXY")):
        if not os.path.exists(os.path.join(d, "traces", f"{case.stations[0][0]}.{case.stations[0][1]}.S2.{ch}.{ext}")):
            continue
        tr = np.zeros((len(case.stations), 1, case.nstep), np.float32)
        for r, (net, sta) in enumerate(case.stations):
            t, v = runner.read_trace(os.path.join(d, "traces", f"{net}.{sta}.S2.{ch}.{ext}"))
            tr[r, 0, : len(v)] = v[: case.nstep]
        traces[ext] = tr
    extra = {}
    if getattr(m, "mat_aniso", None) is not None:
        extra["mat_aniso"] = m.mat_aniso
    if getattr(m, "mat_cosserat", None) is not None:
        extra["mat_cosserat"] = m.mat_cosserat
    if getattr(m, "mat_poro", None) is not None:
        extra["mat_poro"] = m.mat_poro
    nc = runner.nonconforming_records(m)
    if len(nc):
        extra["adjacency"] = nc        # nonconforming records only
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(
        out, nspec=m.nspec, npgeo=m.npgeo, ngnod=m.ngnod, coorg=m.coorg, knods=m.knods,
        kmato=m.kmato, mat_medium=m.mat_medium, mat_rho=m.mat_rho, mat_vp=m.mat_vp,
        mat_vs=m.mat_vs, abs_ispec=m.abs_ispec, abs_type=m.abs_type, free_ispec=m.free_ispec,
        free_type=m.free_type,
        src=np.asarray([[s.x, s.z, s.f0, s.factor, s.tshift, s.angle, 1.0 if s.stf == "dirac" else 0.0,
                         1.0 if s.kind == "moment_tensor" else 0.0, s.mxx, s.mzz, s.mxz,
                         float(STF_CODES.index(s.stf)), s.hdur]
                        for s in case.sources]),
        rec_x=case.rec_x, rec_z=case.rec_z, dt=case.dt, nstep=case.nstep, rec_angle=case.rec_angle,
        stations=np.asarray([f"{n}.{s}" for n, s in case.stations]), traces=traces["semd"],
        **{f"traces_{k}": v for k, v in traces.items() if k != "semd"},
        trace_t0=t0, components=np.asarray(comps), elastic_sh=int(case.elastic_sh), **extra)
    return out


FIXTURE_3D = "HomogeneousHalfspaceSmallNoABCForceSource"


def make3d(ref_root: str) -> str:
    """The 3D fixture: a regular 8 x 6 x 6 hexahedral mesh over 8 x 7 x 7.5 km
    (NEX_XI, NEX_ETA, depth and the single region of its Mesh_Par_file), one
    homogeneous material, no absorbing boundary; stations in the 3D format
    (station, network, y, x, elevation, z); the bytes of its database.bin
    (the 3D mesher's output) and its STATIONS and source files as text, so
    that the 3D configuration driver can be run on the fixture itself."""
    import yaml
    d = os.path.join(ref_root, "tests/unit-tests/displacement_tests/Newmark/serial/dim3", FIXTURE_3D)
    with open(os.path.join(d, "specfem_config.yaml")) as f:
        cfg = yaml.safe_load(f)["parameters"]
    ts = cfg["simulation-setup"]["solver"]["time-marching"]["time-scheme"]
    with open(os.path.join(d, "force.yaml")) as f:
        src = yaml.safe_load(f)["sources"][0]["force"]
    mat = None
    with open(os.path.join(d, "provenance", "specfempp", "Mesh_Par_file")) as f:
        lines = [ln.split("#")[0].strip() for ln in f]
    for i, ln in enumerate(lines):
        if ln.startswith("NMATERIALS"):
            nxt = next(x for x in lines[i + 1:] if x)             # first line after the comments
            mat = [float(v) for v in nxt.split()[1:4]]            # rho vp vs
    names, xyz = [], []
    with open(os.path.join(d, "STATIONS")) as f:
        for ln in f:
            p = ln.split()
            if len(p) >= 6:
                names.append(f"{p[1]}.{p[0]}")
                xyz.append([float(p[3]), float(p[2]), float(p[5])])
    nstep = int(ts["nstep"])
    traces = {}
    t0 = None
    for ext in ("semd", "semv", "sema"):
        tr = np.zeros((len(names), 3, nstep), np.float32)
        for r, nm in enumerate(names):
            for c, comp in enumerate(("BXX", "BXY", "BXZ")):
                t, v = runner.read_trace(os.path.join(d, "traces", f"{nm}.S3.{comp}.{ext}"))
                tr[r, c, : len(v)] = v[:nstep]
                t0 = t[0]
        traces[ext] = tr
    rk = src["Ricker"]
    out = os.path.join(HERE, f"{FIXTURE_3D}.npz")
    np.savez_compressed(out, nex=8, ney=6, nez=6, extent=np.array([0.0, 8000.0, 0.0, 7000.0, -7500.0, 0.0]),
                        material=np.array(mat), src_xyz=np.array([src["x"], src["y"], src["z"]], float),
                        src_force=np.array([src["fx"], src["fy"], src["fz"]], float),
                        src_f0=float(rk["f0"]), src_factor=float(rk["factor"]), src_tshift=float(rk["tshift"]),
                        dt=float(ts["dt"]), nstep=nstep, rec_xyz=np.array(xyz), stations=np.array(names),
                        traces_semd=traces["semd"], traces_semv=traces["semv"], traces_sema=traces["sema"],
                        trace_t0=t0, database=np.frombuffer(open(os.path.join(d, "database.bin"), "rb").read(),
                                                            np.uint8),
                        stations_text=open(os.path.join(d, "STATIONS")).read(),
                        sources_text=open(os.path.join(d, "force.yaml")).read())
    return out


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [FIXTURE ...]  (the SPECFEM++ checkout to read)")
    root = sys.argv[1]
    names = sys.argv[2:] or list(FIXTURES) + [FIXTURE_3D]
    for name in names:
        if name == FIXTURE_3D:
            out = make3d(root)
            print(out, os.path.getsize(out))
            continue
        print(make(root, name, FIXTURES[name]), os.path.getsize(os.path.join(HERE, f"{name}.npz")))
