"""C ABI and host-side assembly checks that need no GPU.

* libsfg.so loads and exports every function declared in include/sfg.h;
* the host assembly (numbering, colouring) agrees with the oracle's;
* the database.bin written by meshgen reads back identically through the
  C++ reader (libsfg) and the oracle's reader;
* error behaviour: missing file, point outside the mesh, calls out of order.
"""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_case


def header_symbols():
    text = open(os.path.join(ROOT, "include", "sfg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sfg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(sfg_lib):
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(sfg_lib, s), s
    from specfempp_b200 import sfg
    assert set(syms) == set(sfg.EXPORTS)


def test_numbering_matches_oracle(sfg_lib, oracle_lib):
    from oracle import runner
    from specfempp_b200 import sfg
    case, _, _ = golden_case("AcousticElasticCoupledDomainVariant2", nstep=10)
    r = runner.run(case, "f64", nthreads=4, want_final=True)
    sim = sfg.Simulation2D(case.mesh, dt=case.dt, nstep=case.nstep)
    ib_p, g2e, g2a = sim.numbering()
    ib_o = r["final"]["ibool"]
    assert sim.info().nglob == r["nglob"]
    # same partition of local points into global points: a bijection between ids
    pairs = np.unique(np.stack([ib_o.ravel(), ib_p.ravel()], 1), axis=0)
    assert len(pairs) == r["nglob"]
    inf = sim.info()
    assert inf.nspec_elastic + inf.nspec_acoustic == case.mesh.nspec
    assert inf.nglob_elastic == (g2e >= 0).sum() and inf.nglob_acoustic == (g2a >= 0).sum()
    assert ((g2e >= 0) & (g2a >= 0)).sum() > 0              # interface points in both media


def test_colouring_is_conflict_free(sfg_lib):
    from specfempp_b200 import meshgen, sfg
    w = meshgen.coupled_400x200(nstep=10, nx=40, nz=20)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep)
    inf = sim.info()
    assert inf.ncolors_elastic == 4 and inf.ncolors_acoustic == 4


def test_database_roundtrip(tmp_path, sfg_lib):
    from oracle.database2d import read_database
    from specfempp_b200 import meshgen, sfg
    w = meshgen.coupled_400x200(nstep=10, nx=40, nz=20)
    p = str(tmp_path / "database.bin")
    meshgen.write_database(w.mesh, p)
    m = read_database(p)
    assert m.nspec == w.mesh.nspec and m.npgeo == w.mesh.npgeo
    assert np.array_equal(m.knods, w.mesh.knods) and np.allclose(m.coorg, w.mesh.coorg)
    assert np.array_equal(m.abs_ispec, w.mesh.abs_ispec) and np.array_equal(m.abs_type, w.mesh.abs_type)
    assert np.array_equal(m.free_ispec, w.mesh.free_ispec) and np.array_equal(m.free_type, w.mesh.free_type)
    assert np.array_equal(m.mat_medium, w.mesh.mat_medium)
    a = sfg.Simulation2D(database=p, dt=w.dt, nstep=10)
    b = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=10)
    ia, ib = a.info(), b.info()
    assert (ia.nglob, ia.nglob_elastic, ia.nglob_acoustic) == (ib.nglob, ib.nglob_elastic, ib.nglob_acoustic)


def test_error_paths(tmp_path, sfg_lib):
    from specfempp_b200 import meshgen, sfg
    with pytest.raises(sfg.SfgError) as e:
        sfg.Simulation2D(database=str(tmp_path / "missing.bin"), dt=1e-3, nstep=10)
    assert e.value.code == -2
    bad = tmp_path / "trunc.bin"
    w = meshgen.elastic_psv_80x60(10)
    meshgen.write_database(w.mesh, str(bad))
    data = open(bad, "rb").read()
    open(bad, "wb").write(data[: len(data) // 2])
    with pytest.raises(sfg.SfgError) as e:
        sfg.Simulation2D(database=str(bad), dt=1e-3, nstep=10)
    assert e.value.code == -2
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=10)
    with pytest.raises(sfg.SfgError) as e:
        sim.set_receivers([1e7], [1e7])
    assert e.value.code == -4
    with pytest.raises(sfg.SfgError) as e:
        sim.run(1)
    assert e.value.code == -5
    with pytest.raises(sfg.SfgError):
        sfg.Simulation2D(w.mesh, dt=-1.0, nstep=10)


def test_library_exports_every_declared_3d_symbol(sfg_lib):
    text = open(os.path.join(ROOT, "include", "sfg3d.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    syms = sorted(set(re.findall(r"\b(sfg3d_[a-z0-9_]+)\s*\(", text)))
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(sfg_lib, s), s
    from specfempp_b200 import sfg3d
    assert set(syms) == set(sfg3d.EXPORTS3D)


def test_3d_create_errors(sfg_lib):
    """Argument checks of the 3D interface that need no GPU."""
    from specfempp_b200 import meshgen, sfg, sfg3d
    m = meshgen.homogeneous_hex_mesh(2, 2, 2, (0, 1000, 0, 1000, -1000, 0), 2700.0, 3000.0, 1732.0)
    with pytest.raises(sfg.SfgError):
        sfg3d.Simulation3D(m, dt=-1.0, nstep=10)
    bad = meshgen.homogeneous_hex_mesh(2, 2, 2, (0, 1000, 0, 1000, -1000, 0), 2700.0, 1000.0, 1732.0)
    with pytest.raises(sfg.SfgError):
        sfg3d.Simulation3D(bad, dt=1e-3, nstep=10)


def test_geometry_export(sfg_lib):
    """sfg_get_geometry: GLL point coordinates and |J| of the library's set-up
    equal the 4-node shape-function geometry; media per element."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.coupled_400x200(nstep=10, nx=40, nz=20)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=10)
    x, z, jac, med = sim.geometry()
    gx, gz, gj = meshgen.gll_geometry(w.mesh)
    assert np.allclose(x, gx, rtol=0, atol=1e-6) and np.allclose(z, gz, rtol=0, atol=1e-6)
    assert np.allclose(jac, gj, rtol=1e-12)
    assert np.array_equal(med, np.asarray(w.mesh.mat_medium)[w.mesh.kmato])


def test_cosserat_mesh_has_three_components(sfg_lib):
    """A mesh with Cosserat materials: the elastic medium carries u_x, u_z and
    the rotation (sfg_info.ncomp_elastic 3)."""
    from conftest import golden_case
    from specfempp_b200 import sfg
    case, _, _ = golden_case("HomogeneousIsotropicCosseratDomain", nstep=10)
    sim = sfg.Simulation2D(case.mesh, dt=case.dt, nstep=10)
    assert sim.info().ncomp_elastic == 3 and sim.ncomp == 3


def test_nonconforming_records_host_side(tmp_path, sfg_lib):
    """Adjacency records survive the database round trip (oracle reader and
    the product's reader agree on the numbering); a nonconforming record
    without its reverse, an out-of-range record and non-overlapping edges
    are refused at creation (host assembly, no GPU)."""
    from oracle.database2d import read_database
    from specfempp_b200 import meshgen, sfg
    w = meshgen.nonconforming_coupled(nx_el=6, nx_ac=9, nz_el=3, nz_ac=3, nstep=5)
    p = str(tmp_path / "database.bin")
    meshgen.write_database(w.mesh, p)
    m = read_database(p)
    assert np.array_equal(m.extra["adjacency"], w.mesh.adjacency)
    a = sfg.Simulation2D(database=p, dt=w.dt, nstep=5)
    b = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=5)
    ia, ib = a.info(), b.info()
    assert (ia.nglob_elastic, ia.nglob_acoustic) == (ib.nglob_elastic, ib.nglob_acoustic)
    # no shared control nodes across the interface: no conforming coupling
    assert ia.nglob_elastic == (6 * 4 + 1) * (3 * 4 + 1)
    adj = w.mesh.adjacency
    nc = np.nonzero(adj[:, 2] == 3)[0]
    w.mesh.adjacency = np.delete(adj, nc[0], axis=0)
    with pytest.raises(sfg.SfgError, match="Non-symmetric"):
        sfg.Simulation2D(w.mesh, dt=w.dt, nstep=5)
    bad = adj.copy()
    bad[nc[0], 1] = w.mesh.nspec
    w.mesh.adjacency = bad
    with pytest.raises(sfg.SfgError, match="adjacency"):
        sfg.Simulation2D(w.mesh, dt=w.dt, nstep=5)
    far = adj.copy()
    e, ac = far[nc[0], 0], far[nc[0], 1]
    back = np.nonzero((far[:, 0] == ac) & (far[:, 1] == e))[0][0]
    far[nc[0], 1] = ac + 8
    far[back, 0] = ac + 8
    w.mesh.adjacency = far
    with pytest.raises(sfg.SfgError, match="intersection"):
        sfg.Simulation2D(w.mesh, dt=w.dt, nstep=5)


def test_poroelastic_host_side(tmp_path, sfg_lib):
    """A poroelastic mesh assembles with four elastic components, also from
    a database.bin with material type 3; Stacey edges, an attenuating Q_mu
    and a mix with isotropic elastic elements are refused (host assembly,
    no GPU)."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.poroelastic_model(nx=6, nz=6, nstep=5, layered=True)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=5)
    inf = sim.info()
    assert inf.ncomp_elastic == 4 and inf.nspec_elastic == 36 and inf.nspec_acoustic == 0
    p = str(tmp_path / "database.bin")
    meshgen.write_database(w.mesh, p)
    from oracle.database2d import read_database
    m = read_database(p)
    assert np.allclose(m.mat_poro, w.mesh.mat_poro)
    assert sfg.Simulation2D(database=p, dt=w.dt, nstep=5).info().ncomp_elastic == 4
    st = meshgen.poroelastic_model(nx=6, nz=6, nstep=5)
    st.mesh.abs_ispec = np.array([0], np.int32)
    st.mesh.abs_type = np.array([0], np.int32)
    with pytest.raises(sfg.SfgError, match="Stacey"):
        sfg.Simulation2D(st.mesh, dt=w.dt, nstep=5)
    q = meshgen.poroelastic_model(nx=6, nz=6, nstep=5)
    q.mesh.mat_poro[0, 12] = 50.0
    with pytest.raises(sfg.SfgError, match="attenuation"):
        sfg.Simulation2D(q.mesh, dt=w.dt, nstep=5)
    mix = meshgen.poroelastic_model(nx=6, nz=6, nstep=5, layered=True)
    mix.mesh.mat_poro[1] = np.nan
    mix.mesh.mat_vp[1], mix.mesh.mat_vs[1], mix.mesh.mat_rho[1] = 3000.0, 1700.0, 2400.0
    with pytest.raises(sfg.SfgError, match="poroelastic"):
        sfg.Simulation2D(mix.mesh, dt=w.dt, nstep=5)
