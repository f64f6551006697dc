"""The 3D configuration front end on CPU: the reference's 3D mesh database
(the fixture's own database.bin and databases written here with permuted
numbering), its mapping onto the library's hexahedral lattice, the 3D
STATIONS and source readers and the trace writer's names."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN
from fixture_dir import write_fixture_dir3d

FIX3D = os.path.join(GOLDEN, "HomogeneousHalfspaceSmallNoABCForceSource.npz")


def test_fixture_database_is_the_golden_lattice():
    """database.bin of the dim3 fixture: 288 8-node elements forming the
    8 x 6 x 6 lattice over 8 x 7 x 7.5 km that the oracle's golden test
    builds, one elastic material, face lists on all six sides."""
    from specfempp_b200 import database3d, meshgen
    z = np.load(FIX3D)
    db = database3d.parse_database3d(z["database"].tobytes())
    assert (db.nspec, db.ngnod, db.ngll) == (288, 8, (5, 5, 5))
    assert {k: len(v[0]) for k, v in db.faces.items()} == {"xmin": 36, "xmax": 36, "ymin": 48, "ymax": 48,
                                                          "zmin": 48, "zmax": 48}
    m = database3d.lattice_mesh(db)
    assert (m.nex, m.ney, m.nez) == (8, 6, 6) and m.absorbing == (0, 0, 0, 0, 0, 0)
    ref = meshgen.homogeneous_hex_mesh(8, 6, 6, z["extent"], *z["material"])
    assert np.abs(m.nodes - ref.nodes).max() < 1e-9
    assert np.allclose(m.rho, 2700.0) and np.allclose(m.vp, 3000.0) and np.allclose(m.vs, 1732.051)
    assert database3d.lattice_mesh(db, absorbing=True).absorbing == (1, 1, 1, 1, 1, 0)


def _distorted(nex, ney, nez, seed):
    from specfempp_b200 import meshgen
    rng = np.random.default_rng(seed)
    nodes = meshgen.hex_lattice(nex, ney, nez, 0.0, 1000.0 * nex, 0.0, 900.0 * ney, -800.0 * nez, 0.0)
    x, y, z = nodes.T
    nodes = nodes + np.stack([60 * np.sin(y / 700.0 + z / 900.0), 50 * np.cos(x / 800.0), 40 * np.sin(x / 600.0)], -1)
    nodes[:, 2] += rng.uniform(-1, 1, len(nodes)) * 5.0
    return meshgen.Mesh3D(nex, ney, nez, nodes, None, None, None)


def test_permuted_database_round_trip():
    """A distorted lattice written with shuffled element records and
    control-node ids, two materials: the reader rebuilds the same lattice,
    node for node and material for material."""
    from specfempp_b200 import database3d
    rng = np.random.default_rng(3)
    m = _distorted(5, 4, 3, 1)
    mats = [(2000.0, 2500.0, 1400.0), (2600.0, 4000.0, 2300.0)]
    mat_of = (np.arange(m.nspec) // (m.nex * m.ney) >= 1).astype(np.int64)
    buf = database3d.database3d_bytes(m, mats, mat_of, element_order=rng.permutation(m.nspec),
                                      node_order=rng.permutation(len(m.nodes)))
    got = database3d.lattice_mesh(database3d.parse_database3d(buf))
    assert (got.nex, got.ney, got.nez) == (5, 4, 3)
    assert np.array_equal(got.nodes, m.nodes)
    want_vp = np.asarray(mats)[mat_of][:, 1]
    assert np.array_equal(got.vp[:, 0], want_vp.astype(np.float32))
    assert np.all(got.vp == got.vp[:, :1]) and got.rho.shape == (m.nspec, 125)


def test_database_refusals():
    """Databases outside the lattice class or the elastic 3D path are refused
    with the reason: an element removed, an acoustic material, a truncated
    file, a PML count."""
    from specfempp_b200 import database3d
    m = _distorted(3, 3, 2, 2)
    mats = [(2000.0, 2500.0, 1400.0)]
    ok = database3d.database3d_bytes(m, mats, np.zeros(m.nspec, np.int64))
    db = database3d.parse_database3d(ok)
    keep = np.arange(db.nspec) != 4
    holed = database3d.Database3D(db.ngnod, db.coords, db.elements[keep], db.material_of[keep], db.materials,
                                  db.ngll, db.faces)
    with pytest.raises(ValueError, match="lattice"):
        database3d.lattice_mesh(holed)
    ac = database3d.database3d_bytes(m, [(1020.0, 1500.0, 0.0)], np.zeros(m.nspec, np.int64))
    with pytest.raises(ValueError, match="acoustic"):
        database3d.lattice_mesh(database3d.parse_database3d(ac))
    with pytest.raises(ValueError):
        database3d.parse_database3d(ok[:-10])
    def rec(fmt, *v):
        b = struct.pack(fmt, *v)
        return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    tail = rec("<i", 0) + rec("<ii", 0, 0) + rec("<i", 0)          # PML, MPI interfaces, adjacency
    assert ok.endswith(tail)
    pml = ok[:-len(tail)] + rec("<i", 1) + rec("<ii", 0, 0) + rec("<i", 0)
    with pytest.raises(ValueError, match="PML"):
        database3d.parse_database3d(pml)


def test_config_inputs(tmp_path):
    """The fixture's run directory through the 3D readers: 26 stations with
    the (y, x) column swap, the force source, the trace names and band code."""
    from specfempp_b200 import io, specfem3d
    cfg_path, z = write_fixture_dir3d(FIX3D, str(tmp_path))
    cfg = io.read_config(cfg_path, str(tmp_path))
    assert (cfg.dt, cfg.nstep) == (float(z["dt"]), int(z["nstep"]))
    names, xyz = specfem3d.read_stations3d(cfg.stations)
    assert [f"{n}.{s}" for n, s in names] == [str(s) for s in z["stations"]]
    assert np.allclose(xyz, z["rec_xyz"])
    (src,) = specfem3d.read_sources3d(cfg.sources)
    assert (src.x, src.y, src.z) == tuple(z["src_xyz"]) and src.comp[:3] == tuple(z["src_force"])
    assert src.f0 == float(z["src_f0"]) and src.kind == "force"
    assert specfem3d.band_code(float(z["dt"])) == "B" and specfem3d.band_code(2e-3) == "C"
    seis = np.arange(2 * 1 * 2 * 3, dtype=np.float32).reshape(2, 1, 2, 3)
    p = specfem3d.write_seismograms3d(str(tmp_path / "tr"), [("XX", "A1"), ("XX", "A2")], seis, ["velocity"],
                                      -1.0, 0.035, 1)
    assert [os.path.basename(q) for q in p[:3]] == ["XX.A1.S3.BXX.semv", "XX.A1.S3.BXY.semv", "XX.A1.S3.BXZ.semv"]
    t, v = np.loadtxt(p[4]).T
    assert np.allclose(t, [-1.0, -0.965]) and np.allclose(v, seis[:, 0, 1, 1])


def _with_hex27(db, bend=0.0):
    """The same mesh with 27-node elements: the 19 extra nodes of every
    element at its edge midpoints, face centres and centre (new control
    nodes, in a shuffled order per element); `bend` moves the centre node of
    element 0 off the trilinear map."""
    from specfempp_b200 import database3d
    rng = np.random.default_rng(5)
    P = db.coords[db.elements[:, :8]]
    coords = [db.coords]
    extra = np.zeros((db.nspec, 19), np.int64)
    nxt = len(db.coords)
    for e in range(db.nspec):
        pts = []
        for a, b, c in database3d._HEX27_REST:
            w = np.array([(a if s[0] else 1 - a) * (b if s[1] else 1 - b) * (c if s[2] else 1 - c)
                          for s in database3d.CORNER_SIGNS])
            pts.append(w @ P[e])
        pts = np.array(pts)
        if e == 0 and bend:
            pts[-1] += bend
        perm = rng.permutation(19)
        coords.append(pts[perm])
        extra[e] = nxt + np.arange(19)
        nxt += 19
    return database3d.Database3D(27, np.concatenate(coords), np.concatenate([db.elements, extra], 1),
                                 db.material_of, db.materials, db.ngll, db.faces)


def test_hex27_straight_accepted_curved_refused():
    """27-node elements whose extra nodes lie on the trilinear map of their
    corners (in any order) give the 8-node lattice; a centre node moved off
    it is refused (the library maps elements trilinearly)."""
    from specfempp_b200 import database3d
    m = _distorted(3, 2, 2, 4)
    db = database3d.parse_database3d(database3d.database3d_bytes(m, [(2000.0, 2500.0, 1400.0)],
                                                                 np.zeros(m.nspec, np.int64)))
    got = database3d.lattice_mesh(_with_hex27(db))
    assert np.array_equal(got.nodes, m.nodes)
    with pytest.raises(ValueError, match="curved"):
        database3d.lattice_mesh(_with_hex27(db, bend=25.0))


def test_sources3d_moment_tensor_and_refusals(tmp_path):
    """Moment-tensor sources keep (Mxx, Myy, Mzz, Mxy, Mxz, Myz); time
    functions other than Ricker and a wrong source count are refused."""
    import yaml
    from specfempp_b200 import specfem3d
    mt = {"x": 1.0, "y": 2.0, "z": -3.0, "Mxx": 1.0, "Myy": 2.0, "Mzz": 3.0, "Mxy": 4.0, "Mxz": 5.0, "Myz": 6.0,
          "Ricker": {"factor": 1e15, "tshift": 0.1, "f0": 2.0}}
    p = tmp_path / "s.yaml"
    p.write_text(yaml.safe_dump({"number-of-sources": 1, "sources": [{"moment-tensor": mt}]}))
    (s,) = specfem3d.read_sources3d(str(p))
    assert s.kind == "moment_tensor" and s.comp == (1.0, 2.0, 3.0, 4.0, 5.0, 6.0) and s.tshift == 0.1
    bad = dict(mt)
    del bad["Ricker"]
    bad["Dirac"] = {"factor": 1.0}
    p.write_text(yaml.safe_dump({"number-of-sources": 1, "sources": [{"moment-tensor": bad}]}))
    with pytest.raises(ValueError, match="Ricker"):
        specfem3d.read_sources3d(str(p))
    p.write_text(yaml.safe_dump({"number-of-sources": 2, "sources": [{"moment-tensor": mt}]}))
    with pytest.raises(ValueError, match="number of sources"):
        specfem3d.read_sources3d(str(p))


def test_seismogram_subsampling(tmp_path):
    """nstep_between_samples: samples of steps 0, nsb, 2 nsb, ... written at
    t0 + k dt nsb."""
    from specfempp_b200 import specfem3d
    seis = np.arange(10 * 1 * 1 * 3, dtype=np.float32).reshape(10, 1, 1, 3)
    sub = specfem3d.subsample(seis, 4)
    assert np.array_equal(sub[:, 0, 0, 0], seis[[0, 4, 8], 0, 0, 0])
    p = specfem3d.write_seismograms3d(str(tmp_path), [("XX", "A")], sub, ["displacement"], -0.5, 0.01, 4)
    t, v = np.loadtxt(p[2]).T
    assert np.allclose(t, [-0.5, -0.46, -0.42]) and np.allclose(v, seis[[0, 4, 8], 0, 0, 2])


def test_stations_as_yaml_sequences(tmp_path):
    """Stations given inline in the configuration (the readers' second form):
    the 3D list gives the same receivers as the fixture's STATIONS file, and
    the 2D reader takes (network, station, x, z) entries."""
    import yaml
    from specfempp_b200 import io, specfem3d
    cfg_path, z = write_fixture_dir3d(FIX3D, str(tmp_path))
    names, xyz = specfem3d.read_stations3d(str(tmp_path / "STATIONS"))
    cfg = yaml.safe_load(open(cfg_path))
    cfg["parameters"]["receivers"]["stations"] = [
        {"network": n, "station": s, "x": float(p[0]), "y": float(p[1]), "z": float(p[2])}
        for (n, s), p in zip(names, xyz)]
    with open(cfg_path, "w") as f:
        yaml.safe_dump(cfg, f)
    c = io.read_config(cfg_path, str(tmp_path))
    n2, xyz2 = specfem3d.read_stations3d(c.stations)
    assert n2 == names and np.array_equal(xyz2, xyz)
    n, x, zz = io.read_stations([{"network": "AA", "station": "S1", "x": 10.0, "z": 20.0},
                                 {"network": "AA", "station": "S2", "x": 30.0, "z": 40.0}])
    assert n == [("AA", "S1"), ("AA", "S2")] and np.array_equal(x, [10.0, 30.0]) and np.array_equal(zz, [20.0, 40.0])
    with pytest.raises(ValueError):
        specfem3d.read_stations3d([])


def test_sources_inline_node(tmp_path):
    """The sources node given inline in the configuration reads like the
    fixture's force.yaml (3D) and like a sources.yaml (2D)."""
    import yaml
    from specfempp_b200 import io, specfem3d
    cfg_path, z = write_fixture_dir3d(FIX3D, str(tmp_path))
    node = yaml.safe_load(open(tmp_path / "force.yaml"))
    cfg = yaml.safe_load(open(cfg_path))
    cfg["parameters"]["sources"] = node
    with open(cfg_path, "w") as f:
        yaml.safe_dump(cfg, f)
    c = io.read_config(cfg_path, str(tmp_path))
    assert specfem3d.read_sources3d(c.sources) == specfem3d.read_sources3d(str(tmp_path / "force.yaml"))
    two = {"number-of-sources": 1, "sources": [{"force": {"x": 1.0, "z": 2.0, "angle": 0.0,
                                                          "Ricker": {"factor": 1e10, "tshift": 0.0, "f0": 5.0}}}]}
    (s,) = io.read_sources(two)
    assert (s.x, s.z, s.f0, s.factor, s.kind) == (1.0, 2.0, 5.0, 1e10, "force")
