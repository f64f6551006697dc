"""Rebuild a reference-style run directory (database.bin, STATIONS,
sources.yaml, specfem_config.yaml) from a committed golden fixture."""
import os

import numpy as np
import yaml


def write_fixture_dir(npz_path, out_dir, types=("displacement",)):
    from specfempp_b200 import meshgen
    z = np.load(npz_path)
    mesh = meshgen.Mesh(nspec=int(z["nspec"]), npgeo=int(z["npgeo"]), ngnod=int(z["ngnod"]), coorg=z["coorg"],
                        knods=z["knods"], kmato=z["kmato"], mat_medium=z["mat_medium"], mat_rho=z["mat_rho"],
                        mat_vp=z["mat_vp"], mat_vs=z["mat_vs"], abs_ispec=z["abs_ispec"], abs_type=z["abs_type"],
                        free_ispec=z["free_ispec"], free_type=z["free_type"],
                        mat_poro=z["mat_poro"] if "mat_poro" in z else None,
                        adjacency=z["adjacency"] if "adjacency" in z else None)
    os.makedirs(out_dir, exist_ok=True)
    meshgen.write_database(mesh, os.path.join(out_dir, "database.bin"))
    with open(os.path.join(out_dir, "STATIONS"), "w") as f:
        for name, x, zz in zip(z["stations"], z["rec_x"], z["rec_z"]):
            net, sta = str(name).split(".")
            f.write(f"{sta} {net} {x:.6f} {zz:.6f} 0.0 0.0\n")
    srcs = []
    codes = ["ricker", "dirac", "gaussian", "gaussian_hdur", "dgaussian", "heaviside"]
    keys = {"ricker": "Ricker", "dirac": "Dirac", "gaussian": "Gaussian", "gaussian_hdur": "Gaussian",
            "dgaussian": "dGaussian", "heaviside": "Heaviside"}
    for s in z["src"]:
        stf = codes[int(s[11])] if len(s) > 11 else ("dirac" if s[6] else "ricker")
        par = {"factor": float(s[3]), "tshift": float(s[4])}
        if stf in ("gaussian_hdur", "heaviside"):
            par["hdur"] = float(s[12])
        else:
            par["f0"] = float(s[2])
        tf = {keys[stf]: par}
        if len(s) > 7 and s[7]:
            srcs.append({"moment-tensor": {"x": float(s[0]), "z": float(s[1]), "Mxx": float(s[8]),
                                           "Mzz": float(s[9]), "Mxz": float(s[10]), **tf}})
        else:
            srcs.append({"force": {"x": float(s[0]), "z": float(s[1]), "angle": float(s[5]), **tf}})
    with open(os.path.join(out_dir, "sources.yaml"), "w") as f:
        yaml.safe_dump({"number-of-sources": len(srcs), "sources": srcs}, f)
    sh = bool(int(z["elastic_sh"])) if "elastic_sh" in z else False
    cfg = {"parameters": {
        "simulation-setup": {
            "elastic-wave": "SH" if sh else "P_SV",
            "quadrature": {"quadrature-type": "GLL4"},
            "solver": {"time-marching": {"type-of-simulation": "forward",
                                         "time-scheme": {"type": "Newmark", "dt": float(z["dt"]),
                                                         "nstep": int(z["nstep"])}}},
            "simulation-mode": {"forward": {"writer": {"seismogram": {"format": "ascii", "directory": "traces"}}}}},
        "receivers": {"stations": "STATIONS", "angle": float(z["rec_angle"]), "seismogram-type": list(types),
                      "nstep_between_samples": 1},
        "databases": {"mesh-database": "database.bin"},
        "sources": "sources.yaml"}}
    path = os.path.join(out_dir, "specfem_config.yaml")
    with open(path, "w") as f:
        yaml.safe_dump(cfg, f)
    return path, z


def write_fixture_dir3d(npz_path, out_dir, types=("displacement", "velocity", "acceleration")):
    """The 3D fixture's run directory: its own database.bin, STATIONS and
    force.yaml (stored verbatim in the npz) plus a specfem_config.yaml with
    the fixture's dt and nstep."""
    z = np.load(npz_path)
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, "database.bin"), "wb") as f:
        f.write(z["database"].tobytes())
    with open(os.path.join(out_dir, "STATIONS"), "w") as f:
        f.write(str(z["stations_text"][()]))
    with open(os.path.join(out_dir, "force.yaml"), "w") as f:
        f.write(str(z["sources_text"][()]))
    cfg = {"parameters": {
        "simulation-setup": {
            "quadrature": {"quadrature-type": "GLL4"},
            "solver": {"time-marching": {"type-of-simulation": "forward",
                                         "time-scheme": {"type": "Newmark", "dt": float(z["dt"]),
                                                         "nstep": int(z["nstep"])}}},
            "simulation-mode": {"forward": {"writer": {"seismogram": {"format": "ascii", "directory": "traces"}}}}},
        "receivers": {"stations": "STATIONS", "angle": 0.0, "seismogram-type": list(types),
                      "nstep_between_samples": 1},
        "run-setup": {"number-of-processors": 1, "number-of-runs": 1},
        "databases": {"mesh-database": "database.bin"},
        "sources": "force.yaml"}}
    path = os.path.join(out_dir, "specfem_config.yaml")
    with open(path, "w") as f:
        yaml.safe_dump(cfg, f)
    return path, z
