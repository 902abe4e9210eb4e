"""Generates the reference-case fixtures of tests/test_reference_cases.py:
inputs files and ASCII material-point files written by the reference's own
pre-processor (Tests/Dam_Break/PreProcess/Generate_MPs_Inputfile_Generic.py:
generate_particle_chunks, write_particles_ascii_streaming :1019-1132 and
write_inputs_file :807-995), run here on small 3-D configurations.

The pre-processor imports h5py and matplotlib for its HDF5 writer and its
plots, neither of which these calls use (and neither is installed here), so
empty stand-in modules satisfy the imports.  The reference tree is read from
EXG_REFERENCE_DIR.  Run from the repository root:

    python tests/golden/make_reference_cases.py

Outputs (committed): tests/golden/refcase_<name>.inp, refcase_<name>.dat and
refcase_<name>.json (the configuration, for the tests' expected values).
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("EXG_REFERENCE_DIR", "/root/reference"))
GEN = REF / "Tests" / "Dam_Break" / "PreProcess" / "Generate_MPs_Inputfile_Generic.py"

CASES = {
    # a fluid column in a box, z periodic as the pre-processor writes every
    # 3-D domain, quadratic B-splines, USL
    "dam_break_3d": {
        "grid": {"xmin": 0.0, "xmax": 0.8, "nx": 16, "ymin": 0.0, "ymax": 0.4, "ny": 8,
                 "zmin": 0.0, "zmax": 1.2, "nz": 24},
        "ppc": [2, 2, 2],
        "body": {"shape": {"type": "block", "xmin": 0.0, "xmax": 0.3, "ymin": 0.0, "ymax": 0.4,
                           "zmin": 0.0, "zmax": 0.6},
                 "constitutive_model": {"type": "fluid", "Bulk_modulus": 2e6, "Gamma_pressure": 7.0,
                                        "Dynamic_viscosity": 1e-3},
                 "initial_velocity": {"type": "uniform", "vx": 0.0, "vy": 0.0, "vz": 0.0},
                 "temperature": {"enabled": False}},
        "density": 1000.0, "CFL": 0.1, "order_scheme": 2, "stress_update_scheme": "USL",
        "alpha_pic_flip": 0.99,
        "simulation": {"final_time": 0.02, "max_steps": 40, "screen_output_time": 0.01,
                       "write_output_time": 0.01, "num_redist": 1, "fixed_timestep": 0, "timestep": 1e-5},
        "gravity": [0.0, -9.81, 0.0],
        "boundary_conditions": {"xlo": {"mom": "slip"}, "xhi": {"mom": "slip"}, "ylo": {"mom": "noslip"},
                                "yhi": {"mom": "slip"}},
        "diagnostics": {"print_diagnostics": 1, "do_calculate_tke_tse": 1, "do_calculate_mwa_velcomp": 1,
                        "do_calculate_mwa_velmag": 1, "do_calculate_minmaxpos": 1,
                        "write_diag_output_time": 0.005},
    },
    # an elastic block moving towards a partial-slip wall, cubic
    # B-splines, MUSL
    "elastic_block_3d": {
        "grid": {"xmin": -0.5, "xmax": 0.5, "nx": 20, "ymin": -0.25, "ymax": 0.25, "ny": 10,
                 "zmin": 0.0, "zmax": 1.2, "nz": 24},
        "ppc": [2, 2, 2],
        "body": {"shape": {"type": "block", "xmin": -0.2, "xmax": 0.2, "ymin": -0.1, "ymax": 0.1,
                           "zmin": 0.2, "zmax": 0.8},
                 "constitutive_model": {"type": "elastic", "E": 1e5, "nu": 0.3},
                 "initial_velocity": {"type": "uniform", "vx": 0.5, "vy": -0.2, "vz": 0.1},
                 "temperature": {"enabled": False}},
        "density": 1200.0, "CFL": 0.2, "order_scheme": 3, "stress_update_scheme": "MUSL",
        "alpha_pic_flip": 0.95,
        "simulation": {"final_time": 0.05, "max_steps": 30, "screen_output_time": 0.01,
                       "write_output_time": 0.01, "num_redist": 1, "fixed_timestep": 1, "timestep": 2e-4},
        "gravity": [0.0, 0.0, -9.81],
        "boundary_conditions": {"xlo": {"mom": "noslip"}, "xhi": {"mom": "partialslip"},
                                "ylo": {"mom": "slip"}, "yhi": {"mom": "slip"}},
        "diagnostics": {"print_diagnostics": 0},
    },
}


def load_generator():
    for name in ("h5py", "matplotlib", "matplotlib.pyplot", "matplotlib.patches"):
        sys.modules.setdefault(name, types.ModuleType(name))
    spec = importlib.util.spec_from_file_location("exagoop_generator", GEN)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    g = load_generator()
    cwd = os.getcwd()
    os.chdir(HERE)
    try:
        for name, cfg in CASES.items():
            body = cfg["body"]
            vel = body["initial_velocity"]
            vx, vy, vz = vel["vx"], vel["vy"], vel["vz"]
            chunks = g.generate_particle_chunks(
                dimensions=3, grid=cfg["grid"], ppc=tuple(cfg["ppc"]),
                constitutive_model=body["constitutive_model"], enable_temperature=False,
                shape_cfg=body["shape"], density=cfg["density"],
                velocity_function=lambda x, y, z: (vx, vy, vz),
                temperature_function=lambda x, y, z: (0.0, 0.0, 0.0, 0.0))
            pfile = f"refcase_{name}.dat"
            n = g.write_particles_ascii_streaming(pfile, chunks, 3)
            g.write_inputs_file(
                grid=cfg["grid"], dimensions=3, order_scheme=cfg["order_scheme"],
                alpha_pic_flip=cfg["alpha_pic_flip"], CFL=cfg["CFL"],
                stress_update_scheme=cfg["stress_update_scheme"], output_tag=f"refcase_{name}",
                constitutive_model=body["constitutive_model"], enable_temperature=False,
                particle_filename=pfile, out_filename=f"refcase_{name}.inp", simulation=cfg["simulation"],
                gravity=cfg["gravity"], boundary_conditions=cfg["boundary_conditions"],
                diagnostics=cfg["diagnostics"], levelset_bodies=[])
            (HERE / f"refcase_{name}.json").write_text(json.dumps({**cfg, "particles": n}, indent=1) + "\n")
            print(name, n, "particles")
    finally:
        os.chdir(cwd)


if __name__ == "__main__":
    main()
