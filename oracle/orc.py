"""ctypes wrapper of the CPU oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The product
library never uses it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from exagoop_b200 import native as nt

ORACLE_DIR = Path(__file__).resolve().parent
LIB = ORACLE_DIR / "_build" / "liborc.so"
LIB_NATIVE = ORACLE_DIR / "_build" / "liborc_native.so"
REFPIN = ORACLE_DIR / "_ref" / "libexg_refpin.so"
_lib = None
_lib_path = None


def build(quiet: bool = True, target: str = "all", force: bool = False):
    cmd = ["make", "-C", str(ORACLE_DIR)] + (["-B"] if force else []) + [target]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def use_native() -> str:
    """Load the oracle built with -march=native for this host (the timed CPU
    baseline) instead of the portable x86-64-v2 build.  Builds it on first
    use; returns a description of the ISA, or of why the portable build is
    used.  Must run before the first lib() call."""
    global _lib_path
    if _lib is not None:
        return "x86-64-v2 (oracle already loaded)"
    try:
        # always rebuilt: a copy built on another host may target another ISA
        build(target="native", force=True)
        _lib_path = LIB_NATIVE
        return "-march=native"
    except Exception as e:  # no compiler on this host: the portable build
        return f"x86-64-v2 (native build failed: {str(e).splitlines()[0][:80]})"


def lib():
    global _lib
    if _lib is not None:
        return _lib
    path = _lib_path or LIB
    if not path.exists():
        build()
    L = C.CDLL(str(path))
    vp, i, d, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "orc_create": (vp, [C.POINTER(nt.Specs)]), "orc_destroy": (None, [vp]),
        "orc_set_threads": (None, [vp, i]),
        "orc_set_particles": (i, [vp, C.POINTER(nt.ParticleSoA)]),
        "orc_get_particles": (i, [vp, C.POINTER(nt.ParticleSoA)]),
        "orc_num_particles": (i64, [vp]), "orc_set_levelset": (i, [vp, i, pd]),
        "orc_get_nodes": (None, [vp, i, pd]), "orc_set_nodes": (None, [vp, i, pd]),
        "orc_init_internal_forces": (None, [vp]), "orc_redistribute": (i, [vp]),
        "orc_calculate_time_step": (d, [vp]), "orc_reset_nodaldata": (None, [vp]),
        "orc_p2g_momentum": (None, [vp, i, i, i]), "orc_backup_current_velocity": (None, [vp]),
        "orc_nodal_time_update_momentum": (None, [vp, d]), "orc_apply_nodal_bcs": (i, [vp, d, d]),
        "orc_g2p_momentum": (None, [vp, i, i, d]), "orc_update_mp_positions": (i, [vp, d]),
        "orc_update_mp_volume": (None, [vp]), "orc_calculate_mp_stress_strain": (None, [vp, d, d]),
        "orc_p2g_temperature": (None, [vp, i, i, i]), "orc_backup_current_temperature": (None, [vp]),
        "orc_nodal_time_update_temperature": (None, [vp, d]),
        "orc_apply_nodal_bcs_temperature": (None, [vp, d, d, i]),
        "orc_store_delta_temperature": (None, [vp]), "orc_g2p_temperature": (None, [vp, i, i]),
        "orc_step": (i, [vp, i]), "orc_get_time": (None, [vp, pd, pd, C.POINTER(i64)]),
        "orc_diagnostics": (None, [vp, C.POINTER(nt.Diag)]),
        "orc_sort_keys": (None, [vp, i, C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
        "orc_fn_spline": (d, [i, i, d]),
        "orc_fn_basis_and_grad": (d, [vp, pi, pi, pd, pd]),
        "orc_fn_interp_two": (None, [vp, i, pd, pi, pi, pi, i, i, pd]),
        "orc_fn_applybc": (i, [pd, pd, d, pd, i]),
        "orc_fn_linear_elastic": (None, [pd, pd, d, d]),
        "orc_fn_newtonian": (None, [pd, pd, d, d]),
        "orc_fn_neo_hookean": (None, [pd, pd, d, d]),
        "orc_fn_defgrad": (None, [pd, pd, d]),
        "orc_fn_levelset": (d, [vp, i, pd, pd]),
        "orc_fn_compute_bounds": (None, [i, i, i, i, i, pi, pi]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class Oracle:
    """The reference step restated on the CPU in FP64 (oracle/exg_oracle.cpp)."""

    def __init__(self, specs: nt.Specs, threads: int = 1):
        self.L = lib()
        self.specs = specs.copy()
        self.h = self.L.orc_create(C.byref(self.specs))
        self.L.orc_set_threads(self.h, threads)
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def upload(self, p: nt.Particles):
        s = p.soa()
        self.L.orc_set_particles(self.h, C.byref(s))
        self.n = p.n

    def download(self) -> nt.Particles:
        p = nt.Particles(self.n)
        s = p.soa()
        self.L.orc_get_particles(self.h, C.byref(s))
        return p

    def nodes(self, comp: int) -> np.ndarray:
        nn = [self.specs.ncells[d] + 1 for d in range(3)]
        out = np.zeros(nn[0] * nn[1] * nn[2])
        self.L.orc_get_nodes(self.h, comp, nt.dptr(out))
        return out

    def set_levelset(self, body: int, phi: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        self.L.orc_set_levelset(self.h, body, nt.dptr(phi))

    def __getattr__(self, name):
        # orc_<name> passthrough with the handle as the first argument
        f = getattr(self.L, "orc_" + name)
        return lambda *a: f(self.h, *a)

    def step(self, n: int = 1) -> int:
        return self.L.orc_step(self.h, n)

    def time(self):
        t, dt, n = C.c_double(), C.c_double(), C.c_int64()
        self.L.orc_get_time(self.h, C.byref(t), C.byref(dt), C.byref(n))
        return t.value, dt.value, n.value

    def diagnostics(self) -> dict:
        d = nt.Diag()
        self.L.orc_diagnostics(self.h, C.byref(d))
        return d.as_dict()

    def sort_keys(self, tile: int):
        keys = np.zeros(self.n, dtype=np.uint32)
        perm = np.zeros(self.n, dtype=np.int32)
        self.L.orc_sort_keys(self.h, tile, keys.ctypes.data_as(C.POINTER(C.c_uint32)),
                             perm.ctypes.data_as(C.POINTER(C.c_int32)))
        return keys, perm
