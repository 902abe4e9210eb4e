"""ctypes binding of libexg.so, the C ABI declared in include/exg.h.

The structures mirror the C layout field for field.  Loading fails loudly
when the shared library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libexg.so"

# status codes (include/exg.h)
EXG_OK = 0
ERRORS = {
    -1: "EXG_ERR_CONFIG", -2: "EXG_ERR_CUDA", -3: "EXG_ERR_ALLOC", -4: "EXG_ERR_NAN",
    -5: "EXG_ERR_DOMAIN", -6: "EXG_ERR_OVERFLOW", -7: "EXG_ERR_TIMEOUT", -8: "EXG_ERR_ARG",
    -9: "EXG_ERR_UNSUPPORTED", -10: "EXG_ERR_IO", -11: "EXG_ERR_NOT_READY", -12: "EXG_ERR_BC",
}
EXG_NREAL = 53
EXG_NINT = 3
EXG_N_NCOMP = 26
EXG_MAX_BODIES = 8
EXG_NOALLOC_MAX_NODES = 262144
PREC_FP64, PREC_MIXED = 0, 1

# realData (Source/mpm_specs.H:17-61) and intData indices
R_RADIUS, R_VEL, R_VEL_PRIME, R_STRAINRATE, R_STRAIN, R_STRESS, R_DEFGRAD = 0, 1, 4, 7, 13, 19, 25
R_VOLUME, R_MASS, R_DENSITY, R_JACOBIAN, R_PRESSURE, R_VOL_INIT = 34, 35, 36, 37, 38, 39
R_E, R_NU, R_BULK, R_GAMMA, R_VISC, R_YACC = 40, 41, 42, 43, 44, 45
R_TEMPERATURE, R_SPHEAT, R_THERMCOND, R_HEATFLUX, R_HEATSRC = 46, 47, 48, 49, 52
I_PHASE, I_RIGID_ID, I_MODEL = 0, 1, 2
# nodal components (constants.H:30-64)
N_MASS, N_VEL, N_FRC, N_DVEL, N_MASS_OLD = 0, 1, 4, 7, 10
N_MASS_SPHEAT, N_MASS_SPHEAT_TEMP, N_TEMPERATURE, N_SOURCE_TEMP, N_DELTA_TEMPERATURE, N_MASS_COND = 20, 21, 22, 23, 24, 25
# thermal wall BC codes (mpm_specs.H bc_temp_*)
BCT_PERIODIC, BCT_ISOTHERMAL, BCT_ADIABATIC, BCT_USERFLUX, BCT_CONVECTION = 0, 1, 2, 3, 4
BC_PERIODIC, BC_NOSLIP, BC_SLIP, BC_PARTIALSLIP, BC_OUTFLOW = 0, 1, 2, 3, 4


class ExgError(RuntimeError):
    """A non-zero status returned through the C ABI."""

    def __init__(self, code: int, where: str, msg: str = ""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} {msg}".strip())


D3 = C.c_double * 3
I3 = C.c_int * 3


class Body(C.Structure):
    _fields_ = [("mom_bc", C.c_int), ("wall_mu", C.c_double), ("wall_vel", D3), ("temp_bc", C.c_int),
                ("T_wall", C.c_double), ("heat_flux", C.c_double), ("h_conv", C.c_double), ("T_inf", C.c_double)]


class Specs(C.Structure):
    _fields_ = [
        ("plo", D3), ("phi", D3), ("ncells", I3), ("periodic", I3), ("gravity", D3),
        ("external_loads", C.c_int), ("force_slab_lo", D3), ("force_slab_hi", D3), ("extforce", D3),
        ("fixed_timestep", C.c_int), ("timestep", C.c_double),
        ("dt_min_limit", C.c_double), ("dt_max_limit", C.c_double), ("cfl", C.c_double),
        ("mass_tolerance", C.c_double), ("alpha_pic_flip", C.c_double),
        ("order_scheme", C.c_int), ("order", I3), ("stress_update_scheme", C.c_int),
        ("calculate_strain_based_on_delta", C.c_int),
        ("applied_strainrate", C.c_double), ("applied_strainrate_time", C.c_double),
        ("bclo", I3), ("bchi", I3), ("wall_mu_lo", D3), ("wall_mu_hi", D3),
        ("wall_vel_lo", C.c_double * 9), ("wall_vel_hi", C.c_double * 9),
        ("udf_wallvel_lo", C.c_void_p * 3), ("udf_wallvel_hi", C.c_void_p * 3),
        ("use_temp", C.c_int), ("bclo_temp", I3), ("bchi_temp", I3),
        ("T_wall_lo", D3), ("T_wall_hi", D3), ("flux_lo", D3), ("flux_hi", D3),
        ("h_lo", D3), ("h_hi", D3), ("Tinf_lo", D3), ("Tinf_hi", D3),
        ("udf_temp_lo", C.c_void_p * 3), ("udf_temp_hi", C.c_void_p * 3),
        ("num_bodies", C.c_int), ("bodies", Body * EXG_MAX_BODIES),
        ("max_steps", C.c_int), ("final_time", C.c_double), ("num_redist", C.c_int),
        ("write_output_time", C.c_double), ("screen_output_time", C.c_double),
        ("write_diag_output_time", C.c_double),
        ("print_diagnostics", C.c_int), ("do_calculate_tke_tse", C.c_int), ("do_calculate_mwa_velcomp", C.c_int),
        ("do_calculate_mwa_velmag", C.c_int), ("do_calculate_minmaxpos", C.c_int),
        ("precision", C.c_int), ("tile", C.c_int), ("autotune", C.c_int),
    ]

    def copy(self) -> "Specs":
        s = Specs()
        C.pointer(s)[0] = self
        return s


class ParticleSoA(C.Structure):
    _fields_ = [("np", C.c_int64), ("pos", C.POINTER(C.c_double)), ("rdata", C.POINTER(C.c_double)),
                ("idata", C.POINTER(C.c_int32))]


class Diag(C.Structure):
    _fields_ = [("tke", C.c_double), ("tse", C.c_double), ("mass", C.c_double), ("momentum", D3),
                ("mwa_vel", D3), ("mwa_velmag", C.c_double), ("minpos", D3), ("maxpos", D3), ("np", C.c_int64)]

    def as_dict(self) -> dict:
        return {"tke": self.tke, "tse": self.tse, "mass": self.mass, "momentum": list(self.momentum),
                "mwa_vel": list(self.mwa_vel), "mwa_velmag": self.mwa_velmag,
                "minpos": list(self.minpos), "maxpos": list(self.maxpos), "np": int(self.np)}


LS_SPHERE, LS_PLANE, LS_CYLINDER, LS_BOX = 1, 2, 3, 4


class LsShape(C.Structure):
    """exg_ls_shape: one analytic level-set shape (sphere, plane, cylinder,
    box), negative inside the solid."""
    _fields_ = [("kind", C.c_int), ("inside", C.c_int), ("dir", C.c_int), ("center", D3), ("normal", D3),
                ("radius", C.c_double), ("height", C.c_double), ("lo", D3), ("hi", D3)]

    @classmethod
    def sphere(cls, center, radius, inside=False):
        return cls(kind=LS_SPHERE, inside=int(inside), center=D3(*center), radius=radius)

    @classmethod
    def plane(cls, point, normal, inside=False):
        return cls(kind=LS_PLANE, inside=int(inside), center=D3(*point), normal=D3(*normal))

    @classmethod
    def cylinder(cls, center, radius, height, direction=2, inside=False):
        return cls(kind=LS_CYLINDER, inside=int(inside), center=D3(*center), radius=radius, height=height,
                   dir=direction)

    @classmethod
    def box(cls, lo, hi, inside=False):
        return cls(kind=LS_BOX, inside=int(inside), lo=D3(*lo), hi=D3(*hi))


# every symbol include/exg.h declares
EXPORTED = [
    "exg_inputs_parse", "exg_inputs_parse_text", "exg_inputs_free", "exg_inputs_get", "exg_specs_from_inputs",
    "exg_specs_default", "exg_levelset_build", "exg_particles_read_ascii", "exg_particles_alloc",
    "exg_particles_free", "exg_ctx_create", "exg_ctx_destroy", "exg_last_error", "exg_check_status",
    "exg_synchronize", "exg_set_levelset", "exg_particles_upload", "exg_particles_download",
    "exg_num_particles", "exg_nodes_download", "exg_init_internal_forces", "exg_redistribute",
    "exg_calculate_time_step", "exg_reset_nodaldata", "exg_p2g_momentum", "exg_backup_current_velocity",
    "exg_nodal_time_update_momentum", "exg_apply_nodal_bcs", "exg_g2p_momentum", "exg_update_mp_positions",
    "exg_update_mp_volume", "exg_calculate_mp_stress_strain", "exg_p2g_temperature",
    "exg_backup_current_temperature", "exg_nodal_time_update_temperature", "exg_apply_nodal_bcs_temperature",
    "exg_store_delta_temperature", "exg_g2p_temperature", "exg_step", "exg_get_time", "exg_set_time",
    "exg_diagnostics", "exg_sort_keys", "exg_tile_size", "exg_set_stage_timing", "exg_last_step_timing",
    "exg_get_stream", "exg_p2g_momentum_noalloc", "exg_batch_create", "exg_batch_destroy", "exg_batch_scene",
    "exg_batch_num_scenes", "exg_batch_step", "exg_batch_last_error", "exg_particles_alloc_pinned",
    "exg_particles_free_pinned", "exg_levelset_shape", "exg_levelset_build_device", "exg_init_levelsets",
    "exg_get_levelset", "exg_autotune", "exg_set_variants", "exg_get_variants", "exg_batch_set_stage_timing",
    "exg_batch_last_step_timing",
]

_lib = None


def lib() -> C.CDLL:
    """Load libexg.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = C.CDLL(str(LIB_PATH))
    vp, i, d, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    pd, pi32 = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    sig = {
        "exg_inputs_parse": (i, [C.c_char_p, i, C.POINTER(C.c_char_p), C.POINTER(vp)]),
        "exg_inputs_parse_text": (i, [C.c_char_p, i, C.POINTER(C.c_char_p), C.POINTER(vp)]),
        "exg_inputs_free": (None, [vp]),
        "exg_inputs_get": (i, [vp, C.c_char_p, C.c_char_p, C.c_size_t]),
        "exg_specs_from_inputs": (i, [vp, C.POINTER(Specs), C.c_char_p, C.c_size_t]),
        "exg_specs_default": (None, [C.POINTER(Specs)]),
        "exg_levelset_build": (i, [vp, C.POINTER(Specs), i, pd]),
        "exg_levelset_shape": (i, [vp, i, C.POINTER(LsShape)]),
        "exg_levelset_build_device": (i, [vp, i, C.POINTER(LsShape), i]),
        "exg_init_levelsets": (i, [vp, vp]),
        "exg_get_levelset": (i, [vp, i, pd]),
        "exg_particles_read_ascii": (i, [C.c_char_p, i, C.POINTER(ParticleSoA)]),
        "exg_particles_alloc": (i, [i64, C.POINTER(ParticleSoA)]),
        "exg_particles_free": (None, [C.POINTER(ParticleSoA)]),
        "exg_particles_alloc_pinned": (i, [i64, C.POINTER(ParticleSoA)]),
        "exg_particles_free_pinned": (None, [C.POINTER(ParticleSoA)]),
        "exg_ctx_create": (i, [C.POINTER(Specs), i, C.POINTER(vp)]),
        "exg_ctx_destroy": (i, [vp]),
        "exg_last_error": (C.c_char_p, [vp]),
        "exg_check_status": (i, [vp]),
        "exg_synchronize": (i, [vp]),
        "exg_set_levelset": (i, [vp, i, pd]),
        "exg_particles_upload": (i, [vp, C.POINTER(ParticleSoA)]),
        "exg_particles_download": (i, [vp, C.POINTER(ParticleSoA)]),
        "exg_num_particles": (i, [vp, C.POINTER(i64)]),
        "exg_nodes_download": (i, [vp, i, pd]),
        "exg_init_internal_forces": (i, [vp]),
        "exg_redistribute": (i, [vp]),
        "exg_calculate_time_step": (i, [vp, pd]),
        "exg_reset_nodaldata": (i, [vp]),
        "exg_p2g_momentum": (i, [vp, i, i, i]),
        "exg_backup_current_velocity": (i, [vp]),
        "exg_nodal_time_update_momentum": (i, [vp, d]),
        "exg_apply_nodal_bcs": (i, [vp, d, d]),
        "exg_g2p_momentum": (i, [vp, i, i, d]),
        "exg_update_mp_positions": (i, [vp, d]),
        "exg_update_mp_volume": (i, [vp]),
        "exg_calculate_mp_stress_strain": (i, [vp, d, d]),
        "exg_p2g_temperature": (i, [vp, i, i, i]),
        "exg_backup_current_temperature": (i, [vp]),
        "exg_nodal_time_update_temperature": (i, [vp, d]),
        "exg_apply_nodal_bcs_temperature": (i, [vp, d, d, i]),
        "exg_store_delta_temperature": (i, [vp]),
        "exg_g2p_temperature": (i, [vp, i, i]),
        "exg_step": (i, [vp, i]),
        "exg_get_time": (i, [vp, pd, pd, C.POINTER(i64)]),
        "exg_set_time": (i, [vp, d, i64]),
        "exg_diagnostics": (i, [vp, C.POINTER(Diag)]),
        "exg_sort_keys": (i, [vp, C.POINTER(C.c_uint32), pi32]),
        "exg_tile_size": (i, [vp, C.POINTER(i)]),
        "exg_set_stage_timing": (i, [vp, i]),
        "exg_last_step_timing": (i, [vp, pd]),
        "exg_get_stream": (i, [vp, C.POINTER(vp)]),
        "exg_p2g_momentum_noalloc": (i, [C.POINTER(Specs), C.POINTER(ParticleSoA), pd, pd, pd, vp]),
        "exg_batch_create": (i, [C.POINTER(Specs), i, i, C.POINTER(vp)]),
        "exg_batch_destroy": (i, [vp]),
        "exg_batch_scene": (vp, [vp, i]),
        "exg_batch_num_scenes": (i, [vp]),
        "exg_batch_step": (i, [vp, i]),
        "exg_batch_last_error": (C.c_char_p, [vp]),
        "exg_autotune": (i, [vp]),
        "exg_batch_set_stage_timing": (i, [vp, i]),
        "exg_batch_last_step_timing": (i, [vp, pd]),
        "exg_set_variants": (i, [vp, i, i]),
        "exg_get_variants": (i, [vp, C.POINTER(i), C.POINTER(i), pd, pd]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Particles:
    """Host particle set in the reference's field layout (FP64 SoA).  With
    pinned=True the arrays live in page-locked memory from
    exg_particles_alloc_pinned (full-speed host transfers; needs a GPU)."""

    def __init__(self, np_: int, pinned: bool = False):
        self._soa = None
        if pinned:
            s = ParticleSoA()
            rc = lib().exg_particles_alloc_pinned(np_, C.byref(s))
            if rc:
                raise ExgError(rc, "exg_particles_alloc_pinned")
            self._soa = s
            self.pos = np.ctypeslib.as_array(s.pos, shape=(3 * max(np_, 1),))[:3 * np_].reshape(3, np_)
            self.rdata = np.ctypeslib.as_array(s.rdata, shape=(EXG_NREAL * max(np_, 1),))[:EXG_NREAL * np_].reshape(
                EXG_NREAL, np_)
            self.idata = np.ctypeslib.as_array(s.idata, shape=(EXG_NINT * max(np_, 1),))[:EXG_NINT * np_].reshape(
                EXG_NINT, np_)
            return
        self.pos = np.zeros((3, np_), dtype=np.float64)
        self.rdata = np.zeros((EXG_NREAL, np_), dtype=np.float64)
        self.idata = np.zeros((EXG_NINT, np_), dtype=np.int32)

    def __del__(self):
        if getattr(self, "_soa", None) is not None:
            try:
                lib().exg_particles_free_pinned(C.byref(self._soa))
            except Exception:
                pass
            self._soa = None

    def view(self, n: int) -> "Particles":
        """A set of n particles laid out (component-major) at the start of
        this page-locked set's memory: a staging area for smaller sets.  It
        shares the memory and frees nothing; keep this set alive while it is
        used."""
        if self._soa is None or not 0 < n <= self.n:
            raise ValueError("view needs a pinned set of at least n particles")
        v = Particles.__new__(Particles)
        v._soa = None
        v._parent = self
        s = self._soa
        v.pos = np.ctypeslib.as_array(s.pos, shape=(3 * n,)).reshape(3, n)
        v.rdata = np.ctypeslib.as_array(s.rdata, shape=(EXG_NREAL * n,)).reshape(EXG_NREAL, n)
        v.idata = np.ctypeslib.as_array(s.idata, shape=(EXG_NINT * n,)).reshape(EXG_NINT, n)
        return v

    def pinned_copy(self) -> "Particles":
        p = Particles(self.n, pinned=True)
        p.pos[:] = self.pos
        p.rdata[:] = self.rdata
        p.idata[:] = self.idata
        return p

    @property
    def n(self) -> int:
        return self.pos.shape[1]

    def soa(self) -> ParticleSoA:
        for a in (self.pos, self.rdata, self.idata):
            assert a.flags.c_contiguous
        return ParticleSoA(self.n, dptr(self.pos), dptr(self.rdata),
                           self.idata.ctypes.data_as(C.POINTER(C.c_int32)))

    def copy(self) -> "Particles":
        p = Particles(self.n)
        p.pos[:] = self.pos
        p.rdata[:] = self.rdata
        p.idata[:] = self.idata
        return p

    def field(self, start: int, ncomp: int = 1) -> np.ndarray:
        return self.rdata[start:start + ncomp]

    @staticmethod
    def read_ascii(path: str, use_temp: bool = False) -> "Particles":
        L = lib()
        s = ParticleSoA()
        rc = L.exg_particles_read_ascii(str(path).encode(), int(use_temp), C.byref(s))
        if rc:
            raise ExgError(rc, "exg_particles_read_ascii", str(path))
        n = s.np
        p = Particles(n)
        p.pos[:] = np.ctypeslib.as_array(s.pos, shape=(3 * n,)).reshape(3, n)
        p.rdata[:] = np.ctypeslib.as_array(s.rdata, shape=(EXG_NREAL * n,)).reshape(EXG_NREAL, n)
        p.idata[:] = np.ctypeslib.as_array(s.idata, shape=(EXG_NINT * n,)).reshape(EXG_NINT, n)
        L.exg_particles_free(C.byref(s))
        return p


def default_specs() -> Specs:
    """exg_specs_default through the C ABI (read_mpm_specs defaults)."""
    s = Specs()
    lib().exg_specs_default(C.byref(s))
    return s


def specs_defaults() -> Specs:
    """The same defaults as exg_specs_default, set in Python without loading
    libexg.so (the CPU-only legs of the benchmark use it, so that timing the
    CPU oracle never maps the GPU library): gravity (0, -9.81, 0)
    (mpm_specs.H:83), num_redist 10, max_steps 1, output times 1e200, order 1
    on every axis, dt limits [1e-12, 1], CFL 0.1, mass_tolerance 1e-8, FLIP
    0.95, USL, slip walls with friction 0.1, adiabatic thermal walls, FP64,
    tile 0 (the library's default), launch-variant autotuning on."""
    s = Specs()  # ctypes zero-fills every field, as the C memset does
    s.gravity[1] = -9.81
    s.num_redist = 10
    s.max_steps = 1
    s.write_output_time = 1e200
    s.write_diag_output_time = 1e200
    s.order_scheme = 1
    for d in range(3):
        s.order[d] = 1
        s.bclo[d] = s.bchi[d] = BC_SLIP
        s.wall_mu_lo[d] = s.wall_mu_hi[d] = 0.1
        s.bclo_temp[d] = s.bchi_temp[d] = BCT_ADIABATIC
    s.dt_max_limit = 1e0
    s.dt_min_limit = 1e-12
    s.cfl = 0.1
    s.mass_tolerance = 1e-8
    s.alpha_pic_flip = 0.95
    s.stress_update_scheme = 0
    s.precision = PREC_FP64
    s.tile = 0
    s.autotune = 1
    return s


class Inputs:
    """A parsed ParmParse-style inputs file plus key=value overrides."""

    def __init__(self, path: str | None = None, text: str | None = None, overrides=()):
        L = lib()
        argv = (C.c_char_p * max(1, len(overrides)))(*[o.encode() for o in overrides])
        h = C.c_void_p()
        if text is not None:
            rc = L.exg_inputs_parse_text(text.encode(), len(overrides), argv, C.byref(h))
        else:
            rc = L.exg_inputs_parse(path.encode() if path else None, len(overrides), argv, C.byref(h))
        if rc:
            raise ExgError(rc, "exg_inputs_parse", str(path))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib().exg_inputs_free(self.h)
            self.h = None

    def get(self, key: str) -> str | None:
        buf = C.create_string_buffer(4096)
        rc = lib().exg_inputs_get(self.h, key.encode(), buf, 4096)
        return None if rc < 0 else buf.value.decode()

    def specs(self) -> Specs:
        s = Specs()
        err = C.create_string_buffer(512)
        rc = lib().exg_specs_from_inputs(self.h, C.byref(s), err, 512)
        if rc:
            raise ExgError(rc, "exg_specs_from_inputs", err.value.decode())
        return s

    def levelset(self, specs: Specs, body: int) -> np.ndarray:
        nn = [specs.ncells[d] + 1 for d in range(3)]
        phi = np.zeros(nn[0] * nn[1] * nn[2], dtype=np.float64)
        rc = lib().exg_levelset_build(self.h, C.byref(specs), body, dptr(phi))
        if rc:
            raise ExgError(rc, "exg_levelset_build")
        return phi

    def levelset_shape(self, body: int) -> LsShape:
        """Analytic shape of body b (ExgError EXG_ERR_UNSUPPORTED for udf_cpp)."""
        sh = LsShape()
        rc = lib().exg_levelset_shape(self.h, body, C.byref(sh))
        if rc:
            raise ExgError(rc, "exg_levelset_shape")
        return sh


class Context:
    """One simulation on one GPU (exg_ctx).  Method names follow the
    reference's L5 step functions (Source/utilities.H:28-79)."""

    def __init__(self, specs: Specs, device: int = 0):
        self.L = lib()
        self.specs = specs.copy()
        self.h = C.c_void_p()
        rc = self.L.exg_ctx_create(C.byref(self.specs), device, C.byref(self.h))
        if rc:
            raise ExgError(rc, "exg_ctx_create")
        self.n = 0

    def close(self):
        if self.h:
            self.L.exg_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, where: str):
        if rc:
            raise ExgError(rc, where, self.L.exg_last_error(self.h).decode(errors="replace"))

    # --- data
    def upload(self, p: Particles):
        self._keep = p.soa()
        self._ck(self.L.exg_particles_upload(self.h, C.byref(self._keep)), "exg_particles_upload")
        self.n = p.n

    def download(self) -> Particles:
        p = Particles(self.n)
        self.download_into(p)
        return p

    def download_into(self, p: Particles):
        """Download into an existing set of this context's size (pinned or not)."""
        s = p.soa()
        self._ck(self.L.exg_particles_download(self.h, C.byref(s)), "exg_particles_download")

    def nodes(self, comp: int) -> np.ndarray:
        nn = [self.specs.ncells[d] + 1 for d in range(3)]
        out = np.zeros(nn[0] * nn[1] * nn[2], dtype=np.float64)
        self._ck(self.L.exg_nodes_download(self.h, comp, dptr(out)), "exg_nodes_download")
        return out

    def set_levelset(self, body: int, phi: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        self._ck(self.L.exg_set_levelset(self.h, body, dptr(phi)), "exg_set_levelset")

    def build_levelset(self, body: int, shapes):
        """Level set of body b as the union of analytic shapes, built on the GPU."""
        shapes = [shapes] if isinstance(shapes, LsShape) else list(shapes)
        arr = (LsShape * len(shapes))(*shapes)
        self._ck(self.L.exg_levelset_build_device(self.h, body, arr, len(shapes)), "exg_levelset_build_device")

    def init_levelsets(self, inputs: "Inputs"):
        """Every body of an inputs file (init_eb): analytic ones on the GPU."""
        self._ck(self.L.exg_init_levelsets(self.h, inputs.h), "exg_init_levelsets")

    def get_levelset(self, body: int) -> np.ndarray:
        nn = [self.specs.ncells[d] + 1 for d in range(3)]
        phi = np.empty(nn[0] * nn[1] * nn[2], dtype=np.float64)
        self._ck(self.L.exg_get_levelset(self.h, body, dptr(phi)), "exg_get_levelset")
        return phi

    # --- L5 step functions
    def Initialise_Internal_Forces(self):
        self._ck(self.L.exg_init_internal_forces(self.h), "exg_init_internal_forces")

    def Redistribute(self):
        self._ck(self.L.exg_redistribute(self.h), "exg_redistribute")

    def Calculate_time_step(self) -> float:
        dt = C.c_double()
        self._ck(self.L.exg_calculate_time_step(self.h, C.byref(dt)), "exg_calculate_time_step")
        return dt.value

    def Reset_Nodaldata_to_Zero(self):
        self._ck(self.L.exg_reset_nodaldata(self.h), "exg_reset_nodaldata")

    def P2G_Momentum(self, update_mass=1, update_vel=1, update_forces=1):
        self._ck(self.L.exg_p2g_momentum(self.h, update_mass, update_vel, update_forces), "exg_p2g_momentum")

    def backup_current_velocity(self):
        self._ck(self.L.exg_backup_current_velocity(self.h), "exg_backup_current_velocity")

    def Nodal_Time_Update_Momentum(self, dt: float):
        self._ck(self.L.exg_nodal_time_update_momentum(self.h, dt), "exg_nodal_time_update_momentum")

    def Apply_Nodal_BCs(self, dt: float, time: float):
        self._ck(self.L.exg_apply_nodal_bcs(self.h, dt, time), "exg_apply_nodal_bcs")

    def G2P_Momentum(self, update_vel: int, update_strainrate: int, dt: float):
        self._ck(self.L.exg_g2p_momentum(self.h, update_vel, update_strainrate, dt), "exg_g2p_momentum")

    def Update_MP_Positions(self, dt: float):
        self._ck(self.L.exg_update_mp_positions(self.h, dt), "exg_update_mp_positions")

    def Update_MP_Volume(self):
        self._ck(self.L.exg_update_mp_volume(self.h), "exg_update_mp_volume")

    def Calculate_MP_Stress_Strain(self, time: float, dt: float):
        self._ck(self.L.exg_calculate_mp_stress_strain(self.h, time, dt), "exg_calculate_mp_stress_strain")

    # --- thermal step functions (Source/utilities.H, USE_TEMP)
    def P2G_Temperature(self, reset=1, update_temp=1, update_source=1):
        self._ck(self.L.exg_p2g_temperature(self.h, reset, update_temp, update_source), "exg_p2g_temperature")

    def backup_current_temperature(self):
        self._ck(self.L.exg_backup_current_temperature(self.h), "exg_backup_current_temperature")

    def Nodal_Time_Update_Temperature(self, dt: float):
        self._ck(self.L.exg_nodal_time_update_temperature(self.h, dt), "exg_nodal_time_update_temperature")

    def Apply_Nodal_BCs_Temperature(self, dt: float, time: float, dirichlet_only: int = 0):
        self._ck(self.L.exg_apply_nodal_bcs_temperature(self.h, dt, time, dirichlet_only),
                 "exg_apply_nodal_bcs_temperature")

    def store_delta_temperature(self):
        self._ck(self.L.exg_store_delta_temperature(self.h), "exg_store_delta_temperature")

    def G2P_Temperature(self, update_temperature: int, update_heatflux: int):
        self._ck(self.L.exg_g2p_temperature(self.h, update_temperature, update_heatflux), "exg_g2p_temperature")

    # --- fused path
    def step(self, nsteps: int = 1):
        self._ck(self.L.exg_step(self.h, nsteps), "exg_step")

    def time(self):
        t, dt, n = C.c_double(), C.c_double(), C.c_int64()
        self._ck(self.L.exg_get_time(self.h, C.byref(t), C.byref(dt), C.byref(n)), "exg_get_time")
        return t.value, dt.value, n.value

    def set_time(self, t: float, nsteps: int = 0):
        self._ck(self.L.exg_set_time(self.h, float(t), int(nsteps)), "exg_set_time")

    def diagnostics(self) -> dict:
        d = Diag()
        self._ck(self.L.exg_diagnostics(self.h, C.byref(d)), "exg_diagnostics")
        return d.as_dict()

    def sort_keys(self):
        keys = np.zeros(self.n, dtype=np.uint32)
        perm = np.zeros(self.n, dtype=np.int32)
        self._ck(self.L.exg_sort_keys(self.h, keys.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      perm.ctypes.data_as(C.POINTER(C.c_int32))), "exg_sort_keys")
        return keys, perm

    def autotune(self):
        """exg_autotune: time the launch variants on the current particles."""
        self._ck(self.L.exg_autotune(self.h), "exg_autotune")

    def set_variants(self, p2g: int = -1, g2p: int = -1):
        self._ck(self.L.exg_set_variants(self.h, p2g, g2p), "exg_set_variants")

    def variants(self) -> dict:
        p, g = C.c_int(), C.c_int()
        pm, gm = (C.c_double * 3)(), (C.c_double * 3)()
        self._ck(self.L.exg_get_variants(self.h, C.byref(p), C.byref(g), pm, gm), "exg_get_variants")
        return {"p2g": p.value, "g2p": g.value, "p2g_ms": list(pm), "g2p_ms": list(gm)}

    def tile(self) -> int:
        t = C.c_int()
        self._ck(self.L.exg_tile_size(self.h, C.byref(t)), "exg_tile_size")
        return t.value

    def stage_timing(self, on: bool):
        self._ck(self.L.exg_set_stage_timing(self.h, int(on)), "exg_set_stage_timing")

    def last_step_timing(self):
        out = np.zeros(5)
        self._ck(self.L.exg_last_step_timing(self.h, dptr(out)), "exg_last_step_timing")
        return out

    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(self.L.exg_get_stream(self.h, C.byref(s)), "exg_get_stream")
        return s.value or 0

    def synchronize(self):
        self._ck(self.L.exg_synchronize(self.h), "exg_synchronize")


class _SceneContext(Context):
    """Context of one scene of a Batch (owned by the batch)."""

    def __init__(self, batch: "Batch", handle: int, specs: Specs):
        self.L = lib()
        self.specs = specs.copy()
        self.h = C.c_void_p(handle)
        self.n = 0
        self._batch = batch

    def close(self):
        self.h = C.c_void_p()  # the batch destroys it


class Batch:
    """Independent scenes advanced together, one launch per hot kernel
    (exg_batch in include/exg.h)."""

    def __init__(self, specs: list, device: int = 0):
        self.L = lib()
        arr = (Specs * len(specs))(*[s.copy() for s in specs])
        self.h = C.c_void_p()
        rc = self.L.exg_batch_create(arr, len(specs), device, C.byref(self.h))
        if rc:
            raise ExgError(rc, "exg_batch_create")
        self.scenes = [_SceneContext(self, self.L.exg_batch_scene(self.h, i), specs[i]) for i in range(len(specs))]

    def stream(self) -> int:
        """The CUDA stream every scene of the batch enqueues on."""
        return self.scenes[0].stream()

    def synchronize(self):
        self.scenes[0].synchronize()

    def step(self, nsteps: int = 1):
        rc = self.L.exg_batch_step(self.h, nsteps)
        if rc:
            raise ExgError(rc, "exg_batch_step", self.L.exg_batch_last_error(self.h).decode(errors="replace"))

    def stage_timing(self, on: bool):
        rc = self.L.exg_batch_set_stage_timing(self.h, int(on))
        if rc:
            raise ExgError(rc, "exg_batch_set_stage_timing")

    def last_step_timing(self):
        """Mean ms per timed step: [sort + bookkeeping, p2g, nodal, g2p, steps]."""
        out = (C.c_double * 5)()
        rc = self.L.exg_batch_last_step_timing(self.h, out)
        if rc:
            raise ExgError(rc, "exg_batch_last_step_timing")
        return list(out)

    def close(self):
        if self.h:
            for sc in self.scenes:
                sc.h = C.c_void_p()
            self.L.exg_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
