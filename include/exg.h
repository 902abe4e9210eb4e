/*
 * exg.h -- C ABI of the B200-native explicit MPM time step.
 *
 * This library replaces the per-step particle/grid path of the ExaGOOP MPM
 * solver (the L5 step functions declared in Source/utilities.H:28-79 and
 * called from Source/main.cpp:88-146).  Every entry point takes plain
 * pointers and sizes; no C++ or torch types cross this boundary.  All entry
 * points return an int status: EXG_OK (0) or a negative EXG_ERR_* code.  The
 * reference reports errors only through amrex::Abort (process exit); here the
 * same conditions come back as status codes and exg_last_error() gives the
 * message.
 *
 * Threading: one host thread per context; every device operation of a context
 * is issued on the context's own CUDA stream.  3-D only (AMREX_SPACEDIM == 3).
 */
#ifndef EXG_H_
#define EXG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define EXG_OK 0
#define EXG_ERR_CONFIG (-1)      /* bad inputs-file value (reference: amrex::Abort in read_mpm_specs) */
#define EXG_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define EXG_ERR_ALLOC (-3)       /* device or host allocation failed */
#define EXG_ERR_NAN (-4)         /* a non-finite value was produced */
#define EXG_ERR_DOMAIN (-5)      /* particles left a non-periodic domain and were dropped */
#define EXG_ERR_OVERFLOW (-6)    /* a fixed-size buffer (sort bucket, fixed-point range) overflowed */
#define EXG_ERR_TIMEOUT (-7)     /* a bounded device-side wait gave up */
#define EXG_ERR_ARG (-8)         /* invalid argument */
#define EXG_ERR_UNSUPPORTED (-9) /* feature outside this library's scope */
#define EXG_ERR_IO (-10)         /* file could not be read or written */
#define EXG_ERR_NOT_READY (-11)  /* call made before its prerequisite (e.g. no particles uploaded) */
#define EXG_ERR_BC (-12)         /* outflow wall BC reached applybc (reference: mpm_kernels.H:103-110 aborts) */

/* -------------------------------------------------------- particle fields */
/* Host particle layout: component-major SoA of doubles whose component index
 * is the reference's realData enum with USE_TEMP (Source/mpm_specs.H:17-61). */
#define EXG_NREAL 53
#define EXG_NINT 3
enum exg_real_field {
    EXG_R_RADIUS = 0,
    EXG_R_VEL = 1,        /* 3 components */
    EXG_R_VEL_PRIME = 4,  /* 3 */
    EXG_R_STRAINRATE = 7, /* 6, packed XX XY XZ YY YZ ZZ (constants.H:80-87) */
    EXG_R_STRAIN = 13,    /* 6 */
    EXG_R_STRESS = 19,    /* 6 */
    EXG_R_DEFGRAD = 25,   /* 9, row-major */
    EXG_R_VOLUME = 34,
    EXG_R_MASS = 35,
    EXG_R_DENSITY = 36,
    EXG_R_JACOBIAN = 37,
    EXG_R_PRESSURE = 38,
    EXG_R_VOL_INIT = 39,
    EXG_R_E = 40,
    EXG_R_NU = 41,
    EXG_R_BULK = 42,
    EXG_R_GAMMA = 43,
    EXG_R_VISC = 44,
    EXG_R_YACC = 45,
    EXG_R_TEMPERATURE = 46,
    EXG_R_SPHEAT = 47,
    EXG_R_THERMCOND = 48,
    EXG_R_HEATFLUX = 49, /* 3 */
    EXG_R_HEATSRC = 52
};
/* intData (Source/mpm_specs.H:63-73) */
enum exg_int_field { EXG_I_PHASE = 0, EXG_I_RIGID_ID = 1, EXG_I_MODEL = 2 };

typedef struct exg_particle_soa {
    int64_t np;      /* number of particles */
    double *pos;     /* [3][np]: x, y, z */
    double *rdata;   /* [EXG_NREAL][np] */
    int32_t *idata;  /* [EXG_NINT][np] */
} exg_particle_soa;

/* --------------------------------------------------------- nodal fields */
/* Nodal component indices of the reference with USE_TEMP (constants.H:30-64). */
enum exg_node_comp {
    EXG_N_MASS = 0,
    EXG_N_VEL = 1,  /* 3 */
    EXG_N_FRC = 4,  /* 3 */
    EXG_N_DVEL = 7, /* 3 */
    EXG_N_MASS_OLD = 10,
    EXG_N_MASS_SPHEAT = 20,
    EXG_N_MASS_SPHEAT_TEMP = 21,
    EXG_N_TEMPERATURE = 22,
    EXG_N_SOURCE_TEMP = 23,
    EXG_N_DELTA_TEMPERATURE = 24,
    EXG_N_MASS_COND = 25,
    EXG_N_NCOMP = 26
};

/* ------------------------------------------------------ boundary codes */
/* constants.H:89-99 */
enum exg_bc { EXG_BC_PERIODIC = 0, EXG_BC_NOSLIP = 1, EXG_BC_SLIP = 2, EXG_BC_PARTIALSLIP = 3, EXG_BC_OUTFLOW = 4 };
enum exg_bc_temp {
    EXG_BCT_PERIODIC = 0,
    EXG_BCT_ISOTHERMAL = 1,
    EXG_BCT_ADIABATIC = 2,
    EXG_BCT_USERFLUX = 3,
    EXG_BCT_CONVECTION = 4
};
enum exg_precision { EXG_PREC_FP64 = 0, EXG_PREC_MIXED = 1 };

#define EXG_MAX_BODIES 8 /* Source/mpm_eb.H:39 EXAGOOP_MAX_LS_BODIES */

/* User-defined functions loaded from shared libraries, same C signatures as
 * the reference (Source/mpm_specs.H:12-13, Source/mpm_udf_loader.H:81). */
typedef void (*exg_wallvel_udf)(double x, double y, double z, double t, double vel[3]);
typedef void (*exg_temp_udf)(double x, double y, double z, double t, double out[2]);
typedef double (*exg_levelset_udf)(double x, double y, double z);

typedef struct exg_body {
    int mom_bc;        /* EXG_BC_NOSLIP / SLIP / PARTIALSLIP (mpm_eb.H:63-73) */
    double wall_mu;
    double wall_vel[3];
    int temp_bc;       /* 0 adiabatic, 1 isothermal, 3 heatflux, 4 convective (mpm_eb.H:92-104) */
    double T_wall, heat_flux, h_conv, T_inf;
} exg_body;

/* Run specification: the fields of MPMspecs (Source/mpm_specs.H:75-221) that
 * the per-step path reads, after read_mpm_specs() and Initialise_Domain()'s
 * per-direction order fallback (Source/mpm_init.cpp:175-268). */
typedef struct exg_specs {
    double plo[3], phi[3];
    int ncells[3];
    int periodic[3];
    double gravity[3];
    int external_loads;
    double force_slab_lo[3], force_slab_hi[3], extforce[3];
    int fixed_timestep;
    double timestep;
    double dt_min_limit, dt_max_limit, cfl;
    double mass_tolerance, alpha_pic_flip;
    int order_scheme;  /* mpm.order_scheme: 1, 2 or 3 */
    int order[3];      /* order_scheme_directional */
    int stress_update_scheme; /* 0 USL, 1 MUSL */
    int calculate_strain_based_on_delta;
    double applied_strainrate, applied_strainrate_time;
    int bclo[3], bchi[3];
    double wall_mu_lo[3], wall_mu_hi[3];
    double wall_vel_lo[9], wall_vel_hi[9]; /* [face dir][component] */
    exg_wallvel_udf udf_wallvel_lo[3], udf_wallvel_hi[3];
    int use_temp;
    int bclo_temp[3], bchi_temp[3];
    double T_wall_lo[3], T_wall_hi[3], flux_lo[3], flux_hi[3], h_lo[3], h_hi[3], Tinf_lo[3], Tinf_hi[3];
    exg_temp_udf udf_temp_lo[3], udf_temp_hi[3];
    int num_bodies;
    exg_body bodies[EXG_MAX_BODIES];
    /* driver-level keys (main.cpp time loop) */
    int max_steps;
    double final_time;
    int num_redist;
    double write_output_time, screen_output_time, write_diag_output_time;
    int print_diagnostics, do_calculate_tke_tse, do_calculate_mwa_velcomp, do_calculate_mwa_velmag,
        do_calculate_minmaxpos;
    /* B200 execution keys (exg.* namespace, no counterpart in the reference) */
    int precision; /* EXG_PREC_FP64 or EXG_PREC_MIXED */
    int tile;      /* tile edge in cells: 0 = the default (8), else 4 or 8 */
    int autotune;  /* 1 (default): exg_step times the launch variants (exg_autotune) after its first step */
} exg_specs;

typedef struct exg_diag {
    double tke, tse;          /* mpm_diagnostics.cpp:23-72 */
    double mass;              /* sum of particle mass (all phases) */
    double momentum[3];       /* sum m v */
    double mwa_vel[3];        /* mass-weighted velocity components (:91-127) */
    double mwa_velmag;        /* (:145-178) */
    double minpos[3], maxpos[3]; /* (:192-216) */
    int64_t np;
} exg_diag;

/* ------------------------------------------------ inputs-file handling */
typedef struct exg_inputs exg_inputs;

/* Parse a ParmParse-style inputs file plus "key=value" overrides (the CLI of
 * the reference executable).  path may be NULL. */
int exg_inputs_parse(const char *path, int argc, const char *const *argv, exg_inputs **out);
/* Same, from an in-memory text. */
int exg_inputs_parse_text(const char *text, int argc, const char *const *argv, exg_inputs **out);
void exg_inputs_free(exg_inputs *in);
/* Raw value of a key (tokens joined by one space); EXG_ERR_ARG if absent. */
int exg_inputs_get(const exg_inputs *in, const char *key, char *buf, size_t buflen);
/* Fill specs from the inputs the way MPMspecs::read_mpm_specs
 * (Source/mpm_specs.H:223-565), init_eb (Source/mpm_eb.cpp:403-547) and
 * Initialise_Domain (Source/mpm_init.cpp:108-299) do.  err gets the message. */
int exg_specs_from_inputs(const exg_inputs *in, exg_specs *specs, char *err, size_t errlen);
void exg_specs_default(exg_specs *specs);
/* Nodal level set of body b on the (ncells+1)^3 node grid, from the eb2.* /
 * <body>.* keys (analytic sphere, plane, box, cylinder or udf_cpp).  The
 * reference builds these in mpm_ebtools::init_eb (Source/mpm_eb.cpp:100-388). */
int exg_levelset_build(const exg_inputs *in, const exg_specs *specs, int body, double *phi_nodes);

/* Analytic level-set shapes (the EB2 implicit functions of
 * build_analytic_levelset, Source/mpm_eb.cpp:150-388): exact signed distance,
 * negative inside the solid; inside = <geom>_has_fluid_inside flips the sign. */
enum exg_ls_kind { EXG_LS_SPHERE = 1, EXG_LS_PLANE = 2, EXG_LS_CYLINDER = 3, EXG_LS_BOX = 4 };
typedef struct exg_ls_shape {
    int kind;          /* exg_ls_kind */
    int inside;        /* fluid inside the shape */
    int dir;           /* cylinder axis 0..2 */
    double center[3];  /* sphere / cylinder centre, plane point */
    double normal[3];  /* plane normal, pointing into the fluid */
    double radius;     /* sphere, cylinder */
    double height;     /* cylinder */
    double lo[3], hi[3]; /* box */
} exg_ls_shape;
/* Shape of body b from its eb2.* / <body>.* keys; EXG_ERR_UNSUPPORTED for
 * udf_cpp and stl bodies, which have no analytic form. */
int exg_levelset_shape(const exg_inputs *in, int body, exg_ls_shape *shape);

/* ASCII particle file of InitParticles (Source/mpm_init.cpp:942-1167).
 * Arrays are allocated with malloc; release with exg_particles_free. */
int exg_particles_read_ascii(const char *path, int use_temp, exg_particle_soa *out);
int exg_particles_alloc(int64_t np, exg_particle_soa *out);
void exg_particles_free(exg_particle_soa *p);
/* The same arrays in page-locked host memory (cudaMallocHost): uploads and
 * downloads from them run at full PCIe speed.  Release with
 * exg_particles_free_pinned. */
int exg_particles_alloc_pinned(int64_t np, exg_particle_soa *out);
void exg_particles_free_pinned(exg_particle_soa *p);

/* ------------------------------------------------------------- context */
typedef struct exg_ctx exg_ctx;

/* Owns all device memory of one simulation on one GPU.  EXG_ERR_CONFIG for
 * specs the step cannot run: periodic axes of fewer than three tiles or not a
 * multiple of the tile edge, more than EXG_MAX_BODIES bodies, or a grid whose
 * tile-padded cell count reaches 2^32 - 1 (32-bit bin keys). */
int exg_ctx_create(const exg_specs *specs, int device, exg_ctx **out);
int exg_ctx_destroy(exg_ctx *ctx);
const char *exg_last_error(const exg_ctx *ctx);
/* Device-side status word accumulated by kernels since the last call. */
int exg_check_status(exg_ctx *ctx);
int exg_synchronize(exg_ctx *ctx);

/* Level set of body b, nodal (ncells+1)^3, x fastest (replaces the lsphi
 * MultiFab of LevelSetBody, Source/mpm_eb.H:45-117). */
int exg_set_levelset(exg_ctx *ctx, int body, const double *phi_nodes);
/* Level set of body b built on the GPU as the union (minimum) of nshapes
 * analytic shapes evaluated at every node: no host grid and no host-to-device
 * copy of it.  Bit-identical to exg_levelset_build for one shape. */
int exg_levelset_build_device(exg_ctx *ctx, int body, const exg_ls_shape *shapes, int nshapes);
/* Every body of the inputs, as mpm_ebtools::init_eb (Source/mpm_eb.cpp:
 * 402-547) builds them: analytic shapes on the GPU, udf_cpp bodies on the
 * host (the UDF is host code) and then uploaded. */
int exg_init_levelsets(exg_ctx *ctx, const exg_inputs *in);
/* Copy of body b's nodal level set to the host ((ncells+1)^3 doubles). */
int exg_get_levelset(exg_ctx *ctx, int body, double *phi_nodes);

/* Upload / download particles (host FP64 SoA).  Download returns particles in
 * upload order. */
int exg_particles_upload(exg_ctx *ctx, const exg_particle_soa *p);
int exg_particles_download(exg_ctx *ctx, exg_particle_soa *p);
int exg_num_particles(exg_ctx *ctx, int64_t *np);
/* Dense nodal component (reference component index) as (ncells+1)^3 doubles,
 * x fastest. */
int exg_nodes_download(exg_ctx *ctx, int comp, double *out);

/* --- step functions: one per reference L5 function (Source/utilities.H) --- */
/* Initialise_Internal_Forces (Source/mpm_init.cpp:368-445). */
int exg_init_internal_forces(exg_ctx *ctx);
/* Redistribute_Fill_Update (Source/utilities.cpp:420-434): cell-key sort,
 * periodic wrap and removal of particles outside a non-periodic domain. */
int exg_redistribute(exg_ctx *ctx);
/* MPMParticleContainer::Calculate_time_step (mpm_particle_timestep.cpp:38-111). */
int exg_calculate_time_step(exg_ctx *ctx, double *dt);
/* Reset_Nodaldata_to_Zero (nodal_data_ops.cpp:924-927). */
int exg_reset_nodaldata(exg_ctx *ctx);
/* P2G_Momentum (utilities.cpp:121-133 -> mpm_particle_grid_ops.cpp:333-628). */
int exg_p2g_momentum(exg_ctx *ctx, int update_mass, int update_vel, int update_forces);
/* backup_current_velocity (nodal_data_ops.cpp:57-81). */
int exg_backup_current_velocity(exg_ctx *ctx);
/* Nodal_Time_Update_Momentum (nodal_data_ops.cpp:451-482). */
int exg_nodal_time_update_momentum(exg_ctx *ctx, double dt);
/* Apply_Nodal_BCs (utilities.cpp:183-204): walls, UDF walls, level sets,
 * then store_delta_velocity. */
int exg_apply_nodal_bcs(exg_ctx *ctx, double dt, double time);
/* G2P_Momentum (utilities.cpp:259-269 -> mpm_particle_grid_ops.cpp:924-1098). */
int exg_g2p_momentum(exg_ctx *ctx, int update_vel, int update_strainrate, double dt);
/* Update_MP_Positions (utilities.cpp:315-334 -> mpm_particle_timestep.cpp:226-578). */
int exg_update_mp_positions(exg_ctx *ctx, double dt);
/* Update_MP_Volume (utilities.cpp:347-350 -> mpm_particle_timestep.cpp:131-182). */
int exg_update_mp_volume(exg_ctx *ctx);
/* Calculate_MP_Stress_Strain (utilities.cpp:372-400 -> mpm_particle_container.cpp:43-142). */
int exg_calculate_mp_stress_strain(exg_ctx *ctx, double time, double dt);
/* Thermal counterparts (main.cpp:99-106, 129-136); need specs.use_temp
 * (EXG_ERR_NOT_READY otherwise). */
/* P2G_Temperature (utilities.cpp:153-164 -> mpm_particle_grid_ops.cpp:656-884);
 * reset must be 1 (the only value the reference passes). */
int exg_p2g_temperature(exg_ctx *ctx, int reset, int update_temp, int update_source);
/* backup_current_temperature (nodal_data_ops.cpp:95-114). */
int exg_backup_current_temperature(exg_ctx *ctx);
/* Nodal_Time_Update_Temperature (nodal_data_ops.cpp:500-527). */
int exg_nodal_time_update_temperature(exg_ctx *ctx, double dt);
/* Apply_Nodal_BCs_Temperature (utilities.cpp:221-240): wall BCs, UDF wall
 * tables at `time`, level-set bodies (isothermal ones only when
 * dirichlet_only). */
int exg_apply_nodal_bcs_temperature(exg_ctx *ctx, double dt, double time, int dirichlet_only);
/* store_delta_temperature (nodal_data_ops.cpp:409-430). */
int exg_store_delta_temperature(exg_ctx *ctx);
/* G2P_Temperature (utilities.cpp:288-298 -> mpm_particle_grid_ops.cpp:1129-1270). */
int exg_g2p_temperature(exg_ctx *ctx, int update_temperature, int update_heatflux);

/* One or more complete explicit steps of main.cpp:83-171 (without output),
 * USL or MUSL, with temperature when specs.use_temp: a fixed launch sequence
 * (sort, P2G, nodal update + BCs, fused G2P/advection/stress) replayed from a
 * CUDA graph when the step has no host-side dependency (UDF wall tables are
 * re-tabulated on the host each step).  dt and time stay on the device. */
int exg_step(exg_ctx *ctx, int nsteps);
int exg_get_time(exg_ctx *ctx, double *time, double *last_dt, int64_t *steps);
int exg_set_time(exg_ctx *ctx, double time, int64_t steps);

/* ------------------------------------------------ batches of scenes
 * Many independent scenes, each with its own grid, particles and
 * parameters, advanced together: every hot kernel of a step (P2G, nodal
 * update, fused G2P) is ONE launch over the tiles of all scenes, taken from
 * a device counter; the per-scene sort and bookkeeping kernels run in the
 * same CUDA graph.  No counterpart in the reference, which runs one scene
 * per process.  All scenes share exg.precision, the B-spline order of every
 * axis and exg.tile, run the USL scheme, and use neither temperature nor
 * UDF wall tables (EXG_ERR_UNSUPPORTED otherwise). */
typedef struct exg_batch exg_batch;
int exg_batch_create(const exg_specs *specs, int nscenes, int device, exg_batch **out);
int exg_batch_destroy(exg_batch *batch);
/* Context of scene i, owned by the batch (never pass it to exg_ctx_destroy):
 * upload, download, exg_init_internal_forces, exg_diagnostics and
 * exg_get_time work on it as on any context. */
exg_ctx *exg_batch_scene(exg_batch *batch, int i);
int exg_batch_num_scenes(const exg_batch *batch);
/* nsteps explicit steps of every scene; each scene keeps its own dt and time. */
int exg_batch_step(exg_batch *batch, int nsteps);
const char *exg_batch_last_error(const exg_batch *batch);
/* Per-stage device timing of batch steps, as exg_set_stage_timing for a
 * context: while enabled, exg_batch_step runs without graph replay and
 * records CUDA events between its stages; exg_batch_last_step_timing
 * returns the mean ms per step since it was enabled: [sort and bookkeeping,
 * p2g, nodal, g2p, steps timed]. */
int exg_batch_set_stage_timing(exg_batch *batch, int on);
int exg_batch_last_step_timing(exg_batch *batch, double *ms5);

/* Deterministic device reductions of Do_All_Diagnostics (utilities.cpp:551-615). */
int exg_diagnostics(exg_ctx *ctx, exg_diag *out);

/* Cell keys and stable sort permutation of the current particle storage
 * order (exposed so the sort can be checked against a CPU stable sort). */
int exg_sort_keys(exg_ctx *ctx, uint32_t *keys, int32_t *perm);
/* Tile edge (cells) the context uses. */
int exg_tile_size(exg_ctx *ctx, int *tile);
/* Per-stage device timing: while enabled, exg_step runs without graph
 * replay and records CUDA events between its kernel stages.
 * exg_last_step_timing returns the mean ms per step since it was enabled:
 * [sort, p2g, nodal, g2p, steps timed]. */
int exg_set_stage_timing(exg_ctx *ctx, int on);
int exg_last_step_timing(exg_ctx *ctx, double *ms5);
/* The CUDA stream (cudaStream_t) the context issues all its work on. */
int exg_get_stream(exg_ctx *ctx, void **stream);

/* ------------------------------------------------ launch-variant autotuner
 * No counterpart in the reference, whose only tiling knob is
 * mpm.max_grid_size (the box size of its BoxArray, Source/mpm_init.cpp:
 * 154-155).  The P2G and the fused G2P kernels each come in EXG_NUM_VARIANTS
 * launch variants (P2G: rows of the stencil slice per pass and threads per
 * block; G2P: threads per block and resident blocks per SM).  Every variant
 * gives bit-identical results; only their speed differs with the GPU, the
 * B-spline order, the precision and the particle distribution.
 * exg_autotune times each variant on the context's current particles (a few
 * launches each, on the context's stream, outside any graph) and keeps the
 * fastest; choices are cached per (device, precision, order, tile, G2P
 * kind, particle-count decade) so later contexts of the same kind reuse them
 * without timing.  With specs.autotune = 1, exg_step calls it once the
 * particles are in the order a fused step leaves them (tile-major, as every
 * later step sees them): after the first step following an upload, which
 * runs with the current variants (a cached choice is applied at once).
 * It leaves the particle state and the step's control block as it found
 * them; nodal data is recomputed by the next step. */
#define EXG_NUM_VARIANTS 3
int exg_autotune(exg_ctx *ctx);
/* Select variants explicitly (0 .. EXG_NUM_VARIANTS-1; -1 keeps the current
 * one); disables the automatic tuning of the next exg_step. */
int exg_set_variants(exg_ctx *ctx, int p2g, int g2p);
/* Current variants and, after a tuning run, each variant's measured ms per
 * launch (arrays of EXG_NUM_VARIANTS; 0 where not measured; either pointer
 * may be NULL). */
int exg_get_variants(exg_ctx *ctx, int *p2g, int *g2p, double *p2g_ms, double *g2p_ms);

/* ------------------------------------------------ P2G without allocation */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running while another component captures a CUDA graph in global
 * capture mode (cudaMalloc is not permitted then), hosts that hand all
 * device memory to their own pool or enforce a fixed device-memory budget,
 * and real-time loops that forbid allocation after start-up.  It computes
 * what exg_p2g_momentum(ctx, 1, 1, 1) computes -- nodal mass, velocity (momentum
 * over mass, zero below mass_tolerance) and force, deterministically in
 * 64-bit fixed point -- without a context and without allocating: its
 * scratch is a static device array of EXG_NOALLOC_MAX_NODES nodes x 7
 * channels x 8 bytes plus one 32-bit count per cell (about 16 MB) that every GPU which loads the library
 * holds until the process exits.
 *   specs          host pointer; grids of more than EXG_NOALLOC_MAX_NODES
 *                  nodes ((ncells+1)^3) are rejected with EXG_ERR_OVERFLOW
 *                  and a message on stderr
 *   dev_particles  host struct whose pos/rdata/idata point to DEVICE arrays
 *                  in the exg_particle_soa layout
 *   node_mass      device, (ncells+1)^3 doubles, x fastest
 *   node_vel, node_frc  device, 3 x (ncells+1)^3 doubles (component-major)
 *   stream         cudaStream_t the work is issued on (NULL = legacy stream)
 * The first call on a device looks up the scratch array's device address and
 * loads the spline tables there; make that first call before any stream
 * capture begins.  All calls share the one array: the part of it a call uses
 * is cleared at the start of that call, and calls that overlap on the GPU
 * (different streams, no ordering between them) race on it.  A non-finite
 * mass, velocity, volume or stress among the phase-0 particles makes every
 * output value NaN (the call itself still returns EXG_OK: it does not wait
 * for the GPU). */
#define EXG_NOALLOC_MAX_NODES 262144
int exg_p2g_momentum_noalloc(const exg_specs *specs, const exg_particle_soa *dev_particles, double *node_mass,
                             double *node_vel, double *node_frc, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EXG_H_ */
