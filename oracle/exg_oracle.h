/*
 * exg_oracle.h -- CPU FP64 oracle of the ExaGOOP per-step MPM path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++ restatement of the
 * reference algorithm, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  The product library
 * (exagoop_b200/libexg.so) never links, loads or calls it.
 *
 * Parity status: the reference cannot be compiled (its AMReX dependency is
 * an empty submodule), so the oracle's step-level arithmetic is "parity
 * unpinned" against reference outputs.  Its shape functions, wall-BC kernel
 * and constitutive models are pinned bit-exactly against the reference's own
 * header-only sources (Source/interpolants.H, Source/mpm_kernels.H,
 * Source/constitutive_models.H) compiled with a small type shim
 * (oracle/ref_pin.cpp), and its physics against the reference's analytic
 * validators (Tests/1D_Axial_Bar_Vibration/PostProcess/validate.py).
 */
#ifndef EXG_ORACLE_H_
#define EXG_ORACLE_H_
#include "../include/exg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const exg_specs *specs);
void orc_destroy(orc_ctx *o);
/* OpenMP threads for the particle loops; 1 (default) = sequential particle
 * order, which makes every nodal sum deterministic. */
void orc_set_threads(orc_ctx *o, int nthreads);
int orc_set_particles(orc_ctx *o, const exg_particle_soa *p);
int orc_get_particles(orc_ctx *o, exg_particle_soa *p);
int64_t orc_num_particles(orc_ctx *o);
int orc_set_levelset(orc_ctx *o, int body, const double *phi_nodes);
void orc_get_nodes(orc_ctx *o, int comp, double *out);
void orc_set_nodes(orc_ctx *o, int comp, const double *in);

void orc_init_internal_forces(orc_ctx *o);
int orc_redistribute(orc_ctx *o);
double orc_calculate_time_step(orc_ctx *o);
void orc_reset_nodaldata(orc_ctx *o);
void orc_p2g_momentum(orc_ctx *o, int update_mass, int update_vel, int update_forces);
void orc_backup_current_velocity(orc_ctx *o);
void orc_nodal_time_update_momentum(orc_ctx *o, double dt);
int orc_apply_nodal_bcs(orc_ctx *o, double dt, double time);
void orc_g2p_momentum(orc_ctx *o, int update_vel, int update_strainrate, double dt);
int orc_update_mp_positions(orc_ctx *o, double dt);
void orc_update_mp_volume(orc_ctx *o);
void orc_calculate_mp_stress_strain(orc_ctx *o, double time, double dt);
void orc_p2g_temperature(orc_ctx *o, int reset, int update_temp, int update_source);
void orc_backup_current_temperature(orc_ctx *o);
void orc_nodal_time_update_temperature(orc_ctx *o, double dt);
void orc_apply_nodal_bcs_temperature(orc_ctx *o, double dt, double time, int dirichlet_only);
void orc_store_delta_temperature(orc_ctx *o);
void orc_g2p_temperature(orc_ctx *o, int update_temperature, int update_heatflux);

/* nsteps iterations of the main.cpp:83-171 loop body (no output). */
int orc_step(orc_ctx *o, int nsteps);
void orc_get_time(orc_ctx *o, double *time, double *last_dt, int64_t *steps);
void orc_diagnostics(orc_ctx *o, exg_diag *out);

/* Cell keys of the tile-major cell ordering the GPU sort uses, and a stable
 * CPU sort permutation of them (std::stable_sort). */
void orc_sort_keys(orc_ctx *o, int tile, uint32_t *keys, int32_t *perm);

#ifdef __cplusplus
}
#endif
#endif
