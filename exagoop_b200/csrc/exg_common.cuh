// exg_common.cuh -- device-side data structures and math of the B200 MPM step.
//
// Shape functions, wall BC and constitutive models follow the reference's
// header-only math (Source/interpolants.H, Source/mpm_kernels.H,
// Source/constitutive_models.H); the citations sit on each function.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/exg.h"

#define EXG_HD __host__ __device__ __forceinline__

namespace exg {

constexpr int kMaxBodies = EXG_MAX_BODIES;
constexpr double kTiny = 1e-20;
// Literal constants of Source/constants.H:9-26; their truncated values are
// part of the arithmetic.
constexpr double kFourByThree = 1.3333333333;
constexpr double kOneBySix = 0.16666666666667;
constexpr double kOneByThree = 0.333333333333;
constexpr double kTwoByThree = 0.6666666666667;

// Device status bits (ORed into Ctl::status by kernels).
enum : unsigned {
    ST_NAN = 1u,
    ST_DOMAIN = 2u,
    ST_OVERFLOW = 4u,
    ST_BC = 8u,
    ST_TIMEOUT = 16u,
    ST_BUCKET = 32u,
    ST_ALIGN = 64u,  // a shared-memory staging buffer was not aligned for TMA (plain loads used)
    ST_BOUNDS = 128u,  // an index failed its range check (the access was skipped)
};

// Fixed-point P2G channels.  Momentum: mass, p(3), f(3).  Thermal: m cp,
// m cp T, m k, source.
enum { CH_M = 0, CH_P = 1, CH_F = 4, CH_MOM_END = 7, CH_MC = 7, CH_MCT = 8, CH_MK = 9, CH_SRC = 10, CH_ALL = 11 };

// Device control block: everything a step reads or produces that must not
// bounce through the host (dt, time, reductions, fixed-point scales).
struct Ctl {
    double dt;            // dt of the current step
    double time;          // simulation time at the start of the current step
    long long steps;
    unsigned status;
    unsigned pad0;
    // reductions produced by the last particle pass (see k_state_reduce)
    unsigned long long dtmin_bits;     // min over phase-0 particles of dxmin/(Cs+|v|), as ordered bits
    unsigned long long bound_bits[CH_ALL];  // max |contribution bound| per channel
    unsigned long long lost;           // particles dropped by the sort
    int maxppc;                        // max particles in one cell (from the sort)
    int pad1;
    double scale[CH_ALL];              // fixed-point scale 2^e per channel
    double inv_scale[CH_ALL];
    int n_active_tiles;
    int n_touched_tiles;
    long long n_sorted;                // particles inside the domain after the sort
    unsigned long long lost_fill;      // next slot for out-of-domain particles in the re-ordered storage
    int next_p2g;                      // dynamic tile counter of the P2G kernel (reset by k_scales)
    int next_g2p;                      // dynamic item counter of the fused G2P (reset by k_nodes)
    int n_g2p_items;                   // work items of the fused G2P (chunks of kG2PChunk particles of a tile)
    int pad2;
};
// Particles of one work item of the fused G2P: a tile of more particles
// (a pile-up) is split into several items, so that no item is much longer
// than an ordinary tile.  Each item stages its tile's node block again, so
// ordinary tiles (8 particles per cell of an 8^3 tile) stay whole: items of
// 1024 made the 9 M-particle sphere step's G2P 5 % slower (FP64, whose node
// block arrives single-buffered, 15 %).
constexpr int kG2PChunk = 4096;

// Per-tile stride of the P2G staging array, in 64-bit words, for nv
// fixed-point values: FP32 state one 64-bit integer per value; FP64 state
// the 64-bit low words, then the 32-bit high words (96-bit values).
template <class R>
EXG_HD constexpr long long stg_stride(long long nv) { return sizeof(R) == 4 ? nv : nv + (nv + 1) / 2; }

// Control block of a batch of independent scenes advanced by one launch per
// kernel: prefix sums of the scenes' tile counts and the batch's dynamic
// tile counters (k_batch_plan fills them before each step's batched
// kernels).
constexpr int kMaxScenes = 1024;
struct BatchCtl {
    int nscenes;
    int next_p2g, next_nodes, next_g2p, next_sort;
    int pre_active[kMaxScenes + 1];   // scene s owns items [pre[s], pre[s+1]) of the active-tile list
    int pre_touched[kMaxScenes + 1];  // the same for the tiles the nodal kernel writes
    // set on the host when the scenes' particle counts change: scene s owns
    // blocks [pre_blocks[s], pre_blocks[s+1]) of the per-particle batched
    // kernels (kBatchThreads particles each, so no block spans two scenes)
    // and tiles [pre_tiles[s], pre_tiles[s+1]) of the per-tile ones
    int pre_blocks[kMaxScenes + 1];
    int pre_tiles[kMaxScenes + 1];
};
constexpr int kBatchThreads = 256;


struct Body {
    int mom_bc;
    double wall_mu;
    double wall_vel[3];
    int temp_bc;
    double T_wall, heat_flux, h_conv, T_inf;
};

// Grid / run parameters passed by value to kernels.
struct Params {
    double plo[3], phi[3], dx[3], dxi[3];
    int nc[3];       // cells
    int nn[3];       // nodes per axis (nc+1)
    long long nnodes;
    int periodic[3];
    int order[3];
    int uniform_order;  // 1,2,3 when all axes share it, else 0
    int dual;           // quadratic: particles binned by nearest node (3-node window per axis)
    int T;              // tile edge (cells, or nearest-node bins when dual)
    int tshift;         // log2(T)
    int ntile[3];
    long long ntiles;
    int hlo, hhi, B;    // node-block halo below/above and edge B = T+hlo+hhi
    double gravity[3];
    int external_loads;
    double slab_lo[3], slab_hi[3], extforce[3];
    double mass_tol, alpha;
    double applied_sr, applied_sr_time;
    int bclo[3], bchi[3];
    double wmu_lo[3], wmu_hi[3];
    double wvel_lo[9], wvel_hi[9];
    int udf_lo[3], udf_hi[3];  // wall-velocity table present
    int fixed_dt;
    double timestep, cfl, dt_min, dt_max, dxmin;
    int num_bodies;
    Body body[kMaxBodies];
    int use_temp;
    int delta_strain;  // calculate_strain_based_on_delta: incremental linear-elastic stress
    // nodal temperatures are stored as T - Tref (FP32 state: a reference near
    // the particles' temperatures keeps their differences resolved; 0 in FP64)
    double Tref;
    // domain-wall thermal BCs (mpm_specs.H bc_temp_* arrays)
    int bclo_temp[3], bchi_temp[3];
    double Twall_lo[3], Twall_hi[3], qflux_lo[3], qflux_hi[3], hc_lo[3], hc_hi[3], Tinf_lo[3], Tinf_hi[3];
    int udfT_lo[3], udfT_hi[3];  // wall-temperature table present
};

// What the batched sort and bookkeeping kernels need of one scene: its grid,
// the positions of the storage the step starts from, its sort buffers, its
// control block and the P2G bounds the step uses.
struct SortDesc {
    Params P;
    double *x[3];
    long long np;
    int cap;  // sort scratch (tiles above the shared-memory cap) starts at bucket + cap
    uint32_t *key;
    int *tile_count, *tile_fill, *tile_start, *active, *slot, *touched, *cell_start, *item_start;
    long long *touched_step;
    int32_t *bucket, *perm;
    Ctl *ctl;
    unsigned long long *bounds_cur;
};

// Particle storage (structure of arrays).  Positions are FP64 in both
// precisions; the deformation gradient is stored as E = F - I so that FP32
// storage keeps J = det F accurate to FP64 level for small strains.
template <class R>
struct Parts {
    double *x[3];
    R *v[3], *vp[3];
    R *sr[6], *eps[6], *sig[6];
    R *E[9];
    R *vol, *mass, *rho, *pres, *vol0, *radius, *yacc;
    double *J;        // det F: FP64 in both precisions
    double *T;        // temperature: FP64 in both precisions (per-step increments
                      // are far below FP32 resolution at a few hundred kelvin)
    R *cp, *kc, *q[3], *Q;
    int32_t *mat;     // index into the material table
    uint8_t *phase;
    int32_t *rigid;
    int32_t *pid;     // upload index (download order)
};

struct Material {
    double E, nu, K, gamma, mu;
    int model;
    int ipow;  // gamma when it is a whole number in 1..16 (the Tait power by multiplication), else 0
    // modulus of the CFL sound speed sqrt(pmod / rho) (Calculate_time_step,
    // mpm_particle_timestep.cpp:55-100): K for the fluid model, lambda + 2 mu
    // otherwise, formed once per material on the host in the reference's
    // expression order
    double pmod;
};

// Dense nodal storage, reference component order, x fastest.
template <class R>
struct Nodes {
    R *c[EXG_N_NCOMP];
    // interleaved copy of the fields the fused G2P reads, written by the
    // nodal kernel of a fused step: per node v(3), dv(3) (FP32 padded to 8
    // words, FP64 6), so one 4-D TMA box fetches a tile's whole node block in
    // the layout the G2P uses; null when the G2P stages nodes itself
    // (periodic axes)
    R *rec;
};
template <class R>
constexpr int rec_words() { return sizeof(R) == 4 ? 8 : 6; }

// ------------------------------------------------------------------ math
template <class R>
EXG_HD R rsqrt_(R x);
template <>
EXG_HD double rsqrt_(double x) { return 1.0 / sqrt(x); }
template <>
EXG_HD float rsqrt_(float x) { return 1.0f / sqrtf(x); }

EXG_HD unsigned long long dbits(double x) {
#ifdef __CUDA_ARCH__
    return (unsigned long long)__double_as_longlong(x);
#else
    unsigned long long u;
    memcpy(&u, &x, 8);
    return u;
#endif
}
EXG_HD double bitsd(unsigned long long u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, 8);
    return x;
#endif
}

// Shape type of basisval*() (interpolants.H:1419-1426).
EXG_HD int shape_type(int idx, int nc, int periodic) {
    if (periodic) return 3;
    return 3 + (idx == 0 || idx == nc) * (1 - 3) + (idx == 1) * (2 - 3) + (idx == nc - 1) * (4 - 3);
}

// compute_bounds, mpm_particle_grid_ops.cpp:255-299.
EXG_HD void stencil_bounds(int ivd, int nc, int order, int periodic, int &bmin, int &bmax) {
    if (order == 1) {
        bmin = 0;
        bmax = 2;
    } else if (periodic) {
        bmin = -1;
        bmax = 3;
    } else if (ivd == 0) {
        bmin = 0;
        bmax = 3;
    } else if (ivd == nc - 1) {
        bmin = -1;
        bmax = 2;
    } else {
        bmin = -1;
        bmax = 3;
    }
}

// Spline tables (interpolants.H:32-183), copied to shared memory by kernels
// that evaluate boundary-aware shape functions.
struct SplineTables {
    double cub[5][4][4];
    double cubd[5][4][3];
    double quad[5][4][3];
    double quadd[5][4][2];
    int qmap[5][6];
};

// 1-D value and derivative (d/dz) of the boundary-aware spline of `order`
// and shape `type` at z, as cubicspline_1d / quadraticspline_1d and their
// derivatives (interpolants.H:215-304).  The cubic interval floor(z)+2 is
// clamped to [0,3]; the reference reads past its table there.  Evaluated in
// FP64 whatever R, from an FP64 offset, as the reference does: the expanded
// pieces cancel to ~1e-16 absolute where they fall to zero, which FP32
// arithmetic would leave at ~1e-7 (R = float rounds the results only).
template <class R>
__device__ __forceinline__ void spline_eval(const SplineTables &t, int order, int type, double z, R &val, R &der) {
    if (order == 3) {
        int iv = (int)floor(z) + 2;
        iv = iv < 0 ? 0 : (iv > 3 ? 3 : iv);
        const double *c = t.cub[type][iv];
        const double *d = t.cubd[type][iv];
        double z2 = z * z, z3 = z2 * z;
        val = (R)(c[0] * z3 + c[1] * z2 + c[2] * z + c[3]);
        der = (R)(d[0] * z2 + d[1] * z + d[2]);
    } else {
        double shift = (type == 2) ? 1.0 : 1.5;
        int raw = (int)floor((z + shift) * 2.0);
        int iv = (raw < 0 || raw >= 6) ? -1 : t.qmap[type][raw];
        if (iv < 0) {
            val = R(0);
            der = R(0);
        } else {
            const double *c = t.quad[type][iv];
            const double *d = t.quadd[type][iv];
            val = (R)(c[0] * z * z + c[1] * z + c[2]);
            der = (R)(d[0] * z + d[1]);
        }
    }
}

// Per-axis weights of one particle: W stencil entries for offsets LO..LO+W-1
// relative to the particle's cell, zero outside compute_bounds.  Value and
// derivative (already scaled by 1/dx) as in basisval_and_grad
// (interpolants.H:1581-1654).
template <class R, int W>
struct AxisW {
    R w[W];
    R dw[W];
};

template <class R, int W, int LO>
__device__ __forceinline__ void axis_weights(const SplineTables &t, const Params &P, int d, double x, int i,
                                             AxisW<R, W> &a) {
    const int od = P.order[d];
    const double dx = P.dx[d];
    const R dxinv = (R)P.dxi[d];
    int bmin, bmax;
    stencil_bounds(i, P.nc[d], od, P.periodic[d], bmin, bmax);
#pragma unroll
    for (int s = 0; s < W; ++s) {
        const int l = LO + s;
        R val = R(0), der = R(0);
        if (l >= bmin && l < bmax) {
            if (od == 1) {
                const double r = (x - (P.plo[d] + i * dx)) * P.dxi[d];
                val = (l == 0) ? (R)(1.0 - r) : (R)r;
                der = (l == 0) ? -dxinv : dxinv;
            } else {
                int ty = shape_type(i + l, P.nc[d], P.periodic[d]);
                const double r = (x - (P.plo[d] + (i + l) * dx)) * P.dxi[d];
                spline_eval<R>(t, od, ty, r, val, der);
                der *= dxinv;
            }
        }
        a.w[s] = val;
        a.dw[s] = der;
    }
}

// applybc, Source/mpm_kernels.H:27-113.  Returns modify_pos (0/1) or -1 for
// the outflow code the reference aborts on.
template <class R>
EXG_HD int applybc(const R in[3], R out[3], R wall_mu, const R n[3], int bc) {
    int modify = 0;
    R veln = in[0] * n[0] + in[1] * n[1] + in[2] * n[2];
    R vt[3];
    for (int d = 0; d < 3; ++d) vt[d] = in[d] - veln * n[d];
    R vtm = sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    if (bc == EXG_BC_NOSLIP) {
        modify = 1;
        for (int d = 0; d < 3; ++d) out[d] = R(0);
    } else if (bc == EXG_BC_SLIP) {
        modify = 1;
        for (int d = 0; d < 3; ++d) out[d] = vt[d];
    } else if (bc == EXG_BC_PARTIALSLIP) {
        if (veln <= R(0)) {
            modify = 1;
            if (vtm <= -wall_mu * veln) {
                for (int d = 0; d < 3; ++d) out[d] = R(0);
            } else {
                R den = vtm + (R)kTiny;
                for (int d = 0; d < 3; ++d) out[d] = (vtm + wall_mu * veln) * (vt[d] / den);
            }
        }
    } else if (bc == EXG_BC_PERIODIC) {
    } else {
        return -1;
    }
    return modify;
}

// Hooke's law, constitutive_models.H:21-54 (3-D branch).
template <class R>
EXG_HD void linear_elastic(const R e[6], R s[6], R E, R nu) {
    R c1 = E / (R(1) + nu) / (R(1) - R(2) * nu);
    R c2 = E / (R(1) + nu);
    s[0] = c1 * ((R(1) - nu) * e[0] + nu * (e[3] + e[5]));
    s[3] = c1 * ((R(1) - nu) * e[3] + nu * (e[0] + e[5]));
    s[5] = c1 * ((R(1) - nu) * e[5] + nu * (e[0] + e[3]));
    s[1] = c2 * e[1];
    s[2] = c2 * e[2];
    s[4] = c2 * e[4];
}
// Newtonian_Fluid, constitutive_models.H:118-159 (3-D branch).
template <class R>
EXG_HD void newtonian(const R ed[6], R s[6], R mu, R p) {
    R tr = ed[0] + ed[3] + ed[5];
    R o3 = R(1) / R(3);
    s[0] = R(2) * mu * (ed[0] - o3 * tr) - p;
    s[3] = R(2) * mu * (ed[3] - o3 * tr) - p;
    s[5] = R(2) * mu * (ed[5] - o3 * tr) - p;
    s[1] = R(2) * mu * ed[1];
    s[2] = R(2) * mu * ed[2];
    s[4] = R(2) * mu * ed[4];
}

// det F in the order of updateVolume (mpm_particle_timestep.cpp:160-163),
// every product and difference rounded on its own (no fused multiply-add),
// as the reference's host build evaluates it.
EXG_HD double det_ref(const double F[9]) {
#ifdef __CUDA_ARCH__
    const double t1 = __dsub_rn(__dmul_rn(F[4], F[8]), __dmul_rn(F[5], F[7]));
    const double t2 = __dsub_rn(__dmul_rn(F[3], F[8]), __dmul_rn(F[5], F[6]));
    const double t3 = __dsub_rn(__dmul_rn(F[3], F[7]), __dmul_rn(F[4], F[6]));
    return __dadd_rn(__dsub_rn(__dmul_rn(F[0], t1), __dmul_rn(F[1], t2)), __dmul_rn(F[2], t3));
#else
    return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
#endif
}

// Node linear index with periodic wrap; -1 outside a non-periodic domain.
EXG_HD long long node_index(const Params &P, int i, int j, int k) {
    int id[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
        if (P.periodic[d]) {
            int n = P.nc[d];
            id[d] %= n;
            if (id[d] < 0) id[d] += n;
        } else if (id[d] < 0 || id[d] > P.nc[d]) {
            return -1;
        }
    }
    return ((long long)id[2] * P.nn[1] + id[1]) * P.nn[0] + id[0];
}

// Cell of a position: floor((x - plo) * dxi) (AMReX getParticleCell).
EXG_HD void cell_of(const Params &P, const double x[3], int iv[3]) {
    for (int d = 0; d < 3; ++d) iv[d] = (int)floor((x[d] - P.plo[d]) * P.dxi[d]);
}

// Nearest-node bin along axis d: every node a quadratic B-spline of the
// particle touches (support 1.5 dx for all boundary types) is bin-1..bin+1.
// Periodic axes wrap bin ncells onto 0.
EXG_HD int dual_bin_raw(const Params &P, int d, double x) { return (int)floor((x - P.plo[d]) * P.dxi[d] + 0.5); }
EXG_HD int dual_bin(const Params &P, int d, double x) {
    int b = dual_bin_raw(P, d, x);
    if (P.periodic[d] && b >= P.nc[d]) b -= P.nc[d];
    return b;
}
// Position used for the weights of a particle whose bin wrapped: shifted
// one period down, so its window bin-1..bin+1 (and the bin's node block)
// holds it.
EXG_HD double dual_x(const Params &P, int d, double x) {
    return (P.dual && P.periodic[d] && dual_bin_raw(P, d, x) >= P.nc[d]) ? x - (P.phi[d] - P.plo[d]) : x;
}

}  // namespace exg
