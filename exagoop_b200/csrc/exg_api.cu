// exg_api.cu -- C ABI of the B200 MPM step: context, particle upload and
// download, one entry point per reference L5 step function, and the fused,
// graph-replayed exg_step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <tuple>
#include <cudaTypedefs.h>
#include "exg_internal.h"
#include "exg_levelset.h"

using namespace exg;

struct exg_ctx {
    Ctx c;
};
struct exg_batch {
    Batch b;
    std::vector<exg_ctx *> ctxs;
    std::string err;
};

namespace {

int fail(exg_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->c.err = msg;
    return code;
}

#define EXG_TRY(ctx, ...)                                          \
    try {                                                          \
        __VA_ARGS__;                                               \
    } catch (const std::exception &e) {                            \
        return fail(ctx, EXG_ERR_CUDA, e.what());                  \
    }

bool fp64(const Ctx &c) { return c.precision == EXG_PREC_FP64; }

// precision dispatch of the launchers
#define DISPATCH(name, ...) (fp64(c) ? name##_fp64(__VA_ARGS__) : name##_fp32(__VA_ARGS__))

template <class T>
T *dalloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    EXG_CUDA_OK(cudaMalloc(&p, n * sizeof(T)));
    return reinterpret_cast<T *>(p);
}

// Host loops over the particles (material table, upload order, download
// expansion) split over the host's cores: at millions of particles they are
// a visible part of an upload or download otherwise.  fn(chunk, begin, end)
// must not throw.
int host_chunks(long long n) {
    if (n < (1ll << 20)) return 1;
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc ? hc : 1u, 32u));
}
template <class F>
void parallel_chunks(long long n, int nchunks, F fn) {
    if (nchunks <= 1) {
        fn(0, 0ll, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nchunks);
    for (int t = 0; t < nchunks; ++t) th.emplace_back(fn, t, n * t / nchunks, n * (t + 1) / nchunks);
    for (auto &x : th) x.join();
}

int ilog2(int v) {
    int s = 0;
    while ((1 << s) < v) ++s;
    return s;
}

}  // namespace

namespace exg {
// Kernel parameters of a run specification.
void build_params_for(const exg_specs &s, Params &P) {
    std::memset(&P, 0, sizeof(P));
    for (int d = 0; d < 3; ++d) {
        P.plo[d] = s.plo[d];
        P.phi[d] = s.phi[d];
        P.nc[d] = s.ncells[d];
        P.nn[d] = s.ncells[d] + 1;
        // AMReX Geometry: dx = (hi - lo) / n, inv_dx = 1 / dx
        P.dx[d] = (s.phi[d] - s.plo[d]) / (double)s.ncells[d];
        P.dxi[d] = 1.0 / P.dx[d];
        P.periodic[d] = s.periodic[d];
        P.order[d] = s.order[d];
        P.gravity[d] = s.gravity[d];
        P.slab_lo[d] = s.force_slab_lo[d];
        P.slab_hi[d] = s.force_slab_hi[d];
        P.extforce[d] = s.extforce[d];
        P.bclo[d] = s.bclo[d];
        P.bchi[d] = s.bchi[d];
        P.wmu_lo[d] = s.wall_mu_lo[d];
        P.wmu_hi[d] = s.wall_mu_hi[d];
        P.udf_lo[d] = s.udf_wallvel_lo[d] != nullptr;
        P.udf_hi[d] = s.udf_wallvel_hi[d] != nullptr;
    }
    for (int i = 0; i < 9; ++i) {
        P.wvel_lo[i] = s.wall_vel_lo[i];
        P.wvel_hi[i] = s.wall_vel_hi[i];
    }
    P.nnodes = (long long)P.nn[0] * P.nn[1] * P.nn[2];
    P.uniform_order = (s.order[0] == s.order[1] && s.order[1] == s.order[2]) ? s.order[0] : 0;
    P.external_loads = s.external_loads;
    P.mass_tol = s.mass_tolerance;
    P.alpha = s.alpha_pic_flip;
    P.applied_sr = s.applied_strainrate;
    P.applied_sr_time = s.applied_strainrate_time;
    P.fixed_dt = s.fixed_timestep == 1;
    P.timestep = s.timestep;
    P.cfl = s.cfl;
    P.dt_min = s.dt_min_limit;
    P.dt_max = s.dt_max_limit;
    P.dxmin = std::min(P.dx[0], std::min(P.dx[1], P.dx[2]));
    P.num_bodies = s.num_bodies;
    for (int b = 0; b < s.num_bodies && b < kMaxBodies; ++b) {
        const exg_body &e = s.bodies[b];
        Body &o = P.body[b];
        o.mom_bc = e.mom_bc;
        o.wall_mu = e.wall_mu;
        for (int d = 0; d < 3; ++d) o.wall_vel[d] = e.wall_vel[d];
        o.temp_bc = e.temp_bc;
        o.T_wall = e.T_wall;
        o.heat_flux = e.heat_flux;
        o.h_conv = e.h_conv;
        o.T_inf = e.T_inf;
    }
    P.use_temp = s.use_temp;
    P.delta_strain = s.calculate_strain_based_on_delta == 1;
    for (int d = 0; d < 3; ++d) {
        P.bclo_temp[d] = s.bclo_temp[d];
        P.bchi_temp[d] = s.bchi_temp[d];
        P.Twall_lo[d] = s.T_wall_lo[d];
        P.Twall_hi[d] = s.T_wall_hi[d];
        P.qflux_lo[d] = s.flux_lo[d];
        P.qflux_hi[d] = s.flux_hi[d];
        P.hc_lo[d] = s.h_lo[d];
        P.hc_hi[d] = s.h_hi[d];
        P.Tinf_lo[d] = s.Tinf_lo[d];
        P.Tinf_hi[d] = s.Tinf_hi[d];
        P.udfT_lo[d] = s.udf_temp_lo[d] != nullptr;
        P.udfT_hi[d] = s.udf_temp_hi[d] != nullptr;
    }
    // tile geometry
    int T = s.tile > 0 ? s.tile : 8;
    P.T = T;
    P.tshift = ilog2(T);
    const bool lin = (P.uniform_order == 1);
    P.dual = (P.uniform_order == 2);
    P.hlo = lin ? 0 : 1;
    P.hhi = lin ? 1 : (P.dual ? 1 : 2);
    P.B = T + P.hlo + P.hhi;
    for (int d = 0; d < 3; ++d)
        P.ntile[d] = s.periodic[d] ? s.ncells[d] / T : (s.ncells[d] + 1 + T - 1) / T;
    P.ntiles = (long long)P.ntile[0] * P.ntile[1] * P.ntile[2];
}
int noalloc_p2g(const exg_specs *specs, const exg_particle_soa *dev, double *mass, double *vel, double *frc,
                cudaStream_t stream, std::string &err);
}  // namespace exg

namespace {

void build_params(Ctx &c) { build_params_for(c.specs, c.P); }

std::string validate(const exg_specs &s) {
    for (int d = 0; d < 3; ++d) {
        if (s.ncells[d] < 1) return "mpm.ncells must be positive";
        if (!(s.phi[d] > s.plo[d])) return "mpm.prob_hi must exceed mpm.prob_lo";
        if (s.order[d] < 1 || s.order[d] > 3) return "order_scheme_directional must be 1, 2 or 3";
    }
    int T = s.tile > 0 ? s.tile : 8;
    if (T != 4 && T != 8) return "exg.tile must be 4 or 8";
    for (int d = 0; d < 3; ++d)
        if (s.periodic[d] && (s.ncells[d] % T != 0 || s.ncells[d] < 3 * T))
            return "periodic axes need ncells to be a multiple of the tile edge and at least three tiles";
    // bin keys are 32-bit (tile index x T^3 + cell in the tile; 0xFFFFFFFF
    // marks a particle outside the domain): the tile grid, as the context
    // lays it out, must keep every key below that
    long long cells = (long long)T * T * T;
    for (int d = 0; d < 3; ++d) cells *= s.periodic[d] ? s.ncells[d] / T : (s.ncells[d] + 1 + T - 1) / T;
    if (cells >= 0xFFFFFFFFll) return "grid too large for the 32-bit bin keys (tile-padded cells must stay below 2^32 - 1)";
    if (s.num_bodies < 0 || s.num_bodies > EXG_MAX_BODIES) return "too many level-set bodies";
    return "";
}

// Particle storage of one orientation.  Fields that no kernel changes and no
// kernel reads (radius, yield acceleration, rigid-body id) live once, in
// upload order, shared by both orientations: the per-step reorder does not
// carry them.
template <class R>
void alloc_parts(Ctx &c, Parts<R> &P, std::vector<void *> &al, long long n, bool temp, const Parts<R> *home) {
    auto A = [&](auto *&ptr) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(ptr)>>;
        ptr = dalloc<T>(n);
        al.push_back(ptr);
    };
    std::memset(&P, 0, sizeof(P));
    for (int d = 0; d < 3; ++d) {
        A(P.x[d]);
        A(P.v[d]);
        A(P.vp[d]);
    }
    for (int k = 0; k < 6; ++k) {
        A(P.sr[k]);
        A(P.eps[k]);
        A(P.sig[k]);
    }
    for (int k = 0; k < 9; ++k) A(P.E[k]);
    A(P.vol);
    A(P.mass);
    A(P.rho);
    A(P.J);
    A(P.pres);
    A(P.vol0);
    if (home) {
        P.radius = home->radius;
        P.yacc = home->yacc;
        P.rigid = home->rigid;
    } else {
        A(P.radius);
        A(P.yacc);
        A(P.rigid);
    }
    if (temp) {
        A(P.T);
        A(P.cp);
        A(P.kc);
        for (int d = 0; d < 3; ++d) A(P.q[d]);
        A(P.Q);
    }
    A(P.mat);
    A(P.phase);
    A(P.pid);
    (void)c;
}

void free_list(std::vector<void *> &al) {
    for (void *p : al) cudaFree(p);
    al.clear();
}

// Host transfers of the particle state: every real field crosses PCIe as the
// caller's FP64 array (pinned when it comes from exg_particles_alloc_pinned)
// and is converted on the device; downloads return to upload order on the
// device (pid), so the host side is contiguous copies only.
template <class R>
void upload_parts(Ctx &c, const exg_particle_soa *h, const std::vector<int32_t> &mat) {
    if (h->np == 0) return;  // an empty set: storage of one slot, nothing to copy
    Parts<R> &P = c.A<R>();
    const long long n = h->np;
    const bool f64 = sizeof(R) == 8;
    auto put_r = [&](R *dst, int field, double sub = 0.0) {
        const double *src = h->rdata + (size_t)field * n;
        f64 ? h2d_field_fp64(c, dst, src, n, sub) : h2d_field_fp32(c, dst, src, n, sub);
    };
    for (int d = 0; d < 3; ++d) {
        EXG_CUDA_OK(cudaMemcpyAsync(P.x[d], h->pos + (size_t)d * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                    c.stream));
        put_r(P.v[d], EXG_R_VEL + d);
        put_r(P.vp[d], EXG_R_VEL_PRIME + d);
    }
    for (int k = 0; k < 6; ++k) {
        put_r(P.sr[k], EXG_R_STRAINRATE + k);
        put_r(P.eps[k], EXG_R_STRAIN + k);
        put_r(P.sig[k], EXG_R_STRESS + k);
    }
    // FP32 state keeps E = F - I, FP64 state F itself
    for (int k = 0; k < 9; ++k) put_r(P.E[k], EXG_R_DEFGRAD + k, (k % 4 == 0 && !fp64(c)) ? 1.0 : 0.0);
    put_r(P.vol, EXG_R_VOLUME);
    put_r(P.mass, EXG_R_MASS);
    put_r(P.rho, EXG_R_DENSITY);
    EXG_CUDA_OK(cudaMemcpyAsync(P.J, h->rdata + (size_t)EXG_R_JACOBIAN * n, sizeof(double) * n,
                                cudaMemcpyHostToDevice, c.stream));
    put_r(P.pres, EXG_R_PRESSURE);
    put_r(P.vol0, EXG_R_VOL_INIT);
    put_r(P.radius, EXG_R_RADIUS);
    put_r(P.yacc, EXG_R_YACC);
    if (c.specs.use_temp) {
        EXG_CUDA_OK(cudaMemcpyAsync(P.T, h->rdata + (size_t)EXG_R_TEMPERATURE * n, sizeof(double) * n,
                                    cudaMemcpyHostToDevice, c.stream));
        put_r(P.cp, EXG_R_SPHEAT);
        put_r(P.kc, EXG_R_THERMCOND);
        for (int d = 0; d < 3; ++d) put_r(P.q[d], EXG_R_HEATFLUX + d);
        put_r(P.Q, EXG_R_HEATSRC);
    }
    EXG_CUDA_OK(cudaMemcpyAsync(P.mat, mat.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, c.stream));
    std::vector<uint8_t> ph(n);
    std::vector<int32_t> pid(n);
    parallel_chunks(n, host_chunks(n), [&](int, long long a, long long b) {
        for (long long i = a; i < b; ++i) {
            ph[i] = (uint8_t)h->idata[(size_t)EXG_I_PHASE * n + i];
            pid[i] = (int32_t)i;
        }
    });
    EXG_CUDA_OK(cudaMemcpyAsync(P.phase, ph.data(), n, cudaMemcpyHostToDevice, c.stream));
    EXG_CUDA_OK(cudaMemcpyAsync(P.rigid, h->idata + (size_t)EXG_I_RIGID_ID * n, sizeof(int32_t) * n,
                                cudaMemcpyHostToDevice, c.stream));
    EXG_CUDA_OK(cudaMemcpyAsync(P.pid, pid.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, c.stream));
    EXG_CUDA_OK(cudaStreamSynchronize(c.stream));  // the host vectors above go out of scope
}

void drop_graphs(Ctx &c);

}  // namespace

bool exg::g2p_lean(const Ctx &c) {
    const exg_specs &s = c.specs;
    if (s.use_temp || s.calculate_strain_based_on_delta || s.num_bodies > 0) return false;
    for (int d = 0; d < 3; ++d)
        if (s.udf_wallvel_lo[d] || s.udf_wallvel_hi[d]) return false;
    for (const Material &m : c.mats)
        if (m.model > 1) return false;
    return true;
}

namespace {

// FP32 state keeps nodal temperatures relative to the mean particle
// temperature, so that differences of a few millikelvin on a few hundred
// kelvin stay resolved; a new reference re-bases the stored nodal values.
void set_tref(Ctx &c, const exg_particle_soa *h) {
    if (!c.specs.use_temp || fp64(c)) return;
    const long long n = h->np;
    double sum = 0.0;
    for (long long i = 0; i < n; ++i) sum += h->rdata[(size_t)EXG_R_TEMPERATURE * n + i];
    const double tref = n ? (double)(float)(sum / n) : 0.0;
    if (tref == c.P.Tref) return;
    c.P.Tref = tref;
    drop_graphs(c);  // the step graphs hold the parameters
    launch_fill_node_fp32(c, EXG_N_TEMPERATURE, -tref);  // untouched nodes: 0 K
}

template <class R>
void download_parts(Ctx &c, exg_particle_soa *h) {
    Parts<R> &P = c.A<R>();
    const long long n = c.np;
    if (n == 0) return;
    const bool f64 = sizeof(R) == 8;
    auto get_r = [&](const R *src, int field, double add = 0.0, bool home = false) {
        double *dst = h->rdata + (size_t)field * n;
        const int32_t *pid = home ? nullptr : P.pid;  // upload-order fields need no reorder
        f64 ? d2h_field_fp64(c, src, pid, dst, n, add) : d2h_field_fp32(c, src, pid, dst, n, add);
    };
    d2h_positions(c, P.x, P.pid, h->pos, n);
    for (int d = 0; d < 3; ++d) {
        get_r(P.v[d], EXG_R_VEL + d);
        get_r(P.vp[d], EXG_R_VEL_PRIME + d);
    }
    for (int k = 0; k < 6; ++k) {
        get_r(P.sr[k], EXG_R_STRAINRATE + k);
        get_r(P.eps[k], EXG_R_STRAIN + k);
        get_r(P.sig[k], EXG_R_STRESS + k);
    }
    for (int k = 0; k < 9; ++k) get_r(P.E[k], EXG_R_DEFGRAD + k, (k % 4 == 0 && !fp64(c)) ? 1.0 : 0.0);
    get_r(P.vol, EXG_R_VOLUME);
    get_r(P.mass, EXG_R_MASS);
    get_r(P.rho, EXG_R_DENSITY);
    d2h_field_fp64(c, P.J, P.pid, h->rdata + (size_t)EXG_R_JACOBIAN * n, n, 0.0);
    get_r(P.pres, EXG_R_PRESSURE);
    get_r(P.vol0, EXG_R_VOL_INIT);
    get_r(P.radius, EXG_R_RADIUS, 0.0, true);
    get_r(P.yacc, EXG_R_YACC, 0.0, true);
    if (c.specs.use_temp) {
        d2h_field_fp64(c, P.T, P.pid, h->rdata + (size_t)EXG_R_TEMPERATURE * n, n, 0.0);
        get_r(P.cp, EXG_R_SPHEAT);
        get_r(P.kc, EXG_R_THERMCOND);
        for (int d = 0; d < 3; ++d) get_r(P.q[d], EXG_R_HEATFLUX + d);
        get_r(P.Q, EXG_R_HEATSRC);
    } else {
        const int tf[7] = {EXG_R_TEMPERATURE, EXG_R_SPHEAT,         EXG_R_THERMCOND, EXG_R_HEATFLUX,
                           EXG_R_HEATFLUX + 1, EXG_R_HEATFLUX + 2, EXG_R_HEATSRC};
        parallel_chunks(n, host_chunks(n), [&](int, long long a, long long b) {
            for (int f : tf) std::fill(h->rdata + (size_t)f * n + a, h->rdata + (size_t)f * n + b, 0.0);
        });
    }
    d2h_int(c, P.phase, 1, P.pid, h->idata + (size_t)EXG_I_PHASE * n, n);
    d2h_int(c, P.rigid, 4, nullptr, h->idata + (size_t)EXG_I_RIGID_ID * n, n);
    // material index in upload order, expanded to the per-particle fields
    std::vector<int32_t> mat(n);
    d2h_int(c, P.mat, 4, P.pid, mat.data(), n);
    EXG_CUDA_OK(cudaStreamSynchronize(c.stream));
    parallel_chunks(n, host_chunks(n), [&](int, long long a, long long b) {
        for (long long j = a; j < b; ++j) {
            const Material &m = c.mats[mat[j]];
            h->rdata[(size_t)EXG_R_E * n + j] = m.E;
            h->rdata[(size_t)EXG_R_NU * n + j] = m.nu;
            h->rdata[(size_t)EXG_R_BULK * n + j] = m.K;
            h->rdata[(size_t)EXG_R_GAMMA * n + j] = m.gamma;
            h->rdata[(size_t)EXG_R_VISC * n + j] = m.mu;
            h->idata[(size_t)EXG_I_MODEL * n + j] = m.model;
        }
    });
}

void sync(Ctx &c) { EXG_CUDA_OK(cudaStreamSynchronize(c.stream)); }

void ctl_pull(Ctx &c) {
    EXG_CUDA_OK(cudaMemcpyAsync(c.ctl_host, c.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c.stream));
    sync(c);
}

// UDF wall tables of compute_udf_wall_vel_at_nodes (nodal_data_ops.cpp:929-1059),
// tabulated on the host at time t and copied to the device.
void tabulate_udf(Ctx &c, double t) {
    for (int side = 0; side < 2; ++side)
        for (int d = 0; d < 3; ++d) {
            exg_wallvel_udf fn = side ? c.specs.udf_wallvel_hi[d] : c.specs.udf_wallvel_lo[d];
            if (!fn) continue;
            const int p0 = (d == 0) ? 1 : 0, p1 = (d == 2) ? 1 : 2;
            const int n0 = c.P.nc[p0] + 1, n1 = c.P.nc[p1] + 1;
            std::vector<double> &tab = c.udf_host[side][d];
            tab.assign((size_t)n0 * n1 * 3, 0.0);
            for (int j = 0; j < n0; ++j)
                for (int k = 0; k < n1; ++k) {
                    double xc[3] = {0, 0, 0};
                    xc[d] = side ? c.P.phi[d] : c.P.plo[d];
                    xc[p0] = c.P.plo[p0] + j * c.P.dx[p0];
                    xc[p1] = c.P.plo[p1] + k * c.P.dx[p1];
                    double vel[3] = {0, 0, 0};
                    fn(xc[0], xc[1], xc[2], t, vel);
                    for (int q = 0; q < 3; ++q) tab[((size_t)j * n1 + k) * 3 + q] = vel[q];
                }
            if (!c.udf_tab[side][d]) c.udf_tab[side][d] = dalloc<double>(tab.size());
            EXG_CUDA_OK(cudaMemcpyAsync(c.udf_tab[side][d], tab.data(), sizeof(double) * tab.size(),
                                        cudaMemcpyHostToDevice, c.stream));
            sync(c);
        }
}
bool has_udf(const Ctx &c) {
    for (int d = 0; d < 3; ++d)
        if (c.specs.udf_wallvel_lo[d] || c.specs.udf_wallvel_hi[d]) return true;
    return false;
}

// UDF wall-temperature tables of compute_udf_temp_at_nodes
// (nodal_data_ops.cpp:1178-1293): two values per face node.
void tabulate_udf_temp(Ctx &c, double t) {
    for (int side = 0; side < 2; ++side)
        for (int d = 0; d < 3; ++d) {
            exg_temp_udf fn = side ? c.specs.udf_temp_hi[d] : c.specs.udf_temp_lo[d];
            if (!fn) continue;
            const int p0 = (d == 0) ? 1 : 0, p1 = (d == 2) ? 1 : 2;
            const int n0 = c.P.nc[p0] + 1, n1 = c.P.nc[p1] + 1;
            std::vector<double> &tab = c.udfT_host[side][d];
            tab.assign((size_t)n0 * n1 * 2, 0.0);
            for (int j = 0; j < n0; ++j)
                for (int k = 0; k < n1; ++k) {
                    double xc[3] = {0, 0, 0};
                    xc[d] = side ? c.P.phi[d] : c.P.plo[d];
                    xc[p0] = c.P.plo[p0] + j * c.P.dx[p0];
                    xc[p1] = c.P.plo[p1] + k * c.P.dx[p1];
                    double out[2] = {0, 0};
                    fn(xc[0], xc[1], xc[2], t, out);
                    tab[((size_t)j * n1 + k) * 2] = out[0];
                    tab[((size_t)j * n1 + k) * 2 + 1] = out[1];
                }
            if (!c.udfT_tab[side][d]) c.udfT_tab[side][d] = dalloc<double>(tab.size());
            EXG_CUDA_OK(cudaMemcpyAsync(c.udfT_tab[side][d], tab.data(), sizeof(double) * tab.size(),
                                        cudaMemcpyHostToDevice, c.stream));
            sync(c);
        }
}
bool has_udf_temp(const Ctx &c) {
    for (int d = 0; d < 3; ++d)
        if (c.specs.udf_temp_lo[d] || c.specs.udf_temp_hi[d]) return true;
    return false;
}

int status_from_ctl(Ctx &c) {
    ctl_pull(c);
    unsigned st = c.ctl_host->status;
    if (st) {
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->status, 0, sizeof(unsigned), c.stream));
        sync(c);
    }
    if (st & ST_BC) {
        c.err = "outflow wall BC reached applybc (the reference aborts here)";
        return EXG_ERR_BC;
    }
    if (st & ST_NAN) {
        c.err = "non-finite particle velocity, stress or Jacobian";
        return EXG_ERR_NAN;
    }
    if (st & ST_OVERFLOW) {
        c.err = "fixed-point range overflow";
        return EXG_ERR_OVERFLOW;
    }
    if (st & ST_TIMEOUT) {
        c.err = "a node-block transfer of the fused G2P did not complete within its wait limit";
        return EXG_ERR_TIMEOUT;
    }
    if (st & ST_BOUNDS) {
        c.err = "internal: a work-item, particle or staging index failed its range check";
        return EXG_ERR_CUDA;
    }
    if (st & ST_ALIGN) {
        c.err = "internal: the fused G2P's node-block buffer was not 128-byte aligned for TMA";
        return EXG_ERR_CUDA;
    }
    return EXG_OK;
}

// Sort by cell key for the current storage order (Redistribute).
void do_sort(Ctx &c, bool touched) {
    launch_keys(c);
    launch_sort_rest(c, touched);
    c.parts_sorted = true;
}

// Fresh particle reductions into the control block accumulators.
void do_reduce(Ctx &c) {
    launch_reset_accum(c, &c.ctl->bound_bits[0], &c.ctl->dtmin_bits);
    DISPATCH(launch_state_reduce, c, &c.ctl->bound_bits[0], &c.ctl->dtmin_bits);
    c.reduce_stale = false;
}

// One fused step, enqueued on c.stream (capturable).
void enqueue_step(Ctx &c) {
    EXG_CUDA_OK(cudaMemcpyAsync(c.bounds_cur, &c.ctl->bound_bits[0], sizeof(unsigned long long) * CH_ALL,
                                cudaMemcpyDeviceToDevice, c.stream));
    launch_dt_finalize(c, true);
    if (c.timing) EXG_CUDA_OK(cudaEventRecord(c.ev[0], c.stream));
    nvtxRangePushA("step: sort (Redistribute)");
    launch_keys(c);
    launch_sort_rest(c, true);
    nvtxRangePop();
    if (c.timing) EXG_CUDA_OK(cudaEventRecord(c.ev[1], c.stream));
    launch_scales_from(c, c.bounds_cur);
    const bool th = c.specs.use_temp != 0;
    const bool musl = c.specs.stress_update_scheme != 0;
    const int tflags = th ? (PF_TEMP | PF_SRC) : 0;
    const int udfT = has_udf_temp(c) ? 1 : 0;
    nvtxRangePushA("step: P2G");
    DISPATCH(launch_p2g, c, PF_MASS | PF_VEL | PF_FORCE | tflags);
    nvtxRangePop();
    if (c.timing) EXG_CUDA_OK(cudaEventRecord(c.ev[2], c.stream));
    DISPATCH(launch_nodes, c, NM_FUSED, PF_MASS | PF_VEL | PF_FORCE | tflags, false);
    if (th) {
        // Apply_Nodal_BCs_Temperature + store_delta_temperature (main.cpp:103-106)
        DISPATCH(launch_temp_bcs, c, TW_MASKED, udfT, 1, musl ? 1 : 0);
        DISPATCH(launch_temp_node_op, c, TN_DELTA, 0.0);
    }
    if (c.timing) EXG_CUDA_OK(cudaEventRecord(c.ev[3], c.stream));
    if (!musl) {
        if (th) DISPATCH(launch_g2p_temp, c, 1, 1);  // G2P_Temperature(1,1) (main.cpp:113)
        DISPATCH(launch_g2p_fused, c, GM_FULL);
    } else {
        if (th) DISPATCH(launch_g2p_temp, c, 1, 0);  // G2P_Temperature(1,0) (main.cpp:132)
        DISPATCH(launch_g2p_fused, c, GM_VEL);
        launch_reset_accum(c, c.bounds2, c.dtmin2);
        DISPATCH(launch_state_reduce, c, c.bounds2, c.dtmin2);
        launch_scales_from(c, c.bounds2);
        // P2G_Momentum(0,1,0) and P2G_Temperature(1,0,1) in one deposit
        DISPATCH(launch_p2g, c, PF_VEL | (th ? PF_SRC : 0));
        DISPATCH(launch_nodes, c, NM_MUSL2, PF_VEL | (th ? PF_SRC : 0), false);
        if (th) {
            DISPATCH(launch_temp_bcs, c, TW_ON, udfT, 1, 0);  // main.cpp:134-135
            DISPATCH(launch_g2p_temp, c, 0, 1);               // G2P_Temperature(0,1) (main.cpp:136)
        }
        DISPATCH(launch_g2p_fused, c, GM_STRAIN);
    }
    DISPATCH(launch_copy_lost, c);
    if (c.timing) EXG_CUDA_OK(cudaEventRecord(c.ev[4], c.stream));
    launch_time_advance(c);
}

void swap_parts(Ctx &c) {
    std::swap(c.pa, c.pb);
    c.orient ^= 1;
}

// Interleaved node records and the tensor map the fused G2P stages its node
// blocks with (one 4-D box: record words x B x B x B).  Skipped on grids
// with a periodic axis (the box cannot wrap) or when EXG_NO_TMA is set; the
// G2P then stages with plain loads.
void setup_node_records(Ctx &c) {
    std::memset(&c.tmap, 0, sizeof(c.tmap));
    c.tma = false;
    if (c.P.periodic[0] || c.P.periodic[1] || c.P.periodic[2] || std::getenv("EXG_NO_TMA")) return;
    const bool f64 = fp64(c);
    const size_t esz = f64 ? 8 : 4, ns = f64 ? rec_words<double>() : rec_words<float>();
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess)
        return;
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    EXG_CUDA_OK(cudaMalloc(&c.rec, esz * ns * c.P.nnodes));
    EXG_CUDA_OK(cudaMemset(c.rec, 0, esz * ns * c.P.nnodes));
    const cuuint64_t dims[4] = {ns, (cuuint64_t)c.P.nn[0], (cuuint64_t)c.P.nn[1], (cuuint64_t)c.P.nn[2]};
    const cuuint64_t strides[3] = {esz * ns, esz * ns * c.P.nn[0], esz * ns * c.P.nn[0] * c.P.nn[1]};
    const cuuint32_t box[4] = {(cuuint32_t)ns, (cuuint32_t)c.P.B, (cuuint32_t)c.P.B, (cuuint32_t)c.P.B};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode(&c.tmap, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                              c.rec, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        cudaFree(c.rec);
        c.rec = nullptr;
        return;
    }
    c.tma = true;
    if (f64)
        reinterpret_cast<Nodes<double> *>(c.nodes)->rec = reinterpret_cast<double *>(c.rec);
    else
        reinterpret_cast<Nodes<float> *>(c.nodes)->rec = reinterpret_cast<float *>(c.rec);
}

void drop_graphs(Ctx &c) {
    for (int k = 0; k < 2; ++k) {
        if (c.gexec[k]) cudaGraphExecDestroy(c.gexec[k]);
        c.gexec[k] = nullptr;
        c.warm[k] = false;
    }
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int exg_ctx_create(const exg_specs *specs, int device, exg_ctx **out) {
    if (!specs || !out) return EXG_ERR_ARG;
    *out = nullptr;
    std::string v = validate(*specs);
    if (!v.empty()) {
        fprintf(stderr, "exg_ctx_create: %s\n", v.c_str());
        return EXG_ERR_CONFIG;
    }
    exg_ctx *ctx = new exg_ctx();
    Ctx &c = ctx->c;
    try {
        c.specs = *specs;
        c.precision = specs->precision;
        c.timing = std::getenv("EXG_STAGE_TIMING") != nullptr;
        c.device = device;
        EXG_CUDA_OK(cudaSetDevice(device));
        EXG_CUDA_OK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        upload_tables_fp64();
        upload_tables_fp32();
        build_params(c);
        const size_t esz = fp64(c) ? 8 : 4;
        // nodes: 26 reference components, dense
        if (fp64(c)) {
            auto *N = new Nodes<double>();
            for (int k = 0; k < EXG_N_NCOMP; ++k) {
                N->c[k] = dalloc<double>(c.P.nnodes);
                c.node_allocs.push_back(N->c[k]);
            }
            c.nodes = N;
        } else {
            auto *N = new Nodes<float>();
            for (int k = 0; k < EXG_N_NCOMP; ++k) {
                N->c[k] = dalloc<float>(c.P.nnodes);
                c.node_allocs.push_back(N->c[k]);
            }
            c.nodes = N;
        }
        for (void *p : c.node_allocs) EXG_CUDA_OK(cudaMemset(p, 0, esz * c.P.nnodes));
        setup_node_records(c);
        c.ctl = dalloc<Ctl>(1);
        EXG_CUDA_OK(cudaMemset(c.ctl, 0, sizeof(Ctl)));
        EXG_CUDA_OK(cudaMallocHost(&c.ctl_host, sizeof(Ctl)));
        c.bounds_cur = dalloc<unsigned long long>(CH_ALL);
        c.bounds2 = dalloc<unsigned long long>(CH_ALL);
        c.dtmin2 = dalloc<unsigned long long>(1);
        c.diag_dev = nullptr;
        // sort and tile buffers
        const long long nt = c.P.ntiles;
        c.sb.tile_count = dalloc<int>(nt);
        c.sb.tile_fill = dalloc<int>(nt);
        c.sb.tile_start = dalloc<int>(nt);
        c.sb.active = dalloc<int>(nt);
        c.sb.slot = dalloc<int>(nt);
        c.sb.touched = dalloc<int>(nt);
        c.sb.touched_step = dalloc<long long>(nt);
        c.sb.cell_start = dalloc<int>((size_t)nt * (c.P.T * c.P.T * c.P.T + 1));
        c.sb.item_start = dalloc<int>(nt + 1);
        EXG_CUDA_OK(cudaMemset(c.sb.touched_step, 0xff, sizeof(long long) * nt));  // -1: never
        EXG_CUDA_OK(cudaMemset(c.sb.slot, 0xff, sizeof(int) * nt));
        c.nch = specs->use_temp ? CH_ALL : CH_MOM_END;
        const long long B3 = (long long)c.P.B * c.P.B * c.P.B;
        c.staging_cap = (size_t)nt;
        c.staging = dalloc<long long>((size_t)nt * (c.precision == EXG_PREC_FP64 ? stg_stride<double>(c.nch * B3)
                                                                                 : stg_stride<float>(c.nch * B3)));
        if (specs->use_temp) {
            // thermal wall pass: one entry per node of each non-periodic face
            c.n_tface = 0;
            for (int d = 0; d < 3; ++d) {
                if (c.P.periodic[d]) continue;
                const int p0 = (d == 0) ? 1 : 0, p1 = (d == 2) ? 1 : 2;
                const long long n0 = c.P.periodic[p0] ? c.P.nc[p0] : c.P.nc[p0] + 1;
                const long long n1 = c.P.periodic[p1] ? c.P.nc[p1] : c.P.nc[p1] + 1;
                c.n_tface += 2 * n0 * n1;
            }
            if (c.n_tface) c.tface = dalloc<double>(c.n_tface);
            c.ttmp = dalloc<unsigned char>(esz * c.P.nnodes);
        }
        for (int k = 0; k < 6; ++k) EXG_CUDA_OK(cudaEventCreate(&c.ev[k]));
        // initial dt accumulators: "no particles"
        launch_reset_accum(c, &c.ctl->bound_bits[0], &c.ctl->dtmin_bits);
        sync(c);
    } catch (const std::exception &e) {
        fprintf(stderr, "exg_ctx_create: %s\n", e.what());
        exg_ctx_destroy(ctx);
        return EXG_ERR_CUDA;
    }
    *out = ctx;
    return EXG_OK;
}

int exg_ctx_destroy(exg_ctx *ctx) {
    if (!ctx) return EXG_OK;
    Ctx &c = ctx->c;
    drop_graphs(c);
    free_list(c.allocs_a);
    free_list(c.allocs_b);
    free_list(c.node_allocs);
    if (c.rec) cudaFree(c.rec);
    c.rec = nullptr;
    if (c.precision == EXG_PREC_FP64) {
        delete reinterpret_cast<Parts<double> *>(c.pa);
        delete reinterpret_cast<Parts<double> *>(c.pb);
        delete reinterpret_cast<Nodes<double> *>(c.nodes);
    } else {
        delete reinterpret_cast<Parts<float> *>(c.pa);
        delete reinterpret_cast<Parts<float> *>(c.pb);
        delete reinterpret_cast<Nodes<float> *>(c.nodes);
    }
    for (double *p : c.ls) cudaFree(p);
    for (auto &row : c.udf_tab)
        for (double *p : row) cudaFree(p);
    for (auto &row : c.udfT_tab)
        for (double *p : row) cudaFree(p);
    cudaFree(c.tface);
    cudaFree(c.ttmp);
    void *bufs[] = {c.sb.key, c.sb.perm, c.sb.bucket, c.sb.tile_count, c.sb.tile_fill, c.sb.tile_start,
                    c.sb.active, c.sb.slot, c.sb.touched, c.sb.touched_step, c.sb.cell_start, c.sb.item_start,
                    c.staging, c.ctl,
                    c.bounds_cur, c.bounds2, c.dtmin2, c.mat_dev, c.diag_dev, c.stage};
    for (void *p : bufs) cudaFree(p);
    if (c.ctl_host) cudaFreeHost(c.ctl_host);
    for (auto &e : c.ev)
        if (e) cudaEventDestroy(e);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete ctx;
    return EXG_OK;
}

const char *exg_last_error(const exg_ctx *ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int exg_synchronize(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    EXG_TRY(ctx, sync(ctx->c));
    return EXG_OK;
}

int exg_check_status(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    EXG_TRY(ctx, return status_from_ctl(ctx->c));
}

}  // extern "C"

namespace {

// Level set of one body as the union of analytic shapes, one thread per node
// (node coordinates plo + i dx as the host builder forms them).
__global__ void k_levelset_shapes(const exg_ls_shape *shapes, int nshapes, int nx, int ny, int nz, double plo0,
                                  double plo1, double plo2, double dx0, double dx1, double dx2, double *phi) {
    const long long nn = (long long)nx * ny * nz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn;
         n += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / ((long long)nx * ny));
        phi[n] = exg_ls_union_eval(shapes, nshapes, exg_ls_node_x(plo0, i, dx0), exg_ls_node_x(plo1, j, dx1),
                                   exg_ls_node_x(plo2, k, dx2));
    }
}

}  // namespace

extern "C" {

int exg_levelset_build_device(exg_ctx *ctx, int body, const exg_ls_shape *shapes, int nshapes) {
    if (!ctx || body < 0 || body >= EXG_MAX_BODIES || !shapes || nshapes < 1) return EXG_ERR_ARG;
    for (int i = 0; i < nshapes; ++i) {
        const exg_ls_shape &sh = shapes[i];
        if (sh.kind < EXG_LS_SPHERE || sh.kind > EXG_LS_BOX) return fail(ctx, EXG_ERR_ARG, "unknown level-set shape");
        if (sh.kind == EXG_LS_CYLINDER && (sh.dir < 0 || sh.dir > 2))
            return fail(ctx, EXG_ERR_ARG, "cylinder_direction must be 0, 1 or 2");
        if (sh.kind == EXG_LS_PLANE && sh.normal[0] == 0.0 && sh.normal[1] == 0.0 && sh.normal[2] == 0.0)
            return fail(ctx, EXG_ERR_ARG, "plane_normal must not be zero");
    }
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        if (!c.ls[body]) c.ls[body] = dalloc<double>(c.P.nnodes);
        struct DevFree {
            void operator()(void *q) const { cudaFree(q); }
        };
        std::unique_ptr<exg_ls_shape, DevFree> dsh(dalloc<exg_ls_shape>(nshapes));
        EXG_CUDA_OK(cudaMemcpyAsync(dsh.get(), shapes, sizeof(exg_ls_shape) * nshapes, cudaMemcpyHostToDevice,
                                    c.stream));
        int nn[3];
        double dx[3];
        for (int d = 0; d < 3; ++d) {
            nn[d] = c.specs.ncells[d] + 1;
            dx[d] = (c.specs.phi[d] - c.specs.plo[d]) / c.specs.ncells[d];
        }
        const long long total = (long long)nn[0] * nn[1] * nn[2];
        const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
        k_levelset_shapes<<<grid, 256, 0, c.stream>>>(dsh.get(), nshapes, nn[0], nn[1], nn[2], c.specs.plo[0],
                                                       c.specs.plo[1], c.specs.plo[2], dx[0], dx[1], dx[2],
                                                       c.ls[body]);
        EXG_CUDA_OK(cudaGetLastError());
        EXG_CUDA_OK(cudaStreamSynchronize(c.stream));
        drop_graphs(c);
    });
    return EXG_OK;
}

int exg_init_levelsets(exg_ctx *ctx, const exg_inputs *in) {
    if (!ctx || !in) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    std::vector<double> host;
    for (int b = 0; b < c.specs.num_bodies; ++b) {
        exg_ls_shape sh;
        const int rc = exg_levelset_shape(in, b, &sh);
        if (rc == EXG_OK) {
            const int r2 = exg_levelset_build_device(ctx, b, &sh, 1);
            if (r2 != EXG_OK) return r2;
        } else if (rc == EXG_ERR_UNSUPPORTED) {
            // udf_cpp: the user's levelset_phi runs on the host
            if (host.empty()) host.resize(c.P.nnodes);
            const int r2 = exg_levelset_build(in, &c.specs, b, host.data());
            if (r2 != EXG_OK) return fail(ctx, r2, "level set of body " + std::to_string(b) + " cannot be built");
            const int r3 = exg_set_levelset(ctx, b, host.data());
            if (r3 != EXG_OK) return r3;
        } else {
            return fail(ctx, rc, "level set of body " + std::to_string(b) + " has a bad geometry");
        }
    }
    return EXG_OK;
}

int exg_get_levelset(exg_ctx *ctx, int body, double *phi) {
    if (!ctx || body < 0 || body >= EXG_MAX_BODIES || !phi) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (!c.ls[body]) return fail(ctx, EXG_ERR_NOT_READY, "body " + std::to_string(body) + " has no level set");
    EXG_TRY(ctx, {
        EXG_CUDA_OK(cudaStreamSynchronize(c.stream));
        EXG_CUDA_OK(cudaMemcpy(phi, c.ls[body], sizeof(double) * c.P.nnodes, cudaMemcpyDeviceToHost));
    });
    return EXG_OK;
}

int exg_set_levelset(exg_ctx *ctx, int body, const double *phi) {
    if (!ctx || body < 0 || body >= EXG_MAX_BODIES || !phi) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        if (!c.ls[body]) c.ls[body] = dalloc<double>(c.P.nnodes);
        EXG_CUDA_OK(cudaMemcpy(c.ls[body], phi, sizeof(double) * c.P.nnodes, cudaMemcpyHostToDevice));
        drop_graphs(c);
    });
    return EXG_OK;
}

int exg_particles_upload(exg_ctx *ctx, const exg_particle_soa *p) {
    EXG_RANGE("exg_particles_upload");
    if (!ctx || !p || p->np < 0) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (p->np > (long long)0x7fffffff) return fail(ctx, EXG_ERR_ARG, "more than 2^31-1 particles");
    EXG_TRY(ctx, {
        const long long n = p->np;
        // material table: one entry per distinct (E, nu, K, gamma, mu, model)
        std::map<std::tuple<double, double, double, double, double, int>, int> idx;
        std::vector<int32_t> mat(n);
        const bool lean_before = g2p_lean(c);
        c.mats.clear();
        using Key = std::tuple<double, double, double, double, double, int>;
        auto key_of = [&](long long i) {
            return std::make_tuple(p->rdata[(size_t)EXG_R_E * n + i], p->rdata[(size_t)EXG_R_NU * n + i],
                                   p->rdata[(size_t)EXG_R_BULK * n + i], p->rdata[(size_t)EXG_R_GAMMA * n + i],
                                   p->rdata[(size_t)EXG_R_VISC * n + i], (int)p->idata[(size_t)EXG_I_MODEL * n + i]);
        };
        // per chunk: its distinct materials in order of first appearance and
        // chunk-local indices (runs of one material need no lookup); the
        // merge in chunk order numbers the materials by first appearance
        const int nch = host_chunks(n);
        std::vector<std::vector<Key>> local(nch);
        parallel_chunks(n, nch, [&](int t, long long a, long long b) {
            std::vector<Key> &keys = local[t];
            Key last;
            int last_id = -1;
            for (long long i = a; i < b; ++i) {
                const Key key = key_of(i);
                if (last_id >= 0 && key == last) {
                    mat[i] = last_id;
                    continue;
                }
                int id = -1;
                for (size_t q = 0; q < keys.size(); ++q)
                    if (keys[q] == key) {
                        id = (int)q;
                        break;
                    }
                if (id < 0) {
                    id = (int)keys.size();
                    keys.push_back(key);
                }
                mat[i] = id;
                last = key;
                last_id = id;
            }
        });
        std::vector<std::vector<int32_t>> trans(nch);
        for (int t = 0; t < nch; ++t)
            for (const Key &key : local[t]) {
                const int model = std::get<5>(key);
                if (model < 0 || model > 2)
                    return fail(ctx, EXG_ERR_UNSUPPORTED, "unknown constitutive model " + std::to_string(model));
                if (model != 0 && c.specs.calculate_strain_based_on_delta == 1)
                    // apply_constitutive_model_delta aborts on these models
                    // (mpm_particle_container.cpp:251-262)
                    return fail(ctx, EXG_ERR_UNSUPPORTED, "calculate_strain_based_on_delta = 1 supports the "
                                                          "linear-elastic model only");
                auto it = idx.find(key);
                if (it == idx.end()) {
                    Material m;
                    std::tie(m.E, m.nu, m.K, m.gamma, m.mu, m.model) = key;
                    m.ipow = (m.gamma >= 1.0 && m.gamma <= 16.0 && m.gamma == std::floor(m.gamma)) ? (int)m.gamma
                                                                                                       : 0;
                    if (m.model == 1) {
                        m.pmod = m.K;
                    } else {
                        const double lambda = m.E * m.nu / ((1 + m.nu) * (1 - 2.0 * m.nu));
                        const double mu = m.E / (2.0 * (1 + m.nu));
                        m.pmod = lambda + 2.0 * mu;
                    }
                    it = idx.emplace(key, (int)c.mats.size()).first;
                    c.mats.push_back(m);
                }
                trans[t].push_back(it->second);
            }
        parallel_chunks(n, nch, [&](int t, long long a, long long b) {
            const std::vector<int32_t> &tr = trans[t];
            for (long long i = a; i < b; ++i) mat[i] = tr[mat[i]];
        });
        if (c.mats.empty()) c.mats.push_back(Material{});
        if (!c.mat_dev || c.mat_cap < c.mats.size()) {
            if (c.mat_dev) cudaFree(c.mat_dev);
            c.mat_dev = dalloc<Material>(c.mats.size());
            c.mat_cap = c.mats.size();
            drop_graphs(c);  // the step graphs hold the table's address
        }
        EXG_CUDA_OK(cudaMemcpy(c.mat_dev, c.mats.data(), sizeof(Material) * c.mats.size(), cudaMemcpyHostToDevice));
        const bool temp = c.specs.use_temp != 0;
        if (g2p_lean(c) != lean_before) drop_graphs(c);  // the graphs hold the other G2P variant
        if (c.pa && n == c.np && n == c.cap) {
            // same particle count: the storage, sort buffers and step graphs stay
            if (fp64(c))
                upload_parts<double>(c, p, mat);
            else
                upload_parts<float>(c, p, mat);
            set_tref(c, p);
            c.parts_sorted = false;
            c.reordered = false;
            c.reduce_stale = true;
            sync(c);
            return EXG_OK;
        }
        // particle storage (re-allocated when the count changes)
        free_list(c.allocs_a);
        free_list(c.allocs_b);
        drop_graphs(c);
        if (c.orient) std::swap(c.pa, c.pb);
        c.orient = 0;
        if (c.stage_cap < n) {  // one FP64 field for the host transfers
            cudaFree(c.stage);
            c.stage = dalloc<double>(n > 0 ? n : 1);
            c.stage_cap = n;
        }
        if (fp64(c)) {
            delete reinterpret_cast<Parts<double> *>(c.pa);
            delete reinterpret_cast<Parts<double> *>(c.pb);
            auto *a = new Parts<double>(), *b = new Parts<double>();
            alloc_parts<double>(c, *a, c.allocs_a, n, temp, nullptr);
            alloc_parts<double>(c, *b, c.allocs_b, n, temp, a);
            c.pa = a;
            c.pb = b;
            c.np = n;
            upload_parts<double>(c, p, mat);
        } else {
            delete reinterpret_cast<Parts<float> *>(c.pa);
            delete reinterpret_cast<Parts<float> *>(c.pb);
            auto *a = new Parts<float>(), *b = new Parts<float>();
            alloc_parts<float>(c, *a, c.allocs_a, n, temp, nullptr);
            alloc_parts<float>(c, *b, c.allocs_b, n, temp, a);
            c.pa = a;
            c.pb = b;
            c.np = n;
            upload_parts<float>(c, p, mat);
        }
        set_tref(c, p);
        c.cap = n;
        cudaFree(c.sb.key);
        cudaFree(c.sb.perm);
        cudaFree(c.sb.bucket);
        c.sb.key = dalloc<uint32_t>(n);
        c.sb.perm = dalloc<int32_t>(n);
        c.sb.bucket = dalloc<int32_t>(2 * n);
        c.parts_sorted = false;
        c.reordered = false;
        c.reduce_stale = true;
        sync(c);
    });
    return EXG_OK;
}

int exg_particles_download(exg_ctx *ctx, exg_particle_soa *p) {
    EXG_RANGE("exg_particles_download");
    if (!ctx || !p) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (p->np != c.np) return fail(ctx, EXG_ERR_ARG, "np mismatch");
    EXG_TRY(ctx, {
        sync(c);
        if (fp64(c))
            download_parts<double>(c, p);
        else
            download_parts<float>(c, p);
    });
    return EXG_OK;
}

int exg_particles_alloc_pinned(int64_t np, exg_particle_soa *p) {
    if (!p || np < 0) return EXG_ERR_ARG;
    p->np = np;
    p->pos = p->rdata = nullptr;
    p->idata = nullptr;
    const size_t n = (size_t)(np > 0 ? np : 1);
    if (cudaMallocHost(&p->pos, 3 * n * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&p->rdata, (size_t)EXG_NREAL * n * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&p->idata, (size_t)EXG_NINT * n * sizeof(int32_t)) != cudaSuccess) {
        exg_particles_free_pinned(p);
        return EXG_ERR_ALLOC;
    }
    std::memset(p->pos, 0, 3 * n * sizeof(double));
    std::memset(p->rdata, 0, (size_t)EXG_NREAL * n * sizeof(double));
    std::memset(p->idata, 0, (size_t)EXG_NINT * n * sizeof(int32_t));
    return EXG_OK;
}

void exg_particles_free_pinned(exg_particle_soa *p) {
    if (!p) return;
    if (p->pos) cudaFreeHost(p->pos);
    if (p->rdata) cudaFreeHost(p->rdata);
    if (p->idata) cudaFreeHost(p->idata);
    p->pos = p->rdata = nullptr;
    p->idata = nullptr;
    p->np = 0;
}

int exg_num_particles(exg_ctx *ctx, int64_t *np) {
    if (!ctx || !np) return EXG_ERR_ARG;
    *np = ctx->c.np;
    return EXG_OK;
}

int exg_nodes_download(exg_ctx *ctx, int comp, double *out) {
    if (!ctx || !out || comp < 0 || comp >= EXG_N_NCOMP) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        sync(c);
        const long long n = c.P.nnodes;
        if (fp64(c)) {
            EXG_CUDA_OK(cudaMemcpy(out, c.N<double>().c[comp], sizeof(double) * n, cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> b(n);
            EXG_CUDA_OK(cudaMemcpy(b.data(), c.N<float>().c[comp], sizeof(float) * n, cudaMemcpyDeviceToHost));
            for (long long i = 0; i < n; ++i) out[i] = b[i];
        }
        // nodal temperatures are stored relative to Tref (FP32 state)
        if (c.P.Tref != 0.0 && (comp == EXG_N_TEMPERATURE || comp == EXG_N_MASS_SPHEAT_TEMP)) {
            std::vector<double> mc;
            if (comp == EXG_N_MASS_SPHEAT_TEMP) {
                std::vector<float> b(n);
                EXG_CUDA_OK(cudaMemcpy(b.data(), c.N<float>().c[EXG_N_MASS_SPHEAT], sizeof(float) * n,
                                       cudaMemcpyDeviceToHost));
                mc.assign(b.begin(), b.end());
            }
            for (long long i = 0; i < n; ++i) out[i] += c.P.Tref * (comp == EXG_N_TEMPERATURE ? 1.0 : mc[i]);
        }
        // periodic axes: node ncells is node 0
        const int *nn = c.P.nn;
        for (int k = 0; k < nn[2]; ++k)
            for (int j = 0; j < nn[1]; ++j)
                for (int i = 0; i < nn[0]; ++i) {
                    int w[3] = {i, j, k};
                    bool alias = false;
                    for (int d = 0; d < 3; ++d)
                        if (c.P.periodic[d] && w[d] == c.P.nc[d]) {
                            w[d] = 0;
                            alias = true;
                        }
                    if (alias)
                        out[((long long)k * nn[1] + j) * nn[0] + i] = out[((long long)w[2] * nn[1] + w[1]) * nn[0] + w[0]];
                }
    });
    return EXG_OK;
}

// ----------------------------------------------------- L5 step functions
int exg_redistribute(exg_ctx *ctx) {
    EXG_RANGE("Redistribute");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->lost, 0, sizeof(unsigned long long), c.stream));
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->maxppc, 0, sizeof(int), c.stream));
        do_sort(c, false);
        ctl_pull(c);
        if (c.ctl_host->lost) {
            c.err = std::to_string(c.ctl_host->lost) + " particles are outside the domain";
            return EXG_ERR_DOMAIN;
        }
    });
    return EXG_OK;
}

int exg_calculate_time_step(exg_ctx *ctx, double *dt) {
    EXG_RANGE("Calculate_time_step");
    if (!ctx || !dt) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        do_reduce(c);
        launch_dt_finalize(c, false);
        ctl_pull(c);
        *dt = c.ctl_host->dt;
    });
    return EXG_OK;
}

int exg_reset_nodaldata(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    EXG_TRY(ctx, launch_node_reset(ctx->c));
    return EXG_OK;
}

int exg_p2g_momentum(exg_ctx *ctx, int update_mass, int update_vel, int update_forces) {
    EXG_RANGE("P2G_Momentum");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (c.np == 0) return fail(ctx, EXG_ERR_NOT_READY, "no particles");
    EXG_TRY(ctx, {
        int flags = (update_mass ? PF_MASS : 0) | (update_vel ? PF_VEL : 0) | (update_forces ? PF_FORCE : 0);
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->maxppc, 0, sizeof(int), c.stream));
        do_sort(c, false);
        launch_reset_accum(c, c.bounds2, c.dtmin2);
        DISPATCH(launch_state_reduce, c, c.bounds2, c.dtmin2);
        launch_scales_from(c, c.bounds2);
        if (flags) {
            DISPATCH(launch_p2g, c, flags);
            DISPATCH(launch_nodes, c, NM_MERGE, flags, true);
        }
        return status_from_ctl(c);
    });
}

int exg_backup_current_velocity(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, DISPATCH(launch_node_backup, c));
    return EXG_OK;
}

int exg_nodal_time_update_momentum(exg_ctx *ctx, double dt) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, DISPATCH(launch_node_time_update, c, dt));
    return EXG_OK;
}

int exg_apply_nodal_bcs(exg_ctx *ctx, double dt, double time) {
    EXG_RANGE("Apply_Nodal_BCs");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    (void)dt;
    EXG_TRY(ctx, {
        tabulate_udf(c, time);
        DISPATCH(launch_node_bcs, c);
        return status_from_ctl(c);
    });
}

int exg_g2p_momentum(exg_ctx *ctx, int update_vel, int update_strainrate, double dt) {
    EXG_RANGE("G2P_Momentum");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        DISPATCH(launch_g2p_simple, c, update_vel, update_strainrate, dt);
        c.reduce_stale = true;
    });
    return EXG_OK;
}

int exg_update_mp_positions(exg_ctx *ctx, double dt) {
    EXG_RANGE("Update_MP_Positions");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        DISPATCH(launch_move, c, dt);
        c.parts_sorted = false;
        c.reduce_stale = true;
        return status_from_ctl(c);
    });
}

int exg_update_mp_volume(exg_ctx *ctx) {
    EXG_RANGE("Update_MP_Volume");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        DISPATCH(launch_volume, c);
        c.reduce_stale = true;
    });
    return EXG_OK;
}

int exg_calculate_mp_stress_strain(exg_ctx *ctx, double time, double dt) {
    EXG_RANGE("Calculate_MP_Stress_Strain");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        DISPATCH(launch_stress, c, time, dt);
        c.reduce_stale = true;
    });
    return EXG_OK;
}

int exg_init_internal_forces(exg_ctx *ctx) {
    EXG_RANGE("Initialise_Internal_Forces");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    int rc = exg_p2g_momentum(ctx, 1, 1, 1);
    if (rc) return rc;
    rc = exg_backup_current_velocity(ctx);
    if (rc) return rc;
    rc = exg_g2p_momentum(ctx, 0, 1, 0.0);
    if (rc) return rc;
    // apply_constitutive_model(dt = 0, applied_strainrate) (mpm_init.cpp:398)
    EXG_TRY(ctx, {
        if (c.np)
            fp64(c) ? launch_stress_fp64(c, -INFINITY, 0.0, true) : launch_stress_fp32(c, -INFINITY, 0.0, true);
        c.reduce_stale = true;
        sync(c);
    });
    if (!c.specs.use_temp) return EXG_OK;
    // thermal prologue (mpm_init.cpp:411-441): deposit without source,
    // backup, domain-wall BCs only (nodal_bcs_temperature), store delta, G2P
    if ((rc = exg_p2g_temperature(ctx, 1, 1, 0))) return rc;
    if ((rc = exg_backup_current_temperature(ctx))) return rc;
    EXG_TRY(ctx, {
        DISPATCH(launch_temp_bcs, c, TW_ON, 0, 0, 0);
        rc = status_from_ctl(c);
    });
    if (rc) return rc;
    if ((rc = exg_store_delta_temperature(ctx))) return rc;
    return exg_g2p_temperature(ctx, 1, 1);
}

static int need_temp(exg_ctx *ctx) {
    return ctx->c.specs.use_temp ? EXG_OK
                                 : fail(ctx, EXG_ERR_NOT_READY, "thermal step function without mpm.use_temp");
}

int exg_p2g_temperature(exg_ctx *ctx, int reset, int update_temp, int update_source) {
    EXG_RANGE("P2G_Temperature");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    if (c.np == 0) return fail(ctx, EXG_ERR_NOT_READY, "no particles");
    if (!reset)
        return fail(ctx, EXG_ERR_UNSUPPORTED, "P2G_Temperature without reset (the reference always resets)");
    EXG_TRY(ctx, {
        const int flags = (update_temp ? PF_TEMP : 0) | (update_source ? PF_SRC : 0);
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->maxppc, 0, sizeof(int), c.stream));
        do_sort(c, false);
        launch_reset_accum(c, c.bounds2, c.dtmin2);
        DISPATCH(launch_state_reduce, c, c.bounds2, c.dtmin2);
        launch_scales_from(c, c.bounds2);
        if (flags) {
            DISPATCH(launch_p2g, c, flags);
            DISPATCH(launch_nodes, c, NM_MERGE, flags, true);
        } else {  // reset only
            const size_t esz = fp64(c) ? 8 : 4;
            for (int comp : {EXG_N_MASS_SPHEAT, EXG_N_MASS_SPHEAT_TEMP, EXG_N_SOURCE_TEMP}) {
                void *a = fp64(c) ? (void *)c.N<double>().c[comp] : (void *)c.N<float>().c[comp];
                EXG_CUDA_OK(cudaMemsetAsync(a, 0, esz * c.P.nnodes, c.stream));
            }
        }
        return status_from_ctl(c);
    });
}
int exg_backup_current_temperature(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    EXG_TRY(ctx, DISPATCH(launch_temp_node_op, c, TN_BACKUP, 0.0));
    return EXG_OK;
}
int exg_nodal_time_update_temperature(exg_ctx *ctx, double dt) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    EXG_TRY(ctx, DISPATCH(launch_temp_node_op, c, TN_TIME_UPDATE, dt));
    return EXG_OK;
}
int exg_apply_nodal_bcs_temperature(exg_ctx *ctx, double dt, double time, int dirichlet_only) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    (void)dt;
    EXG_TRY(ctx, {
        tabulate_udf_temp(c, time);
        DISPATCH(launch_temp_bcs, c, TW_ON, has_udf_temp(c) ? 1 : 0, 1, dirichlet_only ? 1 : 0);
        return status_from_ctl(c);
    });
}
int exg_store_delta_temperature(exg_ctx *ctx) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    EXG_TRY(ctx, DISPATCH(launch_temp_node_op, c, TN_DELTA, 0.0));
    return EXG_OK;
}
int exg_g2p_temperature(exg_ctx *ctx, int update_temperature, int update_heatflux) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (int rc = need_temp(ctx)) return rc;
    EXG_TRY(ctx, {
        DISPATCH(launch_g2p_temp, c, update_temperature, update_heatflux);
        c.reduce_stale = true;
    });
    return EXG_OK;
}

// ------------------------------------------------------------ fused step
}  // extern "C"

namespace {
// Tuning choices shared by the contexts of one process: (device, precision,
// order, tile, lean G2P, particle-count decade) -> (p2g, g2p) variants.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int>, std::pair<int, int>> g_tune_cache;

std::tuple<int, int, int, int, int, int> tune_key(const Ctx &c) {
    const int decade = c.np > 0 ? (int)std::floor(std::log10((double)c.np)) : 0;
    return {c.device, c.precision, c.P.uniform_order, c.P.T, g2p_lean(c) ? 1 : 0, decade};
}

// Mean device ms of `reps` launches of fn() after one untimed launch.
template <class F>
double time_launches(Ctx &c, int reps, F fn) {
    cudaEvent_t e0, e1;
    EXG_CUDA_OK(cudaEventCreate(&e0));
    EXG_CUDA_OK(cudaEventCreate(&e1));
    fn();
    EXG_CUDA_OK(cudaEventRecord(e0, c.stream));
    for (int r = 0; r < reps; ++r) fn();
    EXG_CUDA_OK(cudaEventRecord(e1, c.stream));
    EXG_CUDA_OK(cudaEventSynchronize(e1));
    float ms = 0.f;
    EXG_CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)ms / reps;
}

// Times every P2G and G2P variant on the current particles.  The P2G writes
// only the staging blocks; the nodal pass that follows rebuilds the nodal
// fields the G2P reads; the G2P writes only the re-order target storage and
// the control block's reductions, which are saved before and restored after.
void autotune_impl(Ctx &c) {
    Ctl *saved = nullptr;
    EXG_CUDA_OK(cudaMalloc(&saved, sizeof(Ctl)));
    EXG_CUDA_OK(cudaMemcpyAsync(saved, c.ctl, sizeof(Ctl), cudaMemcpyDeviceToDevice, c.stream));
    const int p2g0 = c.p2g_var, g2p0 = c.g2p_var;
    try {
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->maxppc, 0, sizeof(int), c.stream));
        do_sort(c, true);
        launch_reset_accum(c, c.bounds2, c.dtmin2);
        DISPATCH(launch_state_reduce, c, c.bounds2, c.dtmin2);
        const int flags = PF_MASS | PF_VEL | PF_FORCE;
        for (int v = 0; v < EXG_NUM_VARIANTS; ++v) {
            c.p2g_var = v;
            c.tune_ms[0][v] = time_launches(c, 3, [&] {
                launch_scales_from(c, c.bounds2);  // also resets the P2G tile counter
                DISPATCH(launch_p2g, c, flags);
            });
        }
        DISPATCH(launch_nodes, c, NM_FUSED, flags, false);
        for (int v = 0; v < EXG_NUM_VARIANTS; ++v) {
            c.g2p_var = v;
            c.tune_ms[1][v] = time_launches(c, 3, [&] {
                EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->next_g2p, 0, sizeof(int), c.stream));
                DISPATCH(launch_g2p_fused, c, GM_FULL);
            });
        }
    } catch (...) {
        c.p2g_var = p2g0;
        c.g2p_var = g2p0;
        cudaMemcpyAsync(c.ctl, saved, sizeof(Ctl), cudaMemcpyDeviceToDevice, c.stream);
        cudaStreamSynchronize(c.stream);
        cudaFree(saved);
        throw;
    }
    EXG_CUDA_OK(cudaMemcpyAsync(c.ctl, saved, sizeof(Ctl), cudaMemcpyDeviceToDevice, c.stream));
    EXG_CUDA_OK(cudaStreamSynchronize(c.stream));
    EXG_CUDA_OK(cudaFree(saved));
    c.p2g_var = (int)(std::min_element(c.tune_ms[0], c.tune_ms[0] + EXG_NUM_VARIANTS) - c.tune_ms[0]);
    c.g2p_var = (int)(std::min_element(c.tune_ms[1], c.tune_ms[1] + EXG_NUM_VARIANTS) - c.tune_ms[1]);
    c.parts_sorted = false;
    c.tuned = true;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key(c)] = {c.p2g_var, c.g2p_var};
}

// The choice for this context: the process cache when it holds one for this
// kind of context, otherwise a tuning run, but only on particles in the
// order a fused step leaves them (right after an upload they are in the
// caller's order, whose scattered loads would rank the variants wrongly; the
// first step then runs with the current variants, which give the same
// results).  Graphs captured with other variants are dropped.
void ensure_tuned(Ctx &c) {
    if (c.tuned) return;
    const int p0 = c.p2g_var, g0 = c.g2p_var;
    bool hit = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(tune_key(c));
        if (it != g_tune_cache.end()) {
            c.p2g_var = it->second.first;
            c.g2p_var = it->second.second;
            hit = true;
        }
    }
    if (hit)
        c.tuned = true;
    else if (c.reordered)
        autotune_impl(c);
    if (c.p2g_var != p0 || c.g2p_var != g0) drop_graphs(c);
}
}  // namespace

extern "C" {

int exg_autotune(exg_ctx *ctx) {
    EXG_RANGE("exg_autotune");
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (c.np == 0) return fail(ctx, EXG_ERR_NOT_READY, "no particles");
    EXG_TRY(ctx, {
        const int p0 = c.p2g_var, g0 = c.g2p_var;
        autotune_impl(c);
        if (c.p2g_var != p0 || c.g2p_var != g0) drop_graphs(c);
    });
    return EXG_OK;
}

int exg_set_variants(exg_ctx *ctx, int p2g, int g2p) {
    if (!ctx || p2g < -1 || p2g >= EXG_NUM_VARIANTS || g2p < -1 || g2p >= EXG_NUM_VARIANTS) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    const int p0 = c.p2g_var, g0 = c.g2p_var;
    if (p2g >= 0) c.p2g_var = p2g;
    if (g2p >= 0) c.g2p_var = g2p;
    c.tuned = true;
    EXG_TRY(ctx, if (c.p2g_var != p0 || c.g2p_var != g0) drop_graphs(c));
    return EXG_OK;
}

int exg_get_variants(exg_ctx *ctx, int *p2g, int *g2p, double *p2g_ms, double *g2p_ms) {
    if (!ctx) return EXG_ERR_ARG;
    const Ctx &c = ctx->c;
    if (p2g) *p2g = c.p2g_var;
    if (g2p) *g2p = c.g2p_var;
    for (int v = 0; v < EXG_NUM_VARIANTS; ++v) {
        if (p2g_ms) p2g_ms[v] = c.tune_ms[0][v];
        if (g2p_ms) g2p_ms[v] = c.tune_ms[1][v];
    }
    return EXG_OK;
}

int exg_step(exg_ctx *ctx, int nsteps) {
    EXG_RANGE("exg_step");
    if (!ctx || nsteps < 0) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    if (c.np == 0) return fail(ctx, EXG_ERR_NOT_READY, "no particles");
    EXG_TRY(ctx, {
        const bool tune = c.specs.autotune && nsteps > 0;
        if (tune) ensure_tuned(c);
        if (c.reduce_stale) do_reduce(c);
        const bool host_dep = has_udf(c) || (c.specs.use_temp && has_udf_temp(c));
        const bool use_graph = !host_dep && !c.timing && std::getenv("EXG_NO_GRAPH") == nullptr;
        for (int s = 0; s < nsteps; ++s) {
            if (tune && !c.tuned && c.reordered) ensure_tuned(c);
            if (host_dep) {
                // UDF wall tables depend on the step's start time: tabulate on
                // the host before the step's kernels.
                ctl_pull(c);
                tabulate_udf(c, c.ctl_host->time);
                if (c.specs.use_temp) tabulate_udf_temp(c, c.ctl_host->time);
            }
            if (use_graph) {
                cudaGraphExec_t &g = c.gexec[c.orient];
                if (!g) {
                    if (!c.warm[c.orient]) {
                        // first step of each orientation runs eagerly (kernel
                        // attributes, occupancy queries), later ones replay
                        enqueue_step(c);
                        c.warm[c.orient] = true;
                        swap_parts(c);
                        c.reordered = true;
                        continue;
                    }
                    cudaGraph_t graph = nullptr;
                    EXG_CUDA_OK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
                    enqueue_step(c);
                    EXG_CUDA_OK(cudaStreamEndCapture(c.stream, &graph));
                    EXG_CUDA_OK(cudaGraphInstantiate(&g, graph, 0));
                    cudaGraphDestroy(graph);
                }
                EXG_CUDA_OK(cudaGraphLaunch(g, c.stream));
                swap_parts(c);
                c.reordered = true;
            } else {
                enqueue_step(c);
                swap_parts(c);
                c.reordered = true;
                if (c.timing) {
                    sync(c);
                    float ms[4];
                    for (int k = 0; k < 4; ++k) EXG_CUDA_OK(cudaEventElapsedTime(&ms[k], c.ev[k], c.ev[k + 1]));
                    for (int k = 0; k < 4; ++k) c.stage_ms[k] += ms[k];
                    c.stage_ms[4] += 1.0;
                }
            }
        }
        c.parts_sorted = false;
        int rc = status_from_ctl(c);
        c.host_time = c.ctl_host->time;
        c.host_dt = c.ctl_host->dt;
        c.host_steps = c.ctl_host->steps;
        return rc;
    });
}

int exg_get_time(exg_ctx *ctx, double *time, double *last_dt, int64_t *steps) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        ctl_pull(c);
        if (time) *time = c.ctl_host->time;
        if (last_dt) *last_dt = c.ctl_host->dt;
        if (steps) *steps = c.ctl_host->steps;
    });
    return EXG_OK;
}

int exg_set_time(exg_ctx *ctx, double time, int64_t steps) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        ctl_pull(c);
        c.ctl_host->time = time;
        c.ctl_host->steps = steps;
        EXG_CUDA_OK(cudaMemcpyAsync(&c.ctl->time, &c.ctl_host->time, sizeof(double), cudaMemcpyHostToDevice, c.stream));
        EXG_CUDA_OK(
            cudaMemcpyAsync(&c.ctl->steps, &c.ctl_host->steps, sizeof(long long), cudaMemcpyHostToDevice, c.stream));
        sync(c);
    });
    return EXG_OK;
}

int exg_diagnostics(exg_ctx *ctx, exg_diag *out) {
    EXG_RANGE("Do_All_Diagnostics");
    if (!ctx || !out) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        const long long nb = (std::max<long long>(c.np, 1) + 255) / 256;
        if (!c.diag_dev || (long long)c.staging_cap < 0) c.diag_dev = dalloc<double>(32 + 16 * nb);
        static long long diag_cap = 0;
        if (nb > diag_cap) {
            cudaFree(c.diag_dev);
            c.diag_dev = dalloc<double>(32 + 16 * nb);
            diag_cap = nb;
        }
        DISPATCH(launch_diag, c, c.diag_dev);
        double h[16];
        EXG_CUDA_OK(cudaMemcpyAsync(h, c.diag_dev, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        sync(c);
        std::memset(out, 0, sizeof(*out));
        out->tke = h[0];
        out->tse = h[1];
        out->mass = h[2];
        for (int d = 0; d < 3; ++d) {
            out->momentum[d] = h[3 + d];
            out->mwa_vel[d] = h[3 + d] / h[2];
            out->minpos[d] = h[9 + d];
            out->maxpos[d] = h[12 + d];
        }
        out->mwa_velmag = h[6] / h[2];
        out->np = (int64_t)h[15];
    });
    return EXG_OK;
}

int exg_sort_keys(exg_ctx *ctx, uint32_t *keys, int32_t *perm) {
    if (!ctx) return EXG_ERR_ARG;
    Ctx &c = ctx->c;
    EXG_TRY(ctx, {
        EXG_CUDA_OK(cudaMemsetAsync(&c.ctl->lost, 0, sizeof(unsigned long long), c.stream));
        do_sort(c, false);
        ctl_pull(c);
        const long long n = c.np;
        std::vector<uint32_t> k(n);
        EXG_CUDA_OK(cudaMemcpy(k.data(), c.sb.key, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        if (keys) std::copy(k.begin(), k.end(), keys);
        if (perm) {
            const long long ns = c.ctl_host->n_sorted;
            EXG_CUDA_OK(cudaMemcpy(perm, c.sb.perm, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost));
            long long q = ns;
            for (long long i = 0; i < n; ++i)
                if (k[i] == 0xFFFFFFFFu) perm[q++] = (int32_t)i;
        }
    });
    return EXG_OK;
}

int exg_tile_size(exg_ctx *ctx, int *tile) {
    if (!ctx || !tile) return EXG_ERR_ARG;
    *tile = ctx->c.P.T;
    return EXG_OK;
}

int exg_set_stage_timing(exg_ctx *ctx, int on) {
    if (!ctx) return EXG_ERR_ARG;
    ctx->c.timing = on != 0;
    for (double &v : ctx->c.stage_ms) v = 0.0;
    return EXG_OK;
}

int exg_last_step_timing(exg_ctx *ctx, double *ms5) {
    if (!ctx || !ms5) return EXG_ERR_ARG;
    const double n = ctx->c.stage_ms[4] > 0 ? ctx->c.stage_ms[4] : 1.0;
    for (int k = 0; k < 4; ++k) ms5[k] = ctx->c.stage_ms[k] / n;
    ms5[4] = ctx->c.stage_ms[4];
    return EXG_OK;
}

int exg_p2g_momentum_noalloc(const exg_specs *specs, const exg_particle_soa *dev_particles, double *node_mass,
                             double *node_vel, double *node_frc, void *stream) {
    if (!specs || !dev_particles || !node_mass || !node_vel || !node_frc || dev_particles->np < 0) return EXG_ERR_ARG;
    if (dev_particles->np > 0 && (!dev_particles->pos || !dev_particles->rdata || !dev_particles->idata))
        return EXG_ERR_ARG;
    const std::string v = validate(*specs);
    if (!v.empty()) {
        fprintf(stderr, "exg_p2g_momentum_noalloc: %s\n", v.c_str());
        return EXG_ERR_CONFIG;
    }
    std::string err;
    const int rc = noalloc_p2g(specs, dev_particles, node_mass, node_vel, node_frc, (cudaStream_t)stream, err);
    if (rc) fprintf(stderr, "%s\n", err.c_str());
    return rc;
}

int exg_get_stream(exg_ctx *ctx, void **stream) {
    if (!ctx || !stream) return EXG_ERR_ARG;
    *stream = (void *)ctx->c.stream;
    return EXG_OK;
}

// ------------------------------------------------------------ batches
namespace {
int bfail(exg_batch *B, int code, const std::string &msg) {
    if (B) B->err = msg;
    return code;
}
std::string batch_compatible(const exg_specs *s, int n) {
    for (int i = 0; i < n; ++i) {
        const exg_specs &x = s[i];
        if (x.use_temp) return "scene " + std::to_string(i) + ": batches run without temperature";
        if (x.stress_update_scheme != 0) return "scene " + std::to_string(i) + ": batches run the USL scheme";
        for (int d = 0; d < 3; ++d)
            if (x.udf_wallvel_lo[d] || x.udf_wallvel_hi[d])
                return "scene " + std::to_string(i) + ": UDF wall tables are not supported in batches";
        if (x.precision != s[0].precision) return "scenes must share exg.precision";
        if ((x.tile > 0 ? x.tile : 8) != (s[0].tile > 0 ? s[0].tile : 8)) return "scenes must share exg.tile";
        for (int d = 0; d < 3; ++d)
            if (x.order[d] != s[0].order[d]) return "scenes must share the B-spline order of every axis";
    }
    return "";
}
// One batch step: the batched sort and bookkeeping of every scene, the
// batched P2G, nodal and G2P kernels, the batched end of step -- a fixed
// sequence of launches whatever the number of scenes.
void enqueue_batch_step(exg_batch *B) {
    Batch &b = B->b;
    const bool f64 = b.precision == EXG_PREC_FP64;
    auto mark = [&](int k) {
        if (b.timing) EXG_CUDA_OK(cudaEventRecord(b.ev[k], b.stream));
    };
    mark(0);
    launch_batch_sort(b);
    launch_batch_plan(b);
    mark(1);
    f64 ? launch_batch_p2g_fp64(b) : launch_batch_p2g_fp32(b);
    mark(2);
    f64 ? launch_batch_nodes_fp64(b) : launch_batch_nodes_fp32(b);
    mark(3);
    f64 ? launch_batch_g2p_fp64(b) : launch_batch_g2p_fp32(b);
    f64 ? launch_batch_finish_fp64(b) : launch_batch_finish_fp32(b);
    mark(4);
}
void batch_flip(Batch &b) {
    for (Ctx *c : b.scenes) swap_parts(*c);
    b.parity ^= 1;
}
void batch_drop_graphs(Batch &b) {
    for (int k = 0; k < 2; ++k) {
        if (b.gexec[k]) cudaGraphExecDestroy(b.gexec[k]);
        b.gexec[k] = nullptr;
        b.warm[k] = false;
    }
}
}  // namespace

int exg_batch_create(const exg_specs *specs, int nscenes, int device, exg_batch **out) {
    if (!specs || !out || nscenes < 1 || nscenes > kMaxScenes) return EXG_ERR_ARG;
    *out = nullptr;
    const std::string why = batch_compatible(specs, nscenes);
    if (!why.empty()) {
        fprintf(stderr, "exg_batch_create: %s\n", why.c_str());
        return EXG_ERR_UNSUPPORTED;
    }
    exg_batch *B = new exg_batch();
    Batch &b = B->b;
    b.precision = specs[0].precision;
    try {
        EXG_CUDA_OK(cudaSetDevice(device));
        EXG_CUDA_OK(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
        for (int i = 0; i < nscenes; ++i) {
            exg_ctx *ctx = nullptr;
            const int rc = exg_ctx_create(&specs[i], device, &ctx);
            if (rc) {
                exg_batch_destroy(B);
                return rc;
            }
            // every scene enqueues on the batch's stream
            cudaStreamDestroy(ctx->c.stream);
            ctx->c.stream = b.stream;
            B->ctxs.push_back(ctx);
            b.scenes.push_back(&ctx->c);
        }
        EXG_CUDA_OK(cudaMalloc(&b.bctl, sizeof(BatchCtl)));
        EXG_CUDA_OK(cudaMemset(b.bctl, 0, sizeof(BatchCtl)));
        EXG_CUDA_OK(cudaMemcpy(&b.bctl->nscenes, &nscenes, sizeof(int), cudaMemcpyHostToDevice));
        std::vector<Ctl *> ctls(nscenes);
        for (int i = 0; i < nscenes; ++i) ctls[i] = b.scenes[i]->ctl;
        EXG_CUDA_OK(cudaMalloc(&b.ctls, sizeof(Ctl *) * nscenes));
        EXG_CUDA_OK(cudaMemcpy(b.ctls, ctls.data(), sizeof(Ctl *) * nscenes, cudaMemcpyHostToDevice));
    } catch (const std::exception &e) {
        fprintf(stderr, "exg_batch_create: %s\n", e.what());
        exg_batch_destroy(B);
        return EXG_ERR_CUDA;
    }
    *out = B;
    return EXG_OK;
}

int exg_batch_destroy(exg_batch *B) {
    if (!B) return EXG_OK;
    Batch &b = B->b;
    if (b.stream) cudaStreamSynchronize(b.stream);
    batch_drop_graphs(b);
    for (exg_ctx *ctx : B->ctxs) {
        ctx->c.stream = nullptr;  // the batch's stream
        exg_ctx_destroy(ctx);
    }
    cudaFree(b.bctl);
    cudaFree(b.ctls);
    for (void *d : b.desc) cudaFree(d);
    for (SortDesc *d : b.sdesc) cudaFree(d);
    for (cudaEvent_t e : b.ev)
        if (e) cudaEventDestroy(e);
    if (b.stream) cudaStreamDestroy(b.stream);
    delete B;
    return EXG_OK;
}

int exg_batch_set_stage_timing(exg_batch *B, int on) {
    if (!B) return EXG_ERR_ARG;
    Batch &b = B->b;
    try {
        for (cudaEvent_t &e : b.ev)
            if (!e) EXG_CUDA_OK(cudaEventCreate(&e));
    } catch (const std::exception &e) {
        return bfail(B, EXG_ERR_CUDA, e.what());
    }
    b.timing = on != 0;
    for (double &v : b.stage_ms) v = 0.0;
    return EXG_OK;
}

int exg_batch_last_step_timing(exg_batch *B, double *ms5) {
    if (!B || !ms5) return EXG_ERR_ARG;
    const Batch &b = B->b;
    const double n = b.stage_ms[4] > 0 ? b.stage_ms[4] : 1.0;
    for (int k = 0; k < 4; ++k) ms5[k] = b.stage_ms[k] / n;
    ms5[4] = b.stage_ms[4];
    return EXG_OK;
}

exg_ctx *exg_batch_scene(exg_batch *B, int i) {
    if (!B || i < 0 || i >= (int)B->ctxs.size()) return nullptr;
    return B->ctxs[i];
}

int exg_batch_num_scenes(const exg_batch *B) { return B ? (int)B->ctxs.size() : 0; }

const char *exg_batch_last_error(const exg_batch *B) { return B ? B->err.c_str() : "null batch"; }

int exg_batch_step(exg_batch *B, int nsteps) {
    if (!B || nsteps < 0) return EXG_ERR_ARG;
    Batch &b = B->b;
    for (size_t i = 0; i < b.scenes.size(); ++i)
        if (b.scenes[i]->np == 0) return bfail(B, EXG_ERR_NOT_READY, "scene " + std::to_string(i) + " has no particles");
    try {
        for (Ctx *c : b.scenes)
            if (c->reduce_stale) do_reduce(*c);
        const bool changed = b.precision == EXG_PREC_FP64 ? batch_descriptors_fp64(b) : batch_descriptors_fp32(b);
        int lean = 1;
        for (Ctx *sc : b.scenes) lean = lean && g2p_lean(*sc);
        if (changed || lean != b.lean) batch_drop_graphs(b);
        b.lean = lean;
        const bool use_graph = std::getenv("EXG_NO_GRAPH") == nullptr && !b.timing;
        for (int s = 0; s < nsteps; ++s) {
            cudaGraphExec_t &g = b.gexec[b.parity];
            if (!use_graph || !b.warm[b.parity]) {
                // the first step of each parity runs eagerly (kernel
                // attributes, occupancy queries), later ones replay a graph
                enqueue_batch_step(B);
                if (b.timing) {
                    EXG_CUDA_OK(cudaEventSynchronize(b.ev[4]));
                    float ms[4];
                    for (int k = 0; k < 4; ++k) EXG_CUDA_OK(cudaEventElapsedTime(&ms[k], b.ev[k], b.ev[k + 1]));
                    for (int k = 0; k < 4; ++k) b.stage_ms[k] += ms[k];
                    b.stage_ms[4] += 1.0;
                }
                b.warm[b.parity] = true;
                batch_flip(b);
                continue;
            }
            if (!g) {
                cudaGraph_t graph = nullptr;
                EXG_CUDA_OK(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
                enqueue_batch_step(B);
                EXG_CUDA_OK(cudaStreamEndCapture(b.stream, &graph));
                EXG_CUDA_OK(cudaGraphInstantiate(&g, graph, 0));
                cudaGraphDestroy(graph);
            }
            EXG_CUDA_OK(cudaGraphLaunch(g, b.stream));
            batch_flip(b);
        }
        int rc = EXG_OK;
        for (size_t i = 0; i < b.scenes.size(); ++i) {
            Ctx &c = *b.scenes[i];
            c.parts_sorted = false;
            const int r = status_from_ctl(c);
            c.host_time = c.ctl_host->time;
            c.host_dt = c.ctl_host->dt;
            c.host_steps = c.ctl_host->steps;
            if (r && !rc) {
                rc = r;
                B->err = "scene " + std::to_string(i) + ": " + c.err;
            }
        }
        return rc;
    } catch (const std::exception &e) {
        return bfail(B, EXG_ERR_CUDA, e.what());
    }
}

}  // extern "C"
