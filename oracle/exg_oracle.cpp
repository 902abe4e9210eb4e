// exg_oracle.cpp -- CPU FP64 oracle of the ExaGOOP per-step MPM path.
//
// TEST INFRASTRUCTURE ONLY (see exg_oracle.h).  Each function restates the
// reference routine it names, in the reference's loop and arithmetic order,
// so that the GPU library can be compared against it on the same inputs.
// Semantics the reference inherits from AMReX (un-vendored, version unknown)
// are stated where used and marked "AMReX-unpinned".
#include "exg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Literal constants of Source/constants.H:9-26 (their truncated values are
// part of the arithmetic).
constexpr double kFourByThree = 1.3333333333;
constexpr double kPI = 3.141592654;
constexpr double kOneBySix = 0.16666666666667;
constexpr double kOneByThree = 0.333333333333;
constexpr double kTwoByThree = 0.6666666666667;
constexpr double kTiny = 1e-20;

// ---------------------------------------------------------------------------
// 1-D B-spline pieces.  Coefficient tables restate Source/interpolants.H:
// cubic value  (a z^3 + b z^2 + c z + d) :46-80, derivative (a z^2 + b z + c)
// :85-115, quadratic value (a z^2 + b z + c) :120-149, derivative (a z + b)
// :154-183.  Index [shape type 1..4][interval 0..3].
// ---------------------------------------------------------------------------
const double kCubic[5][4][4] = {
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{kOneBySix, 1.0, 2.0, kFourByThree}, {-kOneBySix, 0.0, 1.0, 1.0}, {kOneBySix, 0.0, -1.0, 1.0},
     {-kOneBySix, 1.0, -2.0, kFourByThree}},
    {{0.0, 0.0, 0.0, 0.0}, {-kOneByThree, -1.0, 0.0, kTwoByThree}, {0.5, -1.0, 0.0, kTwoByThree},
     {-kOneBySix, 1.0, -2.0, kFourByThree}},
    {{kOneBySix, 1.0, 2.0, kFourByThree}, {-0.5, -1.0, 0.0, kTwoByThree}, {0.5, -1.0, 0.0, kTwoByThree},
     {-kOneBySix, 1.0, -2.0, kFourByThree}},
    {{kOneBySix, 1.0, 2.0, kFourByThree}, {-0.5, -1.0, 0.0, kTwoByThree}, {kOneByThree, -1.0, 0.0, kTwoByThree},
     {0.0, 0.0, 0.0, 0.0}}};
const double kCubicDer[5][4][3] = {
    {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{0.5, 2.0, 2.0}, {-0.5, 0.0, 1.0}, {0.5, 0.0, -1.0}, {-0.5, 2.0, -2.0}},
    {{0, 0, 0}, {-1.0, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
    {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
    {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.0, -2.0, 0.0}, {0, 0, 0}}};
const double kQuad[5][4][3] = {
    {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{kTwoByThree, 2.0, 1.5}, {-kFourByThree, 0.0, 1.0}, {-kFourByThree, 0.0, 1.0}, {kTwoByThree, -2.0, 1.5}},
    {{4.0 / 3.0, 8.0 / 3.0, 4.0 / 3.0}, {-7.0 / 6.0, 1.0 / 6.0, 17.0 / 24.0}, {0.5, -1.5, 1.125}, {0, 0, 0}},
    {{0.5, 1.5, 1.125}, {-1.0, 0.0, 0.75}, {0.5, -1.5, 1.125}, {0, 0, 0}},
    {{0.5, 1.5, 1.125}, {-7.0 / 6.0, -1.0 / 6.0, 17.0 / 24.0}, {4.0 / 3.0, -8.0 / 3.0, 4.0 / 3.0}, {0, 0, 0}}};
const double kQuadDer[5][4][2] = {
    {{0, 0}, {0, 0}, {0, 0}, {0, 0}},
    {{4.0 / 3.0, 2.0}, {-8.0 / 3.0, 0.0}, {-8.0 / 3.0, 0.0}, {4.0 / 3.0, -2.0}},
    {{8.0 / 3.0, 8.0 / 3.0}, {-14.0 / 6.0, 1.0 / 6.0}, {1.0, -1.5}, {0, 0}},
    {{2.0 / 2.0, 3.0 / 2.0}, {-2.0, 0.0}, {2.0 / 2.0, -3.0 / 2.0}, {0, 0}},
    {{1.0, 1.5}, {-14.0 / 6.0, -1.0 / 6.0}, {8.0 / 3.0, -8.0 / 3.0}, {0, 0}}};
// Half-interval -> polynomial piece map, interpolants.H:32-38.
const int kQuadMap[5][6] = {
    {-1, -1, -1, -1, -1, -1}, {0, 0, 1, 2, 3, 3}, {0, 1, 1, 2, 2, -1}, {0, 0, 1, 1, 2, 2}, {0, 0, 1, 1, 2, -1}};

// interpolants.H:201-211
int quad_interval(int type, double z) {
    double shift = (type == 2) ? 1.0 : 1.5;
    int raw = static_cast<int>(std::floor((z + shift) * 2));
    if (raw < 0 || raw >= 6) return -1;
    return kQuadMap[type][raw];
}
// The reference indexes the cubic table with floor(z)+2 and no range check
// (interpolants.H:222, :244).  The stencil keeps z inside [-2,2); a z that
// rounds onto 2.0 would read past the table, so the oracle clamps the
// interval to [0,3] (the GPU library does the same).
int cubic_interval(double z) {
    int iv = static_cast<int>(std::floor(z)) + 2;
    return iv < 0 ? 0 : (iv > 3 ? 3 : iv);
}
double cubic1d(int type, double z) {  // interpolants.H:215-226
    double z3 = z * z * z, z2 = z * z;
    const double *c = kCubic[type][cubic_interval(z)];
    return c[0] * z3 + c[1] * z2 + c[2] * z + c[3];
}
double cubic1d_der(int type, double z) {  // interpolants.H:242-250
    double z2 = z * z;
    const double *c = kCubicDer[type][cubic_interval(z)];
    return c[0] * z2 + c[1] * z + c[2];
}
double quad1d(int type, double z) {  // interpolants.H:268-278
    double z2 = z * z;
    int iv = quad_interval(type, z);
    if (iv < 0) return 0.0;
    const double *c = kQuad[type][iv];
    return c[0] * z2 + c[1] * z + c[2];
}
double quad1d_der(int type, double z) {  // interpolants.H:294-304
    int iv = quad_interval(type, z);
    if (iv < 0) return 0.0;
    const double *c = kQuadDer[type][iv];
    return c[0] * z + c[1];
}

// Boundary-aware shape type of basisval*() (interpolants.H:1419-1426):
// 1 at node lo or hi+1, 2 at lo+1, 4 at hi, else 3; periodic -> 3.
int shape_type_additive(int idx, int lo, int hi, int periodic) {
    if (periodic) return 3;
    return 3 + (idx == lo || idx == hi + 1) * (1 - 3) + (idx == lo + 1) * (2 - 3) + (idx == hi) * (4 - 3);
}
// Same classification written as the if-chain of *_interp_two
// (interpolants.H:885-896); identical when ncells >= 3.
int shape_type_chain(int idx, int lo, int hi) {
    if (idx == lo || idx == hi + 1) return 1;
    if (idx == lo + 1) return 2;
    if (idx == hi) return 4;
    return 3;
}

// compute_bounds, Source/mpm_particle_grid_ops.cpp:255-299.
void compute_bounds(int ivd, int lod, int hid, int scheme, int periodic, int &bmin, int &bmax) {
    if (scheme == 1) {
        bmin = 0;
        bmax = 2;
    } else {
        if (periodic) {
            bmin = -1;
            bmax = 3;
        } else if (ivd == lod) {
            bmin = 0;
            bmax = 3;
        } else if (ivd == hid) {
            bmin = -1;
            bmax = 2;
        } else {
            bmin = -1;
            bmax = 3;
        }
    }
}

// applybc, Source/mpm_kernels.H:27-113.  Returns modify_pos, or -1 for the
// outflow code the reference aborts on.
int applybc(const double relvel_in[3], double relvel_out[3], double wall_mu, const double n[3], int bc) {
    int modify_pos = 0;
    double velt[3], velt_hat[3];
    double veln = 0.0;
    for (int d = 0; d < 3; ++d) veln += relvel_in[d] * n[d];
    for (int d = 0; d < 3; ++d) velt[d] = relvel_in[d] - veln * n[d];
    double veltmag = 0.0;
    for (int d = 0; d < 3; ++d) veltmag += velt[d] * velt[d];
    veltmag = std::sqrt(veltmag);
    for (int d = 0; d < 3; ++d) velt_hat[d] = velt[d] / (veltmag + kTiny);
    if (bc == EXG_BC_NOSLIP) {
        modify_pos = 1;
        for (int d = 0; d < 3; ++d) relvel_out[d] = 0.0;
    } else if (bc == EXG_BC_SLIP) {
        modify_pos = 1;
        for (int d = 0; d < 3; ++d) relvel_out[d] = velt[d];
    } else if (bc == EXG_BC_PARTIALSLIP) {
        if (veln <= 0.0) {
            modify_pos = 1;
            if (veltmag <= -wall_mu * veln) {
                for (int d = 0; d < 3; ++d) relvel_out[d] = 0.0;
            } else {
                for (int d = 0; d < 3; ++d) relvel_out[d] = (veltmag + wall_mu * veln) * velt_hat[d];
            }
        }
    } else if (bc == EXG_BC_PERIODIC) {
    } else {
        return -1;
    }
    return modify_pos;
}

// Packed symmetric index order XX XY XZ YY YZ ZZ (constants.H:80-87).
enum { XX = 0, XY = 1, XZ = 2, YY = 3, YZ = 4, ZZ = 5 };

}  // namespace

struct orc_ctx {
    exg_specs s;
    double dx[3], dxi[3], plo[3], phi[3];
    int nc[3], nn[3];
    int lo[3], hi[3];
    int64_t nnodes;
    std::vector<double> node[EXG_N_NCOMP];
    int64_t np = 0;
    std::vector<double> pos[3];
    std::vector<double> r[EXG_NREAL];
    std::vector<int32_t> idat[EXG_NINT];
    std::vector<int64_t> pid;  // upload index; -1 once removed
    std::vector<double> ls[EXG_MAX_BODIES];
    bool has_ls[EXG_MAX_BODIES] = {};
    std::vector<double> udf_lo[3], udf_hi[3], udfT_lo[3], udfT_hi[3];
    int nthreads = 1;
    double time = 0.0, last_dt = 0.0;
    int64_t steps = 0;

    int64_t nidx(int i, int j, int k) const { return ((int64_t)k * nn[1] + j) * nn[0] + i; }
    // Node index with periodic wrap (AMReX ghost nodes filled by FillBoundary
    // with the periodic image; AMReX-unpinned).
    int wrap(int d, int i) const {
        if (!s.periodic[d]) return i;
        int n = nc[d];
        i %= n;
        return i < 0 ? i + n : i;
    }
    int64_t nidx_w(int i, int j, int k) const { return nidx(wrap(0, i), wrap(1, j), wrap(2, k)); }
    double &N(int comp, int64_t n) { return node[comp][n]; }
    double &R(int f, int64_t p) { return r[f][p]; }
    bool alive(int64_t p) const { return pid[p] >= 0; }
    // getParticleCell: floor((x - plo) * dxi) + domain.smallEnd() (AMReX
    // ParticleUtil; AMReX-unpinned).
    void cell(int64_t p, int iv[3]) const {
        for (int d = 0; d < 3; ++d) iv[d] = (int)std::floor((pos[d][p] - plo[d]) * dxi[d]);
    }
};

namespace {

// Per-axis value/derivative of basisval_and_grad (interpolants.H:1581-1654)
// for stencil offset l relative to cell i.
void axis_val_der(const orc_ctx *o, int d, int i, int l, double xp, double &val, double &der) {
    const int od = o->s.order[d];
    const double dx = o->dx[d];
    const double dxinv = 1.0 / dx;
    if (od == 1) {
        double r = (xp - (o->plo[d] + i * dx)) / dx;
        val = (l == 0) ? (1.0 - r) : r;
        der = (l == 0) ? -dxinv : dxinv;
    } else {
        int t = shape_type_additive(i + l, o->lo[d], o->hi[d], o->s.periodic[d]);
        double r = (xp - (o->plo[d] + (i + l) * dx)) / dx;
        if (od == 2) {
            val = quad1d(t, r);
            der = quad1d_der(t, r) * dxinv;
        } else {
            val = cubic1d(t, r);
            der = cubic1d_der(t, r) * dxinv;
        }
    }
}

// basisval_and_grad (interpolants.H:1581-1654).
double basis_and_grad(const orc_ctx *o, const int st[3], const int iv[3], const double xp[3], double grad[3]) {
    double v[3], g[3];
    for (int d = 0; d < 3; ++d) axis_val_der(o, d, iv[d], st[d], xp[d], v[d], g[d]);
    double Nv = 1.0;
    for (int d = 0; d < 3; ++d) Nv *= v[d];
    for (int dir = 0; dir < 3; ++dir) {
        double gg = 1.0;
        for (int d = 0; d < 3; ++d) gg *= (d == dir) ? g[d] : v[d];
        grad[dir] = gg;
    }
    return Nv;
}

// bilin_interp_two / quadratic_interp_two / cubic_interp_two
// (interpolants.H:583-656, 863-1006, 1225-1366) for two nodal components.
void interp_two(const orc_ctx *o, int scheme, const double xp[3], const int iv[3], const int mn[3], const int mx[3],
                const std::vector<double> &c0, const std::vector<double> &c1, double vals[2]) {
    vals[0] = 0.0;
    vals[1] = 0.0;
    if (scheme == 1) {
        int i = iv[0], j = iv[1], k = iv[2];
        double a = (xp[0] - (o->plo[0] + i * o->dx[0])) / o->dx[0];
        double b = (xp[1] - (o->plo[1] + j * o->dx[1])) / o->dx[1];
        double g = (xp[2] - (o->plo[2] + k * o->dx[2])) / o->dx[2];
        double w[8] = {(1.0 - a) * (1.0 - b) * (1.0 - g), a * (1.0 - b) * (1.0 - g), (1.0 - a) * b * (1.0 - g),
                       a * b * (1.0 - g),
                       (1.0 - a) * (1.0 - b) * g,
                       a * (1.0 - b) * g,
                       (1.0 - a) * b * g,
                       a * b * g};
        int64_t n[8] = {o->nidx_w(i, j, k),         o->nidx_w(i + 1, j, k),     o->nidx_w(i, j + 1, k),
                        o->nidx_w(i + 1, j + 1, k), o->nidx_w(i, j, k + 1),     o->nidx_w(i + 1, j, k + 1),
                        o->nidx_w(i, j + 1, k + 1), o->nidx_w(i + 1, j + 1, k + 1)};
        double s0 = w[0] * c0[n[0]], s1 = w[0] * c1[n[0]];
        for (int q = 1; q < 8; ++q) {
            s0 = s0 + w[q] * c0[n[q]];
            s1 = s1 + w[q] * c1[n[q]];
        }
        vals[0] = s0;
        vals[1] = s1;
        return;
    }
    double inv[3] = {1.0 / o->dx[0], 1.0 / o->dx[1], 1.0 / o->dx[2]};
    auto w1d = [&](int d, int idx) {
        int t = o->s.periodic[d] ? 3 : shape_type_chain(idx, o->lo[d], o->hi[d]);
        if (scheme == 2) {
            double rr = (xp[d] - (o->plo[d] + idx * o->dx[d])) / o->dx[d];
            return quad1d(t, rr);
        }
        double rr = (xp[d] - (o->plo[d] + idx * o->dx[d])) * inv[d];
        return cubic1d(t, rr);
    };
    for (int n = mn[2]; n < mx[2]; n++) {
        double nval = w1d(2, iv[2] + n);
        for (int m = mn[1]; m < mx[1]; m++) {
            double mval = w1d(1, iv[1] + m);
            for (int l = mn[0]; l < mx[0]; l++) {
                double lval = w1d(0, iv[0] + l);
                double weight = lval * mval * nval;
                int64_t q = o->nidx_w(iv[0] + l, iv[1] + m, iv[2] + n);
                vals[0] += weight * c0[q];
                vals[1] += weight * c1[q];
            }
        }
    }
}

// get_levelset_value / get_levelset_grad (Source/mpm_eb.H:176-288) with
// lsref = 1 on the coarse nodal grid.  Corner indices are clamped to the
// array bounds (valid nodes plus one ghost layer); ghost nodes outside a
// non-periodic domain read 1.0, the setVal(1.0) of nodal_levelset_bcs
// (nodal_data_ops.cpp:147) (AMReX-unpinned for moveParticles, whose ghosts
// are never set).
double ls_node(const orc_ctx *o, const std::vector<double> &phi, int i, int j, int k) {
    int ii[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
        if (o->s.periodic[d]) {
            ii[d] = o->wrap(d, ii[d]);
        } else if (ii[d] < 0 || ii[d] > o->nc[d]) {
            return 1.0;
        }
    }
    return phi[o->nidx(ii[0], ii[1], ii[2])];
}
void ls_eval(const orc_ctx *o, const std::vector<double> &phi, const double x[3], double *value, double grad[3]) {
    int idx[3];
    for (int d = 0; d < 3; ++d) idx[d] = (int)std::floor((x[d] - o->plo[d] + kTiny) / o->dx[d]);
    double lsval = 0.0;
    double g[3] = {0, 0, 0};
    for (int corner = 0; corner < 8; ++corner) {
        int off[3], c[3];
        for (int d = 0; d < 3; ++d) {
            off[d] = (corner >> d) & 1;
            c[d] = std::min(std::max(idx[d] + off[d], -1), o->nc[d] + 1);
        }
        double ph = ls_node(o, phi, c[0], c[1], c[2]);
        // basisval / basisvalder with order 1, lo = hi = 0, periodic.
        double v[3], dv[3];
        for (int d = 0; d < 3; ++d) {
            double rr = (x[d] - (o->plo[d] + idx[d] * o->dx[d])) / o->dx[d];
            v[d] = (off[d] == 0) ? (1.0 - rr) : rr;
            dv[d] = (off[d] == 0) ? -(1.0 / o->dx[d]) : (1.0 / o->dx[d]);
        }
        double bv = 1.0;
        for (int d = 0; d < 3; ++d) bv *= v[d];
        lsval += ph * bv;
        for (int dir = 0; dir < 3; ++dir) {
            double pr = 1.0;
            for (int d = 0; d < 3; ++d) pr *= (d == dir) ? dv[d] : v[d];
            g[dir] += ph * pr;
        }
    }
    if (value) *value = lsval;
    if (grad)
        for (int d = 0; d < 3; ++d) grad[d] = g[d];
}

// get_deformation_gradient_tensor (interpolants.H:1732-1787): F <- (I + gv dt) F
// unless |gv|^2 >= 1e10.
void defgrad_update(double F[9], const double gv[3][3], double dt) {
    double nrm = 0.0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) nrm += gv[a][b] * gv[a][b];
    if (nrm >= 1.0e10) return;
    double L[3][3], Fo[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            L[a][b] = (a == b) ? 1.0 + gv[a][b] * dt : gv[a][b] * dt;
            Fo[a][b] = F[3 * a + b];
        }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c) acc += L[a][c] * Fo[c][b];
            F[3 * a + b] = acc;
        }
}

void linear_elastic(const double eps[6], double sig[6], double E, double v) {  // constitutive_models.H:21-54
    double const1 = E / (1.0 + v) / (1.0 - 2.0 * v);
    double const2 = E / (1.0 + v);
    sig[XX] = const1 * ((1 - v) * eps[XX] + v * (eps[YY] + eps[ZZ]));
    sig[YY] = const1 * ((1 - v) * eps[YY] + v * (eps[XX] + eps[ZZ]));
    sig[ZZ] = const1 * ((1 - v) * eps[ZZ] + v * (eps[XX] + eps[YY]));
    sig[XY] = const2 * eps[XY];
    sig[XZ] = const2 * eps[XZ];
    sig[YZ] = const2 * eps[YZ];
}
// Compressible neo-Hookean solid, constitutive_models.H:161-250 (3-D):
// b = F F^T, J = max(det F, 1e-12), sigma = (mu/J)(b - I) + (lambda ln J / J) I
// with the Lame constants of E and nu.
void neo_hookean(const double F[9], double sig[6], double E, double v) {
    const double mu = E / (2.0 * (1.0 + v));
    const double lambda = E * v / ((1.0 + v) * (1.0 - 2.0 * v));
    auto row = [&](int i, int j) { return F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2]; };
    const double bxx = row(0, 0), byy = row(1, 1), bxy = row(0, 1), bzz = row(2, 2), bxz = row(0, 2), byz = row(1, 2);
    double detF = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                  F[2] * (F[3] * F[7] - F[4] * F[6]);
    detF = std::max(detF, 1.e-12);
    const double vol = lambda * std::log(detF) / detF;
    const double muJ = mu / detF;
    sig[XX] = muJ * (bxx - 1.0) + vol;
    sig[YY] = muJ * (byy - 1.0) + vol;
    sig[ZZ] = muJ * (bzz - 1.0) + vol;
    sig[XY] = muJ * bxy;
    sig[XZ] = muJ * bxz;
    sig[YZ] = muJ * byz;
}

void newtonian_fluid(const double ed[6], double sig[6], double mu, double p) {  // constitutive_models.H:118-159
    double tr = ed[XX] + ed[YY] + ed[ZZ];
    double o3 = 1.0 / 3.0;
    sig[XX] = 2.0 * mu * (ed[XX] - o3 * tr) - p;
    sig[YY] = 2.0 * mu * (ed[YY] - o3 * tr) - p;
    sig[ZZ] = 2.0 * mu * (ed[ZZ] - o3 * tr) - p;
    sig[XY] = 2.0 * mu * ed[XY];
    sig[XZ] = 2.0 * mu * ed[XZ];
    sig[YZ] = 2.0 * mu * ed[YZ];
}

// Node loop bounds: all (ncells+1) nodes per axis; a periodic axis keeps
// nodes [0, ncells) and mirrors node ncells from node 0 on read-out.
int node_hi(const orc_ctx *o, int d) { return o->s.periodic[d] ? o->nc[d] - 1 : o->nc[d]; }

template <class F>
void for_nodes(orc_ctx *o, F f) {
    for (int k = 0; k <= node_hi(o, 2); ++k)
        for (int j = 0; j <= node_hi(o, 1); ++j)
            for (int i = 0; i <= node_hi(o, 0); ++i) f(i, j, k, o->nidx(i, j, k));
}

template <class F>
void for_particles(orc_ctx *o, F f) {
#ifdef _OPENMP
    if (o->nthreads > 1) {
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
        for (int64_t p = 0; p < o->np; ++p) f(p);
        return;
    }
#endif
    for (int64_t p = 0; p < o->np; ++p) f(p);
}

inline void atomic_add(orc_ctx *o, double &dst, double v) {
#ifdef _OPENMP
    if (o->nthreads > 1) {
#pragma omp atomic
        dst += v;
        return;
    }
#endif
    dst += v;
    (void)o;
}

// UDF wall velocity tables of compute_udf_wall_vel_at_nodes
// (nodal_data_ops.cpp:929-1059): per face, (ncells[p0]+1) x (ncells[p1]+1)
// nodes, p0 = first tangential axis, p1 = second.
void tabulate_udf(orc_ctx *o, double t) {
    for (int d = 0; d < 3; ++d) {
        int p0 = (d == 0) ? 1 : 0;
        int p1 = (d == 2) ? 1 : 2;
        for (int side = 0; side < 2; ++side) {
            exg_wallvel_udf fn = side ? o->s.udf_wallvel_hi[d] : o->s.udf_wallvel_lo[d];
            std::vector<double> &tab = side ? o->udf_hi[d] : o->udf_lo[d];
            if (!fn) {
                tab.clear();
                continue;
            }
            tab.assign((size_t)(o->nc[p0] + 1) * (o->nc[p1] + 1) * 3, 0.0);
            for (int j = 0; j <= o->nc[p0]; ++j)
                for (int k = 0; k <= o->nc[p1]; ++k) {
                    double c[3] = {0, 0, 0};
                    c[d] = side ? o->phi[d] : o->plo[d];
                    c[p0] = o->plo[p0] + j * o->dx[p0];
                    c[p1] = o->plo[p1] + k * o->dx[p1];
                    double vel[3] = {0, 0, 0};
                    fn(c[0], c[1], c[2], t, vel);
                    size_t f = ((size_t)j * (o->nc[p1] + 1) + k) * 3;
                    for (int q = 0; q < 3; ++q) tab[f + q] = vel[q];
                }
        }
    }
}
void tabulate_udf_temp(orc_ctx *o, double t) {  // nodal_data_ops.cpp:1178-1293
    for (int d = 0; d < 3; ++d) {
        int p0 = (d == 0) ? 1 : 0;
        int p1 = (d == 2) ? 1 : 2;
        for (int side = 0; side < 2; ++side) {
            exg_temp_udf fn = side ? o->s.udf_temp_hi[d] : o->s.udf_temp_lo[d];
            std::vector<double> &tab = side ? o->udfT_hi[d] : o->udfT_lo[d];
            if (!fn) {
                tab.clear();
                continue;
            }
            tab.assign((size_t)(o->nc[p0] + 1) * (o->nc[p1] + 1) * 2, 0.0);
            for (int j = 0; j <= o->nc[p0]; ++j)
                for (int k = 0; k <= o->nc[p1]; ++k) {
                    double c[3] = {0, 0, 0};
                    c[d] = side ? o->phi[d] : o->plo[d];
                    c[p0] = o->plo[p0] + j * o->dx[p0];
                    c[p1] = o->plo[p1] + k * o->dx[p1];
                    double out[2] = {0, 0};
                    fn(c[0], c[1], c[2], t, out);
                    size_t f = ((size_t)j * (o->nc[p1] + 1) + k) * 2;
                    tab[f] = out[0];
                    tab[f + 1] = out[1];
                }
        }
    }
}

}  // namespace

extern "C" {

orc_ctx *orc_create(const exg_specs *specs) {
    orc_ctx *o = new orc_ctx();
    o->s = *specs;
    for (int d = 0; d < 3; ++d) {
        o->nc[d] = specs->ncells[d];
        o->nn[d] = specs->ncells[d] + 1;
        o->plo[d] = specs->plo[d];
        o->phi[d] = specs->phi[d];
        // AMReX Geometry: dx = (hi - lo) / ncells, inv_dx = 1 / dx.
        o->dx[d] = (specs->phi[d] - specs->plo[d]) / (double)specs->ncells[d];
        o->dxi[d] = 1.0 / o->dx[d];
        o->lo[d] = 0;
        o->hi[d] = specs->ncells[d] - 1;
    }
    o->nnodes = (int64_t)o->nn[0] * o->nn[1] * o->nn[2];
    for (int c = 0; c < EXG_N_NCOMP; ++c) o->node[c].assign(o->nnodes, 0.0);
    return o;
}

void orc_destroy(orc_ctx *o) { delete o; }
void orc_set_threads(orc_ctx *o, int n) { o->nthreads = n < 1 ? 1 : n; }

int orc_set_particles(orc_ctx *o, const exg_particle_soa *p) {
    o->np = p->np;
    for (int d = 0; d < 3; ++d) o->pos[d].assign(p->pos + d * p->np, p->pos + (d + 1) * p->np);
    for (int f = 0; f < EXG_NREAL; ++f) o->r[f].assign(p->rdata + f * p->np, p->rdata + (f + 1) * p->np);
    for (int f = 0; f < EXG_NINT; ++f) o->idat[f].assign(p->idata + f * p->np, p->idata + (f + 1) * p->np);
    o->pid.resize(o->np);
    for (int64_t i = 0; i < o->np; ++i) o->pid[i] = i;
    return EXG_OK;
}

int orc_get_particles(orc_ctx *o, exg_particle_soa *p) {
    if (p->np != o->np) return EXG_ERR_ARG;
    for (int d = 0; d < 3; ++d) std::copy(o->pos[d].begin(), o->pos[d].end(), p->pos + d * o->np);
    for (int f = 0; f < EXG_NREAL; ++f) std::copy(o->r[f].begin(), o->r[f].end(), p->rdata + f * o->np);
    for (int f = 0; f < EXG_NINT; ++f) std::copy(o->idat[f].begin(), o->idat[f].end(), p->idata + f * o->np);
    return EXG_OK;
}

int64_t orc_num_particles(orc_ctx *o) {
    int64_t n = 0;
    for (int64_t p = 0; p < o->np; ++p) n += o->alive(p);
    return n;
}

int orc_set_levelset(orc_ctx *o, int body, const double *phi_nodes) {
    if (body < 0 || body >= EXG_MAX_BODIES) return EXG_ERR_ARG;
    o->ls[body].assign(phi_nodes, phi_nodes + o->nnodes);
    o->has_ls[body] = true;
    return EXG_OK;
}

void orc_get_nodes(orc_ctx *o, int comp, double *out) {
    std::copy(o->node[comp].begin(), o->node[comp].end(), out);
    // periodic axes: node ncells mirrors node 0
    for (int k = 0; k < o->nn[2]; ++k)
        for (int j = 0; j < o->nn[1]; ++j)
            for (int i = 0; i < o->nn[0]; ++i) {
                int64_t n = o->nidx(i, j, k);
                int64_t w = o->nidx_w(i, j, k);
                if (n != w) out[n] = o->node[comp][w];
            }
}
void orc_set_nodes(orc_ctx *o, int comp, const double *in) { o->node[comp].assign(in, in + o->nnodes); }

// ---------------------------------------------------------------- P2G
// MPMParticleContainer::deposit_onto_grid_momentum,
// Source/mpm_particle_grid_ops.cpp:333-628.  One box covering the domain:
// the tile clamp of :445-451 never binds, and each node receives the full
// sum over particles, the sum AMReX forms with neighbour particles.
void orc_p2g_momentum(orc_ctx *o, int update_mass, int update_vel, int update_forces) {
    for_nodes(o, [&](int, int, int, int64_t n) {  // :368-403
        if (update_mass) o->N(EXG_N_MASS, n) = 0.0;
        if (update_vel)
            for (int d = 0; d < 3; ++d) o->N(EXG_N_VEL + d, n) = 0.0;
        if (update_forces)
            for (int d = 0; d < 3; ++d) o->N(EXG_N_FRC + d, n) = 0.0;
    });
    const exg_specs &s = o->s;
    for_particles(o, [&](int64_t p) {  // :405-588
        if (!o->alive(p)) return;
        if (o->idat[EXG_I_PHASE][p] != 0) return;
        double xp[3] = {o->pos[0][p], o->pos[1][p], o->pos[2][p]};
        int iv[3];
        o->cell(p, iv);
        int mn[3], mx[3];
        for (int d = 0; d < 3; ++d) compute_bounds(iv[d], o->lo[d], o->hi[d], s.order[d], s.periodic[d], mn[d], mx[d]);
        const double m = o->R(EXG_R_MASS, p);
        const double vol = o->R(EXG_R_VOLUME, p);
        double st[9];
        {  // get_tensor (interpolants.H:1673-1688)
            int ind = 0;
            for (int i = 0; i < 3; i++)
                for (int j = i; j < 3; j++) {
                    st[i * 3 + j] = o->R(EXG_R_STRESS + ind, p);
                    st[j * 3 + i] = o->R(EXG_R_STRESS + ind, p);
                    ind++;
                }
        }
        bool in_slab = s.external_loads && xp[0] > s.force_slab_lo[0] && xp[0] < s.force_slab_hi[0] &&
                       xp[1] > s.force_slab_lo[1] && xp[1] < s.force_slab_hi[1] && xp[2] > s.force_slab_lo[2] &&
                       xp[2] < s.force_slab_hi[2];
        for (int n = mn[2]; n < mx[2]; n++)
            for (int mm = mn[1]; mm < mx[1]; mm++)
                for (int l = mn[0]; l < mx[0]; l++) {
                    int stc[3] = {l, mm, n};
                    double grad[3];
                    double bv = basis_and_grad(o, stc, iv, xp, grad);
                    int64_t q = o->nidx_w(iv[0] + l, iv[1] + mm, iv[2] + n);
                    if (update_mass) atomic_add(o, o->N(EXG_N_MASS, q), m * bv);
                    if (update_vel)
                        for (int d = 0; d < 3; ++d) atomic_add(o, o->N(EXG_N_VEL + d, q), m * o->R(EXG_R_VEL + d, p) * bv);
                    if (update_forces) {
                        double bf[3];
                        for (int d = 0; d < 3; ++d) bf[d] = m * s.gravity[d] * bv;
                        if (in_slab)
                            for (int d = 0; d < 3; ++d) bf[d] += s.extforce[d] * bv;
                        double tv[3];  // tensor_vector_pdt (interpolants.H:1804-1817)
                        for (int i = 0; i < 3; i++) {
                            tv[i] = 0.0;
                            for (int j = 0; j < 3; j++) tv[i] += st[i * 3 + j] * grad[j];
                        }
                        for (int d = 0; d < 3; ++d) atomic_add(o, o->N(EXG_N_FRC + d, q), bf[d] + (-vol * tv[d]));
                    }
                }
    });
    for_nodes(o, [&](int, int, int, int64_t n) {  // :590-627
        double mass = o->N(EXG_N_MASS, n);
        if (update_vel && mass > 0.0) {
            for (int d = 0; d < 3; ++d) {
                if (mass >= s.mass_tolerance)
                    o->N(EXG_N_VEL + d, n) /= mass;
                else
                    o->N(EXG_N_VEL + d, n) = 0.0;
            }
        }
    });
}

void orc_backup_current_velocity(orc_ctx *o) {  // nodal_data_ops.cpp:57-81
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS, n) > 0.0) {
            o->N(EXG_N_MASS_OLD, n) = o->N(EXG_N_MASS, n);
            for (int d = 0; d < 3; d++) o->N(EXG_N_DVEL + d, n) = o->N(EXG_N_VEL + d, n);
        }
    });
}

void orc_nodal_time_update_momentum(orc_ctx *o, double dt) {  // nodal_data_ops.cpp:451-482
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS, n) >= o->s.mass_tolerance) {
            for (int d = 0; d < 3; d++) o->N(EXG_N_VEL + d, n) += o->N(EXG_N_FRC + d, n) / o->N(EXG_N_MASS, n) * dt;
        } else {
            for (int d = 0; d < 3; d++) o->N(EXG_N_VEL + d, n) = 0.0;
        }
    });
}

// Apply_Nodal_BCs (Source/utilities.cpp:183-204).
int orc_apply_nodal_bcs(orc_ctx *o, double dt, double time) {
    (void)dt;
    const exg_specs &s = o->s;
    int status = EXG_OK;
    // nodal_bcs, nodal_data_ops.cpp:663-766.  relvel_in accumulates the wall
    // velocities of every face the node lies on; relvel_out persists across
    // directions.
    for_nodes(o, [&](int i, int j, int k, int64_t n) {
        int id[3] = {i, j, k};
        double rin[3], rout[3], wv[3] = {0, 0, 0};
        for (int d = 0; d < 3; d++) {
            rin[d] = o->N(EXG_N_VEL + d, n);
            rout[d] = rin[d];
        }
        for (int dir = 0; dir < 3; ++dir) {
            bool at_lo = id[dir] == o->lo[dir];
            bool at_hi = !at_lo && id[dir] == o->hi[dir] + 1;
            if (!at_lo && !at_hi) continue;
            for (int d = 0; d < 3; ++d) {
                wv[d] = at_lo ? s.wall_vel_lo[dir * 3 + d] : s.wall_vel_hi[dir * 3 + d];
                rin[d] -= wv[d];
            }
            double nd[3] = {0, 0, 0};
            nd[dir] = at_lo ? 1.0 : -1.0;
            int rc = applybc(rin, rout, at_lo ? s.wall_mu_lo[dir] : s.wall_mu_hi[dir], nd, at_lo ? s.bclo[dir] : s.bchi[dir]);
            if (rc < 0) status = EXG_ERR_BC;
            for (int c = 0; c < 3; ++c) o->N(EXG_N_VEL + c, n) = rout[c] + wv[c];
        }
    });
    // UDF walls: compute_udf_wall_vel_at_nodes + apply_udf_nodal_bcs
    // (nodal_data_ops.cpp:929-1175).
    tabulate_udf(o, time);
    bool any_udf = false;
    for (int d = 0; d < 3; ++d) any_udf |= (s.udf_wallvel_lo[d] != nullptr) || (s.udf_wallvel_hi[d] != nullptr);
    if (any_udf) {
        for_nodes(o, [&](int i, int j, int k, int64_t n) {
            int id[3] = {i, j, k};
            for (int dir = 0; dir < 3; ++dir) {
                const std::vector<double> *tab = nullptr;
                int bc = -1;
                if (id[dir] == o->lo[dir] && s.udf_wallvel_lo[dir]) {
                    tab = &o->udf_lo[dir];
                    bc = s.bclo[dir];
                } else if (id[dir] == o->hi[dir] + 1 && s.udf_wallvel_hi[dir]) {
                    tab = &o->udf_hi[dir];
                    bc = s.bchi[dir];
                }
                if (!tab) continue;
                int p0 = (dir == 0) ? 1 : 0;
                int p1 = (dir == 2) ? 1 : 2;
                size_t f = ((size_t)id[p0] * (o->nc[p1] + 1) + id[p1]) * 3;
                if (bc == EXG_BC_NOSLIP) {
                    for (int c = 0; c < 3; ++c) o->N(EXG_N_VEL + c, n) = (*tab)[f + c];
                } else {
                    o->N(EXG_N_VEL + dir, n) = (*tab)[f + dir];
                }
            }
        });
    }
    // nodal_levelset_bcs, nodal_data_ops.cpp:129-220.
    for (int b = 0; b < s.num_bodies; ++b) {
        if (!o->has_ls[b]) continue;
        const exg_body &body = s.bodies[b];
        for_nodes(o, [&](int i, int j, int k, int64_t n) {
            double xp[3] = {o->plo[0] + i * o->dx[0], o->plo[1] + j * o->dx[1], o->plo[2] + k * o->dx[2]};
            double lsval;
            ls_eval(o, o->ls[b], xp, &lsval, nullptr);
            if (lsval >= 0.0 || o->N(EXG_N_MASS, n) <= 0.0) return;
            double nd[3];
            ls_eval(o, o->ls[b], xp, nullptr, nd);
            double gm = 0.0;
            for (int d = 0; d < 3; d++) gm += nd[d] * nd[d];
            gm = std::sqrt(gm);
            if (!(gm >= 1.0e-10)) return;
            for (int d = 0; d < 3; d++) nd[d] /= gm;
            double rin[3], rout[3];
            for (int d = 0; d < 3; d++) {
                rin[d] = o->N(EXG_N_VEL + d, n) - body.wall_vel[d];
                rout[d] = rin[d];
            }
            double veln = 0.0;
            for (int d = 0; d < 3; d++) veln += rin[d] * nd[d];
            if (veln > 0.0) return;
            if (applybc(rin, rout, body.wall_mu, nd, body.mom_bc) < 0) status = EXG_ERR_BC;
            for (int d = 0; d < 3; d++) o->N(EXG_N_VEL + d, n) = rout[d] + body.wall_vel[d];
        });
    }
    // store_delta_velocity, nodal_data_ops.cpp:368-392.
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS, n) > 0.0)
            for (int d = 0; d < 3; d++) o->N(EXG_N_DVEL + d, n) = o->N(EXG_N_VEL + d, n) - o->N(EXG_N_DVEL + d, n);
    });
    return status;
}

// ---------------------------------------------------------------- G2P
// MPMParticleContainer::interpolate_from_grid, mpm_particle_grid_ops.cpp:924-1098.
void orc_g2p_momentum(orc_ctx *o, int update_vel, int update_strainrate, double dt) {
    const exg_specs &s = o->s;
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p)) return;
        if (o->idat[EXG_I_PHASE][p] != 0) return;
        double xp[3] = {o->pos[0][p], o->pos[1][p], o->pos[2][p]};
        int iv[3];
        o->cell(p, iv);
        int mn[3], mx[3];
        for (int d = 0; d < 3; ++d) compute_bounds(iv[d], o->lo[d], o->hi[d], s.order[d], s.periodic[d], mn[d], mx[d]);
        if (update_vel) {  // :1002-1036
            for (int dim = 0; dim < 3; dim++) {
                double vals[2];
                interp_two(o, s.order[dim], xp, iv, mn, mx, o->node[EXG_N_VEL + dim], o->node[EXG_N_DVEL + dim], vals);
                o->R(EXG_R_VEL_PRIME + dim, p) = vals[0];
                o->R(EXG_R_VEL + dim, p) = s.alpha_pic_flip * o->R(EXG_R_VEL + dim, p) + s.alpha_pic_flip * vals[1] +
                                           (1 - s.alpha_pic_flip) * vals[0];
            }
        }
        if (update_strainrate) {  // :1039-1096
            double gv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int n = mn[2]; n < mx[2]; ++n)
                for (int m = mn[1]; m < mx[1]; ++m)
                    for (int l = mn[0]; l < mx[0]; ++l) {
                        int st[3] = {l, m, n};
                        double g[3];
                        basis_and_grad(o, st, iv, xp, g);
                        int64_t q = o->nidx_w(iv[0] + l, iv[1] + m, iv[2] + n);
                        for (int d1 = 0; d1 < 3; ++d1) {
                            double v = o->node[EXG_N_VEL + d1][q];
                            for (int d2 = 0; d2 < 3; ++d2) gv[d1][d2] += v * g[d2];
                        }
                    }
            {
                double F[9];
                for (int q = 0; q < 9; ++q) F[q] = o->R(EXG_R_DEFGRAD + q, p);
                defgrad_update(F, gv, dt);
                for (int q = 0; q < 9; ++q) o->R(EXG_R_DEFGRAD + q, p) = F[q];
            }
            int ind = 0;
            for (int d1 = 0; d1 < 3; ++d1)
                for (int d2 = d1; d2 < 3; ++d2) {
                    o->R(EXG_R_STRAINRATE + ind, p) = 0.5 * (gv[d1][d2] + gv[d2][d1]);
                    ind++;
                }
        }
    });
}

// MPMParticleContainer::moveParticles, mpm_particle_timestep.cpp:226-578.
int orc_update_mp_positions(orc_ctx *o, double dt) {
    const exg_specs &s = o->s;
    int status = EXG_OK;
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p)) return;
        for (int d = 0; d < 3; ++d) o->pos[d][p] += o->R(EXG_R_VEL_PRIME + d, p) * dt;
        double rin[3], rout[3];
        for (int d = 0; d < 3; ++d) {
            rin[d] = o->R(EXG_R_VEL + d, p);
            rout[d] = rin[d];
        }
        if (s.num_bodies > 0 && o->idat[EXG_I_PHASE][p] == 0) {  // :350-402
            double xp[3] = {o->pos[0][p], o->pos[1][p], o->pos[2][p]};
            int hit = -1;
            double min_phi = kTiny;
            for (int b = 0; b < s.num_bodies; ++b) {
                if (!o->has_ls[b]) continue;
                double ph;
                ls_eval(o, o->ls[b], xp, &ph, nullptr);
                if (ph < min_phi) {
                    min_phi = ph;
                    hit = b;
                }
            }
            if (hit >= 0) {
                double nd[3];
                ls_eval(o, o->ls[hit], xp, nullptr, nd);
                double gm = 0.0;
                for (int d = 0; d < 3; ++d) gm += nd[d] * nd[d];
                gm = std::sqrt(gm);
                for (int d = 0; d < 3; ++d) nd[d] /= (gm + kTiny);
                int mp = applybc(rin, rout, s.bodies[hit].wall_mu, nd, s.bodies[hit].mom_bc);
                if (mp < 0) status = EXG_ERR_BC;
                if (mp > 0)
                    for (int d = 0; d < 3; ++d) o->pos[d][p] += 2.0 * std::fabs(min_phi) * nd[d];
                for (int d = 0; d < 3; ++d) o->R(EXG_R_VEL + d, p) = rout[d];
            }
        }
        double wv[3] = {0, 0, 0};
        for (int dir = 0; dir < 3; ++dir) {  // :404-575
            bool lo_hit = o->pos[dir][p] < o->plo[dir];
            bool hi_hit = !lo_hit && o->pos[dir][p] > o->phi[dir];
            if (!lo_hit && !hi_hit) continue;
            for (int d = 0; d < 3; ++d) wv[d] = lo_hit ? s.wall_vel_lo[dir * 3 + d] : s.wall_vel_hi[dir * 3 + d];
            const std::vector<double> &tab = lo_hit ? o->udf_lo[dir] : o->udf_hi[dir];
            bool has_udf = lo_hit ? (s.udf_wallvel_lo[dir] != nullptr) : (s.udf_wallvel_hi[dir] != nullptr);
            if (has_udf && !tab.empty()) {
                int p0 = (dir == 0) ? 1 : 0;
                int p1 = (dir == 2) ? 1 : 2;
                double f0 = (o->pos[p0][p] - o->plo[p0]) / o->dx[p0];
                double f1 = (o->pos[p1][p] - o->plo[p1]) / o->dx[p1];
                f0 = std::max(0.0, std::min((double)o->nc[p0], f0));
                f1 = std::max(0.0, std::min((double)o->nc[p1], f1));
                int j0 = (int)f0, j1 = std::min(j0 + 1, o->nc[p0]);
                int k0 = (int)f1, k1 = std::min(k0 + 1, o->nc[p1]);
                double wx1 = f0 - j0, wx0 = 1.0 - wx1, wy1 = f1 - k0, wy0 = 1.0 - wy1;
                int n1 = o->nc[p1] + 1;
                for (int c = 0; c < 3; ++c)
                    wv[c] = wx0 * wy0 * tab[(j0 * n1 + k0) * 3 + c] + wx0 * wy1 * tab[(j0 * n1 + k1) * 3 + c] +
                            wx1 * wy0 * tab[(j1 * n1 + k0) * 3 + c] + wx1 * wy1 * tab[(j1 * n1 + k1) * 3 + c];
            }
            for (int d = 0; d < 3; ++d) rin[d] -= wv[d];
            double nd[3] = {0, 0, 0};
            nd[dir] = lo_hit ? 1.0 : -1.0;
            int mp = applybc(rin, rout, lo_hit ? s.wall_mu_lo[dir] : s.wall_mu_hi[dir], nd,
                             lo_hit ? s.bclo[dir] : s.bchi[dir]);
            if (mp < 0) status = EXG_ERR_BC;
            if (mp > 0) o->pos[dir][p] = lo_hit ? 2.0 * o->plo[dir] - o->pos[dir][p] : 2.0 * o->phi[dir] - o->pos[dir][p];
            for (int c = 0; c < 3; ++c) o->R(EXG_R_VEL + c, p) = rout[c] + wv[c];
        }
    });
    return status;
}

// MPMParticleContainer::updateVolume, mpm_particle_timestep.cpp:131-182.
void orc_update_mp_volume(orc_ctx *o) {
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p) || o->idat[EXG_I_PHASE][p] != 0) return;
        double F[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) F[a][b] = o->R(EXG_R_DEFGRAD + a * 3 + b, p);
        double det = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
        o->R(EXG_R_JACOBIAN, p) = det;
        o->R(EXG_R_VOLUME, p) = o->R(EXG_R_VOL_INIT, p) * det;
        o->R(EXG_R_DENSITY, p) = o->R(EXG_R_MASS, p) / o->R(EXG_R_VOLUME, p);
    });
}

// Calculate_MP_Stress_Strain (utilities.cpp:372-400) ->
// apply_constitutive_model (mpm_particle_container.cpp:43-142), or with
// calculate_strain_based_on_delta = 1 apply_constitutive_model_delta
// (:178-272): sigma += C : (dt D + applied), linear elastic only (the
// reference aborts on the other models there).
static void stress_strain(orc_ctx *o, double time, double dt, bool total) {
    double asr = (time < o->s.applied_strainrate_time) ? o->s.applied_strainrate : 0.0;
    const bool delta = !total && o->s.calculate_strain_based_on_delta == 1;
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p) || o->idat[EXG_I_PHASE][p] != 0) return;
        for (int d = 0; d < 6; ++d) o->R(EXG_R_STRAIN + d, p) += dt * o->R(EXG_R_STRAINRATE + d, p);
        o->R(EXG_R_STRAIN + XX, p) += dt * asr;
        o->R(EXG_R_STRAIN + YY, p) += dt * asr;
        o->R(EXG_R_STRAIN + ZZ, p) += dt * asr;
        double sr[6], eps[6], sig[6];
        for (int d = 0; d < 6; ++d) {
            sr[d] = o->R(EXG_R_STRAINRATE + d, p);
            eps[d] = o->R(EXG_R_STRAIN + d, p);
        }
        int model = o->idat[EXG_I_MODEL][p];
        if (delta) {
            if (model != 0) return;
            double deps[6], dsig[6];
            for (int d = 0; d < 6; ++d) deps[d] = dt * sr[d];
            deps[XX] += dt * asr;
            deps[YY] += dt * asr;
            deps[ZZ] += dt * asr;
            linear_elastic(deps, dsig, o->R(EXG_R_E, p), o->R(EXG_R_NU, p));  // linear_elastic_delta: same operator
            for (int d = 0; d < 6; ++d) o->R(EXG_R_STRESS + d, p) += dsig[d];
            return;
        }
        if (model == 0) {
            linear_elastic(eps, sig, o->R(EXG_R_E, p), o->R(EXG_R_NU, p));
        } else if (model == 1) {
            const double p_inf = 0.0;
            o->R(EXG_R_PRESSURE, p) =
                o->R(EXG_R_BULK, p) * (std::pow(1.0 / o->R(EXG_R_JACOBIAN, p), o->R(EXG_R_GAMMA, p)) - 1.0) + p_inf;
            newtonian_fluid(sr, sig, o->R(EXG_R_VISC, p), o->R(EXG_R_PRESSURE, p));
        } else if (model == 2) {
            double F[9];
            for (int q = 0; q < 9; ++q) F[q] = o->R(EXG_R_DEFGRAD + q, p);
            neo_hookean(F, sig, o->R(EXG_R_E, p), o->R(EXG_R_NU, p));
        } else {
            return;
        }
        for (int d = 0; d < 6; ++d) o->R(EXG_R_STRESS + d, p) = sig[d];
    });
}
void orc_calculate_mp_stress_strain(orc_ctx *o, double time, double dt) { stress_strain(o, time, dt, false); }

// Calculate_time_step, mpm_particle_timestep.cpp:38-111.
double orc_calculate_time_step(orc_ctx *o) {
    const exg_specs &s = o->s;
    if (s.fixed_timestep == 1) return s.timestep;
    double dt = std::numeric_limits<double>::max();
    double dxmin = o->dx[0];
    for (int d = 1; d < 3; ++d) dxmin = std::min(dxmin, o->dx[d]);
    for (int64_t p = 0; p < o->np; ++p) {
        if (!o->alive(p) || o->idat[EXG_I_PHASE][p] != 0) continue;
        double Cs = 0.0;
        int model = o->idat[EXG_I_MODEL][p];
        if (model == 1) {
            Cs = std::sqrt(o->R(EXG_R_BULK, p) / o->R(EXG_R_DENSITY, p));
        } else {
            double E = o->R(EXG_R_E, p), nu = o->R(EXG_R_NU, p);
            double lambda = E * nu / ((1 + nu) * (1 - 2.0 * nu));
            double mu = E / (2.0 * (1 + nu));
            Cs = std::sqrt((lambda + 2.0 * mu) / o->R(EXG_R_DENSITY, p));
        }
        double vm = 0.0;
        for (int d = 0; d < 3; ++d) vm += o->R(EXG_R_VEL + d, p) * o->R(EXG_R_VEL + d, p);
        vm = std::sqrt(vm);
        dt = std::min(dt, dxmin / (Cs + vm));
    }
    dt = s.cfl * dt;
    dt = std::max(std::min(dt, s.dt_max_limit), s.dt_min_limit);
    return dt;
}

void orc_reset_nodaldata(orc_ctx *o) {  // nodal_data_ops.cpp:924-927
    for (int c = 0; c < EXG_N_NCOMP; ++c) std::fill(o->node[c].begin(), o->node[c].end(), 0.0);
}

// Redistribute (AMReX-unpinned): a periodic axis wraps x into [lo, hi) by
// one period; a particle outside a non-periodic domain, or in the cell
// index ncells, is removed (id = -1).
int orc_redistribute(orc_ctx *o) {
    int status = EXG_OK;
    for (int64_t p = 0; p < o->np; ++p) {
        if (!o->alive(p)) continue;
        for (int d = 0; d < 3; ++d) {
            double L = o->phi[d] - o->plo[d];
            if (o->s.periodic[d]) {
                if (o->pos[d][p] >= o->phi[d])
                    o->pos[d][p] -= L;
                else if (o->pos[d][p] < o->plo[d])
                    o->pos[d][p] += L;
            }
        }
        int iv[3];
        o->cell(p, iv);
        for (int d = 0; d < 3; ++d)
            if (iv[d] < 0 || iv[d] >= o->nc[d]) {
                o->pid[p] = -1;
                status = EXG_ERR_DOMAIN;
                break;
            }
    }
    return status;
}

// ------------------------------------------------------------ thermal
// deposit_onto_grid_temperature, mpm_particle_grid_ops.cpp:656-884.
void orc_p2g_temperature(orc_ctx *o, int reset, int update_temp, int update_source) {
    const exg_specs &s = o->s;
    if (reset)
        for_nodes(o, [&](int, int, int, int64_t n) {
            o->N(EXG_N_MASS_SPHEAT, n) = 0.0;
            o->N(EXG_N_MASS_SPHEAT_TEMP, n) = 0.0;
            o->N(EXG_N_SOURCE_TEMP, n) = 0.0;
            if (update_temp) o->N(EXG_N_MASS_COND, n) = 0.0;
        });
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p) || o->idat[EXG_I_PHASE][p] != 0) return;
        double xp[3] = {o->pos[0][p], o->pos[1][p], o->pos[2][p]};
        int iv[3];
        o->cell(p, iv);
        int mn[3], mx[3];
        for (int d = 0; d < 3; ++d) compute_bounds(iv[d], o->lo[d], o->hi[d], s.order[d], s.periodic[d], mn[d], mx[d]);
        const double m = o->R(EXG_R_MASS, p), cp = o->R(EXG_R_SPHEAT, p), T = o->R(EXG_R_TEMPERATURE, p);
        const double kc = o->R(EXG_R_THERMCOND, p), vol = o->R(EXG_R_VOLUME, p), Q = o->R(EXG_R_HEATSRC, p);
        for (int n = mn[2]; n < mx[2]; n++)
            for (int mm = mn[1]; mm < mx[1]; mm++)
                for (int l = mn[0]; l < mx[0]; l++) {
                    int st[3] = {l, mm, n};
                    double g[3];
                    double bv = basis_and_grad(o, st, iv, xp, g);
                    int64_t q = o->nidx_w(iv[0] + l, iv[1] + mm, iv[2] + n);
                    if (update_temp) {
                        atomic_add(o, o->N(EXG_N_MASS_SPHEAT, q), m * cp * bv);
                        atomic_add(o, o->N(EXG_N_MASS_SPHEAT_TEMP, q), m * cp * T * bv);
                        atomic_add(o, o->N(EXG_N_MASS_COND, q), m * kc * bv);
                    }
                    if (update_source) {
                        double net = 0.0;
                        for (int d = 0; d < 3; d++) net += o->R(EXG_R_HEATFLUX + d, p) * g[d];
                        double is = net * vol;
                        double es = vol * Q * bv;
                        atomic_add(o, o->N(EXG_N_SOURCE_TEMP, q), is + es);
                    }
                }
    });
    // SumBoundary (:846-854) is the identity for the single-box domain.
    for_nodes(o, [&](int, int, int, int64_t n) {
        double mc = o->N(EXG_N_MASS_SPHEAT, n);
        if (update_temp && mc > 0.0) {
            if (mc >= s.mass_tolerance)
                o->N(EXG_N_TEMPERATURE, n) = o->N(EXG_N_MASS_SPHEAT_TEMP, n) / mc;
            else
                o->N(EXG_N_TEMPERATURE, n) = 0.0;
        }
    });
}

void orc_backup_current_temperature(orc_ctx *o) {  // nodal_data_ops.cpp:95-114
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS_SPHEAT, n) > 0.0) o->N(EXG_N_DELTA_TEMPERATURE, n) = o->N(EXG_N_TEMPERATURE, n);
    });
}
void orc_store_delta_temperature(orc_ctx *o) {  // nodal_data_ops.cpp:409-430
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS_SPHEAT, n) > 0.0)
            o->N(EXG_N_DELTA_TEMPERATURE, n) = o->N(EXG_N_TEMPERATURE, n) - o->N(EXG_N_DELTA_TEMPERATURE, n);
    });
}
void orc_nodal_time_update_temperature(orc_ctx *o, double dt) {  // nodal_data_ops.cpp:500-527
    for_nodes(o, [&](int, int, int, int64_t n) {
        if (o->N(EXG_N_MASS_SPHEAT, n) >= o->s.mass_tolerance)
            o->N(EXG_N_TEMPERATURE, n) += o->N(EXG_N_SOURCE_TEMP, n) / o->N(EXG_N_MASS_SPHEAT, n) * dt;
        else
            o->N(EXG_N_TEMPERATURE, n) = 0.0;
    });
}

// Apply_Nodal_BCs_Temperature (utilities.cpp:229-245).  The nodal loops run
// in AMReX's CPU order (k, j, i with i innermost); a boundary node reads its
// inward neighbour's current value, so nodes on high faces see neighbours
// already updated in this pass.
void orc_apply_nodal_bcs_temperature(orc_ctx *o, double dt, double time, int dirichlet_only) {
    (void)dt;
    const exg_specs &s = o->s;
    auto k_node = [&](int64_t n) {
        double mk = o->N(EXG_N_MASS_COND, n), m = o->N(EXG_N_MASS, n);
        return (m > 0.0) ? mk / m : 1.0;
    };
    // nodal_bcs_temperature, nodal_data_ops.cpp:786-910
    for_nodes(o, [&](int i, int j, int k, int64_t n) {
        int id[3] = {i, j, k};
        bool applied = false;
        for (int d = 0; d < 3; ++d) {
            bool is_lo = id[d] == o->lo[d];
            bool is_hi = id[d] == o->hi[d] + 1;
            if (!is_lo && !is_hi) continue;
            int bc = is_lo ? s.bclo_temp[d] : s.bchi_temp[d];
            int sign = is_lo ? 1 : -1;
            int nb[3] = {i, j, k};
            nb[d] += sign;
            if (bc == EXG_BCT_PERIODIC) {
                applied = true;
            } else if (bc == EXG_BCT_ISOTHERMAL) {
                o->N(EXG_N_TEMPERATURE, n) = is_lo ? s.T_wall_lo[d] : s.T_wall_hi[d];
                applied = true;
            } else if (bc == EXG_BCT_ADIABATIC) {
                if (!applied) {
                    o->N(EXG_N_TEMPERATURE, n) = o->N(EXG_N_TEMPERATURE, o->nidx_w(nb[0], nb[1], nb[2]));
                    applied = true;
                }
            } else if (bc == EXG_BCT_USERFLUX) {
                double q = is_lo ? s.flux_lo[d] : s.flux_hi[d];
                o->N(EXG_N_TEMPERATURE, n) = o->N(EXG_N_TEMPERATURE, o->nidx_w(nb[0], nb[1], nb[2])) + q * o->dx[d] / k_node(n);
                applied = true;
            } else if (bc == EXG_BCT_CONVECTION) {
                double hc = is_lo ? s.h_lo[d] : s.h_hi[d];
                double Tinf = is_lo ? s.Tinf_lo[d] : s.Tinf_hi[d];
                double Bi = hc * o->dx[d] / k_node(n);
                o->N(EXG_N_TEMPERATURE, n) = (o->N(EXG_N_TEMPERATURE, o->nidx_w(nb[0], nb[1], nb[2])) + Bi * Tinf) / (1.0 + Bi);
                applied = true;
            }
        }
    });
    // compute_udf_temp_at_nodes + apply_udf_nodal_bcs_temperature
    // (nodal_data_ops.cpp:1178-1446)
    tabulate_udf_temp(o, time);
    bool any = false;
    for (int d = 0; d < 3; ++d) any |= (s.udf_temp_lo[d] != nullptr) || (s.udf_temp_hi[d] != nullptr);
    if (any)
        for_nodes(o, [&](int i, int j, int k, int64_t n) {
            int id[3] = {i, j, k};
            for (int dir = 0; dir < 3; ++dir) {
                const std::vector<double> *tab = nullptr;
                int bc = -1, sign = 0;
                if (id[dir] == o->lo[dir] && s.udf_temp_lo[dir]) {
                    tab = &o->udfT_lo[dir];
                    bc = s.bclo_temp[dir];
                    sign = 1;
                } else if (id[dir] == o->hi[dir] + 1 && s.udf_temp_hi[dir]) {
                    tab = &o->udfT_hi[dir];
                    bc = s.bchi_temp[dir];
                    sign = -1;
                }
                if (!tab) continue;
                int p0 = (dir == 0) ? 1 : 0;
                int p1 = (dir == 2) ? 1 : 2;
                size_t f = ((size_t)id[p0] * (o->nc[p1] + 1) + id[p1]) * 2;
                double v0 = (*tab)[f], v1 = (*tab)[f + 1];
                int nb[3] = {i, j, k};
                nb[dir] += sign;
                if (bc == EXG_BCT_ISOTHERMAL) {
                    o->N(EXG_N_TEMPERATURE, n) = v0;
                } else if (bc == EXG_BCT_USERFLUX) {
                    o->N(EXG_N_TEMPERATURE, n) = o->N(EXG_N_TEMPERATURE, o->nidx_w(nb[0], nb[1], nb[2])) + v0 * o->dx[dir] / k_node(n);
                } else if (bc == EXG_BCT_CONVECTION) {
                    double Bi = v0 * o->dx[dir] / k_node(n);
                    o->N(EXG_N_TEMPERATURE, n) = (o->N(EXG_N_TEMPERATURE, o->nidx_w(nb[0], nb[1], nb[2])) + Bi * v1) / (1.0 + Bi);
                }
            }
        });
    // nodal_levelset_bcs_temperature, nodal_data_ops.cpp:235-349.  The
    // heat-flux and convective forms read a neighbour node that the same
    // pass may write (the reference's ParallelFor races there); neighbours
    // are read as they were before the body's pass.
    for (int b = 0; b < s.num_bodies; ++b) {
        if (!o->has_ls[b]) continue;
        const exg_body &body = s.bodies[b];
        int bc = body.temp_bc;
        if (bc == 0) continue;
        if (dirichlet_only && bc != 1) continue;
        const std::vector<double> Tsnap = o->node[EXG_N_TEMPERATURE];
        for_nodes(o, [&](int i, int j, int k, int64_t n) {
            double xp[3] = {o->plo[0] + i * o->dx[0], o->plo[1] + j * o->dx[1], o->plo[2] + k * o->dx[2]};
            double lsval;
            ls_eval(o, o->ls[b], xp, &lsval, nullptr);
            if (lsval >= 0.0 || o->N(EXG_N_MASS_SPHEAT, n) <= 0.0) return;
            double nd[3];
            ls_eval(o, o->ls[b], xp, nullptr, nd);
            double gm = 0.0;
            for (int d = 0; d < 3; d++) gm += nd[d] * nd[d];
            gm = std::sqrt(gm);
            if (gm < 1.0e-10) return;
            for (int d = 0; d < 3; d++) nd[d] /= gm;
            if (bc == 1) {
                o->N(EXG_N_TEMPERATURE, n) = body.T_wall;
                return;
            }
            int dd = 0;
            for (int d = 1; d < 3; d++)
                if (std::fabs(nd[d]) > std::fabs(nd[dd])) dd = d;
            int nb[3] = {i, j, k};
            nb[dd] += (nd[dd] > 0.0) ? 1 : -1;
            // lsbox.contains(nb): the node box with one ghost layer.  Ghost
            // nodes outside a non-periodic domain hold the 0 of
            // Reset_Nodaldata_to_Zero (AMReX-unpinned).
            if (!o->s.periodic[dd] && (nb[dd] < -1 || nb[dd] > o->nc[dd] + 1)) return;
            double kn = k_node(n);
            bool ghost = !o->s.periodic[dd] && (nb[dd] < 0 || nb[dd] > o->nc[dd]);
            double Tnb = ghost ? 0.0 : Tsnap[o->nidx_w(nb[0], nb[1], nb[2])];
            if (bc == 3)
                o->N(EXG_N_TEMPERATURE, n) = Tnb + body.heat_flux * o->dx[dd] / kn;
            else if (bc == 4) {
                double Bi = body.h_conv * o->dx[dd] / kn;
                o->N(EXG_N_TEMPERATURE, n) = (Tnb + Bi * body.T_inf) / (1.0 + Bi);
            }
        });
    }
}

// interpolate_from_grid_temperature, mpm_particle_grid_ops.cpp:1129-1270.
// The scheme is chosen by the x-direction order (:1192-1213).
void orc_g2p_temperature(orc_ctx *o, int update_temperature, int update_heatflux) {
    const exg_specs &s = o->s;
    for_particles(o, [&](int64_t p) {
        if (!o->alive(p) || o->idat[EXG_I_PHASE][p] != 0) return;
        double xp[3] = {o->pos[0][p], o->pos[1][p], o->pos[2][p]};
        int iv[3];
        o->cell(p, iv);
        int mn[3], mx[3];
        for (int d = 0; d < 3; ++d) compute_bounds(iv[d], o->lo[d], o->hi[d], s.order[d], s.periodic[d], mn[d], mx[d]);
        if (update_temperature) {
            double vals[2];
            interp_two(o, s.order[0], xp, iv, mn, mx, o->node[EXG_N_DELTA_TEMPERATURE], o->node[EXG_N_DELTA_TEMPERATURE], vals);
            o->R(EXG_R_TEMPERATURE, p) += vals[0];
        }
        if (update_heatflux) {
            double gT[3] = {0, 0, 0};
            for (int n = mn[2]; n < mx[2]; ++n)
                for (int m = mn[1]; m < mx[1]; ++m)
                    for (int l = mn[0]; l < mx[0]; ++l) {
                        int st[3] = {l, m, n};
                        double g[3];
                        basis_and_grad(o, st, iv, xp, g);
                        double Tn = o->node[EXG_N_TEMPERATURE][o->nidx_w(iv[0] + l, iv[1] + m, iv[2] + n)];
                        for (int d = 0; d < 3; ++d) gT[d] += Tn * g[d];
                    }
            for (int d = 0; d < 3; ++d) o->R(EXG_R_HEATFLUX + d, p) = -o->R(EXG_R_THERMCOND, p) * gT[d];
        }
    });
}

// Initialise_Internal_Forces, Source/mpm_init.cpp:368-445.
void orc_init_internal_forces(orc_ctx *o) {
    orc_p2g_momentum(o, 1, 1, 1);
    orc_backup_current_velocity(o);
    orc_g2p_momentum(o, 0, 1, 0.0);
    // apply_constitutive_model(dt = 0, applied_strainrate) (:398): always
    // the total formulation
    stress_strain(o, -std::numeric_limits<double>::infinity(), 0.0, true);
    if (o->s.use_temp) {
        orc_p2g_temperature(o, 1, 1, 0);
        orc_backup_current_temperature(o);
        // nodal_bcs_temperature only (:426-432): walls, no UDF, no EB
        exg_specs saved = o->s;
        for (int d = 0; d < 3; ++d) o->s.udf_temp_lo[d] = o->s.udf_temp_hi[d] = nullptr;
        o->s.num_bodies = 0;
        orc_apply_nodal_bcs_temperature(o, 0.0, 0.0, 0);
        o->s = saved;
        orc_store_delta_temperature(o);
        orc_g2p_temperature(o, 1, 1);
    }
}

// One iteration of the main.cpp:83-171 loop body.
int orc_step(orc_ctx *o, int nsteps) {
    int status = EXG_OK;
    const exg_specs &s = o->s;
    for (int it = 0; it < nsteps; ++it) {
        o->steps++;
        int rc = orc_redistribute(o);
        if (rc) status = rc;
        double dt = orc_calculate_time_step(o);
        orc_reset_nodaldata(o);
        orc_p2g_momentum(o, 1, 1, 1);
        orc_backup_current_velocity(o);
        orc_nodal_time_update_momentum(o, dt);
        rc = orc_apply_nodal_bcs(o, dt, o->time);
        if (rc) status = rc;
        if (s.use_temp) {
            orc_p2g_temperature(o, 1, 1, 1);
            orc_backup_current_temperature(o);
            orc_nodal_time_update_temperature(o, dt);
            orc_apply_nodal_bcs_temperature(o, dt, o->time, s.stress_update_scheme == 1);
            orc_store_delta_temperature(o);
        }
        if (s.stress_update_scheme == 0) {
            orc_g2p_momentum(o, 1, 1, dt);
            if (s.use_temp) orc_g2p_temperature(o, 1, 1);
            rc = orc_update_mp_positions(o, dt);
            if (rc) status = rc;
        } else {
            orc_g2p_momentum(o, 1, 0, dt);
            orc_p2g_momentum(o, 0, 1, 0);
            rc = orc_apply_nodal_bcs(o, dt, o->time);
            if (rc) status = rc;
            orc_g2p_momentum(o, 0, 1, dt);
            if (s.use_temp) {
                orc_g2p_temperature(o, 1, 0);
                orc_p2g_temperature(o, 1, 0, 1);
                orc_apply_nodal_bcs_temperature(o, dt, o->time, 0);
                orc_g2p_temperature(o, 0, 1);
            }
            rc = orc_update_mp_positions(o, dt);
            if (rc) status = rc;
        }
        rc = orc_redistribute(o);
        if (rc) status = rc;
        orc_update_mp_volume(o);
        orc_calculate_mp_stress_strain(o, o->time, dt);
        o->time += dt;
        o->last_dt = dt;
    }
    return status;
}

void orc_get_time(orc_ctx *o, double *time, double *last_dt, int64_t *steps) {
    if (time) *time = o->time;
    if (last_dt) *last_dt = o->last_dt;
    if (steps) *steps = o->steps;
}

// Do_All_Diagnostics reductions (Source/mpm_diagnostics.cpp:23-216), over
// every particle in the container (all phases).
void orc_diagnostics(orc_ctx *o, exg_diag *out) {
    std::memset(out, 0, sizeof(*out));
    for (int d = 0; d < 3; ++d) {
        out->minpos[d] = std::numeric_limits<double>::max();
        out->maxpos[d] = -std::numeric_limits<double>::max();
    }
    double mvm = 0.0;
    for (int64_t p = 0; p < o->np; ++p) {
        if (!o->alive(p)) continue;
        out->np++;
        double m = o->R(EXG_R_MASS, p);
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) v2 += o->R(EXG_R_VEL + d, p) * o->R(EXG_R_VEL + d, p);
        out->tke += 0.5 * m * v2;
        double se = o->R(EXG_R_STRESS + XX, p) * o->R(EXG_R_STRAIN + XX, p) +
                    o->R(EXG_R_STRESS + YY, p) * o->R(EXG_R_STRAIN + YY, p) +
                    o->R(EXG_R_STRESS + ZZ, p) * o->R(EXG_R_STRAIN + ZZ, p) +
                    2.0 * (o->R(EXG_R_STRESS + XY, p) * o->R(EXG_R_STRAIN + XY, p) +
                           o->R(EXG_R_STRESS + YZ, p) * o->R(EXG_R_STRAIN + YZ, p) +
                           o->R(EXG_R_STRESS + XZ, p) * o->R(EXG_R_STRAIN + XZ, p));
        out->tse += 0.5 * o->R(EXG_R_VOLUME, p) * se;
        out->mass += m;
        for (int d = 0; d < 3; ++d) out->momentum[d] += m * o->R(EXG_R_VEL + d, p);
        mvm += m * std::sqrt(v2);
        for (int d = 0; d < 3; ++d) {
            out->minpos[d] = std::min(out->minpos[d], o->pos[d][p]);
            out->maxpos[d] = std::max(out->maxpos[d], o->pos[d][p]);
        }
    }
    for (int d = 0; d < 3; ++d) out->mwa_vel[d] = out->momentum[d] / out->mass;
    out->mwa_velmag = mvm / out->mass;
}

// Tile-major cell key: tile index over the node-tile grid (ceil((nc+1)/T)
// tiles per axis, x fastest) times T^3 plus the cell's index inside the tile
// (x fastest).  Particles outside the domain get 0xFFFFFFFF.
void orc_sort_keys(orc_ctx *o, int T, uint32_t *keys, int32_t *perm) {
    // the B200 binning: cells, or with uniform quadratic B-splines the
    // nearest node floor((x - plo) / dx + 1/2) (wrapped on periodic axes);
    // particles outside the domain's cells get the sentinel key
    const bool dual = o->s.order[0] == 2 && o->s.order[1] == 2 && o->s.order[2] == 2;
    int nt[3];
    for (int d = 0; d < 3; ++d) nt[d] = o->s.periodic[d] ? o->nc[d] / T : (o->nc[d] + 1 + T - 1) / T;
    for (int64_t p = 0; p < o->np; ++p) {
        int iv[3];
        o->cell(p, iv);
        bool in = o->alive(p);
        for (int d = 0; d < 3; ++d) in = in && iv[d] >= 0 && iv[d] < o->nc[d];
        if (!in) {
            keys[p] = 0xFFFFFFFFu;
            continue;
        }
        if (dual)
            for (int d = 0; d < 3; ++d) {
                iv[d] = (int)std::floor((o->pos[d][p] - o->plo[d]) * o->dxi[d] + 0.5);
                if (o->s.periodic[d] && iv[d] >= o->nc[d]) iv[d] -= o->nc[d];
            }
        uint32_t tile = (uint32_t)((iv[2] / T) * nt[1] + iv[1] / T) * nt[0] + iv[0] / T;
        uint32_t loc = (uint32_t)(((iv[2] % T) * T + iv[1] % T) * T + iv[0] % T);
        keys[p] = tile * (uint32_t)(T * T * T) + loc;
    }
    std::vector<int32_t> idx(o->np);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return keys[a] < keys[b]; });
    std::copy(idx.begin(), idx.end(), perm);
}

}  // extern "C"

// --------------------------------------------------------- test hooks
// Direct access to the oracle's restated math, for the known-answer tests
// against the reference pin (oracle/ref_pin.cpp) and the golden fixtures.
extern "C" {
double orc_fn_spline(int kind, int type, double z) {
    switch (kind) {
        case 0: return cubic1d(type, z);
        case 1: return cubic1d_der(type, z);
        case 2: return quad1d(type, z);
        default: return quad1d_der(type, z);
    }
}
double orc_fn_basis_and_grad(orc_ctx *o, const int *st, const int *cell, const double *xp, double *grad) {
    return basis_and_grad(o, st, cell, xp, grad);
}
void orc_fn_interp_two(orc_ctx *o, int scheme, const double *xp, const int *cell, const int *mn, const int *mx,
                       int comp0, int comp1, double *vals) {
    interp_two(o, scheme, xp, cell, mn, mx, o->node[comp0], o->node[comp1], vals);
}
int orc_fn_applybc(const double *in, double *out, double mu, const double *n, int bc) {
    return applybc(in, out, mu, n, bc);
}
void orc_fn_linear_elastic(const double *eps, double *sig, double E, double nu) { linear_elastic(eps, sig, E, nu); }
void orc_fn_newtonian(const double *ed, double *sig, double mu, double p) { newtonian_fluid(ed, sig, mu, p); }
void orc_fn_neo_hookean(const double *F, double *sig, double E, double nu) { neo_hookean(F, sig, E, nu); }
void orc_fn_defgrad(double *F, const double *g, double dt) {
    double gv[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) gv[a][b] = g[3 * a + b];
    defgrad_update(F, gv, dt);
}
double orc_fn_levelset(orc_ctx *o, int body, const double *x, double *grad) {
    double v;
    ls_eval(o, o->ls[body], x, &v, grad);
    return v;
}
void orc_fn_compute_bounds(int ivd, int lod, int hid, int scheme, int periodic, int *bmin, int *bmax) {
    compute_bounds(ivd, lod, hid, scheme, periodic, *bmin, *bmax);
}
}
