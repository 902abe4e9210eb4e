// ref_pin.cpp -- exports the reference's own header-only math, compiled
// straight from the reference tree (Source/interpolants.H, mpm_kernels.H,
// constitutive_models.H, mpm_eb.H) with the type shim in ref_shim/, so the
// oracle's restatement can be checked against it bit for bit.  Test
// infrastructure only; built by `make -C oracle refpin` into oracle/_ref/.
#include <AMReX.H>
#include <constants.H>
#include <interpolants.H>
#include <mpm_kernels.H>
#include <constitutive_models.H>
#include <mpm_eb.H>

using amrex::Array4;
using amrex::GpuArray;
using amrex::IntVect;

namespace {
GpuArray<double, 3> ga(const double *a) { return {{a[0], a[1], a[2]}}; }
GpuArray<int, 3> gi(const int *a) { return {{a[0], a[1], a[2]}}; }
IntVect iv(const int *a) { return IntVect(a[0], a[1], a[2]); }
// View of a node array covering indices [lo, hi] (inclusive) per axis,
// x fastest, ncomp components back to back.
Array4<double> view(double *p, const int *lo, const int *hi) {
    Array4<double> a;
    a.p = p;
    a.lo = {lo[0], lo[1], lo[2]};
    a.hi = {hi[0], hi[1], hi[2]};
    return a;
}
}  // namespace

extern "C" {
double ref_cubic1d(int t, double z) { return cubicspline_1d(t, z); }
double ref_cubic1d_der(int t, double z) { return cubicspline_1d_der(t, z); }
double ref_quad1d(int t, double z) { return quadraticspline_1d(t, z); }
double ref_quad1d_der(int t, double z) { return quadraticspline_1d_der(t, z); }

double ref_basisval_and_grad(const int *st, const int *cell, const double *xp, const double *plo, const double *dx,
                             const int *order, const int *periodic, const int *lo, const int *hi, double *grad) {
    double x[3] = {xp[0], xp[1], xp[2]};
    return basisval_and_grad(iv(st), iv(cell), x, ga(plo), ga(dx), gi(order), gi(periodic), lo, hi, grad);
}
double ref_basisval(const int *st, const int *cell, const double *xp, const double *plo, const double *dx,
                    const int *order, const int *periodic, const int *lo, const int *hi) {
    double x[3] = {xp[0], xp[1], xp[2]};
    return basisval(iv(st), iv(cell), x, ga(plo), ga(dx), gi(order), gi(periodic), lo, hi);
}
double ref_basisvalder(int dir, const int *st, const int *cell, const double *xp, const double *plo, const double *dx,
                       const int *order, const int *periodic, const int *lo, const int *hi) {
    double x[3] = {xp[0], xp[1], xp[2]};
    return basisvalder(dir, iv(st), iv(cell), x, ga(plo), ga(dx), gi(order), gi(periodic), lo, hi);
}
// scheme 1/2/3: bilin/quadratic/cubic_interp_two over node data whose
// index box is [alo, ahi] with two components.
void ref_interp_two(int scheme, const double *xp, const int *cell, const int *mn, const int *mx, const double *plo,
                    const double *dx, double *nodes, const int *alo, const int *ahi, const int *periodic,
                    const int *lo, const int *hi, double *vals) {
    double x[3] = {xp[0], xp[1], xp[2]};
    Array4<double> a = view(nodes, alo, ahi);
    if (scheme == 1)
        bilin_interp_two(x, iv(cell), ga(plo), ga(dx), a, 0, 1, vals);
    else if (scheme == 2)
        quadratic_interp_two(x, iv(cell), iv(mn), iv(mx), ga(plo), ga(dx), a, 0, 1, gi(periodic), lo, hi, vals);
    else
        cubic_interp_two(x, iv(cell), iv(mn), iv(mx), ga(plo), ga(dx), a, 0, 1, gi(periodic), lo, hi, vals);
}
int ref_applybc(const double *in, double *out, double mu, const double *n, int bc) {
    double i3[3] = {in[0], in[1], in[2]}, n3[3] = {n[0], n[1], n[2]};
    try {
        return applybc(i3, out, mu, n3, bc);
    } catch (...) {
        return -1;
    }
}
void ref_linear_elastic(const double *eps, double *sig, double E, double nu) {
    double e[6];
    for (int i = 0; i < 6; ++i) e[i] = eps[i];
    linear_elastic(e, sig, E, nu);
}
void ref_neo_hookean(const double *F, double *sig, double E, double nu) {
    double f[9];
    for (int i = 0; i < 9; ++i) f[i] = F[i];
    neo_hookean(sig, f, E, nu);
}
void ref_linear_elastic_delta(const double *deps, double *dsig, double E, double nu) {
    double e[6];
    for (int i = 0; i < 6; ++i) e[i] = deps[i];
    linear_elastic_delta(e, dsig, E, nu);
}
void ref_newtonian(const double *ed, double *sig, double mu, double p) {
    double e[6];
    for (int i = 0; i < 6; ++i) e[i] = ed[i];
    Newtonian_Fluid(e, sig, mu, p);
}
void ref_defgrad_update(double *F, const double *gradv, double dt) {
    MPMParticleContainer::ParticleType p;
    for (int i = 0; i < 9; ++i) p.rdata(25 + i) = F[i];
    double g[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) g[a][b] = gradv[a * 3 + b];
    get_deformation_gradient_tensor(p, 25, g, dt);
    for (int i = 0; i < 9; ++i) F[i] = p.rdata(25 + i);
}
// get_levelset_value / get_levelset_grad with lsref = 1 over a nodal array
// covering [alo, ahi].
double ref_levelset(double *phi, const int *alo, const int *ahi, const double *plo, const double *dx,
                    const double *x, double *grad) {
    double xx[3] = {x[0], x[1], x[2]};
    Array4<double> a = view(phi, alo, ahi);
    get_levelset_grad(a, ga(plo), ga(dx), xx, 1.0, grad);
    return get_levelset_value(a, ga(plo), ga(dx), xx, 1.0);
}
}
