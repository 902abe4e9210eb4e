// Signed distance of one analytic level-set shape, shared by the host
// builder (exg_levelset_build) and the GPU builder (k_levelset_shapes).
//
// The reference builds these bodies with AMReX EB2 implicit functions and
// FillSignedDistance (Source/mpm_eb.cpp:150-388); the functions here are the
// exact signed distances of the same shapes, negative inside the solid, with
// <geom>_has_fluid_inside flipping the sign.  Because the per-step path only
// reads the level set injected onto the coarse nodes (average_down_nodal,
// Source/nodal_data_ops.cpp:147-153, Source/mpm_particle_timestep.cpp:261-277),
// an exact distance evaluated at the coarse nodes is what any ls_refinement
// would give.
#pragma once
#include <math.h>

#include "../../include/exg.h"

#ifdef __CUDACC__
#define EXG_HD __host__ __device__ __forceinline__
#else
#define EXG_HD inline
#endif

EXG_HD double exg_ls_max(double a, double b) { return a > b ? a : b; }
EXG_HD double exg_ls_min(double a, double b) { return a < b ? a : b; }
// Products and sums rounded one by one on both sides (the device compiler
// would otherwise fuse them into FMAs), so the GPU and the host builders
// give the same bits.
#ifdef __CUDA_ARCH__
EXG_HD double exg_ls_mul(double a, double b) { return __dmul_rn(a, b); }
EXG_HD double exg_ls_add(double a, double b) { return __dadd_rn(a, b); }
#else
EXG_HD double exg_ls_mul(double a, double b) { return a * b; }
EXG_HD double exg_ls_add(double a, double b) { return a + b; }
#endif

// Coordinate of node i along an axis: plo + i dx, rounded the same way on
// both sides.
EXG_HD double exg_ls_node_x(double plo, int i, double dx) { return exg_ls_add(plo, exg_ls_mul((double)i, dx)); }

EXG_HD double exg_ls_shape_eval(const exg_ls_shape &s, double x0, double x1, double x2) {
    const double x[3] = {x0, x1, x2};
    double v;
    if (s.kind == EXG_LS_SPHERE) {
        const double a = x[0] - s.center[0], b = x[1] - s.center[1], c = x[2] - s.center[2];
        v = sqrt(exg_ls_add(exg_ls_add(exg_ls_mul(a, a), exg_ls_mul(b, b)), exg_ls_mul(c, c))) - s.radius;
    } else if (s.kind == EXG_LS_PLANE) {
        // the normal points into the fluid: negative on the solid side
        const double nl = sqrt(exg_ls_add(exg_ls_add(exg_ls_mul(s.normal[0], s.normal[0]),
                                                     exg_ls_mul(s.normal[1], s.normal[1])),
                                          exg_ls_mul(s.normal[2], s.normal[2])));
        v = exg_ls_add(exg_ls_add(exg_ls_mul(x[0] - s.center[0], s.normal[0]),
                                  exg_ls_mul(x[1] - s.center[1], s.normal[1])),
                       exg_ls_mul(x[2] - s.center[2], s.normal[2])) /
            nl;
    } else if (s.kind == EXG_LS_CYLINDER) {
        double rr = 0.0;
        for (int d = 0; d < 3; ++d)
            if (d != s.dir) rr = exg_ls_add(rr, exg_ls_mul(x[d] - s.center[d], x[d] - s.center[d]));
        const double q0 = sqrt(rr) - s.radius, q1 = fabs(x[s.dir] - s.center[s.dir]) - 0.5 * s.height;
        const double o0 = exg_ls_max(q0, 0.0), o1 = exg_ls_max(q1, 0.0);
        v = sqrt(exg_ls_add(exg_ls_mul(o0, o0), exg_ls_mul(o1, o1))) + exg_ls_min(exg_ls_max(q0, q1), 0.0);
    } else {  // EXG_LS_BOX
        double o = 0.0, mx = -1e300;
        for (int d = 0; d < 3; ++d) {
            const double cc = 0.5 * (s.lo[d] + s.hi[d]), hh = 0.5 * (s.hi[d] - s.lo[d]);
            const double q = fabs(x[d] - cc) - hh;
            o = exg_ls_add(o, exg_ls_mul(exg_ls_max(q, 0.0), exg_ls_max(q, 0.0)));
            mx = exg_ls_max(mx, q);
        }
        v = sqrt(o) + exg_ls_min(mx, 0.0);
    }
    return s.inside ? -v : v;
}

// Union of shapes: the solid is where any shape is solid, so the level set
// is the minimum of the shapes' signed distances.
EXG_HD double exg_ls_union_eval(const exg_ls_shape *s, int n, double x0, double x1, double x2) {
    double v = 1e300;
    for (int i = 0; i < n; ++i) v = exg_ls_min(v, exg_ls_shape_eval(s[i], x0, x1, x2));
    return v;
}
