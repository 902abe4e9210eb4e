"""Shared comparison rules of the GPU parity tests.

FP64 tolerance: 1e-10 relative to a field's max norm.  Two fields carry a
conditioning term on top of it, both from the reference's own formulas:

* The Tait pressure p = K((1/J)^gamma - 1) (Source/mpm_particle_container.cpp:
  113-120) has absolute sensitivity gamma K J^-(gamma+1) to J.  Near rest
  (J - 1 ~ 1e-6, |p| ~ 10 Pa for water) one ulp of J (2.2e-16) moves p by
  gamma K x 2.2e-16 ~ 3e-9 Pa, above 1e-10 |p|.  The GPU's J and the
  oracle's differ by such ulps (the FP64 GPU path keeps E = F - I and the
  P2G sums in another order), so p, and the stress that contains it
  (Newtonian_Fluid, Source/constitutive_models.H:118-159), are compared within
  1e-10 |p|max plus twice gamma K J^-(gamma+1) |dJ| at the worst particle,
  plus a few ulps of K for the power itself; J itself stays within 1e-10.
* Nodal velocities v = p/m at nodes far lighter than the heaviest: the
  fixed-point nodal sums have absolute precision (2^-61 of the channel
  bound), so v is compared where m >= 1e-6 max m, and the momentum m v
  everywhere.
"""
import numpy as np

import exagoop_b200.native as nt

TOL64 = 1e-10


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def tait_slack(g, r):
    """Absolute pressure slack of the Tait particles (0 without fluid)."""
    fl = r.idata[nt.I_MODEL] == 1
    if not fl.any():
        return 0.0
    K, gam = r.rdata[nt.R_BULK][fl], r.rdata[nt.R_GAMMA][fl]
    J0, J1 = r.rdata[nt.R_JACOBIAN][fl], g.rdata[nt.R_JACOBIAN][fl]
    dJ = np.abs(J1 - J0)
    sens = gam * K * np.minimum(J0, J1) ** (-gam - 1.0)
    return float(2.0 * (sens * dJ).max() + 8.0 * 2.2e-16 * K.max())


def field_errors(g, r, fields):
    """Max error per field relative to its max norm, the pressure and
    stress after removing the Tait slack."""
    slack = tait_slack(g, r)
    out = {}
    for name, f, k in fields:
        a, b = g.rdata[f:f + k], r.rdata[f:f + k]
        scale = max(np.abs(b).max(), 1e-300)
        d = np.abs(a - b).max()
        if name in ("pressure", "stress") and slack > 0.0:
            d = max(0.0, d - slack)
        out[name] = float(d / scale)
    return out


def node_velocity_check(m, v_gpu, v_ref, tol=TOL64):
    """Nodal velocity where the node carries mass >= 1e-6 of the heaviest,
    nodal momentum m v everywhere; returns the two relative errors."""
    heavy = m >= 1e-6 * m.max()
    e_v = rel(v_gpu[heavy], v_ref[heavy]) if heavy.any() else 0.0
    e_p = rel(m * v_gpu, m * v_ref)
    return e_v, e_p
