// exg_inputs.cpp -- inputs-file and particle-file handling of the B200 MPM
// step: a ParmParse-compatible "key = value ..." reader, the mapping of the
// reference's keys onto exg_specs (Source/mpm_specs.H:223-565,
// Source/mpm_init.cpp:175-268, Source/mpm_eb.cpp:403-547), analytic and UDF
// level sets, and the ASCII particle format (Source/mpm_init.cpp:942-1167).
#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/exg.h"
#include "exg_levelset.h"

struct exg_inputs {
    // key -> list of definitions (each a token list); the last one wins, as
    // ParmParse::query returns the last occurrence.
    std::map<std::string, std::vector<std::vector<std::string>>> kv;
    std::vector<void *> dl;  // dlopen handles kept alive for UDF pointers
    ~exg_inputs() {
        for (void *h : dl) dlclose(h);
    }
};

namespace {

std::vector<std::string> tokenize(const std::string &text) {
    std::vector<std::string> out;
    size_t i = 0, n = text.size();
    while (i < n) {
        char ch = text[i];
        if (ch == '#') {
            while (i < n && text[i] != '\n') ++i;
            continue;
        }
        if (std::isspace((unsigned char)ch)) {
            ++i;
            continue;
        }
        if (ch == '=') {
            out.push_back("=");
            ++i;
            continue;
        }
        if (ch == '"') {
            size_t j = text.find('"', i + 1);
            if (j == std::string::npos) j = n;
            out.push_back(text.substr(i + 1, j - i - 1));
            i = j + 1;
            continue;
        }
        size_t j = i;
        while (j < n && !std::isspace((unsigned char)text[j]) && text[j] != '=' && text[j] != '#') ++j;
        out.push_back(text.substr(i, j - i));
        i = j;
    }
    return out;
}

void add_definitions(exg_inputs *in, const std::vector<std::string> &tok) {
    size_t i = 0;
    while (i < tok.size()) {
        if (i + 1 < tok.size() && tok[i + 1] == "=" && tok[i] != "=") {
            std::string key = tok[i];
            i += 2;
            std::vector<std::string> vals;
            while (i < tok.size() && !(i + 1 < tok.size() && tok[i + 1] == "=") && tok[i] != "=") vals.push_back(tok[i++]);
            in->kv[key].push_back(vals);
        } else {
            ++i;
        }
    }
}

int parse_common(const std::string &text, int argc, const char *const *argv, exg_inputs **out) {
    auto *in = new exg_inputs();
    add_definitions(in, tokenize(text));
    std::string cli;
    for (int a = 0; a < argc; ++a) {
        if (!argv[a]) continue;
        cli += argv[a];
        cli += "\n";
    }
    add_definitions(in, tokenize(cli));
    *out = in;
    return EXG_OK;
}

const std::vector<std::string> *last(const exg_inputs *in, const std::string &key) {
    auto it = in->kv.find(key);
    if (it == in->kv.end() || it->second.empty()) return nullptr;
    return &it->second.back();
}

struct Reader {
    const exg_inputs *in;
    std::string err;
    bool has(const std::string &k) const { return last(in, k) != nullptr; }
    bool str(const std::string &k, std::string &v) const {
        auto *p = last(in, k);
        if (!p || p->empty()) return false;
        v = (*p)[0];
        return true;
    }
    bool real(const std::string &k, double &v) {
        auto *p = last(in, k);
        if (!p || p->empty()) return false;
        char *end = nullptr;
        double x = std::strtod((*p)[0].c_str(), &end);
        if (end == (*p)[0].c_str()) {
            err = "cannot read a number from " + k;
            return false;
        }
        v = x;
        return true;
    }
    bool integer(const std::string &k, int &v) {
        double d;
        if (!real(k, d)) return false;
        v = (int)d;
        return true;
    }
    bool boolean(const std::string &k, int &v) {
        auto *p = last(in, k);
        if (!p || p->empty()) return false;
        std::string s = (*p)[0];
        std::transform(s.begin(), s.end(), s.begin(), ::tolower);
        if (s == "true" || s == "t" || s == "1")
            v = 1;
        else if (s == "false" || s == "f" || s == "0")
            v = 0;
        else {
            err = "cannot read a bool from " + k;
            return false;
        }
        return true;
    }
    bool reals(const std::string &k, double *v, int n) {
        auto *p = last(in, k);
        if (!p || (int)p->size() < n) return false;
        for (int i = 0; i < n; ++i) v[i] = std::strtod((*p)[i].c_str(), nullptr);
        return true;
    }
    bool ints(const std::string &k, int *v, int n) {
        auto *p = last(in, k);
        if (!p || (int)p->size() < n) return false;
        for (int i = 0; i < n; ++i) v[i] = (int)std::strtod((*p)[i].c_str(), nullptr);
        return true;
    }
    bool get_reals(const std::string &k, double *v, int n) {
        if (!reals(k, v, n)) {
            if (err.empty()) err = "missing required key " + k;
            return false;
        }
        return true;
    }
    bool get_ints(const std::string &k, int *v, int n) {
        if (!ints(k, v, n)) {
            if (err.empty()) err = "missing required key " + k;
            return false;
        }
        return true;
    }
};

void *load_symbol(exg_inputs *in, const std::string &lib, const std::string &fn, std::string &err) {
    void *h = dlopen(lib.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        err = "cannot dlopen " + lib + ": " + dlerror();
        return nullptr;
    }
    in->dl.push_back(h);
    void *s = dlsym(h, fn.c_str());
    if (!s) err = "symbol " + fn + " not found in " + lib;
    return s;
}

int bc_code(const std::string &s) {  // mpm_specs.H:398-410
    if (s == "periodic") return EXG_BC_PERIODIC;
    if (s == "noslip") return EXG_BC_NOSLIP;
    if (s == "slip") return EXG_BC_SLIP;
    if (s == "partialslip") return EXG_BC_PARTIALSLIP;
    if (s == "outflow") return EXG_BC_OUTFLOW;
    return -1;
}
int bct_code(const std::string &s) {  // mpm_specs.H:475-487
    if (s == "periodic") return EXG_BCT_PERIODIC;
    if (s == "dirichlet") return EXG_BCT_ISOTHERMAL;
    if (s == "adiabatic") return EXG_BCT_ADIABATIC;
    if (s == "heatflux") return EXG_BCT_USERFLUX;
    if (s == "convective") return EXG_BCT_CONVECTION;
    return -1;
}

// Body parameter-prefix list of init_eb (mpm_eb.cpp:410-432): named bodies,
// else one legacy body read from the eb2 namespace, else none.
std::vector<std::string> body_prefixes(const exg_inputs *in, bool &legacy) {
    legacy = false;
    std::vector<std::string> out;
    auto *names = last(in, "eb2.body_names");
    if (names && !names->empty()) return *names;
    std::string g = "all_regular";
    if (auto *p = last(in, "eb2.geom_type"))
        if (!p->empty()) g = (*p)[0];
    if (g == "all_regular") return out;
    legacy = true;
    out.push_back("eb2");
    return out;
}

}  // namespace

extern "C" {

int exg_inputs_parse_text(const char *text, int argc, const char *const *argv, exg_inputs **out) {
    if (!out) return EXG_ERR_ARG;
    return parse_common(text ? text : "", argc, argv, out);
}

int exg_inputs_parse(const char *path, int argc, const char *const *argv, exg_inputs **out) {
    if (!out) return EXG_ERR_ARG;
    std::string text;
    if (path) {
        std::ifstream f(path);
        if (!f.good()) return EXG_ERR_IO;
        std::stringstream ss;
        ss << f.rdbuf();
        text = ss.str();
    }
    return parse_common(text, argc, argv, out);
}

void exg_inputs_free(exg_inputs *in) { delete in; }

int exg_inputs_get(const exg_inputs *in, const char *key, char *buf, size_t buflen) {
    if (!in || !key) return EXG_ERR_ARG;
    auto *p = last(in, key);
    if (!p) return EXG_ERR_ARG;
    std::string s;
    for (size_t i = 0; i < p->size(); ++i) {
        if (i) s += " ";
        s += (*p)[i];
    }
    if (buf && buflen) {
        std::strncpy(buf, s.c_str(), buflen - 1);
        buf[buflen - 1] = 0;
    }
    return (int)s.size();
}

void exg_specs_default(exg_specs *s) {
    std::memset(s, 0, sizeof(*s));
    s->gravity[1] = -9.81;  // mpm_specs.H:83 (0, -ACCG, 0)
    s->num_redist = 10;
    s->max_steps = 1;
    s->write_output_time = 1e200;
    s->write_diag_output_time = 1e200;
    s->order_scheme = 1;
    s->order[0] = s->order[1] = s->order[2] = 1;
    s->dt_max_limit = 1e0;
    s->dt_min_limit = 1e-12;
    s->cfl = 0.1;
    s->mass_tolerance = 1e-8;
    s->alpha_pic_flip = 0.95;
    s->stress_update_scheme = 0;  // the "USL" string default (mpm_specs.H:333)
    for (int d = 0; d < 3; ++d) {
        s->bclo[d] = s->bchi[d] = EXG_BC_SLIP;
        s->wall_mu_lo[d] = s->wall_mu_hi[d] = 0.1;
        s->bclo_temp[d] = s->bchi_temp[d] = EXG_BCT_ADIABATIC;
    }
    s->precision = EXG_PREC_FP64;
    s->tile = 0;
    s->autotune = 1;
}

int exg_specs_from_inputs(const exg_inputs *cin, exg_specs *s, char *errbuf, size_t errlen) {
    exg_inputs *in = const_cast<exg_inputs *>(cin);
    Reader r{in, ""};
    auto bad = [&](const std::string &m) {
        if (errbuf && errlen) {
            std::strncpy(errbuf, m.c_str(), errlen - 1);
            errbuf[errlen - 1] = 0;
        }
        return EXG_ERR_CONFIG;
    };
    exg_specs_default(s);
    if (!r.get_reals("mpm.prob_lo", s->plo, 3) || !r.get_reals("mpm.prob_hi", s->phi, 3) ||
        !r.get_ints("mpm.ncells", s->ncells, 3) || !r.get_ints("mpm.is_it_periodic", s->periodic, 3))
        return bad(r.err);
    int mgs = 0;
    if (!r.integer("mpm.max_grid_size", mgs)) return bad("missing required key mpm.max_grid_size");
    if (!r.integer("mpm.max_steps", s->max_steps)) return bad("missing required key mpm.max_steps");
    if (!r.real("mpm.final_time", s->final_time)) return bad("missing required key mpm.final_time");
    r.reals("mpm.gravity", s->gravity, 3);
    r.integer("mpm.calculate_strain_based_on_delta", s->calculate_strain_based_on_delta);
    s->write_output_time = s->final_time / 10.0;
    r.real("mpm.write_output_time", s->write_output_time);
    s->screen_output_time = s->write_output_time / 10.0;
    r.real("mpm.screen_output_time", s->screen_output_time);
    r.integer("mpm.num_redist", s->num_redist);
    r.integer("mpm.fixed_timestep", s->fixed_timestep);
    std::string sus = "USL";
    r.str("mpm.stress_update_scheme", sus);
    if (sus == "USL")
        s->stress_update_scheme = 0;
    else if (sus == "MUSL")
        s->stress_update_scheme = 1;
    else
        return bad("Stress update scheme should be USL/MUSL. But found " + sus);
    if (s->fixed_timestep == 1) {
        if (!r.real("mpm.timestep", s->timestep)) return bad("missing required key mpm.timestep");
    } else {
        s->timestep = 0.0;
    }
    r.real("mpm.alpha_pic_flip", s->alpha_pic_flip);
    r.real("mpm.dt_max_limit", s->dt_max_limit);
    r.real("mpm.dt_min_limit", s->dt_min_limit);
    r.real("mpm.CFL", s->cfl);
    r.real("mpm.applied_strainrate", s->applied_strainrate);
    s->applied_strainrate_time = s->final_time;
    r.real("mpm.applied_strainrate_time", s->applied_strainrate_time);
    r.integer("mpm.order_scheme", s->order_scheme);
    r.real("mpm.mass_tolerance", s->mass_tolerance);
    r.integer("mpm.external_loads", s->external_loads);
    if (s->external_loads) {
        if (!r.get_reals("mpm.force_slab_lo", s->force_slab_lo, 3) ||
            !r.get_reals("mpm.force_slab_hi", s->force_slab_hi, 3) || !r.get_reals("mpm.extforce", s->extforce, 3))
            return bad(r.err);
    }
    r.integer("mpm.print_diagnostics", s->print_diagnostics);
    if (s->print_diagnostics) {
        r.boolean("mpm.do_calculate_tke_tse", s->do_calculate_tke_tse);
        r.boolean("mpm.do_calculate_mwa_velcomp", s->do_calculate_mwa_velcomp);
        r.boolean("mpm.do_calculate_mwa_velmag", s->do_calculate_mwa_velmag);
        r.boolean("mpm.do_calculate_minmaxpos", s->do_calculate_minmaxpos);
        r.real("mpm.write_diag_output_time", s->write_diag_output_time);
    }
    // momentum wall BCs (mpm_specs.H:383-465)
    const char *ax = "xyz";
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            std::string face = std::string("bc_") + ax[d] + (side ? "hi" : "lo") + "_mom";
            std::string v;
            if (r.str("mpm." + face, v)) {
                int code = bc_code(v);
                if (code < 0) return bad("Unknown BC type: " + v);
                (side ? s->bchi : s->bclo)[d] = code;
            }
            std::string ns = "mpm." + face + ".";
            r.real(ns + "wall_mu", (side ? s->wall_mu_hi : s->wall_mu_lo)[d]);
            double wv[3];
            if (r.reals(ns + "wall_vel", wv, 3))
                for (int c = 0; c < 3; ++c) (side ? s->wall_vel_hi : s->wall_vel_lo)[d * 3 + c] = wv[c];
            std::string lib, fn;
            if (r.str(ns + "udf_lib", lib) && r.str(ns + "udf_func", fn)) {
                std::string e;
                void *sym = load_symbol(in, lib, fn, e);
                if (!sym) return bad(e);
                (side ? s->udf_wallvel_hi : s->udf_wallvel_lo)[d] = reinterpret_cast<exg_wallvel_udf>(sym);
            }
        }
    }
    // thermal (USE_TEMP in the reference; runtime key exg.use_temp here)
    r.boolean("exg.use_temp", s->use_temp);
    for (int d = 0; d < 3; ++d) {
        s->bclo_temp[d] = s->periodic[d] ? EXG_BCT_PERIODIC : EXG_BCT_ADIABATIC;
        s->bchi_temp[d] = s->bclo_temp[d];
        for (int side = 0; side < 2; ++side) {
            std::string face = std::string("bc_") + ax[d] + (side ? "hi" : "lo") + "_temp";
            std::string v;
            if (r.str("mpm." + face, v)) {
                int code = bct_code(v);
                if (code < 0) return bad("Unknown temperature BC type: " + v);
                (side ? s->bchi_temp : s->bclo_temp)[d] = code;
            }
            std::string ns = "mpm." + face + ".";
            r.real(ns + "T_wall", (side ? s->T_wall_hi : s->T_wall_lo)[d]);
            r.real(ns + "flux", (side ? s->flux_hi : s->flux_lo)[d]);
            r.real(ns + "h", (side ? s->h_hi : s->h_lo)[d]);
            r.real(ns + "T_inf", (side ? s->Tinf_hi : s->Tinf_lo)[d]);
            std::string lib, fn;
            if (r.str(ns + "udf_lib", lib) && r.str(ns + "udf_func", fn)) {
                std::string e;
                void *sym = load_symbol(in, lib, fn, e);
                if (!sym) return bad(e);
                (side ? s->udf_temp_hi : s->udf_temp_lo)[d] = reinterpret_cast<exg_temp_udf>(sym);
            }
        }
    }
    // directional order fallback (mpm_init.cpp:175-268)
    if (s->order_scheme == 1) {
        s->order[0] = s->order[1] = s->order[2] = 1;
    } else if (s->order_scheme == 2 || s->order_scheme == 3) {
        for (int d = 0; d < 3; ++d) {
            int nc = s->ncells[d];
            s->order[d] = (s->periodic[d] == 0) ? ((nc < 5) ? 1 : s->order_scheme) : ((nc < 3) ? 1 : s->order_scheme);
        }
    } else {
        return bad("Order scheme not implemented yet (use 1 or 3).");
    }
    // level-set bodies (mpm_eb.cpp:410-547)
    bool legacy = false;
    std::vector<std::string> bodies = body_prefixes(in, legacy);
    if ((int)bodies.size() > EXG_MAX_BODIES) return bad("Number of EB bodies exceeds EXAGOOP_MAX_LS_BODIES");
    s->num_bodies = (int)bodies.size();
    for (size_t b = 0; b < bodies.size(); ++b) {
        const std::string pre = bodies[b] + ".";
        exg_body &bd = s->bodies[b];
        std::string mom = "noslipwall";
        bool has_mom = r.str(pre + "levelset_mom", mom);
        if (!has_mom && legacy) {
            int li = -1;
            if (r.integer("mpm.levelset_bc", li)) mom = (li == 2) ? "slipwall" : (li == 3 ? "partialslip" : "noslipwall");
        }
        if (mom == "noslipwall")
            bd.mom_bc = EXG_BC_NOSLIP;
        else if (mom == "slipwall")
            bd.mom_bc = EXG_BC_SLIP;
        else if (mom == "partialslip")
            bd.mom_bc = EXG_BC_PARTIALSLIP;
        else
            return bad("unknown levelset_mom type '" + mom + "'");
        bd.wall_mu = 0.0;
        if (!r.real(pre + "lset_wall_mu", bd.wall_mu) && legacy) r.real("mpm.levelset_wall_mu", bd.wall_mu);
        r.reals(pre + "lset_wall_vel", bd.wall_vel, 3);
        std::string tb = "adiabatic";
        r.str(pre + "temp_bc_type", tb);
        if (tb == "adiabatic")
            bd.temp_bc = 0;
        else if (tb == "isothermal")
            bd.temp_bc = 1;
        else if (tb == "heatflux")
            bd.temp_bc = 3;
        else if (tb == "convective")
            bd.temp_bc = 4;
        else
            return bad("unknown temp_bc_type '" + tb + "'");
        r.real(pre + "lset_T_wall", bd.T_wall);
        r.real(pre + "lset_heat_flux", bd.heat_flux);
        r.real(pre + "lset_h_conv", bd.h_conv);
        r.real(pre + "lset_T_inf", bd.T_inf);
    }
    // B200 execution keys
    std::string prec = "fp64";
    r.str("exg.precision", prec);
    if (prec == "fp64")
        s->precision = EXG_PREC_FP64;
    else if (prec == "mixed")
        s->precision = EXG_PREC_MIXED;
    else
        return bad("exg.precision must be fp64 or mixed");
    r.integer("exg.tile", s->tile);
    r.integer("exg.autotune", s->autotune);
    if (!r.err.empty()) return bad(r.err);
    return EXG_OK;
}

// Analytic shape of body b from its <geom>_* keys (build_analytic_levelset,
// mpm_eb.cpp:150-388); udf_cpp and stl bodies have none.
int exg_levelset_shape(const exg_inputs *cin, int body, exg_ls_shape *sh) {
    exg_inputs *in = const_cast<exg_inputs *>(cin);
    if (!in || !sh || body < 0) return EXG_ERR_ARG;
    bool legacy = false;
    std::vector<std::string> bodies = body_prefixes(in, legacy);
    if (body >= (int)bodies.size()) return EXG_ERR_ARG;
    Reader r{in, ""};
    const std::string pre = bodies[body] + ".";
    std::string g;
    if (!r.str(pre + "geom_type", g)) return EXG_ERR_CONFIG;
    *sh = exg_ls_shape{};
    sh->center[0] = sh->center[1] = sh->center[2] = 0.5;
    sh->normal[1] = 1.0;
    sh->radius = 1.0;
    sh->height = 1.0;
    sh->dir = 2;
    if (g == "sphere") {
        sh->kind = EXG_LS_SPHERE;
        if (!r.real(pre + "sphere_radius", sh->radius) || !r.reals(pre + "sphere_center", sh->center, 3))
            return EXG_ERR_CONFIG;
        r.boolean(pre + "sphere_has_fluid_inside", sh->inside);
    } else if (g == "plane") {
        sh->kind = EXG_LS_PLANE;
        if (!r.reals(pre + "plane_point", sh->center, 3) || !r.reals(pre + "plane_normal", sh->normal, 3))
            return EXG_ERR_CONFIG;
        r.boolean(pre + "plane_has_fluid_inside", sh->inside);
    } else if (g == "cylinder") {
        sh->kind = EXG_LS_CYLINDER;
        if (!r.real(pre + "cylinder_radius", sh->radius) || !r.reals(pre + "cylinder_center", sh->center, 3))
            return EXG_ERR_CONFIG;
        r.real(pre + "cylinder_height", sh->height);
        r.integer(pre + "cylinder_direction", sh->dir);
        if (sh->dir < 0 || sh->dir > 2) return EXG_ERR_CONFIG;
        r.boolean(pre + "cylinder_has_fluid_inside", sh->inside);
    } else if (g == "box") {
        sh->kind = EXG_LS_BOX;
        if (!r.reals(pre + "box_lo", sh->lo, 3) || !r.reals(pre + "box_hi", sh->hi, 3)) return EXG_ERR_CONFIG;
        r.boolean(pre + "box_has_fluid_inside", sh->inside);
    } else {
        return EXG_ERR_UNSUPPORTED;  // udf_cpp (no analytic form), stl and wedge_hopper (AMReX EB2 only)
    }
    if (!r.err.empty()) return EXG_ERR_CONFIG;
    return EXG_OK;
}

// Nodal level set of body b: phi < 0 inside the solid.  Analytic shapes are
// exact signed distances (the reference builds them with AMReX EB2 and
// FillSignedDistance, whose discrete distance this does not reproduce);
// udf_cpp evaluates the user's levelset_phi at the nodes as
// build_udf_levelset does (mpm_eb.cpp:100-148).
int exg_levelset_build(const exg_inputs *cin, const exg_specs *s, int body, double *phi) {
    exg_inputs *in = const_cast<exg_inputs *>(cin);
    if (!in || !s || !phi || body < 0) return EXG_ERR_ARG;
    bool legacy = false;
    std::vector<std::string> bodies = body_prefixes(in, legacy);
    if (body >= (int)bodies.size()) return EXG_ERR_ARG;
    Reader r{in, ""};
    const std::string pre = bodies[body] + ".";
    std::string g;
    if (!r.str(pre + "geom_type", g)) return EXG_ERR_CONFIG;
    exg_levelset_udf udf = nullptr;
    exg_ls_shape sh{};
    if (g == "udf_cpp") {
        std::string so, e;
        if (!r.str(pre + "udf_so_file", so)) return EXG_ERR_CONFIG;
        void *sym = load_symbol(in, so, "levelset_phi", e);
        if (!sym) return EXG_ERR_IO;
        udf = reinterpret_cast<exg_levelset_udf>(sym);
    } else {
        const int rc = exg_levelset_shape(in, body, &sh);
        if (rc != EXG_OK) return rc;
    }
    int nn[3];
    double dx[3];
    for (int d = 0; d < 3; ++d) {
        nn[d] = s->ncells[d] + 1;
        dx[d] = (s->phi[d] - s->plo[d]) / s->ncells[d];
    }
    for (int k = 0; k < nn[2]; ++k)
        for (int j = 0; j < nn[1]; ++j)
            for (int i = 0; i < nn[0]; ++i) {
                const double x0 = exg_ls_node_x(s->plo[0], i, dx[0]), x1 = exg_ls_node_x(s->plo[1], j, dx[1]),
                             x2 = exg_ls_node_x(s->plo[2], k, dx[2]);
                phi[((long long)k * nn[1] + j) * nn[0] + i] = udf ? udf(x0, x1, x2) : exg_ls_shape_eval(sh, x0, x1, x2);
            }
    return EXG_OK;
}

int exg_particles_alloc(int64_t np, exg_particle_soa *p) {
    if (!p || np < 0) return EXG_ERR_ARG;
    p->np = np;
    size_t n = (size_t)(np > 0 ? np : 1);
    p->pos = (double *)std::calloc(3 * n, sizeof(double));
    p->rdata = (double *)std::calloc(EXG_NREAL * n, sizeof(double));
    p->idata = (int32_t *)std::calloc(EXG_NINT * n, sizeof(int32_t));
    if (!p->pos || !p->rdata || !p->idata) return EXG_ERR_ALLOC;
    return EXG_OK;
}

void exg_particles_free(exg_particle_soa *p) {
    if (!p) return;
    std::free(p->pos);
    std::free(p->rdata);
    std::free(p->idata);
    p->pos = p->rdata = nullptr;
    p->idata = nullptr;
    p->np = 0;
}

// InitParticles (Source/mpm_init.cpp:942-1167), 3-D: header "dim: 3",
// "number_of_material_points: N", one '#' line, then per particle
// phase x y z radius density vx vy vz model (E nu | K gamma mu)
// [T cp k Q].  Derived fields as the reference sets them.
int exg_particles_read_ascii(const char *path, int use_temp, exg_particle_soa *out) {
    if (!path || !out) return EXG_ERR_ARG;
    std::ifstream f(path);
    if (!f.good()) return EXG_ERR_IO;
    std::string label;
    int dim = -1;
    long long np = -1;
    if (!(f >> label >> dim) || label != "dim:" || dim != 3) return EXG_ERR_IO;
    if (!(f >> label >> np) || label != "number_of_material_points:" || np <= 0) return EXG_ERR_IO;
    std::string line;
    std::getline(f, line);
    std::getline(f, line);
    if (line.empty() || line[0] != '#') return EXG_ERR_IO;
    if (exg_particles_alloc(np, out) != EXG_OK) return EXG_ERR_ALLOC;
    const size_t n = (size_t)np;
    auto R = [&](int field, size_t i) -> double & { return out->rdata[(size_t)field * n + i]; };
    auto I = [&](int field, size_t i) -> int32_t & { return out->idata[(size_t)field * n + i]; };
    const double fourbythree = 1.3333333333, pi = 3.141592654;  // constants.H:9-10
    for (size_t i = 0; i < n; ++i) {
        int phase, model;
        double x[3], rad, dens, v[3];
        if (!(f >> phase >> x[0] >> x[1] >> x[2] >> rad >> dens >> v[0] >> v[1] >> v[2] >> model)) {
            exg_particles_free(out);
            return EXG_ERR_IO;
        }
        I(EXG_I_PHASE, i) = phase;
        I(EXG_I_RIGID_ID, i) = -1;
        I(EXG_I_MODEL, i) = model;
        for (int d = 0; d < 3; ++d) {
            out->pos[(size_t)d * n + i] = x[d];
            R(EXG_R_VEL + d, i) = v[d];
        }
        R(EXG_R_RADIUS, i) = rad;
        R(EXG_R_DENSITY, i) = dens;
        if (model == 0 || model == 2) {
            f >> R(EXG_R_E, i) >> R(EXG_R_NU, i);
        } else if (model == 1) {
            f >> R(EXG_R_BULK, i) >> R(EXG_R_GAMMA, i) >> R(EXG_R_VISC, i);
        } else {
            exg_particles_free(out);
            return EXG_ERR_IO;
        }
        if (use_temp) f >> R(EXG_R_TEMPERATURE, i) >> R(EXG_R_SPHEAT, i) >> R(EXG_R_THERMCOND, i) >> R(EXG_R_HEATSRC, i);
        if (!f) {
            exg_particles_free(out);
            return EXG_ERR_IO;
        }
        double vol = fourbythree * pi * std::pow(rad, 3.0);
        R(EXG_R_VOLUME, i) = vol;
        R(EXG_R_MASS, i) = dens * vol;
        R(EXG_R_JACOBIAN, i) = 1.0;
        R(EXG_R_VOL_INIT, i) = vol;
        for (int d = 0; d < 3; ++d) R(EXG_R_DEFGRAD + 4 * d, i) = 1.0;
    }
    return EXG_OK;
}

}  // extern "C"
