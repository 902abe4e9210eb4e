// exg_driver.cpp -- command-line driver of the B200 MPM step, the
// counterpart of the reference executable's main() (Source/main.cpp:19-198).
//
//   exg_driver <inputs file> [key=value ...]
//
// It reads the same inputs file and ASCII particle file, builds the level-set
// bodies, runs Initialise_Internal_Forces, then loops explicit steps
// (exg_step) while steps < mpm.max_steps and time < mpm.final_time, printing
// the reference's "Iteration / Time / Dt / Time/Iter" line every
// screen_output_time, appending the diagnostics files every
// write_diag_output_time, and writing ASCII particle dumps every
// write_output_time when mpm.write_ascii is set.  AMReX plotfiles and
// checkpoints are not produced.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/exg.h"

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int check(int rc, exg_ctx *ctx, const char *what) {
    if (rc) {
        std::fprintf(stderr, "%s failed: status %d %s\n", what, rc, ctx ? exg_last_error(ctx) : "");
        std::exit(1);
    }
    return rc;
}

std::string get_str(exg_inputs *in, const char *key, const std::string &def) {
    char buf[4096];
    return exg_inputs_get(in, key, buf, sizeof buf) >= 0 ? std::string(buf) : def;
}

void mkdirs(const std::string &path) {
    std::string cur;
    std::stringstream ss(path);
    std::string part;
    if (!path.empty() && path[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

// One line per particle: x y z, the real fields in realData order, the
// int fields in intData order (the layout the reference's post-processing
// reads: column = realData index + 3 in 3-D, e.g. build_field_dict in
// Tests/1D_Heat_Conduction/PostProcess/validate.py:40-58 and vx in column 4
// in Tests/1D_Axial_Bar_Vibration/PostProcess/Calculate_Error.py:74-86),
// after five header lines: particle count, real and int field counts of the
// particle struct, and two zero counts of extra runtime fields.  The real
// field count is realData::count of the reference's build: 53 with
// mpm.use_temp, 46 (no thermal fields) without.
void write_ascii(const std::string &file, const exg_particle_soa &p, int use_temp) {
    const int nreal = use_temp ? EXG_NREAL : EXG_R_TEMPERATURE;
    std::ofstream f(file);
    f << p.np << "\n" << nreal << "\n" << EXG_NINT << "\n0\n0\n";
    f << std::setprecision(12);
    for (int64_t i = 0; i < p.np; ++i) {
        for (int d = 0; d < 3; ++d) f << p.pos[d * p.np + i] << ' ';
        for (int k = 0; k < nreal; ++k) f << p.rdata[(size_t)k * p.np + i] << ' ';
        for (int k = 0; k < EXG_NINT; ++k) f << p.idata[(size_t)k * p.np + i] << (k + 1 < EXG_NINT ? ' ' : '\n');
    }
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <inputs file> [key=value ...]\n", argv[0]);
        return 2;
    }
    exg_inputs *in = nullptr;
    if (exg_inputs_parse(argv[1], argc - 2, argv + 2, &in)) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 1;
    }
    exg_specs s;
    char err[512];
    if (exg_specs_from_inputs(in, &s, err, sizeof err)) {
        std::fprintf(stderr, "Error! %s\n", err);
        return 1;
    }
    if (get_str(in, "mpm.use_autogen", "0") != "0") {
        std::fprintf(stderr, "mpm.use_autogen is not supported: give mpm.particle_file\n");
        return 1;
    }
    const std::string pfile = get_str(in, "mpm.particle_file", "mpm_particles.dat");
    exg_particle_soa parts;
    if (exg_particles_read_ascii(pfile.c_str(), s.use_temp, &parts)) {
        std::fprintf(stderr, "cannot read particle file %s\n", pfile.c_str());
        return 1;
    }
    exg_ctx *ctx = nullptr;
    check(exg_ctx_create(&s, 0, &ctx), nullptr, "exg_ctx_create");
    // level-set bodies (init_eb): analytic shapes on the GPU, UDFs on the host
    check(exg_init_levelsets(ctx, in), ctx, "exg_init_levelsets");
    check(exg_particles_upload(ctx, &parts), ctx, "exg_particles_upload");
    check(exg_init_internal_forces(ctx), ctx, "exg_init_internal_forces");

    // diagnostics streams (utilities.cpp:452-535)
    const std::string diag_dir = get_str(in, "mpm.diagnostic_output_folder", "./Diagnostics/");
    std::ofstream ftke, fvel, fmag, fpos;
    if (s.print_diagnostics) {
        mkdirs(diag_dir);
        auto open = [&](std::ofstream &f, const char *name, const char *hdr) {
            f.open(diag_dir + "/" + name, std::ios::out | std::ios::app);
            f.precision(12);
            f << hdr;
        };
        if (s.do_calculate_tke_tse) open(ftke, "Total_Energies.dat", "iter,time,TKE,TSE,TE\n");
        if (s.do_calculate_mwa_velcomp) open(fvel, "VelComponents.dat", "iter,time,xvel,yvel,zvel\n");
        if (s.do_calculate_mwa_velmag) open(fmag, "VelMagnitudes.dat", "iter,time,velmag\n");
        if (s.do_calculate_minmaxpos) open(fpos, "MinMaxPosition.dat", "iter,time,xmin,ymin,xmax,ymax,zmin,zmax\n");
    }
    const int write_ascii_on = get_str(in, "mpm.write_ascii", "0") == "1" || get_str(in, "mpm.write_ascii", "") == "true";
    const std::string ascii_dir = "./Solution/ascii_files/";
    const std::string ascii_prefix = get_str(in, "mpm.prefix_asciifilename", "matpnt");
    const int digits = std::atoi(get_str(in, "mpm.num_of_digits_in_filenames", "6").c_str());
    auto dump = [&](double t) {
        if (!write_ascii_on) return;
        check(exg_particles_download(ctx, &parts), ctx, "exg_particles_download");
        std::ostringstream oss;
        oss << ascii_dir << ascii_prefix << "_t" << std::fixed << std::setprecision(digits) << t;
        // the prefix may hold folders of its own (the reference's
        // pre-processor writes "<tag>/matpnt")
        const std::string path = oss.str();
        mkdirs(path.substr(0, path.find_last_of('/') + 1));
        write_ascii(path, parts, s.use_temp);
    };

    int steps = 0;
    double time = 0.0, dt = 0.0;
    double output_time = 0.0, output_print = 0.0, diag_print = 0.0;
    dump(time);
    const double run_start = now();
    std::printf("\n Timestepping begins\n");
    while (steps < s.max_steps && time < s.final_time) {  // main.cpp:83-187
        steps++;
        const double t0 = now();
        check(exg_step(ctx, 1), ctx, "exg_step");
        int64_t nsteps;
        double tnew;
        check(exg_get_time(ctx, &tnew, &dt, &nsteps), ctx, "exg_get_time");
        if (diag_print >= s.write_diag_output_time) {
            exg_diag d;
            check(exg_diagnostics(ctx, &d), ctx, "exg_diagnostics");
            if (ftke.is_open()) ftke << steps << " " << time << " " << d.tke << " " << d.tse << " " << d.tke + d.tse << "\n";
            if (fvel.is_open())
                fvel << steps << " " << time << " " << d.mwa_vel[0] << " " << d.mwa_vel[1] << " " << d.mwa_vel[2] << "\n";
            if (fmag.is_open()) fmag << steps << " " << time << " " << d.mwa_velmag << "\n";
            if (fpos.is_open())
                fpos << steps << " " << time << " " << d.minpos[0] << " " << d.maxpos[0] << " " << d.minpos[1] << " "
                     << d.maxpos[1] << " " << d.minpos[2] << " " << d.maxpos[2] << "\n";
            diag_print = 0.0;
        }
        if (std::fabs(output_time - s.write_output_time) < dt * 0.5) {
            dump(time);
            output_time = 0.0;
        }
        time = tnew;
        output_time += dt;
        output_print += dt;
        diag_print += dt;
        const double per_iter = now() - t0;
        if (output_print >= s.screen_output_time) {
            std::printf(" Iteration: %10d,\tTime: %.10f,\tDt = %.5e,\t Time/Iter = %.10f\n", steps, time, dt, per_iter);
            output_print = 0.0;
        }
    }
    std::printf("\nSimulation run time = %f\n", now() - run_start);
    dump(time);
    exg_ctx_destroy(ctx);
    exg_particles_free(&parts);
    exg_inputs_free(in);
    return 0;
}
