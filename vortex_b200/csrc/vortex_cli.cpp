// vortex_cli.cpp — command-line driver with the reference program's
// interface (src/main.c of grechkin-pogrebnyakov/vortex) on the native API:
//
//   vortex -c file.conf [-l level] [-o log_file]
//
// Reads the same .conf keys and profile file, restarts from a Kadr frame
// (kadr_file, the step number taken from the file name), and writes the same
// outputs in the same formats and at the same points of the step:
//   output/kadrs/Kadr%06d.txt   every saving_step after the birth, and at the end
//   output/vels/contr_Vel%06d.txt  velocities at 500 control points
//                               (x = -0.15, y = 0.01 + 0.002 i) of the steps
//                               since the previous save
//   output/F_p.txt              step, Fx, Fy, M of the previous step, per step
//                               and once more at the end
//   timings_file (or stdout)    step, N, cumulative birth / velocity / step
//                               seconds
//   L.txt, M.txt                the panel system and its inverse when the
//                               matrix is generated (matrix_load 0); with
//                               matrix_load 1 the inverse is read from M.txt
// Each step runs as three device stages (birth; velocity with both
// diffusions; convection, compaction and collapse) with the outputs in
// between, as the reference orders them.
//
// Tracers (second_points_file, with rel_t): two copies of the points file are
// carried, inertial ("second": velocity relaxed towards the carrier velocity
// with time constant rel_t) and passive ("first": moved with the carrier
// velocity), each step after the outputs and before the vortices' velocity;
// they are written to output/second and output/first on saving steps and at
// the end, their velocities to output/vels/Vel%06d_4.txt (carrier) and
// _5.txt (as the reference: the passive set's file replaces the inertial
// set's), and reloaded from output/second and output/first on a restart when
// both frames of the start step exist (src/main.c:480-505, 606-648, 731-752).
// steady_flow: the vortices stay as loaded (no birth, velocity or
// convection, no vortex outputs); only the tracers move.
#include <sys/stat.h>

#include <cerrno>
#include <cstdarg>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "vortex_b200.h"
#include "vortex_b200_unit1.h"

namespace {

int g_level = 3;
FILE *g_log = nullptr;

void logm(int lev, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void logm(int lev, const char *fmt, ...) {
    if (lev > g_level) return;
    va_list ap;
    va_start(ap, fmt);
    FILE *f = g_log ? g_log : stderr;
    std::vfprintf(f, fmt, ap);
    std::fputc('\n', f);
    std::fflush(f);
    va_end(ap);
}

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

bool ensure_dir(const char *d) {
    struct stat st;
    if (stat(d, &st) == 0) return S_ISDIR(st.st_mode);
    return mkdir(d, 0777) == 0;
}

bool check(vx_status st, const char *what) {
    if (st == VX_OK) return true;
    logm(0, "%s failed: %s (%s)", what, vx_status_str(st), vx_last_error());
    return false;
}

bool save_kadr(vx_sim *s, int step) {
    int64_t n = 0;
    if (!check(vx_get_count(s, &n), "vx_get_count")) return false;
    std::vector<double> x(n), y(n), g(n);
    if (n > 0 && !check(vx_get_particles(s, x.data(), y.data(), g.data(), n, &n), "vx_get_particles")) return false;
    char name[256];
    std::snprintf(name, sizeof(name), "output/kadrs/Kadr%06d.txt", step);
    FILE *f = std::fopen(name, "w");
    if (!f) { logm(0, "cannot open %s: %s", name, std::strerror(errno)); return false; }
    std::fprintf(f, "%zu\n", (size_t)n);
    for (int64_t i = 0; i < n; ++i)
        std::fprintf(f, "%zu %lf %lf %lf %lf %lf %lf %lf\n", (size_t)i, 0.008, x[i], y[i], 0.0, 0.0, 0.0, g[i]);
    std::fclose(f);
    return true;
}

bool save_points(const char *folder, int step, const std::vector<double> &x, const std::vector<double> &y,
                 const std::vector<double> &g) {
    char name[256];
    std::snprintf(name, sizeof(name), "output/%s/Kadr%06d.txt", folder, step);
    FILE *f = std::fopen(name, "w");
    if (!f) { logm(0, "cannot open %s: %s", name, std::strerror(errno)); return false; }
    std::fprintf(f, "%zu\n", x.size());
    for (size_t i = 0; i < x.size(); ++i)
        std::fprintf(f, "%zu %lf %lf %lf %lf %lf %lf %lf\n", i, 0.008, x[i], y[i], 0.0, 0.0, 0.0, g[i]);
    std::fclose(f);
    return true;
}

void save_vel(int step, int stage, const std::vector<double> &x, const std::vector<double> &y,
              const std::vector<double> &u, const std::vector<double> &v) {
    char name[256];
    std::snprintf(name, sizeof(name), "output/vels/Vel%06d_%d.txt", step, stage);
    FILE *f = std::fopen(name, "w");
    if (!f) return;
    std::fprintf(f, "%zu\n", x.size());
    for (size_t i = 0; i < x.size(); ++i) std::fprintf(f, "%zu %lf %lf %lf %lf\n", i, x[i], y[i], u[i], v[i]);
    std::fclose(f);
}

bool file_exists(const char *name) {
    struct stat st;
    return stat(name, &st) == 0 && !S_ISDIR(st.st_mode);
}

bool load_kadr(const char *name, std::vector<double> &x, std::vector<double> &y, std::vector<double> &g) {
    FILE *f = std::fopen(name, "r");
    if (!f) { logm(0, "cannot open %s: %s", name, std::strerror(errno)); return false; }
    size_t n = 0;
    if (std::fscanf(f, "%zu", &n) != 1) { std::fclose(f); return false; }
    x.resize(n); y.resize(n); g.resize(n);
    for (size_t i = 0; i < n; ++i)
        if (std::fscanf(f, "%*u %*f %lf %lf %*f %*f %*f %lf", &x[i], &y[i], &g[i]) != 3) {
            logm(0, "%s: bad record %zu", name, i);
            std::fclose(f);
            return false;
        }
    std::fclose(f);
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    std::string cfg, logname;
    for (int i = 1; i < argc; ++i) {
        if (argv[i][0] != '-' || i + 1 >= argc) continue;
        switch (argv[i][1]) {
        case 'c': cfg = argv[++i]; break;
        case 'l': g_level = std::atoi(argv[++i]); break;
        case 'o': logname = argv[++i]; break;
        default: break;
        }
    }
    if (cfg.empty()) {
        std::printf("Usage:\nvortex -c file.conf\n");
        return 1;
    }
    if (!logname.empty()) g_log = std::fopen(logname.c_str(), "a");
    vx_conf c;
    vx_conf_default(&c);
    if (!check(vx_conf_read(cfg.c_str(), &c), "reading the configuration")) return 1;
    // tracers: inertial (second) and passive (first) copies of the points
    std::vector<double> x2, y2, g2, x1, y1, g1;
    if (c.second_points_file[0]) {
        if (c.rel_t == 0.0) { logm(0, "rel_t is necessary if the second component is set"); return 1; }
        if (!load_kadr(c.second_points_file, x2, y2, g2)) return 1;
        x1 = x2; y1 = y2; g1 = g2;
    } else if (c.steady_flow) {
        logm(0, "steady_flow and no second component");
        return 1;
    }
    const bool steady = c.steady_flow != 0;
    for (const char *d : {"output", "output/kadrs", "output/vels", "output/second", "output/first"})
        if (!ensure_dir(d)) { logm(0, "cannot create %s", d); return 1; }

    // profile, padded to a multiple of 32 for the matrix files
    int64_t P = 0;
    if (!check(vx_profile_read(c.pr_file, nullptr, 0, &P), "reading the profile")) return 1;
    const int64_t P32 = (P + 31) / 32 * 32;
    std::vector<vx_panel> pan((size_t)P32);
    std::memset(pan.data(), 0, sizeof(vx_panel) * (size_t)P32);
    if (!check(vx_profile_read(c.pr_file, pan.data(), P, &P), "reading the profile")) return 1;

    vx_sim *sim = nullptr;
    if (!check(vx_create(&c, pan.data(), P, 0, &sim), "vx_create")) return 1;
    const size_t S1 = (size_t)P + 1;
    if (!c.matrix_load) {
        // write L.txt / M.txt as the reference does; the device system is the same
        double *M = matr_creation(pan.data(), (size_t)P, (size_t)P32);
        if (!M) { logm(0, "Matrix creation error!"); return 1; }
        std::free(M);
    } else {
        size_t p = 0;
        double *M = load_matrix(&p);
        if (!M) { logm(0, "Matrix loading error!"); return 1; }
        if (p != (size_t)P) { logm(0, "matrix and profile mismatch"); std::free(M); return 1; }
        const size_t B1 = (size_t)P32 + 1;
        std::vector<double> Mu(S1 * S1);
        for (size_t i = 0; i < S1; ++i)
            for (size_t j = 0; j < S1; ++j) Mu[i * S1 + j] = M[i * B1 + j];
        std::free(M);
        if (!check(vx_set_matrix(sim, Mu.data()), "vx_set_matrix")) return 1;
    }

    int first = 0;
    int64_t steps = c.steps;
    if (c.kadr_file[0]) {
        std::vector<double> x, y, g;
        if (!load_kadr(c.kadr_file, x, y, g)) return 1;
        if (!check(vx_set_particles(sim, x.data(), y.data(), g.data(), (int64_t)x.size()), "vx_set_particles"))
            return 1;
        const char *k = std::strstr(c.kadr_file, "Kadr");
        int num = 0;
        if (k && std::sscanf(k + 4, "%d", &num) == 1) {
            first = num;
            steps += num;
        }
    }
    if (!check(vx_set_step_index(sim, first), "vx_set_step_index")) return 1;
    if (steady && (int64_t)first < c.v_inf_incr_steps) {
        logm(0, "steady_flow while the V_inf ramp (v_inf_incr_steps) is still running is not driven here");
        return 1;
    }
    if (first && !x2.empty()) {   // restart: the tracer frames of the start step, if both were saved
        char sname[256], fname[256];
        std::snprintf(sname, sizeof(sname), "output/second/Kadr%06d.txt", first);
        std::snprintf(fname, sizeof(fname), "output/first/Kadr%06d.txt", first);
        if (file_exists(sname) && file_exists(fname)) {
            if (!load_kadr(sname, x2, y2, g2) || !load_kadr(fname, x1, y1, g1)) return 1;
            if (x1.size() != x2.size()) { logm(0, "%s and %s hold different counts", sname, fname); return 1; }
        }
    }
    const size_t nt = x2.size();
    std::vector<double> ue(nt), ve(nt), u2(nt, 0.0), v2(nt, 0.0), u1(nt), v1(nt);

    const int NC = 500;
    std::vector<double> cpx(NC), cpy(NC);
    for (int i = 0; i < NC; ++i) { cpx[i] = -0.15; cpy[i] = 0.01 + 0.002 * i; }
    const size_t saving = c.saving_step > 0 ? (size_t)c.saving_step : 1;
    std::vector<double> vcx(NC * saving, 0.0), vcy(NC * saving, 0.0);
    size_t vc_blocks = 0;

    FILE *tim = c.timings_file[0] ? std::fopen(c.timings_file, "w") : stdout;
    if (!tim) { logm(0, "cannot open %s", c.timings_file); return 1; }
    FILE *fp = steady ? nullptr : std::fopen("output/F_p.txt", "w");   // no forces in a steady-flow run
    if (!steady && !fp) { logm(0, "unable to output forces: %s", std::strerror(errno)); return 1; }

    double t_birth = 0.0, t_speed = 0.0, t_step = 0.0;
    double f[4];
    int64_t n = 0;
    for (int k = first; k < steps; ++k) {
        double t0 = now_s();
        if (!steady) {
            if (!check(vx_stage(sim, VX_STAGE_BIRTH), "birth")) return 1;
            t_birth += now_s() - t0;
        }
        vx_get_count(sim, &n);
        std::fprintf(tim, "%d\tN = %zu\tCreation time = %f\tSpeed time = %f\tStep time = %f\n", k, (size_t)n,
                     t_birth, t_speed, t_step);
        std::fflush(tim);
        if ((size_t)k % saving == 0 && !steady) {
            char name[256];
            std::snprintf(name, sizeof(name), "output/vels/contr_Vel%06d.txt", k);
            FILE *o = std::fopen(name, "w");
            if (o) {
                for (size_t i = 0; i < (size_t)NC * saving; ++i)
                    std::fprintf(o, "%zu %lf %lf %lf %lf\n", i, cpx[i % NC], cpy[i % NC], vcx[i], vcy[i]);
                std::fclose(o);
            }
            vc_blocks = 0;
            if (!save_kadr(sim, k)) return 1;
        }
        if ((size_t)k % saving == 0 && nt) {
            if (!save_points("second", k, x2, y2, g2) || !save_points("first", k, x1, y1, g1)) return 1;
        }
        if (nt) {
            // inertial tracers: carrier velocity, relaxation towards it (the
            // previous velocity taken in FP32, as the reference), convection
            if (!check(vx_probe(sim, x2.data(), y2.data(), (int64_t)nt, ue.data(), ve.data()), "tracer velocity"))
                return 1;
            if (k == first) { u2 = ue; v2 = ve; }
            save_vel(k, 4, x2, y2, ue, ve);
            for (size_t i = 0; i < nt; ++i) {
                if (g2[i] == 0.0) { u2[i] = 0.0; v2[i] = 0.0; continue; }
                const float pu = (float)u2[i], pv = (float)v2[i];
                u2[i] = (ue[i] - pu) / c.rel_t * c.dt + pu;
                v2[i] = (ve[i] - pv) / c.rel_t * c.dt + pv;
            }
            save_vel(k, 5, x2, y2, u2, v2);
            if (!check(vx_move_points(sim, x2.data(), y2.data(), g2.data(), u2.data(), v2.data(), (int64_t)nt),
                       "tracer convection"))
                return 1;
            // passive tracers
            if (!check(vx_probe(sim, x1.data(), y1.data(), (int64_t)nt, u1.data(), v1.data()), "tracer velocity"))
                return 1;
            save_vel(k, 5, x1, y1, u1, v1);
            if (!check(vx_move_points(sim, x1.data(), y1.data(), g1.data(), u1.data(), v1.data(), (int64_t)nt),
                       "tracer convection"))
                return 1;
        }
        if (steady) {
            if (!check(vx_set_step_index(sim, k + 1), "vx_set_step_index")) return 1;
            continue;
        }
        if (vc_blocks < saving) {
            if (!check(vx_probe(sim, cpx.data(), cpy.data(), NC, &vcx[vc_blocks * NC], &vcy[vc_blocks * NC]),
                       "control velocities"))
                return 1;
            ++vc_blocks;
        }
        vx_get_forces(sim, f);
        std::fprintf(fp, "%d %lf %lf %lf\n", k, f[1], f[2], f[3]);
        std::fflush(fp);
        t0 = now_s();
        if (!check(vx_stage(sim, VX_STAGE_VELOCITY | VX_STAGE_DIFFUSION | VX_STAGE_WALL), "velocity")) return 1;
        t_speed += now_s() - t0;
        t0 = now_s();
        if (!check(vx_stage(sim, VX_STAGE_ADVECT | VX_STAGE_COMPACT | VX_STAGE_COLLAPSE1 | VX_STAGE_COLLAPSE2),
                   "step"))
            return 1;
        t_step += now_s() - t0;
        if (!check(vx_set_step_index(sim, k + 1), "vx_set_step_index")) return 1;
    }
    vx_get_count(sim, &n);
    std::fprintf(tim, "%d\tN = %zu\tCreation time = %f\tSpeed time = %f\tStep time = %f\n", (int)steps, (size_t)n,
                 t_birth, t_speed, t_step);
    if (!steady) {
        if (!save_kadr(sim, (int)steps)) return 1;
        vx_get_forces(sim, f);
        std::fprintf(fp, "%d %lf %lf %lf\n", (int)steps, f[1], f[2], f[3]);
    }
    if (fp) std::fclose(fp);
    if (nt && (!save_points("second", (int)steps, x2, y2, g2) || !save_points("first", (int)steps, x1, y1, g1)))
        return 1;
    if (tim != stdout) std::fclose(tim);
    vx_destroy(sim);
    if (g_log) std::fclose(g_log);
    return 0;
}
