// tsuner_run.cpp -- the drop-in TSUNER() whole-run entry point, the data.dat
// parser, and the NetCDF output with the reference layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <string>
#include <vector>

#include "cdf1.h"
#include "tsuner_b200.h"

namespace {

// Output file with the variables, dimensions and attributes of the
// reference writer (fgennc, GPU/netcdf.cu:38-242): dims x, y, time
// (unlimited); vars x, y, b(time,y,x), hmax, bmin, eta_max (y,x), time,
// eta, ux, uy, c (time,y,x); fill -1e30; CF-1.0 global attributes.
struct Output {
    tsu::cdf1::File f;
    int x_id = -1, y_id = -1, b_id = -1, hmax_id = -1, bmin_id = -1, etamax_id = -1, time_id = -1;
    int eta_id = -1, ux_id = -1, uy_id = -1, c_id = -1;
    int npx = 0, npy = 0;

    int open(const char *prefix, const SimParams &p) {
        npx = p.npx;
        npy = p.npy;
        std::string name = std::string(prefix) + ".nc";
        if (f.create(name.c_str())) return -1;
        int xd, yd, td;
        f.def_dim("x", npx, &xd);
        f.def_dim("y", npy, &yd);
        f.def_dim("time", 0, &td);
        f.def_var("x", tsu::cdf1::NC_DOUBLE_T, 1, &xd, &x_id);
        f.def_var("y", tsu::cdf1::NC_DOUBLE_T, 1, &yd, &y_id);
        int g2[2] = {yd, xd}, g3[3] = {td, yd, xd};
        f.def_var("b", tsu::cdf1::NC_DOUBLE_T, 3, g3, &b_id);
        f.def_var("hmax", tsu::cdf1::NC_DOUBLE_T, 2, g2, &hmax_id);
        f.def_var("bmin", tsu::cdf1::NC_DOUBLE_T, 2, g2, &bmin_id);
        f.def_var("eta_max", tsu::cdf1::NC_DOUBLE_T, 2, g2, &etamax_id);
        f.def_var("time", tsu::cdf1::NC_DOUBLE_T, 1, &td, &time_id);
        f.def_var("eta", tsu::cdf1::NC_DOUBLE_T, 3, g3, &eta_id);
        text(eta_id, "units", "meters");
        text(eta_id, "long_name", "Depth");
        f.def_var("ux", tsu::cdf1::NC_DOUBLE_T, 3, g3, &ux_id);
        text(ux_id, "units", "meters/second");
        text(ux_id, "long_name", "x-velocity");
        f.def_var("uy", tsu::cdf1::NC_DOUBLE_T, 3, g3, &uy_id);
        text(uy_id, "units", "meters/second");
        text(uy_id, "long_name", "y-velocity");
        f.def_var("c", tsu::cdf1::NC_DOUBLE_T, 3, g3, &c_id);
        text(c_id, "units", "adimensional");
        text(c_id, "long_name", "Volumetric Sediment Concentration");
        const double fill = -1e+30;
        fillatt(c_id, fill);
        text(hmax_id, "long_name", "hmax");
        text(hmax_id, "standard_name", "hmax");
        text(hmax_id, "units", "meters");
        fillatt(hmax_id, fill);
        text(bmin_id, "long_name", "bmin");
        text(bmin_id, "standard_name", "bmin");
        text(bmin_id, "units", "meters");
        fillatt(bmin_id, fill);
        text(etamax_id, "long_name", "eta_max");
        text(etamax_id, "standard_name", "eta_max");
        text(etamax_id, "units", "meters");
        fillatt(etamax_id, fill);
        text(x_id, "long_name", "x dim");
        text(x_id, "units", "meters");
        text(y_id, "long_name", "y dim");
        text(y_id, "units", "meters");
        text(time_id, "long_name", "Time");
        text(time_id, "units", "seconds");
        fillatt(eta_id, fill);
        fillatt(ux_id, fill);
        fillatt(uy_id, fill);
        text(-1, "Conventions", "CF-1.0");
        text(-1, "title", "TSUNER NOAA PMEL model output");
        text(-1, "creator_name", "Ernesto Guerrero Fernandez");
        text(-1, "institution", "NOAA/NCTR/UW");
        text(-1, "Paper", "https://repository.library.noaa.gov/view/noaa/67438/noaa_67438_DS1.pdf");
        text(-1, "Github", "https://github.com/ErnestoGuerreroFernandez");
        char date[32];
        std::time_t now = std::time(nullptr);
        std::strftime(date, sizeof(date), "%Y-%m-%d %H:%M:%S", std::localtime(&now));
        text(-1, "history", date);
        dbl(-1, "simulation_time", p.total_time);
        dbl(-1, "Sediment_relative_density", p.R);
        dbl(-1, "Sediment_mean_diameter", p.DS);
        dbl(-1, "Friction", p.FR * 8.0);
        dbl(-1, "Sediment_porosity", p.porosity);
        dbl(-1, "Sediment_critical_theta", p.OC);
        dbl(-1, "Geometric_mean_size_of_suspended_sediment", p.Dsg);
        if (f.enddef()) return -1;
        // cell-centre coordinates (initNC, GPU/netcdf.cu:263-277)
        std::vector<double> xg(npx), yg(npy);
        double dx = (p.xmax - p.xmin) / npx, dy = (p.ymax - p.ymin) / npy;
        for (int i = 0; i < npx; i++) xg[i] = p.xmin + (i + 0.5) * dx;
        for (int j = 0; j < npy; j++) yg[j] = p.ymin + (j + 0.5) * dy;
        if (f.put_var_double(x_id, xg.data()) || f.put_var_double(y_id, yg.data())) return -1;
        return 0;
    }
    void text(int v, const char *n, const char *s) { f.put_att_text(v, n, std::strlen(s), s); }
    void dbl(int v, const char *n, double d) { f.put_att_double(v, n, 1, &d); }
    void fillatt(int v, double fill) {
        f.put_att_double(v, "missing_value", 1, &fill);
        f.put_att_double(v, "_FillValue", 1, &fill);
    }
    int frame(int num, double t, const double *V, std::vector<double> &vec) {
        // saveNetCDF, GPU/netcdf.cu:379-435
        const size_t n = (size_t)npx * npy;
        const double eps = 2.220446049250313080847e-16;  // DBL_EPSILON
        size_t one = 1, st1 = (size_t)num;
        int r = f.put_vara_double(time_id, &st1, &one, &t);
        size_t start[3] = {(size_t)num, 0, 0}, count[3] = {1, (size_t)npy, (size_t)npx};
        for (size_t i = 0; i < n; i++) vec[i] = V[i] - V[3 * n + i];
        r |= f.put_vara_double(eta_id, start, count, vec.data());
        r |= f.sync();
        for (size_t i = 0; i < n; i++) vec[i] = V[n + i] / (V[i] + eps);
        r |= f.put_vara_double(ux_id, start, count, vec.data());
        r |= f.sync();
        for (size_t i = 0; i < n; i++) vec[i] = V[2 * n + i] / (V[i] + eps);
        r |= f.put_vara_double(uy_id, start, count, vec.data());
        r |= f.sync();
        for (size_t i = 0; i < n; i++) vec[i] = -V[3 * n + i];
        r |= f.put_vara_double(b_id, start, count, vec.data());
        r |= f.sync();
        for (size_t i = 0; i < n; i++) vec[i] = V[4 * n + i] / (V[i] + eps);
        r |= f.put_vara_double(c_id, start, count, vec.data());
        r |= f.sync();
        return r;
    }
};

bool g_quiet() {
    const char *q = std::getenv("TSU_QUIET");
    return q && *q && *q != '0';
}

}  // namespace

// data.dat reader (Problem_loader.cxx:264-342): a leading comment line, then
// for each value a "# label" line followed by the value line.
extern "C" int tsu_parse_data_dat(const char *path, SimParams *p, char *prefix, char *bathy_file, char *ic_file,
                                  char *mask_file, double *slr, char *tides_file, size_t cap) {
    if (!path || !p) return TSU_ERR_INVALID;
    std::ifstream in(path);
    if (!in) return TSU_ERR_IO;
    std::vector<std::string> vals;
    std::string line;
    bool first = true;
    while (std::getline(in, line)) {
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos) continue;
        if (line[a] == '#') {
            first = false;
            continue;
        }
        if (first) continue;
        size_t b = line.find_last_not_of(" \t\r");
        vals.push_back(line.substr(a, b - a + 1));
    }
    // 22 values: box (4), times (2), npx, npy, CFL, epsilon_h, R, DS, friction,
    // porosity, theta_c, Dsg, output prefix, bathymetry, IC, mask, SLR, tides
    if (vals.size() < 22) return TSU_ERR_INVALID;
    SimParams q{};
    try {
        q.xmin = std::stod(vals[0]);
        q.xmax = std::stod(vals[1]);
        q.ymin = std::stod(vals[2]);
        q.ymax = std::stod(vals[3]);
        q.total_time = std::stod(vals[4]);
        q.save_time = std::stod(vals[5]);
        q.npx = std::stoi(vals[6]);
        q.npy = std::stoi(vals[7]);
        q.CFL = std::stod(vals[8]);
        q.epsilon_h = std::stod(vals[9]);
        q.R = std::stod(vals[10]);
        q.DS = std::stod(vals[11]);
        double fr = std::stod(vals[12]);
        q.porosity = std::stod(vals[13]);
        q.OC = std::stod(vals[14]);
        q.Dsg = std::stod(vals[15]);
        if (slr) *slr = std::stod(vals[20]);
        tsu_derive_params(&q, fr);
    } catch (...) {
        return TSU_ERR_INVALID;
    }
    q.nvol = q.npx * q.npy;
    q.vmax = 10.0;
    q.dx = (q.xmax - q.xmin) / q.npx;  // Problem_loader.cxx:631-632
    q.dy = (q.ymax - q.ymin) / q.npy;
    *p = q;
    auto cp = [&](char *dst, const std::string &s) {
        if (dst && cap) {
            std::strncpy(dst, s.c_str(), cap - 1);
            dst[cap - 1] = 0;
        }
    };
    cp(prefix, vals[16]);
    cp(bathy_file, vals[17]);
    cp(ic_file, vals[18]);
    cp(mask_file, vals[19]);
    cp(tides_file, vals[21]);
    return TSU_OK;
}

// Whole run (GPU/main_TSUNER.cu:21-222 contract).
extern "C" int TSUNER(double *dVh, tsu_double2 *dVhu, double *dVH, int *fixH, SimParams params, char *input_prefix,
                      double *d, double *CC, double *tCC, unsigned long timeCC, double *dyrup, float *time_dyrup,
                      double &tiempo, int CudaDevice, double *tides_bd, float *tides_time, int tidesNPT) {
    (void)d;
    (void)dyrup;
    (void)time_dyrup;
    (void)tides_bd;
    (void)tides_time;
    (void)tidesNPT;
    TsuSwitches sw;
    tsu_get_default_switches(&sw);
    params.nvol = params.npx * params.npy;
    const size_t n = (size_t)params.nvol;
    std::vector<double> V, vec, plane;
    try {
        V.resize(5 * n);
        vec.resize(n);
    } catch (...) {
        return TSU_ERR_HOST_OOM;
    }
    for (size_t i = 0; i < n; i++) {  // SoA packing, GPU/main_TSUNER.cu:104-111
        V[i] = dVh[i];
        V[n + i] = dVhu[i].x;
        V[2 * n + i] = dVhu[i].y;
        V[3 * n + i] = dVH[i];
        V[4 * n + i] = 0.0;
    }
    TsuSolver *s = nullptr;
    int rc = tsu_create(&s, &params, &sw, CudaDevice);
    if (rc) return rc == TSU_ERR_GPU_OOM ? 1 : rc;
    struct Guard {
        TsuSolver *s;
        ~Guard() { tsu_destroy(s); }
    } guard{s};
    if ((rc = tsu_set_state(s, &V[0], &V[n], &V[2 * n], &V[3 * n], &V[4 * n]))) return rc;
    if ((rc = tsu_set_mask(s, fixH))) return rc;
    if (sw.read_files && (rc = tsu_set_boundary_series(s, CC, tCC, timeCC))) return rc;
    Output out;
    if (out.open(input_prefix, params)) return TSU_ERR_HOST_OOM;  // the reference returns 2 when initNC fails
    if ((rc = tsu_reset(s))) return rc;
    double t = 0, dt = 0;
    long steps = 0;
    tsu_get_time(s, &t, &dt, &steps);
    const bool quiet = g_quiet();
    if (!quiet) std::fprintf(stdout, "Initial deltaT = %e sec\n", dt);
    auto c0 = std::chrono::steady_clock::now();
    int niters = 0;
    double next_save = 0.0;
    std::vector<double> hm(n), em(n), bm(n);
    while (t < params.total_time) {
        if (params.save_time >= 0.0 && t >= next_save) {
            if ((rc = tsu_get_state(s, V.data())) || (rc = tsu_get_extrema(s, hm.data(), nullptr, em.data())))
                return rc;
            out.f.put_var_double(out.hmax_id, hm.data());
            out.f.put_var_double(out.etamax_id, em.data());
            out.frame(niters, t, V.data(), vec);
            niters++;
            next_save += params.save_time;
        }
        double stop = params.total_time;
        if (params.save_time >= 0.0) stop = std::min(stop, next_save);
        long before = steps;
        if (t < stop) {
            long done = 0;
            if ((rc = tsu_run_until(s, stop, 1L << 40, &done))) return rc;
        } else {
            if ((rc = tsu_step(s, 1))) return rc;  // the reference always steps after a save
        }
        tsu_get_time(s, &t, &dt, &steps);
        if (!quiet)
            std::fprintf(stdout, "Iterations %ld-%ld, deltaT = %e sec, Time = %g sec\n", before + 1, steps, dt, t);
    }
    if ((rc = tsu_get_state(s, V.data())) || (rc = tsu_get_extrema(s, hm.data(), bm.data(), em.data()))) return rc;
    out.frame(niters, t, V.data(), vec);
    out.f.put_var_double(out.hmax_id, hm.data());
    out.f.put_var_double(out.etamax_id, em.data());
    for (size_t i = 0; i < n; i++) bm[i] = -bm[i];  // GPU/main_TSUNER.cu:207-209
    out.f.put_var_double(out.bmin_id, bm.data());
    if (out.f.close()) return TSU_ERR_IO;
    tiempo = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
    return TSU_OK;
}
