// nctr.cpp -- the arithmetic of the reference's Read_files == 1 input
// pipeline (Problem_loader.cxx:355-625 with interpolations.cxx and
// tides.cxx): gridded bathymetry, non-erodible-bed and NCTR free-surface /
// velocity grids in geographic coordinates are interpolated onto the
// simulation grid, turned into the boundary series CC, mapped to Cartesian
// coordinates and assigned to the initial state.
//
// The reference reads its grids from NetCDF4 files; here the caller passes
// the grids as arrays (read by whatever NetCDF reader it has), and every
// expression follows the reference's operation order, so that the results
// are the reference's to the last bit (the unit is built without floating-
// point contraction, like the reference's host code).  Host code only: no
// device is touched.  Large loops run on the library's host thread pool.
// Positions are 64-bit; where the reference's int arithmetic or an index
// below 0 would leave its arrays (undefined there) the index is clamped.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hostio.h"
#include "tsuner_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;  // Sim_parameters.hxx:30
constexpr double kRe = 6371e3;                  // Sim_parameters.hxx:37
constexpr double kUnits = 0.01;                 // Sim_parameters.hxx:42 (NCTR centimetres -> metres)

// Lagrange basis on the reference interval [-1, 1] (interpolations.cxx:46-54)
inline double lag0(double x) { return x / 2.0 * (x - 1); }
inline double lag1(double x) { return 1 - x * x; }
inline double lag2(double x) { return x / 2.0 * (x + 1); }
// on three nodes (interpolations.cxx:67-75)
inline double node0(double x, double x0, double x1, double x2) { return ((x - x1) * (x - x2)) / ((x0 - x1) * (x0 - x2)); }
inline double node1(double x, double x0, double x1, double x2) { return ((x - x0) * (x - x2)) / ((x1 - x0) * (x1 - x2)); }
inline double node2(double x, double x0, double x1, double x2) { return ((x - x0) * (x - x1)) / ((x2 - x0) * (x2 - x1)); }
// tides.cxx:155-163
inline double tide0(double x, double xi, double xip, double, double dx) { return ((x - xi) * (x - xip) / (2 * dx * dx)); }
inline double tide1(double x, double, double xip, double xim, double dx) { return ((x - xim) * (x - xip) / (-dx * dx)); }
inline double tide2(double x, double xi, double, double xim, double dx) { return ((x - xim) * (x - xi) / (2 * dx * dx)); }

// the 3 x 3 neighbours of grid point (ig, jg) of an nx x ny grid, with the
// point itself standing in beyond the grid's edges
struct Stencil {
    long long c, L, R, U, D, LU, LD, RU, RD;
};
inline Stencil stencil_clamped(long long base, int ig, int jg, int nx, int ny) {
    Stencil s;
    s.c = base + (long long)jg * nx + ig;
    s.L = s.c - 1;
    s.R = s.c + 1;
    s.U = s.c + nx;
    s.D = s.c - nx;
    s.LU = s.U - 1;
    s.LD = s.D - 1;
    s.RU = s.U + 1;
    s.RD = s.D + 1;
    if (ig == 0) s.L = s.LU = s.LD = s.c;
    if (ig == nx - 1) s.R = s.RD = s.RU = s.c;
    if (jg == 0) s.D = s.LD = s.RD = s.c;
    if (jg == ny - 1) s.U = s.LU = s.RU = s.c;
    return s;
}
// the same as interpolate_CC writes it (interpolations.cxx:496-504): offsets
// switched off at the edges, diagonal points built from the clamped ones
inline Stencil stencil_offsets(long long base, int ig, int jg, int nx, int ny) {
    Stencil s;
    s.c = base + (long long)nx * jg + ig;
    s.L = s.c - 1 * (ig > 0);
    s.R = s.c + 1 * (ig < nx - 1);
    s.U = s.c + (long long)nx * (jg < ny - 1);
    s.D = s.c - (long long)nx * (jg > 0);
    s.LD = s.D - 1 * (ig > 0);
    s.RD = s.D + 1 * (ig < nx - 1);
    s.LU = s.U - 1 * (ig > 0);
    s.RU = s.U + 1 * (ig < nx - 1);
    return s;
}

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// the nine-point sum in the reference's order
inline double sum9(const double *f, const Stencil &s, const double N[9]) {
    return f[s.LD] * N[0] + f[s.D] * N[1] + f[s.RD] * N[2] + f[s.L] * N[3] + f[s.c] * N[4] + f[s.R] * N[5] +
           f[s.LU] * N[6] + f[s.U] * N[7] + f[s.RU] * N[8];
}
inline double sum9_weights_first(const double *f, const Stencil &s, const double N[9]) {
    return N[0] * f[s.LD] + N[1] * f[s.D] + N[2] * f[s.RD] + N[3] * f[s.L] + N[4] * f[s.c] + N[5] * f[s.R] +
           N[6] * f[s.LU] + N[7] * f[s.U] + N[8] * f[s.RU];
}

// rows [0, n) in parallel chunks
template <typename F>
void rows_parallel(int n, F &&fn) {
    const int parts = std::max(1, std::min(n, 8 * tsu::host_threads()));
    tsu::host_parallel(parts, [&](int q) {
        const int a = (int)((long long)n * q / parts), b = (int)((long long)n * (q + 1) / parts);
        for (int r = a; r < b; r++) fn(r);
    });
}

// One boundary sample of interpolate_CC (interpolations.cxx:475-540 and the
// three copies after it): the biquadratic interpolation of (ha, ua, va) of
// time slice t at (x, y), scaled to metres, the sea-level rise added to the
// free surface, the bed depth Hb attached, and fill values replaced.
void cc_sample(const double *ha, const double *ua, const double *va, long long tslice, int nxg, int nyg,
               double xmin_g, double ymin_g, double dx_g, double dy_g, double x, double y, double Hb, double slr,
               double *out4) {
    int ig = int((x - xmin_g - 0.5 * dx_g) / dx_g);
    if (ig > nxg - 1) ig = nxg - 1;
    int jg = int((y - ymin_g - 0.5 * dy_g) / dy_g);
    if (jg > nyg - 1) jg = nyg - 1;
    ig = std::max(ig, 0);
    jg = std::max(jg, 0);
    const Stencil s = stencil_offsets(tslice, ig, jg, nxg, nyg);
    const double x1 = xmin_g + 0.5 * dx_g + ig * dx_g, x0 = x1 - dx_g, x2 = x1 + dx_g;
    const double y1 = ymin_g + 0.5 * dy_g + jg * dy_g, y0 = y1 - dy_g, y2 = y1 + dy_g;
    const double N[9] = {node0(x, x0, x1, x2) * node0(y, y0, y1, y2), node1(x, x0, x1, x2) * node0(y, y0, y1, y2),
                         node2(x, x0, x1, x2) * node0(y, y0, y1, y2), node0(x, x0, x1, x2) * node1(y, y0, y1, y2),
                         node1(x, x0, x1, x2) * node1(y, y0, y1, y2), node2(x, x0, x1, x2) * node1(y, y0, y1, y2),
                         node0(x, x0, x1, x2) * node2(y, y0, y1, y2), node1(x, x0, x1, x2) * node2(y, y0, y1, y2),
                         node2(x, x0, x1, x2) * node2(y, y0, y1, y2)};
    out4[0] = sum9_weights_first(ha, s, N);
    out4[1] = sum9_weights_first(ua, s, N);
    out4[2] = sum9_weights_first(va, s, N);
    out4[0] *= kUnits;
    out4[1] *= kUnits;
    out4[2] *= kUnits;
    out4[0] += slr;
    out4[3] = Hb;
    if (out4[0] < -1e20) out4[0] = Hb;
    if (out4[1] < -1e20) out4[1] = 0.0;
    if (out4[2] < -1e20) out4[2] = 0.0;
    if (out4[0] > 1e20) out4[0] = Hb;
    if (out4[1] > 1e20) out4[1] = 0.0;
    if (out4[2] > 1e20) out4[2] = 0.0;
}

// one point of spheric2cartesian_CC: three-node blend of the segment samples
inline void cc_blend(const double *CC, long long pos, long long pos0, long long pos1, double N0, double N1, double N2,
                     double *out) {
    for (int k = 0; k < 4; k++) out[k] = N0 * CC[pos0 + k] + N1 * CC[pos + k] + N2 * CC[pos1 + k];
}

}  // namespace

extern "C" int tsu_nctr_interp_grid(double xmin, double xmax, double ymin, double ymax, double xmin_f, double ymin_f,
                                    int npx_f, int npy_f, double dx_f, double dy_f, int npx, int npy, const double *fun,
                                    double *sol) {
    if (!fun || !sol || npx < 1 || npy < 1 || npx_f < 1 || npy_f < 1) return TSU_ERR_INVALID;
    // interpolate_spherics, interpolations.cxx:779-865
    const double dx = (xmax - xmin) / (npx), dy = (ymax - ymin) / (npy);
    rows_parallel(npy, [&](int j) {
        for (int i = 0; i < npx; i++) {
            const double x = xmin + 0.5 * dx + i * dx;
            const double y = ymin + 0.5 * dy + j * dy;
            const double xt = 1.0 / (xmax - xmin) * (2 * x - (xmax + xmin));
            const double yt = 1.0 / (ymax - ymin) * (2 * y - (ymax + ymin));
            int ig = int((x - xmin_f - 0.5 * dx_f) / dx_f);
            int jg = int((y - ymin_f - 0.5 * dy_f) / dy_f);
            ig = clampi(ig, 0, npx_f - 1);
            jg = clampi(jg, 0, npy_f - 1);
            const Stencil s = stencil_clamped(0, ig, jg, npx_f, npy_f);
            const double N[9] = {lag0(xt) * lag0(yt), lag1(xt) * lag0(yt), lag2(xt) * lag0(yt),
                                 lag0(xt) * lag1(yt), lag1(xt) * lag1(yt), lag2(xt) * lag1(yt),
                                 lag0(xt) * lag2(yt), lag1(xt) * lag2(yt), lag2(xt) * lag2(yt)};
            sol[(long long)j * npx + i] = sum9(fun, s, N);
        }
    });
    return TSU_OK;
}

extern "C" int tsu_nctr_fix_eta(double *eta, const double *H, int npx, int npy, double slr) {
    if (!eta || !H || npx < 1 || npy < 1) return TSU_ERR_INVALID;
    // fix_eta, interpolations.cxx:867-876
    const long long n = (long long)npx * npy;
    for (long long p = 0; p < n; p++) {
        eta[p] -= slr;
        if (eta[p] < -1e20) eta[p] = H[p];
        if (eta[p] > 1e20) eta[p] = H[p];
    }
    return TSU_OK;
}

extern "C" int tsu_nctr_boundary_series(const double *ha, const double *ua, const double *va, unsigned long ntime,
                                        int nxg, int nyg, double xmin_g, double ymin_g, double dx_g, double dy_g,
                                        int npx, int npy, double xmin, double xmax, double ymin, double ymax,
                                        const double *H, double slr, double *CC) {
    if (!ha || !ua || !va || !H || !CC || ntime < 1 || nxg < 1 || nyg < 1 || npx < 1 || npy < 1)
        return TSU_ERR_INVALID;
    // interpolate_CC, interpolations.cxx:368-775 (the biquadratic form the
    // reference compiles); segments bottom i | right npx+j | top npx+npy+i |
    // left 2npx+npy+j, 4 values each (eta, u, v, H)
    const double dx = (xmax - xmin) / npx, dy = (ymax - ymin) / npy;
    const long long nseg4 = (long long)(2 * npx + 2 * npy) * 4, slice = (long long)nxg * nyg;
    tsu::host_parallel((int)ntime, [&](int t) {
        const long long posC = t * nseg4, ts = t * slice;
        for (int i = 0; i < npx; i++) {
            const double x = xmin + 0.5 * dx + i * dx;
            cc_sample(ha, ua, va, ts, nxg, nyg, xmin_g, ymin_g, dx_g, dy_g, x, ymin, H[i], slr, CC + posC + i * 4);
            cc_sample(ha, ua, va, ts, nxg, nyg, xmin_g, ymin_g, dx_g, dy_g, x, ymax, H[(long long)(npy - 1) * npx + i],
                      slr, CC + posC + (long long)(npx + npy + i) * 4);
        }
        for (int j = 0; j < npy; j++) {
            const double y = ymin + 0.5 * dy + j * dy;
            cc_sample(ha, ua, va, ts, nxg, nyg, xmin_g, ymin_g, dx_g, dy_g, xmin, y, H[(long long)j * npx], slr,
                      CC + posC + (long long)(2 * npx + npy + j) * 4);
            cc_sample(ha, ua, va, ts, nxg, nyg, xmin_g, ymin_g, dx_g, dy_g, xmax, y, H[(long long)j * npx + npx - 1],
                      slr, CC + posC + (long long)(npx + j) * 4);
        }
    });
    return TSU_OK;
}

extern "C" int tsu_nctr_sphere_metrics(double ymin, double dy, int npy, double xmax, double xmin, double dx,
                                       double *dxE, double *dy_unit, double *dmax) {
    if (!dxE || !dy_unit || !dmax || npy < 1) return TSU_ERR_INVALID;
    // dy_transform / dx_transform, interpolations.cxx:79-94
    *dy_unit = (2 * kPi * kRe) / 360;
    double m = -1.0;
    for (int i = 0; i < npy; i++) {
        const double lat = ymin + 0.5 * dy + i * dy;
        dxE[i] = (2 * kPi * kRe * cos(lat * kPi / 180)) / 360;
        m = std::max(m, dxE[i] * (xmax - xmin));
        dxE[i] *= dx;
    }
    *dmax = m;
    return TSU_OK;
}

extern "C" int tsu_nctr_to_cartesian(double xmin, double xmax, double ymin, double ymax, const double *dxE, double dyE,
                                     int npx, int npy, const double *fun, double *sol) {
    if (!dxE || !fun || !sol || npx < 1 || npy < 1) return TSU_ERR_INVALID;
    // spheric2cartesian, interpolations.cxx:879-968
    const double dxG = (xmax - xmin) / npx, dyG = (ymax - ymin) / npy;
    rows_parallel(npy, [&](int j) {
        for (int i = 0; i < npx; i++) {
            const double x = xmin + 0.5 * dxG + i * dxG;
            const double y = ymin + 0.5 * dyG + j * dyG;
            const double xt = 1.0 / (xmax - xmin) * (2 * x - (xmax + xmin));
            const double yt = 1.0 / (ymax - ymin) * (2 * y - (ymax + ymin));
            int jg = int((y - ymin - 0.5 * dyE) / dyE);
            jg = clampi(jg, 0, npy - 1);
            const double xminE = 0 + (xmax - dxE[jg] * npx) / 2;
            int ig = int((x - xminE - 0.5 * dxE[jg]) / dxE[jg]);
            ig = clampi(ig, 0, npx - 1);
            const Stencil s = stencil_clamped(0, ig, jg, npx, npy);
            const double N[9] = {lag0(xt) * lag0(yt), lag1(xt) * lag0(yt), lag2(xt) * lag0(yt),
                                 lag0(xt) * lag1(yt), lag1(xt) * lag1(yt), lag2(xt) * lag1(yt),
                                 lag0(xt) * lag2(yt), lag1(xt) * lag2(yt), lag2(xt) * lag2(yt)};
            sol[(long long)j * npx + i] = sum9(fun, s, N);
        }
    });
    return TSU_OK;
}

extern "C" int tsu_nctr_to_cartesian_series(double xmin, double xmax, double ymin, double ymax, const double *dxE,
                                            double dyE, int npx, int npy, unsigned long ntime, double *CC) {
    if (!dxE || !CC || npx < 1 || npy < 1) return TSU_ERR_INVALID;
    // spheric2cartesian_CC, interpolations.cxx:970-1097 (in place, one time
    // slice at a time; the right boundary's upper neighbour test compares
    // with npx - 1 as the reference does)
    const double dx = (xmax - xmin) / npx, dy = (ymax - ymin) / npy;
    const long long nseg = 2LL * npx + 2LL * npy;
    tsu::host_parallel((int)ntime, [&](int t) {
        std::vector<double> aux((size_t)nseg * 4, 0.0);
        const long long base = t * nseg * 4;
        for (int i = 0; i < npx; i++) {
            const double x = xmin + 0.5 * dx + i * dx;
            const double xt = 1.0 / (xmax - xmin) * (2 * x - (xmax + xmin));
            const double N0 = lag0(xt), N1 = lag1(xt), N2 = lag2(xt);
            double xminE = 0 + (xmax - dxE[0] * npx) / 2;
            int ig = clampi(int((x - xminE - 0.5 * dxE[0]) / dxE[0]), 0, npx - 1);
            long long pos = base + (long long)ig * 4;
            cc_blend(CC, pos, pos - 4 * (ig > 0), pos + 4 * (ig < npx - 1), N0, N1, N2, &aux[(size_t)i * 4]);
            xminE = 0 + (xmax - dxE[npy - 1] * npx) / 2;
            ig = clampi(int((x - xminE - 0.5 * dxE[npy - 1]) / dxE[npy - 1]), 0, npx - 1);
            pos = base + (long long)(npx + npy) * 4 + (long long)ig * 4;
            cc_blend(CC, pos, pos - 4 * (ig > 0), pos + 4 * (ig < npx - 1), N0, N1, N2,
                     &aux[(size_t)(npx + npy + i) * 4]);
        }
        for (int j = 0; j < npy; j++) {
            const double y = ymin + 0.5 * dy + j * dy;
            const double yt = 1.0 / (ymax - ymin) * (2 * y - (ymax + ymin));
            const double N0 = lag0(yt), N1 = lag1(yt), N2 = lag2(yt);
            const double yminE = 0 + (ymax - dyE * npy) / 2;
            const int jg = clampi(int((y - yminE - 0.5 * dyE) / dyE), 0, npy - 1);
            long long pos = base + (long long)(npx * 2 + npy) * 4 + (long long)jg * 4;
            cc_blend(CC, pos, pos - 4 * (jg > 0), pos + 4 * (jg < npy - 1), N0, N1, N2,
                     &aux[(size_t)(npx * 2 + npy + j) * 4]);
            pos = base + (long long)npx * 4 + (long long)jg * 4;
            long long pos1 = pos + 4 * (jg < npx - 1);
            if (pos1 >= base + nseg * 4) pos1 = pos;  // beyond the series (the reference reads past it)
            cc_blend(CC, pos, pos - 4 * (jg > 0), pos1, N0, N1, N2, &aux[(size_t)(npx + j) * 4]);
        }
        std::memcpy(CC + base, aux.data(), aux.size() * sizeof(double));
    });
    return TSU_OK;
}

extern "C" int tsu_nctr_assign_state(const double *H_cart, const double *eta_cart, const double *fix_cart, int npx,
                                     int npy, double slr, double *h, tsu_double2 *hu, double *H, int *fixH) {
    if (!H_cart || !eta_cart || !h || !hu || !H || !fixH || npx < 1 || npy < 1) return TSU_ERR_INVALID;
    // value assignment, Problem_loader.cxx:576-605
    rows_parallel(npy, [&](int j) {
        for (int i = 0; i < npx; i++) {
            const long long pos = (long long)j * npx + i;
            H[pos] = (double)(H_cart[pos]);
            h[pos] = (double)(eta_cart[pos]) * kUnits + H[pos] + slr;
            h[pos] *= (h[pos] >= 0.0);
            hu[pos].x = 0.0;
            hu[pos].y = 0.0;
            fixH[pos] = fix_cart ? (fix_cart[pos] >= 0.5 ? 1 : 0) : 1;
        }
    });
    return TSU_OK;
}

extern "C" int tsu_nctr_prepare(int nxb, int nyb, const double *xb, const double *yb, const double *bathy, int nxf,
                                int nyf, const double *xf, const double *yf, const double *fix, int nxc, int nyc,
                                const double *xc, const double *yc, unsigned long ntime, const double *tgrid,
                                const double *ha, const double *ua, const double *va, int npx, int npy, double slr,
                                SimParams *p, double *h, tsu_double2 *hu, double *H, int *fixH, double *CC,
                                double *tCC) {
    if (!xb || !yb || !bathy || !xc || !yc || !tgrid || !ha || !ua || !va || !p || !h || !hu || !H || !fixH || !CC ||
        !tCC || nxb < 2 || nyb < 2 || nxc < 2 || nyc < 2 || ntime < 1 || npx < 1 || npy < 1 ||
        (fix && (!xf || !yf || nxf < 2 || nyf < 2)))
        return TSU_ERR_INVALID;
    // Problem_loader.cxx:355-625 (SPL == 0), step by step
    const long long n = (long long)npx * npy;
    std::vector<double> Hs(n), fs(fix ? n : 0), es(n), dxE(npy);
    // bathymetry grid -> simulation grid (:396-438): the box is the grid's
    // cell-centre range widened by half a cell
    const double dxg = (xb[nxb - 1] - xb[0]) / (nxb - 1), dyg = (yb[nyb - 1] - yb[0]) / (nyb - 1);
    double xmin = xb[0] - 0.5 * dxg, xmax = xb[nxb - 1] + 0.5 * dxg;
    double ymin = yb[0] - 0.5 * dyg, ymax = yb[nyb - 1] + 0.5 * dyg;
    tsu_nctr_interp_grid(xmin, xmax, ymin, ymax, xmin, ymin, nxb, nyb, dxg, dyg, npx, npy, bathy, Hs.data());
    // non-erodible-bed grid (:441-471): placed by its first cell centre
    if (fix) {
        const double dxf = (xf[nxf - 1] - xf[0]) / (nxf - 1), dyf = (yf[nyf - 1] - yf[0]) / (nyf - 1);
        tsu_nctr_interp_grid(xmin, xmax, ymin, ymax, xf[0], yf[0], nxf, nyf, dxf, dyf, npx, npy, fix, fs.data());
    }
    // initial free surface: time slice 0 of the NCTR grid (:473-507); its
    // spacing divides by the point count, as the reference does
    const double dxc = (xc[nxc - 1] - xc[0]) / nxc, dyc = (yc[nyc - 1] - yc[0]) / nyc;
    tsu_nctr_interp_grid(xmin, xmax, ymin, ymax, xc[0], yc[0], nxc, nyc, dxc, dyc, npx, npy, ha, es.data());
    tsu_nctr_fix_eta(es.data(), Hs.data(), npx, npy, slr);
    // boundary series (:510-527)
    std::memcpy(tCC, tgrid, ntime * sizeof(double));
    tsu_nctr_boundary_series(ha, ua, va, ntime, nxc, nyc, xc[0], yc[0], dxc, dyc, npx, npy, xmin, xmax, ymin, ymax,
                             Hs.data(), slr, CC);
    // geographic -> Cartesian metres (:530-571)
    double dx = (xmax - xmin) / (npx), dy = (ymax - ymin) / npy;
    double dy_unit, dmax;
    tsu_nctr_sphere_metrics(ymin, dy, npy, xmax, xmin, dx, dxE.data(), &dy_unit, &dmax);
    xmin = 0;
    xmax = dmax;
    ymax = dy_unit * (ymax - ymin);
    ymin = 0;
    const double dyE = dy * dy_unit;
    std::vector<double> Hc(n), ec(n), fc(fix ? n : 0);
    tsu_nctr_to_cartesian(xmin, xmax, ymin, ymax, dxE.data(), dyE, npx, npy, Hs.data(), Hc.data());
    if (fix) tsu_nctr_to_cartesian(xmin, xmax, ymin, ymax, dxE.data(), dyE, npx, npy, fs.data(), fc.data());
    tsu_nctr_to_cartesian(xmin, xmax, ymin, ymax, dxE.data(), dyE, npx, npy, es.data(), ec.data());
    tsu_nctr_to_cartesian_series(xmin, xmax, ymin, ymax, dxE.data(), dyE, npx, npy, ntime, CC);
    // the state and the grid (:575-625)
    dx = (xmax - xmin) / (npx);
    dy = (ymax - ymin) / npy;
    tsu_nctr_assign_state(Hc.data(), ec.data(), fix ? fc.data() : nullptr, npx, npy, slr, h, hu, H, fixH);
    p->xmin = xmin;
    p->xmax = xmax;
    p->ymin = ymin;
    p->ymax = ymax;
    p->npx = npx;
    p->npy = npy;
    p->nvol = (int)n;
    p->dx = dx;
    p->dy = dy;
    return TSU_OK;
}

extern "C" int tsu_nctr_tides(const double *tides, int nxt, int nyt, unsigned long npt, const double *xp, int npx,
                              int npy, double xmin, double xmax, double ymin, double ymax, double *tides_bd) {
    if (!tides || !xp || !tides_bd || nxt < 1 || nyt < 1 || npx < 1 || npy < 1) return TSU_ERR_INVALID;
    // tides_prep, tides.cxx:170-291: quadratic interpolation of the tide grid
    // along the four boundaries, [npt][2npx + 2npy] (bottom i | right npx+j |
    // top npx+npy+i | left 2npx+npy+j), values above 1e5 in magnitude zeroed
    const double dx = (xmax - xmin) / npx, dy = (ymax - ymin) / npy;
    const double dxt = (xmax - xmin) / (nxt), dyt = (ymax - ymin) / (nyt);
    const long long nseg = 2LL * npx + 2LL * npy, slice = (long long)nxt * nyt;
    for (unsigned long t = 0; t < npt; t++) {
        for (int i = 0; i < npx; i++) {
            const double x = xmin + 0.5 * dx + i * dx;
            long long post = int((x - xmin - 0.5 * dxt) / dxt);
            long long postm = post - 1 * (post > 0), postp = post + 1 * (post < nxt - 1);
            const double xt = xp[0] + 0.5 * dxt + post * dxt, xtm = xt - dxt, xtp = xt + dxt;
            post += t * slice;
            postm += t * slice;
            postp += t * slice;
            const double a = tide0(x, xt, xtp, xtm, dxt), b = tide1(x, xt, xtp, xtm, dxt), c = tide2(x, xt, xtp, xtm, dxt);
            tides_bd[i + nseg * t] = tides[postm] * a + tides[post] * b + tides[postp] * c;
            const long long top = slice - nxt;
            tides_bd[(npx + npy) + i + nseg * t] = tides[postm + top] * a + tides[post + top] * b + tides[postp + top] * c;
        }
        for (int j = 0; j < npy; j++) {
            const double y = ymin + 0.5 * dy + j * dy;
            long long post = int((y - ymin - 0.5 * dyt) / dyt);
            long long postm = post - 1 * (post > 0), postp = post + 1 * (post < nyt - 1);
            const double yt = ymin + 0.5 * dyt + post * dyt, ytm = yt - dyt, ytp = yt + dyt;
            post *= nxt;
            postm *= nxt;
            postp *= nxt;
            post += t * slice;
            postm += t * slice;
            postp += t * slice;
            const double a = tide0(y, yt, ytp, ytm, dyt), b = tide1(y, yt, ytp, ytm, dyt), c = tide2(y, yt, ytp, ytm, dyt);
            tides_bd[npx + j + nseg * t] =
                tides[postm + nxt - 1] * a + tides[post + nxt - 1] * b + tides[postp + nxt - 1] * c;
            tides_bd[(2 * npx + npy) + j + nseg * t] = tides[postm] * a + tides[post] * b + tides[postp] * c;
        }
    }
    for (long long i = 0; i < (long long)npt * 2 * (npx + npy); i++)
        if (std::fabs(tides_bd[i]) > 1e5) tides_bd[i] = 0.0;
    return TSU_OK;
}
