/*
 * ref_interp_shim.cpp -- C entry points into the REFERENCE's own input
 * interpolation code (interpolations.cxx, tides.cxx), compiled unmodified
 * from the reference checkout together with fake_netcdf.c into
 * oracle/_ref/interp/libref_interp.so.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the product's input pipeline
 * (tsuner_b200/csrc/nctr.cpp); never linked into the product.  Each ref_*
 * call forwards to the reference function of the same role; the reference
 * signatures take std::string and references, which a C caller cannot pass.
 */
#include "TSUNER.h"

extern "C" {

void ref_interpolate_spherics(double xmin, double xmax, double ymin, double ymax, double xmin_fun, double ymin_fun,
                              int npx_fun, int npy_fun, double dx_fun, double dy_fun, int npx, int npy, double *fun,
                              double *sol)
{
    interpolate_spherics(xmin, xmax, ymin, ymax, xmin_fun, ymin_fun, npx_fun, npy_fun, dx_fun, dy_fun, npx, npy, fun,
                         sol);
}

void ref_fix_eta(double *p, double *H, int npx, int npy, double slr) { fix_eta(p, H, npx, npy, slr); }

/* `file` is the free-surface file name; interpolate_CC derives the velocity
 * files' names from it and opens them, `id` is the open free-surface file */
void ref_interpolate_CC(const char *file, double *CC, double *tCC, int npx, int npy, double xmin, double xmax,
                        double ymin, double ymax, double xmin_grid, double ymin_grid, unsigned long time,
                        double dx_grid, double dy_grid, double *H, int id, double slr)
{
    interpolate_CC(std::string(file), CC, tCC, npx, npy, xmin, xmax, ymin, ymax, xmin_grid, ymin_grid, time, dx_grid,
                   dy_grid, H, id, slr);
}

void ref_spheric2cartesian(double xmin, double xmax, double ymin, double ymax, double *dx, double dy, int npx,
                           int npy, double *fun, double *sol)
{
    spheric2cartesian(xmin, xmax, ymin, ymax, dx, dy, npx, npy, fun, sol);
}

void ref_spheric2cartesian_CC(double xmin, double xmax, double ymin, double ymax, double *dxE, double dyE, int npx,
                              int npy, int time_grid, double *CC)
{
    spheric2cartesian_CC(xmin, xmax, ymin, ymax, dxE, dyE, npx, npy, time_grid, CC);
}

void ref_transforms(double ymin, double dy, int tam, double xmax, double xmin, double *dx, double dx_cartesianas,
                    double *dmax, double *dy_unit)
{
    double m = 0.0, u = 0.0;
    dx_transform(ymin, dy, tam, xmax, xmin, dx, dx_cartesianas, m);
    dy_transform(u);
    *dmax = m;
    *dy_unit = u;
}

/* tides_prep reads the tide file `file` (registered with the fake netCDF);
 * returns the number of time points and copies the boundary values */
int ref_tides_prep(double *eta_aux, const char *file, int npx, int npy, double xmin, double xmax, double ymin,
                   double ymax, double *tides_bd_out, size_t cap)
{
    double *bd = 0;
    float *tt = 0;
    int npt = 0;
    tides_prep(eta_aux, &bd, &tt, npx, npy, std::string(file), xmin, xmax, ymin, ymax, npt);
    size_t n = (size_t)npt * (2 * npx + 2 * npy);
    if (n > cap) n = cap;
    for (size_t k = 0; k < n; k++) tides_bd_out[k] = bd[k];
    delete[] bd;
    delete[] tt;
    return npt;
}

} /* extern "C" */
