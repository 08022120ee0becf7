/*
 * fake_netcdf.c -- an in-memory stand-in for the few libnetcdf read calls
 * the reference's input pipeline makes (interpolations.cxx interpolate_CC,
 * tides.cxx tides_prep), so that those unmodified reference functions can
 * run on arrays a test provides: the image has no libnetcdf or HDF5.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/interp/libref_interp.so
 * (the reference checker of the product's input pipeline), never into the
 * product library.
 *
 * A test registers datasets by path (fake_nc_dataset), their dimensions
 * (fake_nc_dim) and double variables (fake_nc_var); nc_open of that path
 * then opens it, and nc_inq_dimid / nc_inq_dimlen / nc_inq_varid /
 * nc_get_var(a)_double / nc_get_var_float / nc_get_att_int serve the
 * registered values (a hyperslab read copies the leading elements).
 */
#include <stdlib.h>
#include <string.h>

#include "netcdf.h"

#define MAXDS 16
#define MAXITEM 16

typedef struct {
    char name[64];
    size_t len;
} Dim;

typedef struct {
    char name[64];
    const double *data;
    size_t n;
} Var;

typedef struct {
    char path[512];
    int ndims, nvars;
    Dim dims[MAXITEM];
    Var vars[MAXITEM];
    int boundaries;
} Dataset;

static Dataset g_ds[MAXDS];
static int g_nds = 0;

void fake_nc_clear(void) { g_nds = 0; }

/* a path registered again replaces the earlier dataset */
int fake_nc_dataset(const char *path) {
    int k = 0;
    while (k < g_nds && strcmp(g_ds[k].path, path)) k++;
    if (k == g_nds) {
        if (g_nds >= MAXDS) return -1;
        g_nds++;
    }
    Dataset *d = &g_ds[k];
    memset(d, 0, sizeof(*d));
    strncpy(d->path, path, sizeof(d->path) - 1);
    return k;
}

int fake_nc_dim(int ds, const char *name, size_t len) {
    if (ds < 0 || ds >= g_nds || g_ds[ds].ndims >= MAXITEM) return -1;
    Dim *m = &g_ds[ds].dims[g_ds[ds].ndims];
    strncpy(m->name, name, sizeof(m->name) - 1);
    m->len = len;
    return g_ds[ds].ndims++;
}

int fake_nc_var(int ds, const char *name, const double *data, size_t n) {
    if (ds < 0 || ds >= g_nds || g_ds[ds].nvars >= MAXITEM) return -1;
    Var *v = &g_ds[ds].vars[g_ds[ds].nvars];
    strncpy(v->name, name, sizeof(v->name) - 1);
    v->data = data;
    v->n = n;
    return g_ds[ds].nvars++;
}

void fake_nc_set_boundaries(int ds, int value) {
    if (ds >= 0 && ds < g_nds) g_ds[ds].boundaries = value;
}

static Dataset *get(int ncid) { return (ncid >= 1 && ncid <= g_nds) ? &g_ds[ncid - 1] : NULL; }

const char *nc_strerror(int ncerr) { return ncerr ? "fake netCDF: not found" : "no error"; }

int nc_open(const char *path, int mode, int *ncidp) {
    (void)mode;
    for (int k = 0; k < g_nds; k++)
        if (!strcmp(g_ds[k].path, path)) {
            *ncidp = k + 1;
            return NC_NOERR;
        }
    return NC_ENOTNC;
}

int nc_close(int ncid) { return get(ncid) ? NC_NOERR : NC_EBADID; }

int nc_inq_dimid(int ncid, const char *name, int *idp) {
    Dataset *d = get(ncid);
    if (!d) return NC_EBADID;
    for (int k = 0; k < d->ndims; k++)
        if (!strcmp(d->dims[k].name, name)) {
            *idp = k;
            return NC_NOERR;
        }
    return -46; /* NC_EBADDIM */
}

int nc_inq_dimlen(int ncid, int dimid, size_t *lenp) {
    Dataset *d = get(ncid);
    if (!d || dimid < 0 || dimid >= d->ndims) return NC_EBADID;
    *lenp = d->dims[dimid].len;
    return NC_NOERR;
}

int nc_inq_varid(int ncid, const char *name, int *varidp) {
    Dataset *d = get(ncid);
    if (!d) return NC_EBADID;
    for (int k = 0; k < d->nvars; k++)
        if (!strcmp(d->vars[k].name, name)) {
            *varidp = k;
            return NC_NOERR;
        }
    return -49; /* NC_ENOTVAR */
}

static const Var *var(int ncid, int varid) {
    Dataset *d = get(ncid);
    return (d && varid >= 0 && varid < d->nvars) ? &d->vars[varid] : NULL;
}

int nc_get_var_double(int ncid, int varid, double *ip) {
    const Var *v = var(ncid, varid);
    if (!v) return -49;
    memcpy(ip, v->data, v->n * sizeof(double));
    return NC_NOERR;
}

int nc_get_vara_double(int ncid, int varid, const size_t *startp, const size_t *countp, double *ip) {
    const Var *v = var(ncid, varid);
    (void)startp;
    (void)countp;
    if (!v) return -49;
    /* the reference reads whole variables from the origin; a test registers
     * exactly the values read */
    memcpy(ip, v->data, v->n * sizeof(double));
    return NC_NOERR;
}

int nc_get_var_float(int ncid, int varid, float *ip) {
    const Var *v = var(ncid, varid);
    if (!v) return -49;
    for (size_t k = 0; k < v->n; k++) ip[k] = (float)v->data[k];
    return NC_NOERR;
}

int nc_get_att_int(int ncid, int varid, const char *name, int *ip) {
    Dataset *d = get(ncid);
    (void)varid;
    if (!d || strcmp(name, "boundaries")) return -43; /* NC_ENOTATT */
    *ip = d->boundaries;
    return NC_NOERR;
}
