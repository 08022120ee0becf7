/*
 * Minimal declaration of the libnetcdf C API subset that the reference
 * TSUNER sources call (GPU/netcdf.cu, Problem_loader.cxx, interpolations.cxx,
 * tides.cxx).  The image has no libnetcdf; this header lets the reference
 * kernels compile unmodified for the parity harness: the kernel sources the
 * harness builds (GPU/Reconstructor.cu, VolumeSolver.cu, Volume_kernel.cu,
 * Reduction_kernel_min.cu) include it through GPU/GPU_kernels.cuh and
 * TSUNER.h but call none of its functions, so no implementation is linked.
 *
 * TEST INFRASTRUCTURE ONLY: used to build the reference checker under
 * oracle/_ref/, never by the product library.
 */
#ifndef TSU_REF_NETCDF_STUB_H
#define TSU_REF_NETCDF_STUB_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int nc_type;

#define NC_NOERR      0
#define NC_ENOTNC   (-51)
#define NC_EBADID   (-33)
#define NC_NOWRITE    0x0000
#define NC_WRITE      0x0001
#define NC_CLOBBER    0x0000
#define NC_UNLIMITED  0L
#define NC_GLOBAL    (-1)
#define NC_BYTE       1
#define NC_CHAR       2
#define NC_SHORT      3
#define NC_INT        4
#define NC_FLOAT      5
#define NC_DOUBLE     6

const char *nc_strerror(int ncerr);
int nc_create(const char *path, int cmode, int *ncidp);
int nc_open(const char *path, int mode, int *ncidp);
int nc_close(int ncid);
int nc_sync(int ncid);
int nc_enddef(int ncid);
int nc_def_dim(int ncid, const char *name, size_t len, int *idp);
int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp);
int nc_put_att_text(int ncid, int varid, const char *name, size_t len, const char *op);
int nc_put_att_double(int ncid, int varid, const char *name, nc_type xtype, size_t len, const double *op);
int nc_put_var_double(int ncid, int varid, const double *op);
int nc_put_vara_double(int ncid, int varid, const size_t *startp, const size_t *countp, const double *op);
int nc_inq_dimid(int ncid, const char *name, int *idp);
int nc_inq_dimlen(int ncid, int dimid, size_t *lenp);
int nc_inq_varid(int ncid, const char *name, int *varidp);
int nc_get_var_double(int ncid, int varid, double *ip);
int nc_get_vara_double(int ncid, int varid, const size_t *startp, const size_t *countp, double *ip);
int nc_get_var_float(int ncid, int varid, float *ip);
int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip);
int nc_inq_var(int ncid, int varid, char *name, nc_type *xtypep, int *ndimsp, int *dimidsp, int *nattsp);
int nc_get_att_int(int ncid, int varid, const char *name, int *ip);

#ifdef __cplusplus
}
#endif
#endif
