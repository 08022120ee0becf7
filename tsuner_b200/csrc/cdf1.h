// cdf1.h -- minimal NetCDF classic (CDF-1) writer.
//
// The reference writes its output through libnetcdf with NC_CLOBBER
// (GPU/netcdf.cu:54), i.e. the classic CDF-1 format.  libnetcdf is not part
// of this image, so the library carries this small writer for the subset the
// output needs: fixed and one unlimited (record) dimension, NC_CHAR and
// NC_DOUBLE attributes, NC_DOUBLE variables, whole-variable and
// hyperslab writes, prefill with _FillValue.  Format: NetCDF classic file
// format specification (big-endian header, 4-byte aligned, 32-bit offsets).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace tsu {
namespace cdf1 {

enum { NC_CHAR_T = 2, NC_DOUBLE_T = 6 };
constexpr double kDefaultFillDouble = 9.9692099683868690e+36;

class File {
public:
    ~File();
    int create(const char *path);  // 0 on success
    int def_dim(const char *name, size_t len, int *id);  // len 0 = record dim
    int def_var(const char *name, int type, int ndims, const int *dimids, int *id);
    int put_att_text(int varid, const char *name, size_t len, const char *text);  // varid -1 = global
    int put_att_double(int varid, const char *name, size_t n, const double *v);
    int enddef();
    int put_var_double(int varid, const double *v);
    int put_vara_double(int varid, const size_t *start, const size_t *count, const double *v);
    int sync();
    int close();
    bool is_open() const { return f_ != nullptr; }

private:
    struct Att {
        std::string name;
        int type;
        std::vector<char> text;
        std::vector<double> d;
    };
    struct Dim {
        std::string name;
        size_t len;
    };
    struct Var {
        std::string name;
        int type;
        std::vector<int> dims;
        std::vector<Att> atts;
        uint64_t vsize = 0;
        uint64_t begin = 0;
        bool rec = false;
    };
    std::vector<unsigned char> header() const;
    size_t nelems_fixed(const Var &v) const;
    double fill_of(const Var &v) const;
    int write_doubles(uint64_t off, const double *v, size_t n);
    int fill_record(size_t rec);

    FILE *f_ = nullptr;
    bool define_ = true;
    std::vector<Dim> dims_;
    std::vector<Att> gatts_;
    std::vector<Var> vars_;
    size_t numrecs_ = 0;
    uint64_t recsize_ = 0;
};

}  // namespace cdf1
}  // namespace tsu
