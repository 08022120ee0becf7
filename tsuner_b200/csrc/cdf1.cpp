// cdf1.cpp -- see cdf1.h.
#include "cdf1.h"

#include <cstring>

namespace tsu {
namespace cdf1 {

namespace {
enum : uint32_t { TAG_DIM = 0x0A, TAG_VAR = 0x0B, TAG_ATT = 0x0C };

void put32(std::vector<unsigned char> &b, uint32_t v) {
    b.push_back((unsigned char)(v >> 24));
    b.push_back((unsigned char)(v >> 16));
    b.push_back((unsigned char)(v >> 8));
    b.push_back((unsigned char)v);
}
void pad4(std::vector<unsigned char> &b) {
    while (b.size() % 4) b.push_back(0);
}
void put_name(std::vector<unsigned char> &b, const std::string &s) {
    put32(b, (uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    pad4(b);
}
void be_double(unsigned char *o, double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    for (int i = 0; i < 8; i++) o[i] = (unsigned char)(u >> (56 - 8 * i));
}
uint64_t round4(uint64_t x) { return (x + 3) & ~uint64_t(3); }
}  // namespace

File::~File() { close(); }

int File::create(const char *path) {
    close();
    f_ = std::fopen(path, "wb+");
    if (!f_) return -1;
    define_ = true;
    dims_.clear();
    gatts_.clear();
    vars_.clear();
    numrecs_ = 0;
    return 0;
}

int File::def_dim(const char *name, size_t len, int *id) {
    if (!f_ || !define_) return -1;
    if (len == 0)
        for (auto &d : dims_)
            if (d.len == 0) return -1;  // one record dimension at most
    dims_.push_back({name, len});
    if (id) *id = (int)dims_.size() - 1;
    return 0;
}

int File::def_var(const char *name, int type, int ndims, const int *dimids, int *id) {
    if (!f_ || !define_ || type != NC_DOUBLE_T) return -1;
    Var v;
    v.name = name;
    v.type = type;
    for (int i = 0; i < ndims; i++) {
        if (dimids[i] < 0 || dimids[i] >= (int)dims_.size()) return -1;
        if (dims_[dimids[i]].len == 0 && i != 0) return -1;  // record dim must lead
        v.dims.push_back(dimids[i]);
    }
    v.rec = ndims > 0 && dims_[v.dims[0]].len == 0;
    vars_.push_back(v);
    if (id) *id = (int)vars_.size() - 1;
    return 0;
}

int File::put_att_text(int varid, const char *name, size_t len, const char *text) {
    if (!f_ || !define_) return -1;
    Att a;
    a.name = name;
    a.type = NC_CHAR_T;
    a.text.assign(text, text + len);
    if (varid == -1) gatts_.push_back(a);
    else if (varid >= 0 && varid < (int)vars_.size()) vars_[varid].atts.push_back(a);
    else return -1;
    return 0;
}

int File::put_att_double(int varid, const char *name, size_t n, const double *v) {
    if (!f_ || !define_) return -1;
    Att a;
    a.name = name;
    a.type = NC_DOUBLE_T;
    a.d.assign(v, v + n);
    if (varid == -1) gatts_.push_back(a);
    else if (varid >= 0 && varid < (int)vars_.size()) vars_[varid].atts.push_back(a);
    else return -1;
    return 0;
}

size_t File::nelems_fixed(const Var &v) const {
    size_t n = 1;
    for (size_t i = v.rec ? 1 : 0; i < v.dims.size(); i++) n *= dims_[v.dims[i]].len;
    return n;
}

double File::fill_of(const Var &v) const {
    for (auto &a : v.atts)
        if (a.name == "_FillValue" && a.type == NC_DOUBLE_T && !a.d.empty()) return a.d[0];
    return kDefaultFillDouble;
}

std::vector<unsigned char> File::header() const {
    std::vector<unsigned char> b;
    b.push_back('C');
    b.push_back('D');
    b.push_back('F');
    b.push_back(1);
    put32(b, (uint32_t)numrecs_);
    if (dims_.empty()) {
        put32(b, 0);
        put32(b, 0);
    } else {
        put32(b, TAG_DIM);
        put32(b, (uint32_t)dims_.size());
        for (auto &d : dims_) {
            put_name(b, d.name);
            put32(b, (uint32_t)d.len);
        }
    }
    auto atts = [&](const std::vector<Att> &as) {
        if (as.empty()) {
            put32(b, 0);
            put32(b, 0);
            return;
        }
        put32(b, TAG_ATT);
        put32(b, (uint32_t)as.size());
        for (auto &a : as) {
            put_name(b, a.name);
            put32(b, (uint32_t)a.type);
            if (a.type == NC_CHAR_T) {
                put32(b, (uint32_t)a.text.size());
                b.insert(b.end(), a.text.begin(), a.text.end());
                pad4(b);
            } else {
                put32(b, (uint32_t)a.d.size());
                for (double d : a.d) {
                    unsigned char o[8];
                    be_double(o, d);
                    b.insert(b.end(), o, o + 8);
                }
            }
        }
    };
    atts(gatts_);
    if (vars_.empty()) {
        put32(b, 0);
        put32(b, 0);
    } else {
        put32(b, TAG_VAR);
        put32(b, (uint32_t)vars_.size());
        for (auto &v : vars_) {
            put_name(b, v.name);
            put32(b, (uint32_t)v.dims.size());
            for (int d : v.dims) put32(b, (uint32_t)d);
            atts(v.atts);
            put32(b, (uint32_t)v.type);
            put32(b, (uint32_t)v.vsize);
            put32(b, (uint32_t)v.begin);
        }
    }
    return b;
}

int File::write_doubles(uint64_t off, const double *v, size_t n) {
    std::vector<unsigned char> buf(n * 8);
    for (size_t i = 0; i < n; i++) be_double(&buf[i * 8], v[i]);
    if (std::fseek(f_, (long)off, SEEK_SET) != 0) return -1;
    if (std::fwrite(buf.data(), 1, buf.size(), f_) != buf.size()) return -1;
    return 0;
}

int File::enddef() {
    if (!f_ || !define_) return -1;
    for (auto &v : vars_) v.vsize = round4(nelems_fixed(v) * 8);
    // header size does not depend on the offsets' values (fixed width)
    uint64_t off = header().size();
    for (auto &v : vars_)
        if (!v.rec) {
            v.begin = off;
            off += v.vsize;
        }
    recsize_ = 0;
    for (auto &v : vars_)
        if (v.rec) {
            v.begin = off + recsize_;
            recsize_ += v.vsize;
        }
    if (off + recsize_ > 0xFFFFFFFFull) return -1;  // CDF-1 offsets are 32-bit
    define_ = false;
    std::vector<unsigned char> h = header();
    std::fseek(f_, 0, SEEK_SET);
    if (std::fwrite(h.data(), 1, h.size(), f_) != h.size()) return -1;
    for (auto &v : vars_)  // prefill fixed-size variables
        if (!v.rec) {
            std::vector<double> fill(nelems_fixed(v), fill_of(v));
            if (write_doubles(v.begin, fill.data(), fill.size())) return -1;
        }
    return 0;
}

int File::fill_record(size_t rec) {
    for (auto &v : vars_)
        if (v.rec) {
            std::vector<double> fill(nelems_fixed(v), fill_of(v));
            if (write_doubles(v.begin + rec * recsize_, fill.data(), fill.size())) return -1;
        }
    return 0;
}

int File::put_var_double(int varid, const double *v) {
    if (!f_ || define_ || varid < 0 || varid >= (int)vars_.size()) return -1;
    Var &var = vars_[varid];
    if (var.rec) return -1;
    return write_doubles(var.begin, v, nelems_fixed(var));
}

int File::put_vara_double(int varid, const size_t *start, const size_t *count, const double *v) {
    if (!f_ || define_ || varid < 0 || varid >= (int)vars_.size()) return -1;
    Var &var = vars_[varid];
    const size_t nd = var.dims.size();
    std::vector<size_t> shape(nd);
    for (size_t i = 0; i < nd; i++) shape[i] = dims_[var.dims[i]].len;
    if (var.rec) {
        size_t last = start[0] + count[0];
        while (numrecs_ < last) {
            if (fill_record(numrecs_)) return -1;
            numrecs_++;
        }
    }
    for (size_t i = (var.rec ? 1 : 0); i < nd; i++)
        if (start[i] + count[i] > shape[i]) return -1;
    if (nd == 0) return write_doubles(var.begin, v, 1);
    // iterate over all index tuples of the hyperslab except the innermost run
    const size_t inner = count[nd - 1];
    size_t nouter = 1;
    for (size_t i = 0; i + 1 < nd; i++) nouter *= count[i];
    std::vector<size_t> idx(nd, 0);
    for (size_t o = 0; o < nouter; o++) {
        size_t rem = o;
        for (size_t i = nd - 1; i-- > 0;) {
            idx[i] = start[i] + rem % count[i];
            rem /= count[i];
        }
        idx[nd - 1] = start[nd - 1];
        uint64_t off = var.begin;
        uint64_t lin = 0;
        for (size_t i = var.rec ? 1 : 0; i < nd; i++) lin = lin * shape[i] + idx[i];
        off += lin * 8;
        if (var.rec) off += (uint64_t)idx[0] * recsize_;
        if (write_doubles(off, v + o * inner, inner)) return -1;
    }
    return 0;
}

int File::sync() {
    if (!f_) return -1;
    if (!define_) {
        std::vector<unsigned char> h = header();
        std::fseek(f_, 4, SEEK_SET);
        std::fwrite(&h[4], 1, 4, f_);  // numrecs
    }
    return std::fflush(f_) == 0 ? 0 : -1;
}

int File::close() {
    if (!f_) return 0;
    if (define_) enddef();
    int r = sync();
    std::fclose(f_);
    f_ = nullptr;
    return r;
}

}  // namespace cdf1
}  // namespace tsu
