// tsuner_main.cpp -- tsuner.exe, the command-line front end.
//
//   tsuner.exe data.dat [cudaDevice] [options]
//
// Same contract as the reference front end (main_TSUNER.cxx:22-107): reads a
// data.dat (Problem_loader.cxx:264-342 format), checks the GPU, builds the
// initial state, calls TSUNER() and writes <output prefix>.nc with the
// reference NetCDF layout.
//
// Initial state sources:
//   default        the analytic initial condition of the reference's
//                  Read_files == 0 path (Problem_loader.cxx:628-697) with the
//                  functions shipped in cini.cxx:22-61 (Gaussian hump and pit
//                  over a beach), evaluated at cell centres;
//   --raw PREFIX   raw little-endian arrays PREFIX_h.f64, PREFIX_H.f64 (nvol
//                  doubles each, row-major [npy][npx]) and optionally
//                  PREFIX_mask.i32 (nvol int32, 1 = erodible).
// The NetCDF4/HDF5 inputs of the reference's Read_files == 1 path cannot be
// read here (no libnetcdf/HDF5 in the image).
//
// Options (run-time form of Sim_parameters.hxx:45-54; defaults = shipped):
//   --order 1|2  --wbc 0|1|2  --bedload 0|1  --suspension 0|1
//   --fp32 (precision form, still-water level = SLR of data.dat)  --grass A_g
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "tsuner_b200.h"

namespace {

// cini.cxx:22-61 (shipped analytic initial condition)
double ic_bathy(double x, double y) {
    double H = -2.5 * std::exp(-5.0 * ((x + 0) * (x + 0) + (y - 0) * (y - 0)));
    H += -x * (x > 0.0);
    return H;
}
double ic_depth(double x, double y) {
    double h = ic_bathy(x, y) + 2.0 + 6 * std::exp(-5.0 * ((x + 2) * (x + 2) + (y - 0) * (y - 0)));
    return h * (h > 0.0);
}

bool read_raw(const std::string &path, void *dst, size_t bytes) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.read(static_cast<char *>(dst), (std::streamsize)bytes);
    return (size_t)f.gcount() == bytes;
}

bool file_exists(const char *p) {
    std::ifstream f(p);
    return (bool)f;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s data.dat [cudaDevice] [--raw PREFIX] [--order N] [--wbc N] "
                             "[--bedload N] [--suspension N] [--fp32] [--grass A]\n", argv[0]);
        return EXIT_FAILURE;
    }
    const char *input = argv[1];
    int dev = 0;
    int a = 2;
    if (argc > 2 && argv[2][0] != '-') {
        dev = std::atoi(argv[2]);
        a = 3;
    }
    TsuSwitches sw;
    tsu_switches_default(&sw);
    sw.read_files = 0;  // analytic / raw initial state: no boundary series
    std::string raw;
    bool fp32 = false;
    for (; a < argc; a++) {
        std::string o = argv[a];
        auto val = [&](void) -> const char * { return (a + 1 < argc) ? argv[++a] : "0"; };
        if (o == "--raw") raw = val();
        else if (o == "--order") sw.order = std::atoi(val());
        else if (o == "--wbc") sw.wbc = std::atoi(val());
        else if (o == "--bedload") sw.bedload = std::atoi(val());
        else if (o == "--suspension") sw.suspension = std::atoi(val());
        else if (o == "--grass") {
            sw.bedload_law = 1;
            sw.grass_ag = std::atof(val());
        } else if (o == "--fp32") fp32 = true;
        else {
            std::fprintf(stderr, "unknown option %s\n", o.c_str());
            return EXIT_FAILURE;
        }
    }
    if (!file_exists(input)) {  // main_TSUNER.cxx:51-54
        std::fprintf(stderr, "Error: Folder not found. '%s'\n", input);
        return EXIT_FAILURE;
    }
    switch (checkCUDAsupport(dev)) {  // main_TSUNER.cxx:57-71
        case 1: std::fprintf(stderr, "Error: There is no GPU\n"); return EXIT_FAILURE;
        case 2: std::fprintf(stderr, "Error: There is no GPU that supports CUDA\n"); return EXIT_FAILURE;
        case 3: std::fprintf(stderr, "N. Device erroneo\n"); return EXIT_FAILURE;
        default: break;
    }
    initializeGPU();

    SimParams p;
    char prefix[512], bathy[512], ic[512], maskf[512], tides[512];
    double slr = 0.0;
    int rc = tsu_parse_data_dat(input, &p, prefix, bathy, ic, maskf, &slr, tides, sizeof(prefix));
    if (rc) {
        std::fprintf(stderr, "Error: cannot parse %s (%s)\n", input, tsu_strerror(rc));
        return EXIT_FAILURE;
    }
    if (fp32) {
        sw.precision = 1;
        sw.eta0 = slr;
    }
    const size_t n = (size_t)p.npx * p.npy;
    std::vector<double> h(n), H(n);
    std::vector<tsu_double2> q(n);
    std::vector<int> fix(n, 1);
    if (!raw.empty()) {
        if (!read_raw(raw + "_h.f64", h.data(), n * 8) || !read_raw(raw + "_H.f64", H.data(), n * 8)) {
            std::fprintf(stderr, "Error: cannot read %s_h.f64 / %s_H.f64\n", raw.c_str(), raw.c_str());
            return EXIT_FAILURE;
        }
        read_raw(raw + "_mask.i32", fix.data(), n * 4);
        for (size_t i = 0; i < n; i++) q[i].x = q[i].y = 0.0;
    } else {
        // Problem_loader.cxx:662-685: values at cell centres
        for (int j = 0; j < p.npy; j++)
            for (int i = 0; i < p.npx; i++) {
                const size_t pos = (size_t)j * p.npx + i;
                const double x = p.xmin + 0.5 * p.dx + i * p.dx, y = p.ymin + 0.5 * p.dy + j * p.dy;
                h[pos] = ic_depth(x, y);
                H[pos] = ic_bathy(x, y);
                q[pos].x = q[pos].y = 0.0;
            }
    }
    tsu_set_default_switches(&sw);
    std::printf("%i\n", p.nvol);  // main_TSUNER.cxx:88
    double tiempo = 0.0;
    rc = TSUNER(h.data(), q.data(), H.data(), fix.data(), p, prefix, nullptr, nullptr, nullptr, 0, nullptr, nullptr,
                tiempo, dev, nullptr, nullptr, -1);
    if (rc) {  // main_TSUNER.cxx:91-98
        if (rc == 1) std::fprintf(stderr, "Error: Not enough GPU memory\n");
        else if (rc == 2) std::fprintf(stderr, "Error: Not enough CPU memory\n");
        else std::fprintf(stderr, "Error: %s (%s)\n", tsu_strerror(rc), tsu_last_error());
        return EXIT_FAILURE;
    }
    std::printf("\nTotal simulation time: %e sec.\n", tiempo);
    std::printf("Normal End.\n");
    return EXIT_SUCCESS;
}
