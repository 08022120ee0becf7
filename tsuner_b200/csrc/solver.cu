// solver.cu -- TsuSolver: device buffers, stepping and the tsu_* C ABI.
//
// Device layout (HBM): each field is a plane of npy rows with a row pitch
// rounded up to 32 elements (256 B in FP64, 128 B in FP32), planes
// consecutive:
//   bufA  [5][npy][pitch]  U^n at step entry / U^{n+1} at exit
//   bufB  [5][npy][pitch]  U* (intermediate RK stage)
//   hmax, bmin, eta_max [npy][pitch], mask [npy][pitch] uint8
// FP64 plain form (planes h, qx, qy, H, hc): ~105 B per cell.  FP32 form
// (planes z = eta - eta0, H, qx, qy, hc): ~53 B per cell plus an FP64
// staging area used only by uploads/downloads.  The reference allocates
// ~796 B per cell (GPU/main_TSUNER.cu:57-91).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "hostio.h"
#include "solver.h"
#include "stage32.h"
#include "stage64.h"
#include "tsuner_b200.h"

using namespace tsu;

namespace {
thread_local char g_err[512] = "";
std::mutex g_defaults_mu;
TsuSwitches g_defaults = {2, 1, 1, 1, 1, 1, 0, 0, 1e-3, 0.0};

int cuda_fail(cudaError_t e, const char *what) {
    snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
    return (e == cudaErrorMemoryAllocation) ? TSU_ERR_GPU_OOM : TSU_ERR_CUDA;
}
#define CK(call)                                            \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #call); \
    } while (0)

__global__ void set_scal_kernel(double *scal, int i, double v) { scal[i] = v; }
}  // namespace

const char *tsu_last_error_detail() { return g_err; }
void tsu_set_error_detail(const char *text) { snprintf(g_err, sizeof(g_err), "%s", text); }

// Status words the kernels leave in the scalar block (the stream must be
// synchronised): TSU_ERR_CUDA if a bounded wait expired, TSU_ERR_NONFINITE if
// a cell became NaN / infinite.  Either one makes the solver need a
// tsu_reset (after a new tsu_set_state for a non-finite state) before it steps
// again: an expired wait leaves the step it happened in unfinished.
int tsu_device_flags(TsuSolver *s, const double *sc) {
    if (sc[SC_ERR] != 0.0) {
        s->ready = false;
        s->fault = TSU_ERR_CUDA;
        snprintf(g_err, sizeof(g_err), "a bounded device wait for a tile load expired (step %.0f); tsu_reset "
                 "before stepping again", sc[SC_STEPS]);
        return TSU_ERR_CUDA;
    }
    if (sc[SC_NAN] != 0.0) {
        s->ready = false;
        s->fault = TSU_ERR_NONFINITE;
        snprintf(g_err, sizeof(g_err), "the state holds a NaN or an infinite value (detected at step %.0f)",
                 sc[SC_STEPS]);
        return TSU_ERR_NONFINITE;
    }
    return TSU_OK;
}

// a solver whose kernels reported an error steps again only after tsu_reset;
// until then stepping calls return that error
static int fault_refuses(TsuSolver *s, const char *what) {
    snprintf(g_err, sizeof(g_err), "%s: the last steps reported %s; tsu_reset (after tsu_set_state for a "
             "non-finite state) before stepping again", what, tsu_strerror(s->fault));
    return s->fault;
}

static int device_flags(TsuSolver *s) {
    double sc[SC_N];
    CK(cudaMemcpy(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost));
    return tsu_device_flags(s, sc);
}

static int validate(const SimParams *p, const TsuSwitches *sw) {
    if (!p || !sw) return TSU_ERR_INVALID;
    if (p->npx < 1 || p->npy < 1 || (long long)p->npx * p->npy > (1LL << 31) - 1) return TSU_ERR_INVALID;
    if (!(p->dx > 0) || !(p->dy > 0) || !(p->CFL > 0)) return TSU_ERR_INVALID;
    if (sw->order != 1 && sw->order != 2) return TSU_ERR_INVALID;
    if (sw->rk != 0 && sw->rk != 1) return TSU_ERR_INVALID;
    if (sw->manning != 0 && sw->manning != 1) return TSU_ERR_INVALID;
    // MUSCL-Hancock and the Manning branch exist in the FP64 plain form only
    if (sw->precision == 1 && (sw->rk == 0 || sw->manning)) return TSU_ERR_INVALID;
    if (sw->wbc < 0 || sw->wbc > 2) return TSU_ERR_INVALID;
    if (sw->bedload_law < 0 || sw->bedload_law > 1) return TSU_ERR_INVALID;
    if (sw->precision != 0 && sw->precision != 1) return TSU_ERR_INVALID;
    if (!std::isfinite(sw->eta0)) return TSU_ERR_INVALID;
    return TSU_OK;
}

extern "C" int tsu_switches_default(TsuSwitches *sw) {
    if (!sw) return TSU_ERR_INVALID;
    TsuSwitches d = {2, 1, 1, 1, 1, 1, 0, 0, 1e-3, 0.0};
    *sw = d;
    return TSU_OK;
}
extern "C" int tsu_set_default_switches(const TsuSwitches *sw) {
    if (!sw) return TSU_ERR_INVALID;
    std::lock_guard<std::mutex> g(g_defaults_mu);
    g_defaults = *sw;
    return TSU_OK;
}
extern "C" int tsu_get_default_switches(TsuSwitches *sw) {
    if (!sw) return TSU_ERR_INVALID;
    std::lock_guard<std::mutex> g(g_defaults_mu);
    *sw = g_defaults;
    return TSU_OK;
}

extern "C" int tsu_derive_params(SimParams *p, double friction_datdat) {
    if (!p) return TSU_ERR_INVALID;
    p->FR = friction_datdat / 8.0;  // Problem_loader.cxx:337-339 (Chezy)
    p->HQB = 5.0 * p->DS;
    p->Q = p->DS * sqrt(9.81 * (p->R - 1.0) * p->DS) / (1.0 - p->porosity);
    p->Opar = p->FR / ((p->R - 1.0) * 9.81 * p->DS);
    return TSU_OK;
}

static void free_all(TsuSolver *s) {
    s->invalidate_graph();
    cudaFree(s->A);
    cudaFree(s->B);
    cudaFree(s->K);
    cudaFree(s->hmax);
    cudaFree(s->bmin);
    cudaFree(s->eta);
    cudaFree(s->stage64);
    cudaFree(s->mask);
    cudaFree(s->CC);
    cudaFree(s->tCC);
    cudaFree(s->scal);
    cudaFree(s->partials);
    cudaFree(s->ticket);
    cudaFree(s->dconsts);
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    if (s->own_st) cudaStreamDestroy(s->own_st);
}

// TSU_DRY_SKIP=0 evaluates the Riemann solver on dry-dry edges too (for
// measurement; the results are the same values)
static int dry_skip_enabled() {
    const char *e = std::getenv("TSU_DRY_SKIP");
    return (e && e[0] == '0') ? 0 : 1;
}

static void fill_phys(TsuSolver *s) {
    const SimParams *p = &s->p;
    const TsuSwitches *sw = &s->sw;
    Phys64 &P = s->phys;
    P.FR = p->FR;
    P.eps_h = p->epsilon_h;
    P.Opar = p->Opar;
    P.OC = p->OC;
    P.Q = p->Q;
    P.HQB = p->HQB;
    P.porosity = p->porosity;
    P.CFL = p->CFL;
    P.dx = p->dx;
    P.dy = p->dy;
    P.inv_dx = 1.0 / p->dx;  // GPU/main_TSUNER.cu:43-44
    P.inv_dy = 1.0 / p->dy;
    P.k = s->hconsts;
    P.npx = p->npx;
    P.npy = p->npy;
    P.order = sw->order;
    P.wbc = sw->wbc;
    P.bedload = sw->bedload;
    P.suspension = sw->suspension;
    P.read_files = sw->read_files;
    P.bedload_law = sw->bedload_law;
    P.grass_ag = sw->grass_ag;
    P.rk = sw->rk;
    P.manning = sw->manning;
    P.ny_glob = s->ny_glob;
    P.j0 = s->j0;
    P.gs = s->gs;
    P.gn = s->gn;
    P.dry_skip = dry_skip_enabled();
    Phys32 &Q = s->phys32;
    Q.eta0 = sw->eta0;
    Q.eta0f = (float)sw->eta0;
    Q.FR = (float)p->FR;
    Q.eps_h = (float)p->epsilon_h;
    Q.Opar = (float)p->Opar;
    Q.OC = (float)p->OC;
    Q.Q = (float)p->Q;
    Q.HQB = (float)p->HQB;
    Q.porosity = (float)p->porosity;
    Q.CFL = (float)p->CFL;
    Q.dx = (float)p->dx;
    Q.dy = (float)p->dy;
    Q.inv_dx = (float)(1.0 / p->dx);
    Q.inv_dy = (float)(1.0 / p->dy);
    Q.vs = (float)s->hconsts.vs;
    Q.inv_vs = (float)(1.0 / s->hconsts.vs);
    Q.A_er = (float)s->hconsts.A_er;
    Q.sqrt_FR = (float)s->hconsts.sqrt_FR;
    Q.VP = (float)s->hconsts.VP;
    Q.K_dep = (float)s->hconsts.K_dep;
    Q.sqrt_OC = (float)s->hconsts.sqrt_OC;
    Q.DS5 = (float)s->hconsts.DS5;
    Q.npx = p->npx;
    Q.npy = p->npy;
    Q.order = sw->order;
    Q.wbc = sw->wbc;
    Q.bedload = sw->bedload;
    Q.suspension = sw->suspension;
    Q.read_files = sw->read_files;
    Q.bedload_law = sw->bedload_law;
    Q.grass_ag = (float)sw->grass_ag;
    Q.dry_skip = dry_skip_enabled();
}

// A solver for global rows [j0, j1) of the grid p (the whole grid: 0, npy),
// storing gs / gn ghost rows below / above them.
static int create_solver(TsuSolver **out, const SimParams *pg, const TsuSwitches *sw, int device, int j0, int j1,
                         int gs, int gn) {
    if (!out) return TSU_ERR_INVALID;
    *out = nullptr;
    int rc = validate(pg, sw);
    if (rc) {
        snprintf(g_err, sizeof(g_err), "invalid parameters or switches");
        return rc;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        snprintf(g_err, sizeof(g_err), "no CUDA device");
        return TSU_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return TSU_ERR_NO_DEVICE;
    CK(cudaSetDevice(device));
    TsuSolver *s = new (std::nothrow) TsuSolver();
    if (!s) return TSU_ERR_HOST_OOM;
    s->p = *pg;
    s->p.npy = j1 - j0;  // the owned rows
    s->p.nvol = pg->npx * s->p.npy;
    s->slab = (j0 != 0 || j1 != pg->npy || gs || gn);
    s->j0 = j0;
    s->gs = gs;
    s->gn = gn;
    s->ny_glob = pg->npy;
    const SimParams *p = &s->p;
    s->sw = *sw;
    s->device = device;
    s->fp32 = (sw->precision == 1);
    s->pitch = ((long long)p->npx + 31) / 32 * 32;
    const int nstore = gs + p->npy + gn;
    s->plane = s->pitch * nstore;
    const size_t pl = (size_t)s->plane * s->elem();
    cudaError_t e = cudaSuccess;
#define AL(ptr, bytes) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&(ptr), (bytes));
    AL(s->A, 5 * pl);
    AL(s->B, 5 * pl);
    if (sw->rk == 0) AL(s->K, 5 * pl);
    AL(s->hmax, pl);
    AL(s->bmin, pl);
    AL(s->eta, pl);
    AL(s->mask, (size_t)s->plane);
    AL(s->scal, SC_N * sizeof(double));
    s->npartials = partials_needed(p->npx, p->npy);
    AL(s->partials, 3 * s->npartials * sizeof(double));
    AL(s->ticket, sizeof(unsigned));
    AL(s->dconsts, sizeof(TsuConsts));
#undef AL
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->own_st, cudaStreamNonBlocking);
    s->st = s->own_st;
    if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
    if (e == cudaSuccess) e = s->fp32 ? stage32_prepare() : stage64_prepare();
    if (e == cudaSuccess) e = cudaMemsetAsync(s->A, 0, 5 * pl, s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->B, 0, 5 * pl, s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->mask, 1, (size_t)s->plane, s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->scal, 0, SC_N * sizeof(double), s->st);
    if (e == cudaSuccess) e = consts_launch(s->p, s->dconsts, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&s->hconsts, s->dconsts, sizeof(TsuConsts), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    // TSU_STAGE_TMA=0 makes every tile load with ordinary instructions
    const char *tma_env = std::getenv("TSU_STAGE_TMA");
    const bool tma_allowed = !(tma_env && tma_env[0] == '0');
    if (e == cudaSuccess && tma_allowed) {
        if (s->fp32) {
            Tma32 t32{};
            s->tma = stage32_tma_maps(-1, (const float *)s->A, (const float *)s->B, s->mask, s->pitch, s->plane,
                                      p->npx, p->npy, &t32);
            s->tmA = t32.a;
            s->tmB = t32.b;
            s->tmM = t32.m;
        } else {
            // the maps cover every stored row (ghost rows included)
            const double *ext[3] = {(const double *)s->hmax, (const double *)s->bmin, (const double *)s->eta};
            s->tma = stage64_tma_maps((const double *)s->A, (const double *)s->B, s->mask, ext, s->pitch, s->plane,
                                      p->npx, nstore, &s->tmA, &s->tmB, &s->tmM, &s->tmO, s->tmE);
        }
    }
    if (e != cudaSuccess) {
        int r = cuda_fail(e, "tsu_create");
        free_all(s);
        delete s;
        return r;
    }
    fill_phys(s);
    *out = s;
    return TSU_OK;
}

extern "C" int tsu_create(TsuSolver **out, const SimParams *p, const TsuSwitches *sw, int device) {
    if (!p) return TSU_ERR_INVALID;
    return create_solver(out, p, sw, device, 0, p->npy, 0, 0);
}

extern "C" int tsu_slab_create(TsuSolver **out, const SimParams *p, const TsuSwitches *sw, int j0, int j1,
                               int device) {
    if (out) *out = nullptr;
    if (!p || !sw || !out) return TSU_ERR_INVALID;
    if (j0 < 0 || j1 > p->npy || j1 - j0 < 2 || (j0 == 0 && j1 == p->npy)) {
        snprintf(g_err, sizeof(g_err), "slab rows [%d, %d) of a %d-row grid: a slab owns at least 2 rows and not "
                 "the whole grid", j0, j1, p->npy);
        return TSU_ERR_INVALID;
    }
    if (sw->precision != 0 || sw->order != 2 || sw->rk != 1) {
        snprintf(g_err, sizeof(g_err), "row slabs are built for the FP64 plain form with order 2 and RK2");
        return TSU_ERR_INVALID;
    }
    const bool periodic = (sw->wbc == 2);
    const int gs = (j0 > 0 || periodic) ? 2 : 0, gn = (j1 < p->npy || periodic) ? 2 : 0;
    return create_solver(out, p, sw, device, j0, j1, gs, gn);
}

extern "C" int tsu_destroy(TsuSolver *s) {
    if (!s) return TSU_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->st);
    free_all(s);
    delete s;
    return TSU_OK;
}

// FP64 staging planes of the FP32 form (allocated on first use).
static int staging(TsuSolver *s) {
    if (!s->stage64) CK(cudaMalloc((void **)&s->stage64, 5 * (size_t)s->plane * sizeof(double)));
    return TSU_OK;
}

extern "C" int tsu_set_state(TsuSolver *s, const double *h, const double *qx, const double *qy, const double *H,
                             const double *hc) {
    if (!s || !h || !qx || !qy || !H) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    int r = s->fp32 ? staging(s) : TSU_OK;
    if (r) return r;
    double *base = s->fp32 ? s->stage64 : (double *)s->A;
    const double *src[5] = {h, qx, qy, H, hc};
    void *dst[5];
    const void *from[5];
    int n = 0;
    for (int f = 0; f < 5; f++) {
        if (src[f]) {
            dst[n] = base + f * s->plane + s->own_off();
            from[n++] = src[f];
        } else {
            CK(cudaMemsetAsync(base + f * s->plane, 0, (size_t)s->plane * sizeof(double), s->st));  // ghost rows too
        }
    }
    CK(tsu::planes_h2d(n, dst, s->pitch * sizeof(double), from, s->p.npx * sizeof(double), s->p.npx * sizeof(double),
                       s->p.npy, s->st));
    if (s->fp32)
        CK(to32_launch(s->stage64, s->pitch, s->plane, s->p.npx, s->p.npy, s->sw.eta0, (float *)s->A, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->has_state = true;
    s->ready = false;
    return TSU_OK;
}

extern "C" int tsu_set_mask(TsuSolver *s, const int *fixH) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    if (!fixH) {
        CK(cudaMemsetAsync(s->mask, 1, (size_t)s->plane, s->st));
        CK(cudaStreamSynchronize(s->st));
        return TSU_OK;
    }
    const size_t npx = s->p.npx, npy = s->p.npy;
    // Validate first (the mask is left as it was on a bad value), in parallel
    // row ranges; the first bad index is the first one of the lowest range.
    const int parts = (int)std::min<size_t>(npy, 4 * (size_t)tsu::host_threads());
    std::vector<long long> bad(parts, -1);
    tsu::host_parallel(parts, [&](int q) {
        const size_t a = npy * q / parts * npx, b = npy * (q + 1) / parts * npx;
        for (size_t i = a; i < b; i++)
            if (fixH[i] != 0 && fixH[i] != 1) {
                bad[q] = (long long)i;
                return;
            }
    });
    for (int q = 0; q < parts; q++)
        if (bad[q] >= 0) {
            snprintf(g_err, sizeof(g_err), "mask value %d at %lld is not 0 or 1", fixH[bad[q]], bad[q]);
            return TSU_ERR_INVALID;
        }
    void *dst[1] = {s->mask + s->own_off()};
    const void *from[1] = {fixH};
    CK(tsu::planes_h2d(1, dst, s->pitch, from, npx * sizeof(int), npx, npy, s->st,
                       [&](int, size_t r0, size_t nr, unsigned char *out) {
                           const int *in = fixH + r0 * npx;
                           for (size_t i = 0; i < nr * npx; i++) out[i] = (unsigned char)in[i];
                       }));
    return TSU_OK;
}

extern "C" int tsu_set_boundary_series(TsuSolver *s, const double *CC, const double *tCC, unsigned long timeCC) {
    if (!s || !CC || !tCC || timeCC < 2) return TSU_ERR_INVALID;
    // GPU/VolumeSolver.cu:172-215 assumes a uniform series; check it so that
    // interpolation indices stay inside the arrays.
    double dtc = tCC[1] - tCC[0];
    if (!(dtc > 0)) return TSU_ERR_INVALID;
    for (unsigned long q = 1; q < timeCC; q++)
        if (fabs((tCC[q] - tCC[0]) - q * dtc) > 1e-9 * fabs(dtc) * q) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    // The buffers are kept and only grown: a free + allocate pair per call
    // occasionally took hundreds of milliseconds.  The copies below are
    // ordered on the solver's stream after any steps still in flight.  Until
    // the new series has arrived the solver has none (a failed upload leaves
    // it unable to step rather than holding half of a series).
    s->timeCC = 0;
    s->invalidate_graph();
    size_t n = (size_t)(2 * s->p.npx + 2 * s->p.npy) * 4 * timeCC;
    if (n > s->CC_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(s->CC);
        s->CC = nullptr;
        s->CC_cap = 0;
        CK(cudaMalloc((void **)&s->CC, n * sizeof(double)));
        s->CC_cap = n;
    }
    if (timeCC > s->tCC_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(s->tCC);
        s->tCC = nullptr;
        s->tCC_cap = 0;
        CK(cudaMalloc((void **)&s->tCC, timeCC * sizeof(double)));
        s->tCC_cap = timeCC;
    }
    CK(tsu::bytes_h2d(s->CC, CC, n * sizeof(double), s->st));
    CK(tsu::bytes_h2d(s->tCC, tCC, timeCC * sizeof(double), s->st));
    s->timeCC = timeCC;
    s->invalidate_graph();
    return TSU_OK;
}

Stage64Args TsuSolver::args() const {
    Stage64Args a;
    // the kernels address the owned rows from row 0; a slab's ghost rows
    // lie below (negative offsets) and above them
    const long long o = own_off();
    a.bufA = (double *)A + o;
    a.bufB = (double *)B + o;
    a.bufK = K ? (double *)K + o : nullptr;
    a.mask = mask + o;
    a.CC = CC;
    a.tCC = tCC;
    a.timeCC = timeCC;
    a.hmax = (double *)hmax + o;
    a.bmin = (double *)bmin + o;
    a.eta_max = (double *)eta + o;
    a.scal = scal;
    a.partials = partials;
    a.ticket = ticket;
    a.pitch = pitch;
    a.plane = plane;
    a.phys = phys;
    a.tmA = tmA;
    a.tmB = tmB;
    a.tmM = tmM;
    a.tmO = tmO;
    for (int k = 0; k < 3; k++) a.tmE[k] = tmE[k];
    a.tma = tma ? 1 : 0;
    return a;
}

Stage32Args TsuSolver::args32() const {
    Stage32Args a;
    a.bufA = (float *)A;
    a.bufB = (float *)B;
    a.mask = mask;
    a.CC = CC;
    a.tCC = tCC;
    a.timeCC = timeCC;
    a.hmax = (float *)hmax;
    a.bmin = (float *)bmin;
    a.eta_max = (float *)eta;
    a.scal = scal;
    a.partials = partials;
    a.ticket = ticket;
    a.pitch = pitch;
    a.plane = plane;
    a.phys = phys32;
    return a;
}

void TsuSolver::invalidate_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
}

extern "C" int tsu_reset(TsuSolver *s) {
    if (!s || !s->has_state) return TSU_ERR_INVALID;
    if (s->sw.read_files && s->timeCC < 2) {
        snprintf(g_err, sizeof(g_err), "read_files is set but no boundary series was given");
        return TSU_ERR_INVALID;
    }
    CK(cudaSetDevice(s->device));
    s->ready = false;
    s->fault = 0;
    const size_t state_bytes = 5 * (size_t)s->plane * s->elem();
    if (s->single_stage()) {
        // the state may sit in B after an odd number of single-stage steps:
        // bring it to A, where a reset run starts
        CK(cudaStreamSynchronize(s->st));
        if (s->current() == s->B) CK(cudaMemcpyAsync(s->A, s->B, state_bytes, cudaMemcpyDeviceToDevice, s->st));
    }
    if (s->K) CK(cudaMemcpyAsync(s->K, s->A, state_bytes, cudaMemcpyDeviceToDevice, s->st));  // Vk = V
    double init[SC_N] = {0.0, -1.0, HUGE_VAL, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    CK(cudaMemcpyAsync(s->scal, init, sizeof(init), cudaMemcpyHostToDevice, s->st));
    // the end-of-step ticket: a step whose tiles stopped early (an expired
    // wait) leaves it short of the tile count
    CK(cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), s->st));
    if (s->fp32) {
        CK(fill32_launch((float *)s->hmax, s->plane, -1e30f, s->st));
        CK(fill32_launch((float *)s->bmin, s->plane, -1e30f, s->st));
        CK(fill32_launch((float *)s->eta, s->plane, -1e30f, s->st));
        CK(initial_dt32_launch((const float *)s->A, s->pitch, s->plane, s->phys32, s->partials, s->ticket, s->scal,
                               s->st));
    } else {
        CK(fill_launch((double *)s->hmax, s->plane, -1e30, s->st));  // GPU/Volume_kernel.cu:112-137
        CK(fill_launch((double *)s->bmin, s->plane, -1e30, s->st));
        CK(fill_launch((double *)s->eta, s->plane, -1e30, s->st));
        CK(initial_dt_launch((const double *)s->A + s->own_off(), s->pitch, s->plane, s->phys, s->partials, s->ticket, s->scal,
                             s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    int rc = device_flags(s);  // e.g. a NaN in the uploaded state
    if (rc) return rc;
    s->ready = true;
    return TSU_OK;
}

// FP64 host planes -> the FP32 form's float extrema (exact for values that
// came from float extrema)
__global__ void narrow_kernel(const double *__restrict__ a, float *__restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

extern "C" int tsu_resume(TsuSolver *s, double t, long steps, const double *hmax, const double *bmin_rawH,
                          const double *eta_max) {
    if (!s || !s->ready || s->slab || steps < 0 || !(t >= 0.0) || !std::isfinite(t)) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    const double *src[3] = {hmax, bmin_rawH, eta_max};
    void *ext[3] = {s->hmax, s->bmin, s->eta};
    if (s->fp32) {
        int r = staging(s);
        if (r) return r;
    }
    for (int f = 0; f < 3; f++) {
        if (!src[f]) continue;
        double *d = s->fp32 ? s->stage64 + f * s->plane : (double *)ext[f];
        void *dst[1] = {d + s->own_off()};
        const void *from[1] = {src[f]};
        CK(tsu::planes_h2d(1, dst, s->pitch * sizeof(double), from, s->p.npx * sizeof(double),
                           s->p.npx * sizeof(double), s->p.npy, s->st));
        if (s->fp32) {
            narrow_kernel<<<1184, 256, 0, s->st>>>(d, (float *)ext[f], s->plane);
            CK(cudaGetLastError());
        }
    }
    const double ts[2] = {t, (double)steps};
    CK(cudaMemcpyAsync(s->scal + SC_T, &ts[0], sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->scal + SC_STEPS, &ts[1], sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return TSU_OK;
}

int TsuSolver::launch_steps(long n) {
    if (fp32) {
        Stage32Args a = args32();
        Tma32 tm;
        tm.a = tmA;
        tm.b = tmB;
        tm.m = tmM;
        tm.on = tma ? 1 : 0;
        for (long i = 0; i < n; i++)
            for (int k = 0; k < sw.order; k++) CK(stage32_launch(sw.order, k, a, tm, st));
    } else {
        Stage64Args a = args();
        for (long i = 0; i < n; i++)
            for (int k = 0; k < stages(); k++) CK(stage64_launch(sw.order, k, a, st));
    }
    return TSU_OK;
}

static int slab_refuses(TsuSolver *s, const char *what) {
    snprintf(g_err, sizeof(g_err), "%s: a row slab steps stage by stage (tsu_slab_stage) with its halo exchange "
             "in between", what);
    return TSU_ERR_INVALID;
}

extern "C" int tsu_step(TsuSolver *s, long nsteps) {
    if (!s || nsteps < 0) return TSU_ERR_INVALID;
    if (s->slab) return slab_refuses(s, "tsu_step");
    if (s->fault) return fault_refuses(s, "tsu_step");
    if (s->sw.read_files && s->timeCC < 2) {  // e.g. the last series upload failed
        snprintf(g_err, sizeof(g_err), "read_files is set but no boundary series is loaded");
        return TSU_ERR_INVALID;
    }
    if (!s->ready) {
        int r = tsu_reset(s);
        if (r) return r;
    }
    CK(cudaSetDevice(s->device));
    long n = nsteps;
    const long K = TsuSolver::kGraphSteps;
    if (n >= K && !s->graph_exec) {  // host-side setup, once: before the timed region
        CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
        int r = s->launch_steps(K);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->st, &g);
        if (r) return r;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        s->graph = g;
        CK(cudaGraphInstantiate(&s->graph_exec, g, 0));
    }
    CK(cudaEventRecord(s->e0, s->st));
    while (n >= K && s->graph_exec) {
        CK(cudaGraphLaunch(s->graph_exec, s->st));
        n -= K;
    }
    int r = s->launch_steps(n);
    if (r) return r;
    CK(cudaEventRecord(s->e1, s->st));
    s->last_launches = nsteps * s->stages();
    s->timed = true;
    return TSU_OK;
}

extern "C" int tsu_sync(TsuSolver *s) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    return device_flags(s);
}

// ------------------------------------------------------------- row slabs
extern "C" int tsu_set_stream(TsuSolver *s, void *stream) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));  // work issued so far completes first
    s->invalidate_graph();
    s->st = static_cast<cudaStream_t>(stream);
    return TSU_OK;
}

extern "C" int tsu_slab_info(TsuSolver *s, int *j0, int *rows, int *ghost_south, int *ghost_north) {
    if (!s) return TSU_ERR_INVALID;
    if (j0) *j0 = s->j0;
    if (rows) *rows = s->p.npy;
    if (ghost_south) *ghost_south = s->gs;
    if (ghost_north) *ghost_north = s->gn;
    return TSU_OK;
}

extern "C" int tsu_slab_stage(TsuSolver *s, int k) {
    if (!s || !s->slab || k < 0 || k >= s->stages()) return TSU_ERR_INVALID;
    if (s->fault) return fault_refuses(s, "tsu_slab_stage");
    if (!s->ready) {
        snprintf(g_err, sizeof(g_err), "tsu_slab_stage: tsu_reset the slab first");
        return TSU_ERR_INVALID;
    }
    if (s->sw.read_files && s->timeCC < 2) {
        snprintf(g_err, sizeof(g_err), "read_files is set but no boundary series is loaded");
        return TSU_ERR_INVALID;
    }
    CK(cudaSetDevice(s->device));
    CK(stage64_launch(s->sw.order, k, s->args(), s->st));
    return TSU_OK;
}

// which: 0 = buffer A (the state a step starts from), 1 = buffer B (the
// intermediate RK2 state), 2 = the mask; side: 0 = south, 1 = north
static int halo_geometry(TsuSolver *s, int which, int side, size_t *elem, int *planes) {
    if (!s || !s->slab || which < 0 || which > 2 || side < 0 || side > 1 || s->p.npy < 2) return TSU_ERR_INVALID;
    *elem = (which == 2) ? 1 : s->elem();
    *planes = (which == 2) ? 1 : 5;
    return TSU_OK;
}

extern "C" int tsu_slab_halo_bytes(TsuSolver *s, int which, size_t *bytes) {
    size_t el;
    int np;
    if (!bytes || halo_geometry(s, which, 0, &el, &np)) return TSU_ERR_INVALID;
    *bytes = (size_t)np * 2 * s->p.npx * el;
    return TSU_OK;
}

// the two owned rows next to `side` -> d_dst [planes][2][npx] (contiguous)
extern "C" int tsu_slab_pack(TsuSolver *s, int which, int side, void *d_dst) {
    size_t el;
    int np;
    if (!d_dst || halo_geometry(s, which, side, &el, &np)) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    char *base = static_cast<char *>(which == 2 ? (void *)s->mask : which == 0 ? s->A : s->B);
    const long long row = s->gs + (side == 0 ? 0 : s->p.npy - 2);  // stored row of the first one
    const size_t w = (size_t)s->p.npx * el, sp = (size_t)s->pitch * el;
    for (int f = 0; f < np; f++)
        CK(cudaMemcpy2DAsync(static_cast<char *>(d_dst) + (size_t)f * 2 * w, w,
                             base + ((size_t)f * s->plane + (size_t)row * s->pitch) * el, sp, w, 2,
                             cudaMemcpyDeviceToDevice, s->st));
    return TSU_OK;
}

// d_src [planes][2][npx] -> the two ghost rows beyond `side`
extern "C" int tsu_slab_unpack(TsuSolver *s, int which, int side, const void *d_src) {
    size_t el;
    int np;
    if (!d_src || halo_geometry(s, which, side, &el, &np)) return TSU_ERR_INVALID;
    if ((side == 0 && s->gs < 2) || (side == 1 && s->gn < 2)) {
        snprintf(g_err, sizeof(g_err), "tsu_slab_unpack: the slab has no ghost rows on side %d", side);
        return TSU_ERR_INVALID;
    }
    CK(cudaSetDevice(s->device));
    char *base = static_cast<char *>(which == 2 ? (void *)s->mask : which == 0 ? s->A : s->B);
    const long long row = (side == 0) ? 0 : s->gs + s->p.npy;  // stored row of the first ghost row
    const size_t w = (size_t)s->p.npx * el, sp = (size_t)s->pitch * el;
    for (int f = 0; f < np; f++)
        CK(cudaMemcpy2DAsync(base + ((size_t)f * s->plane + (size_t)row * s->pitch) * el, sp,
                             static_cast<const char *>(d_src) + (size_t)f * 2 * w, w, w, 2, cudaMemcpyDeviceToDevice,
                             s->st));
    return TSU_OK;
}

extern "C" int tsu_get_dt_device(TsuSolver *s, double *d_dt) {
    if (!s || !d_dt) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(d_dt, s->scal + SC_DT, sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    return TSU_OK;
}

extern "C" int tsu_set_dt_device(TsuSolver *s, const double *d_dt) {
    if (!s || !d_dt) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(s->scal + SC_DT, d_dt, sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    return TSU_OK;
}

extern "C" int tsu_set_wait_limit_ns(unsigned long long ns) {
    if (ns == 0) ns = kDefaultWaitNs;
    CK(set_wait_limit_stage64(ns));
    CK(set_wait_limit_stage32(ns));
    CK(set_wait_limit_corrector(ns));
    return TSU_OK;
}

extern "C" int tsu_run_until(TsuSolver *s, double t_end, long max_steps, long *steps_done) {
    if (!s || max_steps < 0) return TSU_ERR_INVALID;
    if (s->slab) return slab_refuses(s, "tsu_run_until");
    if (s->fault) return fault_refuses(s, "tsu_run_until");
    if (s->sw.read_files && s->timeCC < 2) {  // e.g. the last series upload failed
        snprintf(g_err, sizeof(g_err), "read_files is set but no boundary series is loaded");
        return TSU_ERR_INVALID;
    }
    if (!s->ready) {
        int r = tsu_reset(s);
        if (r) return r;
    }
    CK(cudaSetDevice(s->device));
    double sc[SC_N];
    CK(cudaMemcpyAsync(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const double steps0 = sc[SC_STEPS];
    set_scal_kernel<<<1, 1, 0, s->st>>>(s->scal, SC_TEND, t_end);
    CK(cudaGetLastError());
    long left = max_steps;
    int rf = TSU_OK;
    while (left > 0) {
        long chunk = left < 64 ? left : 64;
        int r = tsu_step(s, chunk);
        if (r) return r;
        left -= chunk;
        CK(cudaMemcpyAsync(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        if ((rf = tsu_device_flags(s, sc)) != TSU_OK) break;  // an expired wait or a non-finite state
        if (!(sc[SC_T] < t_end)) break;
    }
    set_scal_kernel<<<1, 1, 0, s->st>>>(s->scal, SC_TEND, HUGE_VAL);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->st));
    if (steps_done) *steps_done = (long)(sc[SC_STEPS] - steps0);
    return rf;
}

void *TsuSolver::current() const {
    if (!single_stage()) return A;
    double sc[SC_N];
    if (cudaMemcpy(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost) != cudaSuccess) return A;
    return sc[SC_PAR] != 0.0 ? B : A;
}

extern "C" int tsu_get_state(TsuSolver *s, double *V) {
    if (!s || !V) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    const double *cur = (const double *)s->current();
    if (s->fp32) {
        int r = staging(s);
        if (r) return r;
        CK(to64_launch((const float *)s->current(), s->pitch, s->plane, s->p.npx, s->p.npy, s->sw.eta0, s->stage64,
                       s->st));
        cur = s->stage64;
    }
    const size_t n = (size_t)s->p.npx * s->p.npy;
    void *dst[5];
    const void *from[5];
    for (int f = 0; f < 5; f++) {
        dst[f] = V + f * n;
        from[f] = cur + f * s->plane + s->own_off();
    }
    CK(tsu::planes_d2h(5, dst, s->p.npx * sizeof(double), from, s->pitch * sizeof(double), s->p.npx * sizeof(double),
                       s->p.npy, s->st));
    return TSU_OK;
}

extern "C" int tsu_get_extrema(TsuSolver *s, double *hmax, double *bmin, double *eta_max) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    void *src[3] = {s->hmax, s->bmin, s->eta};
    double *want[3] = {hmax, bmin, eta_max};
    void *dst[3];
    const void *from[3];
    int n = 0;
    if (s->fp32) {
        int r = staging(s);
        if (r) return r;
    }
    for (int f = 0; f < 3; f++) {
        if (!want[f]) continue;
        const double *d = (const double *)src[f];
        if (s->fp32) {  // widen into the FP64 staging planes, one per field
            CK(widen_launch((const float *)src[f], s->stage64 + f * s->plane, s->plane, s->st));
            d = s->stage64 + f * s->plane;
        }
        dst[n] = want[f];
        from[n++] = d + s->own_off();
    }
    CK(tsu::planes_d2h(n, dst, s->p.npx * sizeof(double), from, s->pitch * sizeof(double), s->p.npx * sizeof(double),
                       s->p.npy, s->st));
    return TSU_OK;
}

extern "C" int tsu_get_time(TsuSolver *s, double *t, double *dt, long *steps) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    double sc[SC_N];
    CK(cudaMemcpy(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost));
    if (t) *t = sc[SC_T];
    if (dt) *dt = sc[SC_DT];
    if (steps) *steps = (long)sc[SC_STEPS];
    return tsu_device_flags(s, sc);
}

extern "C" int tsu_get_sums(TsuSolver *s, double *water, double *sediment) {
    if (!s || !s->fp32) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    double sc[SC_N];
    CK(cudaMemcpy(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost));
    if (water) *water = sc[SC_MASS];
    if (sediment) *sediment = sc[SC_SED];
    return TSU_OK;
}

extern "C" int tsu_get_consts(TsuSolver *s, TsuConsts *k) {
    if (!s || !k) return TSU_ERR_INVALID;
    *k = s->hconsts;
    return TSU_OK;
}

extern "C" int tsu_last_step_ms(TsuSolver *s, double *ms) {
    if (!s || !ms || !s->timed) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaEventSynchronize(s->e1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, s->e0, s->e1));
    *ms = f;
    return TSU_OK;
}

extern "C" int tsu_last_step_launches(TsuSolver *s, long *launches) {
    if (!s || !launches) return TSU_ERR_INVALID;
    *launches = s->last_launches;
    return TSU_OK;
}

extern "C" int tsu_state_device(TsuSolver *s, void **ptr, long *pitch_elems, long *plane_elems, int *elem_bytes) {
    if (!s) return TSU_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    if (ptr) *ptr = static_cast<char *>(s->current()) + s->own_off() * (long long)s->elem();
    if (pitch_elems) *pitch_elems = (long)s->pitch;
    if (plane_elems) *plane_elems = (long)s->plane;
    if (elem_bytes) *elem_bytes = (int)s->elem();
    return TSU_OK;
}

extern "C" const char *tsu_strerror(int code) {
    switch (code) {
        case TSU_OK: return "ok";
        case TSU_ERR_GPU_OOM: return "not enough GPU memory";
        case TSU_ERR_HOST_OOM: return "not enough CPU memory";
        case TSU_ERR_INVALID: return "invalid argument";
        case TSU_ERR_CUDA: return "CUDA runtime error";
        case TSU_ERR_NO_DEVICE: return "no usable CUDA device";
        case TSU_ERR_NONFINITE: return "non-finite state";
        case TSU_ERR_IO: return "output file error";
        default: return "unknown error";
    }
}

extern "C" const char *tsu_last_error(void) { return g_err; }

extern "C" int tsu_struct_sizes(size_t out[3]) {
    if (!out) return TSU_ERR_INVALID;
    out[0] = sizeof(SimParams);
    out[1] = sizeof(TsuSwitches);
    out[2] = sizeof(TsuConsts);
    return TSU_OK;
}

extern "C" const char *tsu_version(void) { return "tsuner_b200 0.2 (sm_100a)"; }

// GPU/CheckCUDASupport.cu:21-44 contract: 0 ok, 1 no GPU, 2 no CUDA GPU, 3 bad index.
extern "C" int checkCUDAsupport(int cudaDevice) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    if (n == 0) return 1;
    if (cudaDevice < 0 || cudaDevice >= n) return 3;
    for (int d = 0; d < n; d++) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major >= 1) return 0;
    }
    return 2;
}

extern "C" void initializeGPU(void) { cudaFree(0); }
