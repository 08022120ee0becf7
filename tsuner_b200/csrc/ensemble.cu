// ensemble.cu -- batched ensemble of FP32-form grids of uneven size.
//
// Each member is an ordinary FP32-form solver (its own buffers, time, dt,
// extrema, sums, boundary series); stepping the ensemble launches, per RK
// stage, ONE persistent kernel (ens32_kernel) whose CTAs walk the tile list
// of all members, so small and large members share the GPU without a launch
// per member.  Each member's dt comes from a segmented min-reduction: the
// last CTA to finish a member's tiles reduces that member's partials.  Steps
// are replayed from a captured CUDA graph.  The tile shape, the schedule
// (static stride vs a dynamic work counter) and the number of resident CTAs
// are chosen by tsu_ens_autotune(), which times every candidate on the
// ensemble itself and restores the members' state afterwards.
// No counterpart in the reference (single grid only).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "solver.h"
#include "stage32.h"
#include "tsuner_b200.h"

using namespace tsu;

struct TsuEnsemble {
    int device = 0;
    int n = 0;
    std::vector<TsuSolver *> m;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // current configuration
    int variant = 0, dynamic = 0, ctas = 0;
    // device tables for the current tile shape
    std::vector<EnsMember> h_members;  // last uploaded member descriptors
    EnsMember *d_members = nullptr;
    Tma32 *d_tmas = nullptr;  // per member TMA descriptors for the current tile shape
    int *d_tile_member = nullptr;
    unsigned *d_work = nullptr;
    unsigned ntiles = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long last_launches = 0;
    bool timed = false;
    int num_sms = 148;
};

namespace {
__global__ void set_tend_kernel(const EnsMember *members, int n, double t_end) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        members[i].g.scal[SC_TEND] = t_end;
}
// 1 if every member's time has reached t_end
__global__ void all_done_kernel(const EnsMember *members, int n, double t_end, int *done) {
    __shared__ int s_not;
    if (threadIdx.x == 0) s_not = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (members[i].g.scal[SC_T] < t_end) s_not = 1;
    __syncthreads();
    if (threadIdx.x == 0) *done = !s_not;
}

// error detail, reported through tsu_last_error()
void ens_error(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
void ens_error(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    tsu_set_error_detail(buf);
}
#define ECK(call)                                                                    \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess) {                                                     \
            ens_error("%s: %s", #call, cudaGetErrorString(_e));                      \
            return _e == cudaErrorMemoryAllocation ? TSU_ERR_GPU_OOM : TSU_ERR_CUDA; \
        }                                                                            \
    } while (0)

void drop_graph(TsuEnsemble *E) {
    if (E->graph_exec) cudaGraphExecDestroy(E->graph_exec);
    if (E->graph) cudaGraphDestroy(E->graph);
    E->graph_exec = nullptr;
    E->graph = nullptr;
}

// Rebuilds the member descriptors and the global tile list for `variant`.
int build_tables(TsuEnsemble *E, int variant) {
    int tx, ty, minb;
    stage32_tile_shape(variant, &tx, &ty, &minb);
    std::vector<EnsMember> mem(E->n);
    std::vector<int> tm;
    unsigned tile0 = 0;
    for (int i = 0; i < E->n; i++) {
        TsuSolver *s = E->m[i];
        EnsMember &M = mem[i];
        M.g = s->args32();
        M.ntx = (s->p.npx + tx - 1) / tx;
        const int nty = (s->p.npy + ty - 1) / ty;
        M.ntiles = (unsigned)M.ntx * nty;
        M.tile0 = tile0;
        tile0 += M.ntiles;
        tm.insert(tm.end(), M.ntiles, i);
    }
    // TMA descriptors of every member's state buffers for this tile shape
    // (a member whose grid is too small for the box loads without TMA)
    std::vector<Tma32> tmas(E->n);
    const char *tma_env = std::getenv("TSU_STAGE_TMA");
    const bool tma_allowed = !(tma_env && tma_env[0] == '0');
    for (int i = 0; i < E->n; i++) {
        TsuSolver *s = E->m[i];
        tmas[i].on = tma_allowed && stage32_tma_maps(variant, (const float *)s->A, (const float *)s->B, s->mask,
                                                     s->pitch, s->plane, s->p.npx, s->p.npy, &tmas[i]);
    }
    cudaFree(E->d_members);
    cudaFree(E->d_tile_member);
    cudaFree(E->d_tmas);
    E->d_members = nullptr;
    E->d_tile_member = nullptr;
    E->d_tmas = nullptr;
    ECK(cudaMalloc((void **)&E->d_members, sizeof(EnsMember) * E->n));
    ECK(cudaMalloc((void **)&E->d_tile_member, sizeof(int) * tm.size()));
    ECK(cudaMalloc((void **)&E->d_tmas, sizeof(Tma32) * E->n));
    ECK(cudaMemcpy(E->d_members, mem.data(), sizeof(EnsMember) * E->n, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(E->d_tile_member, tm.data(), sizeof(int) * tm.size(), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(E->d_tmas, tmas.data(), sizeof(Tma32) * E->n, cudaMemcpyHostToDevice));
    E->h_members.swap(mem);
    E->ntiles = tile0;
    E->variant = variant;
    drop_graph(E);
    return TSU_OK;
}

bool same_buffers(const Stage32Args &a, const Stage32Args &b) {
    return a.bufA == b.bufA && a.bufB == b.bufB && a.mask == b.mask && a.CC == b.CC && a.tCC == b.tCC &&
           a.timeCC == b.timeCC && a.hmax == b.hmax && a.bmin == b.bmin && a.eta_max == b.eta_max &&
           a.scal == b.scal && a.partials == b.partials && a.ticket == b.ticket && a.pitch == b.pitch &&
           a.plane == b.plane;
}

// The member descriptors hold the members' device pointers, and some of
// those (the boundary series) are allocated after the ensemble is created.
// Before stepping, every descriptor is compared with its member's current
// buffers and the table is re-uploaded, in stream order, when one changed.
int refresh_members(TsuEnsemble *E) {
    bool changed = false;
    for (int i = 0; i < E->n; i++) {
        const Stage32Args g = E->m[i]->args32();
        if (!same_buffers(g, E->h_members[i].g)) {
            E->h_members[i].g = g;
            changed = true;
        }
    }
    if (changed)
        ECK(cudaMemcpyAsync(E->d_members, E->h_members.data(), sizeof(EnsMember) * E->n, cudaMemcpyHostToDevice,
                            E->st));
    return TSU_OK;
}

EnsArgs ens_args(const TsuEnsemble *E) {
    EnsArgs a;
    a.members = E->d_members;
    a.tile_member = E->d_tile_member;
    a.ntiles = E->ntiles;
    a.dynamic = E->dynamic;
    a.work = E->d_work;
    a.tmas = E->d_tmas;
    return a;
}

int launch_steps(TsuEnsemble *E, long nsteps) {
    const EnsArgs a = ens_args(E);
    const int order = E->m[0]->sw.order;
    for (long i = 0; i < nsteps; i++)
        for (int k = 0; k < order; k++) ECK(ens32_launch(E->variant, order, k, a, E->m[0]->phys32, E->ctas, E->st));
    return TSU_OK;
}

int default_ctas(TsuEnsemble *E, int variant) {
    int per = ens32_max_ctas_per_sm(variant);
    if (per < 1) per = 1;
    return std::max(1, std::min<int>((int)E->ntiles, per * E->num_sms));
}
}  // namespace

extern "C" int tsu_ens_create(TsuEnsemble **out, int nmembers, const SimParams *params, const TsuSwitches *sw,
                              int device) {
    if (!out || nmembers < 1 || !params || !sw) return TSU_ERR_INVALID;
    for (int i = 0; i < nmembers; i++)  // FP32 form, one scheme order for the whole batch
        if (sw[i].precision != 1 || sw[i].order != sw[0].order) return TSU_ERR_INVALID;
    *out = nullptr;
    TsuEnsemble *E = new (std::nothrow) TsuEnsemble();
    if (!E) return TSU_ERR_HOST_OOM;
    E->device = device;
    E->n = nmembers;
    E->m.assign(nmembers, nullptr);
    for (int i = 0; i < nmembers; i++) {
        int rc = tsu_create(&E->m[i], &params[i], &sw[i], device);
        if (rc) {
            for (int j = 0; j < i; j++) tsu_destroy(E->m[j]);
            delete E;
            return rc;
        }
    }
    for (int i = 1; i < nmembers; i++)
        if (!phys32_shared(E->m[0]->phys32, E->m[i]->phys32)) {
            ens_error("tsu_ens_create: member %d differs from member 0 in a physical parameter other than the grid, "
                      "the still-water level, WBC and Read_files",
                      i);
            for (int j = 0; j < nmembers; j++) tsu_destroy(E->m[j]);
            delete E;
            return TSU_ERR_INVALID;
        }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) E->num_sms = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&E->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&E->e1);
    if (e == cudaSuccess) e = cudaMalloc((void **)&E->d_work, sizeof(unsigned));
    if (e != cudaSuccess) {
        for (int j = 0; j < nmembers; j++) tsu_destroy(E->m[j]);
        delete E;
        return TSU_ERR_CUDA;
    }
    int rc = build_tables(E, 0);
    if (rc) return rc;
    E->ctas = default_ctas(E, 0);
    *out = E;
    return TSU_OK;
}

extern "C" int tsu_ens_destroy(TsuEnsemble *E) {
    if (!E) return TSU_OK;
    cudaSetDevice(E->device);
    cudaStreamSynchronize(E->st);
    drop_graph(E);
    cudaFree(E->d_members);
    cudaFree(E->d_tile_member);
    cudaFree(E->d_tmas);
    cudaFree(E->d_work);
    if (E->e0) cudaEventDestroy(E->e0);
    if (E->e1) cudaEventDestroy(E->e1);
    if (E->st) cudaStreamDestroy(E->st);
    for (TsuSolver *s : E->m) tsu_destroy(s);
    delete E;
    return TSU_OK;
}

extern "C" int tsu_ens_member(TsuEnsemble *E, int i, TsuSolver **solver) {
    if (!E || i < 0 || i >= E->n || !solver) return TSU_ERR_INVALID;
    cudaSetDevice(E->device);
    cudaStreamSynchronize(E->st);
    *solver = E->m[i];
    return TSU_OK;
}

extern "C" int tsu_ens_reset(TsuEnsemble *E) {
    if (!E) return TSU_ERR_INVALID;
    ECK(cudaSetDevice(E->device));
    ECK(cudaStreamSynchronize(E->st));
    for (TsuSolver *s : E->m) {
        int rc = tsu_reset(s);
        if (rc) return rc;
        ECK(cudaStreamSynchronize(s->st));
    }
    return refresh_members(E);
}

extern "C" int tsu_ens_set_config(TsuEnsemble *E, int variant, int dynamic, int ctas) {
    if (!E || variant < 0 || variant >= stage32_num_tiles()) return TSU_ERR_INVALID;
    ECK(cudaSetDevice(E->device));
    ECK(cudaStreamSynchronize(E->st));
    if (variant != E->variant) {
        int rc = build_tables(E, variant);
        if (rc) return rc;
    }
    E->dynamic = dynamic ? 1 : 0;
    E->ctas = ctas > 0 ? std::min<int>(ctas, (int)E->ntiles) : default_ctas(E, variant);
    drop_graph(E);
    return TSU_OK;
}

extern "C" int tsu_ens_get_config(TsuEnsemble *E, int *variant, int *tx, int *ty, int *dynamic, int *ctas,
                                  long *ntiles) {
    if (!E) return TSU_ERR_INVALID;
    int a, b, c;
    stage32_tile_shape(E->variant, &a, &b, &c);
    if (variant) *variant = E->variant;
    if (tx) *tx = a;
    if (ty) *ty = b;
    if (dynamic) *dynamic = E->dynamic;
    if (ctas) *ctas = E->ctas;
    if (ntiles) *ntiles = (long)E->ntiles;
    return TSU_OK;
}

extern "C" int tsu_ens_step(TsuEnsemble *E, long nsteps) {
    if (!E || nsteps < 0) return TSU_ERR_INVALID;
    for (TsuSolver *s : E->m)
        if (!s->ready) return TSU_ERR_INVALID;  // tsu_ens_reset first
    ECK(cudaSetDevice(E->device));
    int rc0 = refresh_members(E);
    if (rc0) return rc0;
    const long K = TsuSolver::kGraphSteps;
    long n = nsteps;
    if (n >= K && !E->graph_exec) {  // host-side setup, once: before the timed region
        ECK(cudaStreamBeginCapture(E->st, cudaStreamCaptureModeThreadLocal));
        int rc = launch_steps(E, K);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(E->st, &g);
        if (rc) return rc;
        ECK(e);
        E->graph = g;
        ECK(cudaGraphInstantiate(&E->graph_exec, g, 0));
    }
    ECK(cudaEventRecord(E->e0, E->st));
    while (n >= K && E->graph_exec) {
        ECK(cudaGraphLaunch(E->graph_exec, E->st));
        n -= K;
    }
    int rc = launch_steps(E, n);
    if (rc) return rc;
    ECK(cudaEventRecord(E->e1, E->st));
    E->last_launches = nsteps * E->m[0]->sw.order * (E->dynamic ? 2 : 1);
    E->timed = true;
    return TSU_OK;
}

extern "C" int tsu_ens_sync(TsuEnsemble *E) {
    if (!E) return TSU_ERR_INVALID;
    ECK(cudaSetDevice(E->device));
    ECK(cudaStreamSynchronize(E->st));
    // every member's status words (an expired wait, a non-finite state)
    int rc = TSU_OK;
    for (TsuSolver *s : E->m) {
        double sc[SC_N];
        ECK(cudaMemcpy(sc, s->scal, sizeof(sc), cudaMemcpyDeviceToHost));
        const int r = tsu_device_flags(s, sc);
        if (r && !rc) rc = r;
    }
    return rc;
}

extern "C" int tsu_ens_last_step_ms(TsuEnsemble *E, double *ms) {
    if (!E || !ms || !E->timed) return TSU_ERR_INVALID;
    ECK(cudaEventSynchronize(E->e1));
    float f = 0.f;
    ECK(cudaEventElapsedTime(&f, E->e0, E->e1));
    *ms = f;
    return TSU_OK;
}

extern "C" int tsu_ens_last_step_launches(TsuEnsemble *E, long *launches) {
    if (!E || !launches) return TSU_ERR_INVALID;
    *launches = E->last_launches;
    return TSU_OK;
}

// Snapshot / restore of every member's device state used by the autotuner.
namespace {
struct Snapshot {
    std::vector<void *> bufs;
};
int snapshot(TsuEnsemble *E, Snapshot &S, bool save) {
    for (int i = 0; i < E->n; i++) {
        TsuSolver *s = E->m[i];
        const size_t pl = (size_t)s->plane * s->elem();
        void *src[5] = {s->A, s->hmax, s->bmin, s->eta, s->scal};
        const size_t sz[5] = {5 * pl, pl, pl, pl, SC_N * sizeof(double)};
        for (int f = 0; f < 5; f++) {
            const size_t k = (size_t)i * 5 + f;
            if (save) {
                void *p = nullptr;
                ECK(cudaMalloc(&p, sz[f]));
                S.bufs.push_back(p);
                ECK(cudaMemcpyAsync(p, src[f], sz[f], cudaMemcpyDeviceToDevice, E->st));
            } else {
                ECK(cudaMemcpyAsync(src[f], S.bufs[k], sz[f], cudaMemcpyDeviceToDevice, E->st));
            }
        }
    }
    ECK(cudaStreamSynchronize(E->st));
    return TSU_OK;
}
}  // namespace

// Times every (tile shape, schedule, resident CTAs) candidate over `steps`
// steps after one warm-up step, keeps the fastest and restores the members'
// state.  Writes a one-line-per-candidate report when `report` is given.
extern "C" int tsu_ens_autotune(TsuEnsemble *E, int steps, char *report, size_t cap) {
    if (!E || steps < 1) return TSU_ERR_INVALID;
    ECK(cudaSetDevice(E->device));
    for (TsuSolver *s : E->m)
        if (!s->ready) return TSU_ERR_INVALID;  // tsu_ens_reset first
    int rc = refresh_members(E);
    if (rc) return rc;
    ECK(cudaStreamSynchronize(E->st));
    Snapshot S;
    rc = snapshot(E, S, true);
    if (rc) return rc;
    std::string rep;
    double best = 1e30;
    int bv = 0, bd = 0, bc = 0;
    for (int v = 0; v < stage32_num_tiles(); v++) {
        for (int dyn = 0; dyn < 2; dyn++) {
            int per = ens32_max_ctas_per_sm(v);
            for (int mult = per; mult >= 1; mult = (mult > 1 ? mult / 2 : 0)) {
                rc = tsu_ens_set_config(E, v, dyn, mult * E->num_sms);
                if (rc) return rc;
                rc = launch_steps(E, 1);
                if (rc) return rc;
                ECK(cudaEventRecord(E->e0, E->st));
                rc = launch_steps(E, steps);
                if (rc) return rc;
                ECK(cudaEventRecord(E->e1, E->st));
                ECK(cudaEventSynchronize(E->e1));
                float ms = 0.f;
                ECK(cudaEventElapsedTime(&ms, E->e0, E->e1));
                int tx, ty, mb;
                stage32_tile_shape(v, &tx, &ty, &mb);
                char line[160];
                snprintf(line, sizeof(line), "tile %dx%d %s ctas %d: %.3f ms/step\n", tx, ty, dyn ? "dynamic" : "static",
                         E->ctas, ms / steps);
                rep += line;
                if (ms < best) {
                    best = ms;
                    bv = v;
                    bd = dyn;
                    bc = E->ctas;
                }
                rc = snapshot(E, S, false);
                if (rc) return rc;
                if (mult == 1) break;
            }
        }
        // one CTA per tile (no persistence)
        rc = tsu_ens_set_config(E, v, 0, (int)E->ntiles);
        if (rc) return rc;
        rc = launch_steps(E, 1);
        if (rc) return rc;
        ECK(cudaEventRecord(E->e0, E->st));
        rc = launch_steps(E, steps);
        if (rc) return rc;
        ECK(cudaEventRecord(E->e1, E->st));
        ECK(cudaEventSynchronize(E->e1));
        float ms = 0.f;
        ECK(cudaEventElapsedTime(&ms, E->e0, E->e1));
        int tx, ty, mb;
        stage32_tile_shape(v, &tx, &ty, &mb);
        char line[160];
        snprintf(line, sizeof(line), "tile %dx%d one-CTA-per-tile ctas %d: %.3f ms/step\n", tx, ty, E->ctas, ms / steps);
        rep += line;
        if (ms < best) {
            best = ms;
            bv = v;
            bd = 0;
            bc = E->ctas;
        }
        rc = snapshot(E, S, false);
        if (rc) return rc;
    }
    for (void *p : S.bufs) cudaFree(p);
    rc = tsu_ens_set_config(E, bv, bd, bc);
    if (rc) return rc;
    if (report && cap) {
        std::strncpy(report, rep.c_str(), cap - 1);
        report[cap - 1] = 0;
    }
    return TSU_OK;
}

extern "C" int tsu_ens_run_until(TsuEnsemble *E, double t_end, long max_steps, long *steps_done) {
    if (!E || max_steps < 0) return TSU_ERR_INVALID;
    for (TsuSolver *s : E->m)
        if (!s->ready) return TSU_ERR_INVALID;  // tsu_ens_reset first
    ECK(cudaSetDevice(E->device));
    int rc = refresh_members(E);
    if (rc) return rc;
    int *d_done = nullptr, *h_done = nullptr;
    ECK(cudaMalloc((void **)&d_done, sizeof(int)));
    if (cudaMallocHost((void **)&h_done, sizeof(int)) != cudaSuccess) {
        cudaFree(d_done);
        return TSU_ERR_HOST_OOM;
    }
    set_tend_kernel<<<1, 256, 0, E->st>>>(E->d_members, E->n, t_end);
    cudaError_t e = cudaGetLastError();
    long done_steps = 0;
    while (e == cudaSuccess && !rc && done_steps < max_steps) {
        const long chunk = std::min<long>(64, max_steps - done_steps);
        rc = tsu_ens_step(E, chunk);
        if (rc) break;
        done_steps += chunk;
        all_done_kernel<<<1, 256, 0, E->st>>>(E->d_members, E->n, t_end, d_done);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(h_done, d_done, sizeof(int), cudaMemcpyDeviceToHost, E->st)) != cudaSuccess) break;
        if ((e = cudaStreamSynchronize(E->st)) != cudaSuccess) break;
        if (*h_done) break;
    }
    if (e == cudaSuccess && !rc) {
        set_tend_kernel<<<1, 256, 0, E->st>>>(E->d_members, E->n, HUGE_VAL);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->st);
    }
    cudaFree(d_done);
    cudaFreeHost(h_done);
    if (e != cudaSuccess) {
        ens_error("tsu_ens_run_until: %s", cudaGetErrorString(e));
        return TSU_ERR_CUDA;
    }
    if (rc) return rc;
    if (steps_done) *steps_done = done_steps;
    return tsu_ens_sync(E);  // the members' status words
}
