// stage64.h -- launch interface of the FP64 fused stage kernels.
#pragma once
#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>
#include <math_constants.h>

#include "physics64.cuh"

#ifndef S64_TX
#define S64_TX 32
#endif
#ifndef S64_TY
#define S64_TY 8
#endif

namespace tsu {

// Device scalars (double slots of Stage64Args::scal):
//   [0] simulated time t      [1] dt of the next step
//   [2] t_end of run_until (steps execute only while t < t_end)
//   [3] steps taken           [4] order-1 ping-pong parity
//   [5] FP32 form: sum of water depth after the last step (FP64)
//   [6] FP32 form: sum of H + hc after the last step (FP64)
//   [7] non-zero when a bounded device wait expired (reported by the host)
//   [8] non-zero when a cell of the state became NaN or infinite (set by the
//       last stage of a step and by the initial-dt kernel; reported by the host)
enum {
    SC_T = 0,
    SC_DT = 1,
    SC_TEND = 2,
    SC_STEPS = 3,
    SC_PAR = 4,
    SC_MASS = 5,
    SC_SED = 6,
    SC_ERR = 7,
    SC_NAN = 8,
    SC_N = 9
};

struct Stage64Args {
    // TMA descriptors of the two state buffers as 3-D tensors [5][npy][npx]
    // (boxes = the loaded tile with its halo); used for tiles whose halo lies
    // inside the grid when `tma` is set
    CUtensorMap tmA, tmB;
    CUtensorMap tmM;  // the uint8 mask [npy][pitch] (box origin x0 - 16)
    // boxes of the owned cells (TX x TY): U^n in bufA [5][npy][npx] and the
    // running extrema hmax, bmin, eta_max [npy][npx]
    CUtensorMap tmO;
    CUtensorMap tmE[3];
    int tma;
    double *bufA;           // U^n at step entry (and U^{n+1} at exit, order 2)
    double *bufB;           // U* (order 2) / ping-pong partner (order 1, MUSCL-Hancock)
    double *bufK;           // MUSCL-Hancock: the unfiltered working state carried between steps
    const unsigned char *mask;
    const double *CC;
    const double *tCC;
    unsigned long timeCC;
    double *hmax, *bmin, *eta_max;
    double *scal;
    double *partials;
    unsigned *ticket;
    long long pitch, plane;  // elements
    Phys64 phys;
};

// dt finalisation of MinReduction<double> (GPU/Reduction_kernel_min.cu:
// 155-196): above 4096 cells every device compare is fminf on doubles, so
// the minimum is rounded to float; the host loop starts from 1e30.
__device__ __forceinline__ double finalize_dt(double m, long long ncells) {
    if (ncells > 4096) m = (double)__double2float_rn(m);
    if (!(m < 1e30)) m = 1e30;
    return m;
}

size_t stage64_smem_bytes();
cudaError_t stage64_prepare();
dim3 stage64_grid(int npx, int npy);
cudaError_t stage64_launch(int order, int stage, const Stage64Args &a, cudaStream_t st);
cudaError_t initial_dt_launch(const double *V, long long pitch, long long plane, const Phys64 &P, double *partials,
                              unsigned *ticket, double *scal, cudaStream_t st);
cudaError_t fill_launch(double *p, long long n, double v, cudaStream_t st);
cudaError_t consts_launch(const SimParams &p, TsuConsts *k, cudaStream_t st);
size_t partials_needed(int npx, int npy);
// Limit of the ordinary bounded device waits of each kernel unit (the stage
// kernels of stage64.cu / stage32.cu, the convolutions of corrector.cu), on
// the current device; the error-path drain waits always keep the full limit.
cudaError_t set_wait_limit_stage64(unsigned long long ns);
cudaError_t set_wait_limit_stage32(unsigned long long ns);
cudaError_t set_wait_limit_corrector(unsigned long long ns);
constexpr unsigned long long kDefaultWaitNs = 500000000ull;  // async.cuh kWaitNs
// encodes the TMA descriptors of the two FP64 state buffers for the current
// tile shape; false if the driver cannot (the kernels then load with
// ordinary instructions)
// (tmO, tmE[3]: the owned-cell boxes of bufA and of the extrema hmax, bmin,
// eta_max)
bool stage64_tma_maps(const double *bufA, const double *bufB, const unsigned char *mask, const double *const ext[3],
                      long long pitch, long long plane, int npx, int npy, CUtensorMap *tmA, CUtensorMap *tmB,
                      CUtensorMap *tmM, CUtensorMap *tmO, CUtensorMap tmE[3]);

}  // namespace tsu
