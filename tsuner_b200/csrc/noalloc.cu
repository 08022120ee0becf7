// noalloc.cu -- CFL time step of a caller-owned FP64 state without any
// device allocation by the library.
//
// Some callers cannot let a library call cudaMalloc: code that runs inside a
// host framework which owns all device memory through its own pool (an
// allocation behind its back can fail or fragment that pool), or embedded and
// long-running services that forbid allocation after start-up so that memory
// use stays fixed and no call can fail for lack of memory mid-run.
// For them tsu_cfl_dt_noalloc() computes the reference's CFL step
// (GetDeltaT + MinReduction, GPU/Volume_kernel.cu:19-43 and
// GPU/Reduction_kernel_min.cu:155-196) of a state they already hold on the
// device and writes it to a device double they provide.  The per-CTA partial
// minima and the arrival counter live in the file-scope array below: a fixed
// 16384 partials + 1 counter (about 128 KiB), held by every GPU that loads
// this library until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "physics64.cuh"
#include "solver.h"
#include "stage64.h"
#include "tsuner_b200.h"

namespace tsu {
namespace {

constexpr int kNoallocMaxCtas = 16384;   // capacity of the partial minima
constexpr int kNoallocBx = 32, kNoallocBy = 8;

// [0, kNoallocMaxCtas): partial minima; [kNoallocMaxCtas]: arrival counter
// (as the bits of a double slot, used through an unsigned pointer).
static __device__ __align__(256) double g_noalloc_scratch[kNoallocMaxCtas + 1];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void __launch_bounds__(kNoallocBx *kNoallocBy)
    cfl_dt_noalloc_kernel(const double *__restrict__ h, const double *__restrict__ qx, const double *__restrict__ qy,
                          long long pitch, Phys64 P, double *__restrict__ scratch, double *__restrict__ dt_out) {
    __shared__ double sRed[8];
    __shared__ int sLast;
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + kNoallocMaxCtas);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int gi = blockIdx.x * blockDim.x + threadIdx.x, gj = blockIdx.y * blockDim.y + threadIdx.y;
    double m = CUDART_INF;
    if (gi < P.npx && gj < P.npy) {
        const long long g = (long long)gj * pitch + gi;
        const double d = cfl_dt(P, h[g], qx[g], qy[g]);
        if (!isnan(d)) m = d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) sRed[tid >> 5] = m;
    __syncthreads();
    const unsigned nb = gridDim.x * gridDim.y;
    if (tid == 0) {
        for (int w = 1; w < 8; w++) m = fmin(m, sRed[w]);
        scratch[blockIdx.y * gridDim.x + blockIdx.x] = m;
        __threadfence();
        sLast = (atomicAdd(ticket, 1u) == nb - 1);
    }
    __syncthreads();
    if (sLast) {
        __threadfence();
        double mm = CUDART_INF;
        for (unsigned i = tid; i < nb; i += kNoallocBx * kNoallocBy) mm = fmin(mm, __ldcg(scratch + i));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mm = fmin(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        __syncthreads();
        if ((tid & 31) == 0) sRed[tid >> 5] = mm;
        __syncthreads();
        if (tid == 0) {
            for (int w = 0; w < 8; w++) mm = fmin(mm, sRed[w]);
            *dt_out = finalize_dt(mm, (long long)P.npx * P.npy);
            *ticket = 0u;
        }
    }
}

}  // namespace
}  // namespace tsu

using namespace tsu;

extern "C" int tsu_cfl_dt_noalloc(const double *d_h, const double *d_qx, const double *d_qy, long pitch_elems,
                                  const SimParams *p, double *d_dt, void *stream) {
    if (!d_h || !d_qx || !d_qy || !p || !d_dt || p->npx < 1 || p->npy < 1 || pitch_elems < p->npx ||
        !(p->dx > 0) || !(p->dy > 0))
        return TSU_ERR_INVALID;
    const long long ctas = (long long)((p->npx + kNoallocBx - 1) / kNoallocBx) * ((p->npy + kNoallocBy - 1) / kNoallocBy);
    if (ctas > kNoallocMaxCtas) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "tsu_cfl_dt_noalloc: a %d x %d grid needs %lld partial minima; the fixed scratch holds %d "
                      "(at most %d cells); use tsu_create/tsu_reset for larger grids",
                      p->npx, p->npy, ctas, kNoallocMaxCtas, kNoallocMaxCtas * kNoallocBx * kNoallocBy);
        tsu_set_error_detail(msg);
        std::fprintf(stderr, "%s\n", msg);
        return TSU_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TSU_ERR_NO_DEVICE;
    double *scratch = nullptr;
    {
        // set-up once per device, with that device current: the host-side name
        // of the array is not a device address, so look the address up
        std::lock_guard<std::mutex> g(g_setup_mu);
        if (!g_scratch_ptr[dev]) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                char msg[256];
                std::snprintf(msg, sizeof(msg), "tsu_cfl_dt_noalloc: cudaGetSymbolAddress failed: %s",
                              cudaGetErrorString(e));
                tsu_set_error_detail(msg);
                std::fprintf(stderr, "%s\n", msg);
                return TSU_ERR_CUDA;
            }
            g_scratch_ptr[dev] = static_cast<double *>(ptr);
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the arrival counter must start at zero; the partials need no clearing
    if (cudaMemsetAsync(scratch + kNoallocMaxCtas, 0, sizeof(double), st) != cudaSuccess) return TSU_ERR_CUDA;
    Phys64 P{};
    P.CFL = p->CFL;
    P.dx = p->dx;
    P.dy = p->dy;
    P.npx = p->npx;
    P.npy = p->npy;
    dim3 b(kNoallocBx, kNoallocBy), g((p->npx + kNoallocBx - 1) / kNoallocBx, (p->npy + kNoallocBy - 1) / kNoallocBy);
    cfl_dt_noalloc_kernel<<<g, b, 0, st>>>(d_h, d_qx, d_qy, (long long)pitch_elems, P, scratch, d_dt);
    return cudaGetLastError() == cudaSuccess ? TSU_OK : TSU_ERR_CUDA;
}
