// stage32.h -- launch interface of the FP32 precision-form kernels.
#pragma once
#include <cuda_runtime.h>

#include "physics32.cuh"
#include "stage64.h"

namespace tsu {

struct Stage32Args {
    float *bufA;  // planes z, H, qx, qy, hc (U^n at step entry / U^{n+1} at exit)
    float *bufB;  // U* / ping-pong partner
    const unsigned char *mask;
    const double *CC;
    const double *tCC;
    unsigned long timeCC;
    float *hmax, *bmin, *eta_max;
    double *scal;
    double *partials;  // 3 x number of CTAs (dt, water, sediment)
    unsigned *ticket;
    long long pitch, plane;
    Phys32 phys;
};

size_t stage32_smem_bytes();
cudaError_t stage32_prepare();
dim3 stage32_grid(int npx, int npy);
cudaError_t stage32_launch(int order, int stage, const Stage32Args &a, cudaStream_t st);
cudaError_t to32_launch(const double *V64, long long pitch, long long plane, int npx, int npy, double eta0, float *V32,
                        cudaStream_t st);
cudaError_t to64_launch(const float *V32, long long pitch, long long plane, int npx, int npy, double eta0, double *V64,
                        cudaStream_t st);
cudaError_t widen_launch(const float *a, double *b, long long n, cudaStream_t st);
cudaError_t fill32_launch(float *p, long long n, float v, cudaStream_t st);
cudaError_t initial_dt32_launch(const float *V, long long pitch, long long plane, const Phys32 &P, double *partials,
                                unsigned *ticket, double *scal, cudaStream_t st);

}  // namespace tsu
