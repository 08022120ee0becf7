// stage32.h -- launch interface of the FP32 precision-form kernels (single
// grid and batched ensemble).
#pragma once
#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include "physics32.cuh"
#include "stage64.h"

namespace tsu {

// Everything one RK stage needs about one grid.
struct Stage32Args {
    float *bufA;  // planes z, H, qx, qy, hc (U^n at step entry / U^{n+1} at exit)
    float *bufB;  // U* / ping-pong partner
    const unsigned char *mask;
    const double *CC;
    const double *tCC;
    unsigned long timeCC;
    float *hmax, *bmin, *eta_max;
    double *scal;
    double *partials;  // 3 x number of tiles (dt, water, sediment)
    unsigned *ticket;
    long long pitch, plane;
    Phys32 phys;
};

// One ensemble member: its grid and its slice of the global tile list.
struct EnsMember {
    Stage32Args g;
    unsigned tile0;   // first entry in the global tile list
    unsigned ntiles;  // tiles of this member for the current tile shape
    int ntx;          // tiles per row
};

// TMA descriptors of a single grid's two FP32 state buffers as 3-D tensors
// [5][npy][npx] (boxes = the loaded tile); `on` = 0 means ordinary loads.
struct Tma32 {
    CUtensorMap a, b;
    CUtensorMap m;  // the uint8 mask [npy][pitch] (box origin x0 - 16: 16-byte aligned)
    int on;
};

struct EnsArgs {
    const EnsMember *members;
    const int *tile_member;  // global tile -> member
    unsigned ntiles;
    int dynamic;     // 0: static stride over the tile list, 1: work counter
    unsigned *work;  // work counter (dynamic schedule)
    // per member: TMA descriptors for the current tile shape, in device
    // memory (written before the launch), or null
    const Tma32 *tmas;
};

size_t stage32_smem_bytes();
cudaError_t stage32_prepare();
dim3 stage32_grid(int npx, int npy);
cudaError_t stage32_launch(int order, int stage, const Stage32Args &a, const Tma32 &tm, cudaStream_t st);
// TMA descriptors of two FP32 state buffers with the boxes of tile variant
// `variant` (-1: the single-grid variant); false if they cannot be made
bool stage32_tma_maps(int variant, const float *bufA, const float *bufB, const unsigned char *mask, long long pitch,
                      long long plane, int npx, int npy, Tma32 *out);
// tile-shape variants available to the ensemble kernel
int stage32_num_tiles();
void stage32_tile_shape(int variant, int *tx, int *ty, int *minb);
// common: physical parameters shared by all members (grid fields ignored)
cudaError_t ens32_launch(int variant, int order, int stage, const EnsArgs &e, const Phys32 &common, int ctas,
                         cudaStream_t st);
// true if two members may share one ensemble launch (equal non-grid fields)
bool phys32_shared(const Phys32 &a, const Phys32 &b);
int ens32_max_ctas_per_sm(int variant);
cudaError_t to32_launch(const double *V64, long long pitch, long long plane, int npx, int npy, double eta0, float *V32,
                        cudaStream_t st);
cudaError_t to64_launch(const float *V32, long long pitch, long long plane, int npx, int npy, double eta0, double *V64,
                        cudaStream_t st);
cudaError_t widen_launch(const float *a, double *b, long long n, cudaStream_t st);
cudaError_t fill32_launch(float *p, long long n, float v, cudaStream_t st);
cudaError_t initial_dt32_launch(const float *V, long long pitch, long long plane, const Phys32 &P, double *partials,
                                unsigned *ticket, double *scal, cudaStream_t st);

}  // namespace tsu
