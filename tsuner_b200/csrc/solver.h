// solver.h -- internal definition of the opaque TsuSolver handle.
#pragma once
#include <cuda_runtime.h>

#include "stage32.h"
#include "stage64.h"
#include "tsuner_b200.h"

struct TsuSolver {
    static constexpr long kGraphSteps = 16;  // steps per captured CUDA graph

    SimParams p{};
    TsuSwitches sw{};
    int device = 0;
    bool fp32 = false;
    cudaStream_t st = nullptr;     // the stream all work is issued on
    cudaStream_t own_st = nullptr;  // the solver's own stream (st unless tsu_set_stream chose another)
    long long pitch = 0, plane = 0;  // elements; a plane holds the stored rows
    // Row slab of a decomposed grid (tsu_slab_create): p describes the owned
    // rows only (p.npy of them, global rows j0 .. j0 + p.npy - 1 of a grid of
    // ny_glob rows); gs / gn ghost rows are stored below / above them.  A
    // whole grid has slab = false, j0 = gs = gn = 0, ny_glob = p.npy.
    bool slab = false;
    int j0 = 0, gs = 0, gn = 0, ny_glob = 0;
    long long own_off() const { return (long long)gs * pitch; }  // elements to owned row 0
    // FP64 plain form: planes h, qx, qy, H, hc.  FP32 form: z, H, qx, qy, hc.
    void *A = nullptr, *B = nullptr;
    void *K = nullptr;  // MUSCL-Hancock (rk == 0) only: the unfiltered working state Vk
    void *hmax = nullptr, *bmin = nullptr, *eta = nullptr;
    double *stage64 = nullptr;  // FP32 form: FP64 staging planes for upload/download
    unsigned char *mask = nullptr;
    double *CC = nullptr, *tCC = nullptr;
    size_t CC_cap = 0, tCC_cap = 0;  // allocated elements (kept across series)
    unsigned long timeCC = 0;
    double *scal = nullptr, *partials = nullptr;
    size_t npartials = 0;
    unsigned *ticket = nullptr;
    TsuConsts *dconsts = nullptr;
    TsuConsts hconsts{};
    tsu::Phys64 phys{};
    tsu::Phys32 phys32{};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long last_launches = 0;
    bool has_state = false, ready = false, timed = false;
    int fault = 0;  // status a kernel reported (TSU_ERR_CUDA / TSU_ERR_NONFINITE) until the next tsu_reset
    // TMA descriptors of A and B (interior tiles stage their loads by TMA)
    CUtensorMap tmA{}, tmB{};
    CUtensorMap tmM{};  // the mask (uint8 [npy][pitch])
    CUtensorMap tmO{};  // FP64: the owned-cell boxes of A and of the extrema
    CUtensorMap tmE[3]{};
    bool tma = false;

    tsu::Stage64Args args() const;
    tsu::Stage32Args args32() const;
    int launch_steps(long n);
    void invalidate_graph();
    void *current() const;
    size_t elem() const { return fp32 ? sizeof(float) : sizeof(double); }
    // one kernel per step whose state alternates between A and B (order 1, MUSCL-Hancock)
    bool single_stage() const { return sw.order == 1 || sw.rk == 0; }
    int stages() const { return single_stage() ? 1 : sw.order; }
};

// status of the scalar block sc (a host copy of s->scal): TSU_OK, TSU_ERR_CUDA
// (an expired device wait) or TSU_ERR_NONFINITE (a NaN / Inf state cell);
// on an error the solver needs a tsu_reset before it steps again
int tsu_device_flags(TsuSolver *s, const double *sc);
const char *tsu_last_error_detail();
// sets the detail text that tsu_last_error() returns on this thread
void tsu_set_error_detail(const char *text);
