// solver.h -- internal definition of the opaque TsuSolver handle.
#pragma once
#include <cuda_runtime.h>

#include "stage64.h"
#include "tsuner_b200.h"

struct TsuSolver {
    static constexpr long kGraphSteps = 16;  // steps per captured CUDA graph

    SimParams p{};
    TsuSwitches sw{};
    int device = 0;
    cudaStream_t st = nullptr;
    long long pitch = 0, plane = 0;  // elements
    double *A = nullptr, *B = nullptr;
    double *hmax = nullptr, *bmin = nullptr, *eta = nullptr;
    unsigned char *mask = nullptr;
    double *CC = nullptr, *tCC = nullptr;
    unsigned long timeCC = 0;
    double *scal = nullptr, *partials = nullptr;
    size_t npartials = 0;
    unsigned *ticket = nullptr;
    TsuConsts *dconsts = nullptr;
    TsuConsts hconsts{};
    tsu::Phys64 phys{};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long last_launches = 0;
    bool has_state = false, ready = false, timed = false;

    tsu::Stage64Args args() const;
    int launch_steps(long n);
    void invalidate_graph();
    double *current() const;
};

const char *tsu_last_error_detail();
