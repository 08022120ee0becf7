/*
 * ref_harness.cu -- drives the REFERENCE TSUNER CUDA kernels, unmodified, for
 * an exact number of time steps on caller-supplied inputs.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference's own GPU sources (GPU/Reconstructor.cu, GPU/VolumeSolver.cu,
 * GPU/Volume_kernel.cu, GPU/Reduction_kernel_min.cu, built with the reference
 * flags -O2 -fmad=false -rdc=true -dlto) into oracle/_ref/<variant>/
 * libtsuner_ref.so.  It is the parity checker for the product and the
 * reference arm of bench.py; it is never linked into the product.
 *
 * The reference has no step-count mode (its loop runs `while t < T`,
 * GPU/main_TSUNER.cu:157), so this harness restates the loop body of
 * GPU/main_TSUNER.cu:142-197 with a step counter:
 *   init extrema (:142-144) -> GetDeltaT + MinReduction (:147-148) ->
 *   repeat { for k < order: reconstructor, VolumeSolver, states_updater
 *   (:169-183); t += dt (:185); hmax/bmin/eta_max (:187-189);
 *   GetDeltaT + MinReduction (:190-192) }.
 * Buffers are allocated as in GPU/main_TSUNER.cu:57-91 (minus the unused
 * dynamic-rupture arrays) and the SoA packing follows :104-115.
 */
#include "GPU_kernels.cuh"
#include <vector>

extern "C" {

/* Number of CUDA devices this build can see (0 on error), so that callers can
 * probe for a GPU without loading any other library. */
int ref_device_count(int *n)
{
    int k = 0;
    if (cudaGetDeviceCount(&k) != cudaSuccess) {
        cudaGetLastError();
        k = 0;
    }
    *n = k;
    return 0;
}

/* Compile-time switches of this build (Sim_parameters.hxx values). */
int ref_switches(int *out6)
{
    out6[0] = order;
    out6[1] = RK;
    out6[2] = WBC;
    out6[3] = BEDLOAD;
    out6[4] = SUSPENSION;
    out6[5] = Read_files;
    return 0;
}

/*
 * Runs `nsteps` steps (nsteps < 0: run while t < params.total_time, as the
 * reference loop does).  V is 5*nvol doubles SoA (h, qx, qy, H, hc), in/out.
 * hmax/bmin/eta_max receive the running extrema (bmin as the raw running max
 * of H, i.e. before the sign flip of GPU/main_TSUNER.cu:208).
 * t_out/dt_out: simulated time after the run and the dt of the next step.
 * ms_out: device time of the step loop in milliseconds (CUDA events).
 * Returns 0 on success, 1 on device allocation failure, 3 on CUDA error,
 * 4 when the boundary series is missing or not uniform (Read_files == 1).
 */
int ref_run(SimParams params, double *V, const int *fixH, const double *CC,
            const double *tCC, unsigned long timeCC, long nsteps,
            double *hmax, double *bmin, double *eta_max, double *t_out,
            double *dt_out, long *steps_out, double *ms_out, int device)
{
    cudaSetDevice(device);
    const int nvol = params.nvol;
    const size_t plane = (size_t)nvol * sizeof(double);
    double *d_V = 0, *d_V0 = 0, *d_Vk = 0, *d_hmax = 0, *d_bmin = 0, *d_eta = 0;
    double *rL = 0, *rR = 0, *rU = 0, *rD = 0, *FL = 0, *FR = 0, *FU = 0, *FD = 0;
    double *d_dt = 0, *d_CC = 0, *d_tCC = 0, *d_d = 0, *d_dyrup = 0;
    float *d_tdyrup = 0;
    int *d_fixH = 0;
    int err = 0;
    err += cudaMalloc((void **)&d_hmax, plane);
    err += cudaMalloc((void **)&d_bmin, plane);
    err += cudaMalloc((void **)&d_eta, plane);
    err += cudaMalloc((void **)&d_V, 5 * plane);
    err += cudaMalloc((void **)&d_V0, 5 * plane);
    err += cudaMalloc((void **)&d_Vk, 5 * plane);
    err += cudaMalloc((void **)&d_fixH, (size_t)nvol * sizeof(int));
    err += cudaMalloc((void **)&d_dt, plane);
    err += cudaMalloc((void **)&rL, 5 * plane);
    err += cudaMalloc((void **)&rR, 5 * plane);
    err += cudaMalloc((void **)&rU, 5 * plane);
    err += cudaMalloc((void **)&rD, 5 * plane);
    err += cudaMalloc((void **)&FL, 5 * plane);
    err += cudaMalloc((void **)&FR, 5 * plane);
    err += cudaMalloc((void **)&FU, 5 * plane);
    err += cudaMalloc((void **)&FD, 5 * plane);
    size_t ccn = (size_t)(2 * params.npx + 2 * params.npy) * 4 * (timeCC ? timeCC : 1);
    err += cudaMalloc((void **)&d_CC, ccn * sizeof(double));
    err += cudaMalloc((void **)&d_tCC, (timeCC ? timeCC : 1) * sizeof(double));
    err += cudaMalloc((void **)&d_d, 8);
    err += cudaMalloc((void **)&d_dyrup, 8);
    err += cudaMalloc((void **)&d_tdyrup, 8);
    int rc = 0;
    if (err) { rc = 1; goto done; }
#if Read_files == 1
    /* GPU/VolumeSolver.cu:249 reads d_tCC[timeCC - 2] on every boundary edge
     * and GPU/VolumeSolver.cu:172-215 assumes a uniform series: refuse
     * inputs that would make those reads leave the arrays. */
    if (timeCC < 2) { rc = 4; goto done; }
    for (unsigned long q = 1; q < timeCC; q++) {
        double dtc = tCC[1] - tCC[0];
        if (!(dtc > 0.0) || fabs((tCC[q] - tCC[0]) - q * dtc) > 1e-9 * fabs(dtc) * q) { rc = 4; goto done; }
    }
#endif
    {
        cudaMemcpy(d_V, V, 5 * plane, cudaMemcpyHostToDevice);
        cudaMemcpy(d_Vk, d_V, 5 * plane, cudaMemcpyDeviceToDevice);
        cudaMemcpy(d_V0, d_V, 5 * plane, cudaMemcpyDeviceToDevice);
        cudaMemcpy(d_fixH, fixH, (size_t)nvol * sizeof(int), cudaMemcpyHostToDevice);
        if (timeCC) {
            cudaMemcpy(d_CC, CC, ccn * sizeof(double), cudaMemcpyHostToDevice);
            cudaMemcpy(d_tCC, tCC, timeCC * sizeof(double), cudaMemcpyHostToDevice);
        }
        dim3 gE(iDivUp(params.npx, NUM_THREADS_HORIZONTAL_VOL), iDivUp(params.npy, NUM_THREADS_VERTICAL_VOL));
        dim3 gR(iDivUp(params.npx + 1, NUM_THREADS_HORIZONTAL_VOL), iDivUp(params.npy + 1, NUM_THREADS_VERTICAL_VOL));
        dim3 tB(NUM_THREADS_HORIZONTAL_VOL, NUM_THREADS_VERTICAL_VOL);
        double inv_dx = 1.0 / params.dx, inv_dy = 1.0 / params.dy;

        set_inicializacion<<<gE, tB>>>(d_hmax, params.npx, params.npy);
        set_inicializacion_bmin<<<gE, tB>>>(d_bmin, params.npx, params.npy);
        set_inicializacion_eta_max<<<gE, tB>>>(d_eta, params.npx, params.npy);
        GetDeltaT<<<gE, tB>>>(d_V, d_dt, params);
        double delta_T = MinReduction<double>(d_dt, nvol);
        double current_time = 0.0;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        long it = 0;
        while (nsteps >= 0 ? it < nsteps : current_time < params.total_time) {
#if RK == 1
            for (int k = 0; k < order; k++) {
#else
            int k = 0;
            {
#endif
                reconstructor<<<gE, tB>>>(d_V, rL, rR, rD, rU, delta_T, inv_dx, inv_dy, params, d_Vk, d_V0);
                VolumeSolver<<<gR, tB>>>(d_fixH, current_time, params, rL, rR, rD, rU, FL, FR, FU, FD, d_CC, d_tCC, timeCC, 0, 0, -1);
                states_updater<<<gE, tB>>>(d_Vk, d_V0, d_V, params.npx, params.npy, k, params.epsilon_h, delta_T * inv_dx, delta_T * inv_dy, FL, FR, FU, FD, d_d, current_time, d_CC, d_tCC, timeCC, d_dyrup, d_tdyrup);
            }
            current_time += delta_T;
            hmax_calculator<<<gE, tB>>>(d_hmax, d_V, params.epsilon_h, params.npx, params.npy);
            bmin_calculator<<<gE, tB>>>(d_bmin, d_V, params.npx, params.npy);
            eta_max_calculator<<<gE, tB>>>(d_eta, d_V, params.epsilon_h, params.npx, params.npy);
            GetDeltaT<<<gE, tB>>>(d_V, d_dt, params);
            delta_T = MinReduction<double>(d_dt, nvol);
            it++;
        }
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaMemcpy(V, d_V, 5 * plane, cudaMemcpyDeviceToHost);
        if (hmax) cudaMemcpy(hmax, d_hmax, plane, cudaMemcpyDeviceToHost);
        if (bmin) cudaMemcpy(bmin, d_bmin, plane, cudaMemcpyDeviceToHost);
        if (eta_max) cudaMemcpy(eta_max, d_eta, plane, cudaMemcpyDeviceToHost);
        if (t_out) *t_out = current_time;
        if (dt_out) *dt_out = delta_T;
        if (steps_out) *steps_out = it;
        if (ms_out) *ms_out = ms;
        if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = 3;
    }
done:
    cudaFree(d_hmax); cudaFree(d_bmin); cudaFree(d_eta);
    cudaFree(d_V); cudaFree(d_V0); cudaFree(d_Vk); cudaFree(d_fixH); cudaFree(d_dt);
    cudaFree(rL); cudaFree(rR); cudaFree(rU); cudaFree(rD);
    cudaFree(FL); cudaFree(FR); cudaFree(FU); cudaFree(FD);
    cudaFree(d_CC); cudaFree(d_tCC); cudaFree(d_d); cudaFree(d_dyrup); cudaFree(d_tdyrup);
    return rc;
}

/* Initial dt exactly as GPU/main_TSUNER.cu:147-148 (GetDeltaT + MinReduction). */
int ref_initial_dt(SimParams params, const double *V, double *dt_out, int device)
{
    cudaSetDevice(device);
    const size_t plane = (size_t)params.nvol * sizeof(double);
    double *d_V = 0, *d_dt = 0;
    if (cudaMalloc((void **)&d_V, 5 * plane) != cudaSuccess) return 1;
    if (cudaMalloc((void **)&d_dt, plane) != cudaSuccess) { cudaFree(d_V); return 1; }
    cudaMemcpy(d_V, V, 5 * plane, cudaMemcpyHostToDevice);
    dim3 gE(iDivUp(params.npx, NUM_THREADS_HORIZONTAL_VOL), iDivUp(params.npy, NUM_THREADS_VERTICAL_VOL));
    dim3 tB(NUM_THREADS_HORIZONTAL_VOL, NUM_THREADS_VERTICAL_VOL);
    GetDeltaT<<<gE, tB>>>(d_V, d_dt, params);
    *dt_out = MinReduction<double>(d_dt, params.nvol);
    int rc = (cudaDeviceSynchronize() == cudaSuccess) ? 0 : 3;
    cudaFree(d_V);
    cudaFree(d_dt);
    return rc;
}

} /* extern "C" */
