// stage64.cu -- FP64 plain form: one fused kernel per RK stage.
//
// Replaces the reference chain reconstructor (GPU/Reconstructor.cu:90) ->
// VolumeSolver (GPU/VolumeSolver.cu:217) -> states_updater
// (GPU/Volume_kernel.cu:180) and, on the last stage of a step, also
// hmax/bmin/eta_max_calculator (GPU/Volume_kernel.cu:79-110), GetDeltaT
// (:19-43) and MinReduction (GPU/Reduction_kernel_min.cu:155-196).
//
// A CTA owns a TX x TY tile of cells.  Phases, separated by __syncthreads():
//   1. stage state (5 planes) + mask of the tile and a 2-cell halo -> smem
//      (halo indices clamped -- which reproduces the reference's im/ip/jm/jp
//      clamping -- or wrapped for periodic boundaries);
//   2. per-cell velocity and concentration, once per cell;
//   3. MUSCL faces (x: L/R, y: D/U) of the tile plus one halo cell per side,
//      positivity-filtered, and the hydrostatic slopes for the source term;
//   4. every edge of the tile evaluated once (boundary ghosts / CC series /
//      periodic seam as in GPU/VolumeSolver.cu:217-408) -> fluctuations;
//   5. per cell: pressure source, friction, erosion/deposition, flux
//      divergence, RK combine, positivity filter, store; on the last stage
//      also the running extrema and the CFL dt partial, with the global
//      minimum finished by the last CTA to arrive (no host round trip).
// Face states and fluxes never touch global memory: per cell-step the
// kernel moves the 250 algorithmic bytes instead of the reference's ~2 KB.
#include <cuda_runtime.h>

#include "physics64.cuh"
#include "stage64.h"

namespace tsu {

namespace {

constexpr int TX = S64_TX, TY = S64_TY, NT = TX * TY;
constexpr int LX = TX + 4, LY = TY + 4;  // loaded tile with a 2-cell halo
constexpr int FXW = TX + 2;              // x faces: tile columns -1..TX
constexpr int FYH = TY + 2;              // y faces: tile rows -1..TY

// shared-memory carve-up (doubles); region A (state + per-cell velocity) is
// dead once the faces exist and is reused for the fluxes.
constexpr int kSV = 5 * LY * LX;
constexpr int kSUC = 3 * LY * LX;
constexpr int kFlux = 4 * 5 * TY * TX;
constexpr int kRegA = (kSV + kSUC) > kFlux ? (kSV + kSUC) : kFlux;
constexpr int kFx = 2 * 5 * TY * FXW;
constexpr int kFy = 2 * 5 * FYH * TX;
constexpr int kDeta = 2 * TY * TX;
constexpr int kDoubles = kRegA + kFx + kFy + kDeta;
constexpr int kRed = NT / 32;
}  // namespace

size_t stage64_smem_bytes() { return sizeof(double) * (kDoubles + kRed) + LY * LX + 16; }

__device__ __forceinline__ int wrap_clamp(int g, int n, bool periodic) {
    if (periodic) {
        g %= n;
        return g < 0 ? g + n : g;
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

// MUSCL reconstruction of one cell along one direction, GPU/Reconstructor.cu
// :124-194 (x) / :207-271 (y).  c/l/r index the centre and its two
// neighbours in the smem tile.  Returns the two filtered faces (minus side,
// plus side) and the hydrostatic slope deta.
__device__ __forceinline__ void reconstruct_dir(const double *sV, const double *sUC, int c, int l, int r,
                                                bool xdir, State5 &fm, State5 &fp, double &deta) {
    constexpr int PS = LY * LX;
    const double hi = sV[c], Hi = sV[3 * PS + c];
    const double hl = sV[l], Hl = sV[3 * PS + l];
    const double hr = sV[r], Hr = sV[3 * PS + r];
    const double ci = sUC[2 * PS + c], cl = sUC[2 * PS + l], cr = sUC[2 * PS + r];
    const double uix = sUC[c], uiy = sUC[PS + c];
    const double ulx = sUC[l], uly = sUC[PS + l];
    const double urx = sUC[r], ury = sUC[PS + r];

    double dl = hi - hl, dr = hr - hi;
    double dh = limiter(dl, dr);
    if (0.5 * fabs(dh) > hi) dh = 2.0 * hi * sgn(dh);
    fm.h = hi - 0.5 * dh;
    fp.h = hi + 0.5 * dh;

    double zm = fmin(Hl, Hi);
    dl = fmax(hi - Hi + zm, 0.0) - fmax(hl - Hl + zm, 0.0);
    zm = fmin(Hr, Hi);
    dr = fmax(hr - Hr + zm, 0.0) - fmax(hi - Hi + zm, 0.0);
    deta = limiter(dl, dr);
    double dz = dh - deta;
    fm.H = Hi - 0.5 * dz;
    fp.H = Hi + 0.5 * dz;

    const double qxi = sV[PS + c], qyi = sV[2 * PS + c];
    dl = uix - ulx;
    dr = urx - uix;
    double du = limiter(dl, dr);
    double dq = hi * du + uix * dh;
    fm.qx = qxi - 0.5 * dq;
    fp.qx = qxi + 0.5 * dq;
    dl = uiy - uly;
    dr = ury - uiy;
    du = limiter(dl, dr);
    dq = hi * du + uiy * dh;
    fm.qy = qyi - 0.5 * dq;
    fp.qy = qyi + 0.5 * dq;

    dl = ci - cl;
    dr = cr - ci;
    du = limiter(dl, dr);
    fm.hc = (ci - 0.5 * du) * fm.h;
    fp.hc = (ci + 0.5 * du) * fp.h;

    positivity_filter(fm.h, fm.qx, fm.qy, fm.hc);
    positivity_filter(fp.h, fp.qx, fp.qy, fp.hc);
    (void)xdir;
}

__device__ __forceinline__ void put5(double *base, int stride, const State5 &s) {
    base[0] = s.h;
    base[stride] = s.qx;
    base[2 * stride] = s.qy;
    base[3 * stride] = s.H;
    base[4 * stride] = s.hc;
}
__device__ __forceinline__ State5 get5(const double *base, int stride) {
    State5 s;
    s.h = base[0];
    s.qx = base[stride];
    s.qy = base[2 * stride];
    s.H = base[3 * stride];
    s.hc = base[4 * stride];
    return s;
}
__device__ __forceinline__ void put5a(double *base, int stride, const double D[5]) {
#pragma unroll
    for (int f = 0; f < 5; f++) base[f * stride] = D[f];
}

template <int ORDER, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT, 2) stage64_kernel(Stage64Args A) {
    extern __shared__ __align__(16) double smem[];
    const Phys64 &P = A.phys;
    double *sV = smem;                       // [5][LY][LX]
    double *sUC = smem + kSV;                // [3][LY][LX]  (ux, uy, c)
    double *sFlux = smem;                    // [4][5][TY][TX] aliases sV/sUC
    double *sFx = smem + kRegA;              // [2][5][TY][FXW]
    double *sFy = sFx + kFx;                 // [2][5][FYH][TX]
    double *sDeta = sFy + kFy;               // [2][TY][TX]
    double *sRed = sDeta + kDeta;            // [NT/32]
    unsigned char *sM = reinterpret_cast<unsigned char *>(sRed + kRed);  // [LY][LX]
    __shared__ int sLast;

    const double t = A.scal[0];
    if (!(t < A.scal[2])) return;            // run_until predicate (uniform)
    const double dt = A.scal[1];

    const int npx = P.npx, npy = P.npy;
    const bool periodic = (P.wbc == 2);
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const long long pitch = A.pitch, plane = A.plane;

    // buffers of this stage
    const double *Vin;
    const double *V0;
    double *Vout;
    int par = 0;
    if (ORDER == 2) {
        Vin = FIRST ? A.bufA : A.bufB;
        V0 = A.bufA;
        Vout = FIRST ? A.bufB : A.bufA;
    } else {
        par = (int)A.scal[4];
        Vin = par ? A.bufB : A.bufA;
        V0 = Vin;
        Vout = par ? A.bufA : A.bufB;
    }

    // ---- phase 1: tile + halo -> smem
    for (int idx = tid; idx < LY * LX; idx += NT) {
        int ly = idx / LX, lx = idx - ly * LX;
        int gx = wrap_clamp(x0 + lx - 2, npx, periodic);
        int gy = wrap_clamp(y0 + ly - 2, npy, periodic);
        long long g = (long long)gy * pitch + gx;
#pragma unroll
        for (int f = 0; f < 5; f++) sV[f * LY * LX + idx] = Vin[f * plane + g];
        sM[idx] = A.mask[g];
    }
    const int tx = tid % TX, ty = tid / TX;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool own = (gi < npx) && (gj < npy);
    const long long gown = (long long)(own ? gj : 0) * pitch + (own ? gi : 0);
    // U^n at the owned cell for friction / erosion / RK combine
    double v0[5];
    if (!FIRST) {
#pragma unroll
        for (int f = 0; f < 5; f++) v0[f] = V0[f * plane + gown];
    }
    __syncthreads();

    const int cidx = (ty + 2) * LX + (tx + 2);
    double vc[5];
#pragma unroll
    for (int f = 0; f < 5; f++) vc[f] = sV[f * LY * LX + cidx];
    if (FIRST) {
#pragma unroll
        for (int f = 0; f < 5; f++) v0[f] = vc[f];
    }

    // ---- phase 2: per-cell velocity and concentration
    if (ORDER == 2) {
        for (int idx = tid; idx < LY * LX; idx += NT) {
            double h = sV[idx];
            double ux, uy;
            velocity(h, sV[LY * LX + idx], sV[2 * LY * LX + idx], ux, uy);
            sUC[idx] = ux;
            sUC[LY * LX + idx] = uy;
            sUC[2 * LY * LX + idx] = sV[4 * LY * LX + idx] / (h + kEpsilon);
        }
        __syncthreads();
    }

    // ---- phase 3: faces
    constexpr int NXI = FXW * TY, NYI = TX * FYH;
    for (int item = tid; item < NXI + NYI; item += NT) {
        State5 fm, fp;
        double deta = 0.0;
        if (item < NXI) {
            int r = item / FXW, cx = item - r * FXW;  // tile col cx-1
            int c = (r + 2) * LX + (cx + 1);
            if (ORDER == 2) {
                reconstruct_dir(sV, sUC, c, c - 1, c + 1, true, fm, fp, deta);
                int tc = cx - 1;
                if (tc >= 0 && tc < TX) sDeta[r * TX + tc] = deta;
            } else {
                fm = get5(sV + c, LY * LX);
                fp = fm;
            }
            put5(sFx + (0 * 5 * TY + r) * FXW + cx, TY * FXW, fm);
            put5(sFx + (1 * 5 * TY + r) * FXW + cx, TY * FXW, fp);
        } else {
            int it = item - NXI;
            int ry = it / TX, cc = it - ry * TX;  // tile row ry-1
            int c = (ry + 1) * LX + (cc + 2);
            if (ORDER == 2) {
                reconstruct_dir(sV, sUC, c, c - LX, c + LX, false, fm, fp, deta);
                int tr = ry - 1;
                if (tr >= 0 && tr < TY) sDeta[TY * TX + tr * TX + cc] = deta;
            } else {
                fm = get5(sV + c, LY * LX);
                fp = fm;
            }
            put5(sFy + (0 * 5 * FYH + ry) * TX + cc, FYH * TX, fm);
            put5(sFy + (1 * 5 * FYH + ry) * TX + cc, FYH * TX, fp);
        }
    }
    __syncthreads();

    // ---- phase 4: edges (each once per tile)
    const bool series_on = P.read_files && (t < A.tCC[A.timeCC - 2]);
    constexpr int NV = (TX + 1) * TY, NH = TX * (TY + 1);
    constexpr int FS = TY * TX;  // flux plane stride
    for (int item = tid; item < NV + NH; item += NT) {
        double Dm[5], Dp[5];
        if (item < NV) {
            int r = item / (TX + 1), e = item - r * (TX + 1);
            int ex = x0 + e, ey = y0 + r;
            if (ey >= npy || ex > npx) continue;
            const int ly = r + 2;
            // R face of tile col e-1 sits at sFx col e; L face of tile col e at col e+1
            const double *Rf = sFx + (1 * 5 * TY + r) * FXW + e;
            const double *Lf = sFx + (0 * 5 * TY + r) * FXW + (e + 1);
            if (periodic && (ex == 0 || ex == npx)) {
                State5 a = get5(Rf, TY * FXW), b = get5(Lf, TY * FXW);
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, npx + ey, b);
                    else b.qx = -a.qx;
                }
                edge_flux(P, a, b, 1, 0, sM[ly * LX + e + 1], Dm, Dp);
                if (e >= 1) put5a(sFlux + (1 * 5) * FS + r * TX + (e - 1), FS, Dm);
                if (e < TX) put5a(sFlux + (0 * 5) * FS + r * TX + e, FS, Dp);
            } else if (ex == 0) {
                State5 a = get5(Lf, TY * FXW), b = a;
                if (P.wbc == 1) b.qx = -a.qx;
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, 2 * npx + npy + ey, b);
                    else b.qx = -a.qx;
                }
                edge_flux(P, a, b, -1, 0, sM[ly * LX + e + 2], Dm, Dp);
                put5a(sFlux + (0 * 5) * FS + r * TX + e, FS, Dm);
            } else if (ex == npx) {
                State5 a = get5(Rf, TY * FXW), b = a;
                if (P.wbc == 1) b.qx = -a.qx;
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, npx + ey, b);
                    else b.qx = -a.qx;
                }
                edge_flux(P, a, b, 1, 0, sM[ly * LX + e + 1], Dm, Dp);
                put5a(sFlux + (1 * 5) * FS + r * TX + (e - 1), FS, Dm);
            } else {
                State5 a = get5(Rf, TY * FXW), b = get5(Lf, TY * FXW);
                int fixed = (int)sM[ly * LX + e + 1] * (int)sM[ly * LX + e + 2];
                edge_flux(P, a, b, 1, 0, fixed, Dm, Dp);
                if (e >= 1) put5a(sFlux + (1 * 5) * FS + r * TX + (e - 1), FS, Dm);
                if (e < TX) put5a(sFlux + (0 * 5) * FS + r * TX + e, FS, Dp);
            }
        } else {
            int it = item - NV;
            int e = it / TX, c = it - e * TX;
            int ex = x0 + c, ey = y0 + e;
            if (ex >= npx || ey > npy) continue;
            // U face of tile row e-1 sits at sFy row e; D face of tile row e at row e+1
            const double *Uf = sFy + (1 * 5 * FYH + e) * TX + c;
            const double *Df = sFy + (0 * 5 * FYH + e + 1) * TX + c;
            if (periodic && (ey == 0 || ey == npy)) {
                State5 a = get5(Uf, FYH * TX), b = get5(Df, FYH * TX);
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, npx + npy + ex, b);
                    else b.qy = -a.qy;
                }
                edge_flux(P, a, b, 0, 1, sM[(e + 1) * LX + c + 2], Dm, Dp);
                if (e >= 1) put5a(sFlux + (3 * 5) * FS + (e - 1) * TX + c, FS, Dm);
                if (e < TY) put5a(sFlux + (2 * 5) * FS + e * TX + c, FS, Dp);
            } else if (ey == 0) {
                State5 a = get5(Df, FYH * TX), b = a;
                if (P.wbc == 1) b.qy = -a.qy;
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, ex, b);
                    else b.qy = -a.qy;
                }
                edge_flux(P, a, b, 0, -1, sM[(e + 2) * LX + c + 2], Dm, Dp);
                put5a(sFlux + (2 * 5) * FS + e * TX + c, FS, Dm);
            } else if (ey == npy) {
                State5 a = get5(Uf, FYH * TX), b = a;
                if (P.wbc == 1) b.qy = -a.qy;
                if (P.read_files) {
                    if (series_on) series_state(A.CC, A.tCC, t, npx, npy, npx + npy + ex, b);
                    else b.qy = -a.qy;
                }
                edge_flux(P, a, b, 0, 1, sM[(e + 1) * LX + c + 2], Dm, Dp);
                put5a(sFlux + (3 * 5) * FS + (e - 1) * TX + c, FS, Dm);
            } else {
                State5 a = get5(Uf, FYH * TX), b = get5(Df, FYH * TX);
                int fixed = (int)sM[(e + 1) * LX + c + 2] * (int)sM[(e + 2) * LX + c + 2];
                edge_flux(P, a, b, 0, 1, fixed, Dm, Dp);
                if (e >= 1) put5a(sFlux + (3 * 5) * FS + (e - 1) * TX + c, FS, Dm);
                if (e < TY) put5a(sFlux + (2 * 5) * FS + e * TX + c, FS, Dp);
            }
        }
    }
    __syncthreads();

    // ---- phase 5: cell update
    double dtcell = CUDART_INF;
    if (own) {
        double vk[5];
#pragma unroll
        for (int f = 0; f < 5; f++) vk[f] = vc[f];
        if (ORDER == 2) {
            // pressure source, GPU/Reconstructor.cu:197,274
            const double dtax = dt * P.inv_dx, dtay = dt * P.inv_dy;
            vk[1] -= dtax * kG * vc[0] * sDeta[ty * TX + tx];
            vk[2] -= dtay * kG * vc[0] * sDeta[TY * TX + ty * TX + tx];
        }
        // friction (GPU/Reconstructor.cu:33-55) and erosion/deposition
        // (:57-88) from U^n; one velocity evaluation serves both.
        {
            double ux, uy;
            velocity(v0[0], v0[1], v0[2], ux, uy);
            double modu = sqrt(ux * ux + uy * uy);
            double cf = dt * P.FR * modu / (v0[0] + kEpsilon);
            vk[1] /= (1.0 + cf);
            vk[2] /= (1.0 + cf);
            double c = v0[4] / (v0[0] + P.eps_h);
            double Z = P.k.A_er * (modu * P.k.sqrt_FR) / P.k.vs;
            double Z5 = Z * Z * Z * Z * Z;
            double Es = (1.3e-7 * Z5) / (1 + 4.3e-7 * Z5);
            double Fe = P.k.VP * Es;
            if (Fe > 0.1) Fe = 0.1;
            Fe = Fe * (double)(Fe > 0.0);
            double Cb = P.k.K_dep * c;
            double Fd = P.k.vs * Cb;
            if (Fd > 0.1) Fd = 0.1;
            Fd = Fd * (double)(Fd > 0.0);
            double phi = (Fe - Fd) * (double)P.suspension;
            vk[3] -= dt * phi;
            vk[4] += dt * phi;
        }
        // flux divergence, GPU/Volume_kernel.cu:191-195
        const double invx = dt * P.inv_dx, invy = dt * P.inv_dy;
        const int cell = ty * TX + tx;
#pragma unroll
        for (int f = 0; f < 5; f++) {
            double FL = sFlux[(0 * 5 + f) * FS + cell], FR = sFlux[(1 * 5 + f) * FS + cell];
            double FD = sFlux[(2 * 5 + f) * FS + cell], FU = sFlux[(3 * 5 + f) * FS + cell];
            vk[f] -= invx * (FL + FR) + invy * (FD + FU);
        }
        // RK combine + filter, GPU/Volume_kernel.cu:244-281
        const int k = (ORDER == 2 && !FIRST) ? 1 : 0;
        const double coef0 = 0.0 * (double)(k == 0) + 0.5 * (double)(k == 1);
        const double coef1 = 1.0 - coef0;
        double h = coef0 * v0[0] + coef1 * vk[0];
        double qx = coef0 * v0[1] + coef1 * vk[1];
        double qy = coef0 * v0[2] + coef1 * vk[2];
        double z = coef0 * v0[3] + coef1 * vk[3];
        double hc = coef0 * v0[4] + coef1 * vk[4];
        positivity_filter(h, qx, qy, hc);
        Vout[gown] = h;
        Vout[plane + gown] = qx;
        Vout[2 * plane + gown] = qy;
        Vout[3 * plane + gown] = z;
        Vout[4 * plane + gown] = hc;
        if (LAST) {
            const double eps_h = P.eps_h;
            if (h > eps_h) A.hmax[gown] = fmax(A.hmax[gown], h);
            A.bmin[gown] = fmax(A.bmin[gown], z);
            if (h > eps_h) A.eta_max[gown] = fmax(A.eta_max[gown], h - z);
            double d = cfl_dt(P, h, qx, qy);
            if (!isnan(d)) dtcell = d;
        }
    }

    if (LAST) {
        // CTA minimum with warp shuffles, then the last CTA finishes the
        // global minimum and advances t (GPU/main_TSUNER.cu:185,190-192).
        double m = dtcell;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((tid & 31) == 0) sRed[tid >> 5] = m;
        __syncthreads();
        if (tid < 32) {
            m = (tid < kRed) ? sRed[tid] : CUDART_INF;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (tid == 0) {
                const unsigned nb = gridDim.x * gridDim.y;
                const unsigned b = blockIdx.y * gridDim.x + blockIdx.x;
                A.partials[b] = m;
                __threadfence();
                unsigned tk = atomicAdd(A.ticket, 1u);
                sLast = (tk == nb - 1);
            }
        }
        __syncthreads();
        if (sLast) {
            __threadfence();
            const unsigned nb = gridDim.x * gridDim.y;
            double mm = CUDART_INF;
            for (unsigned i = tid; i < nb; i += NT) mm = fmin(mm, __ldcg(A.partials + i));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mm = fmin(mm, __shfl_xor_sync(0xffffffffu, mm, o));
            if ((tid & 31) == 0) sRed[tid >> 5] = mm;
            __syncthreads();
            if (tid == 0) {
                for (int w = 0; w < kRed; w++) mm = fmin(mm, sRed[w]);
                A.scal[0] = t + dt;
                A.scal[1] = finalize_dt(mm, (long long)npx * npy);
                A.scal[3] += 1.0;
                if (ORDER == 1) A.scal[4] = (double)(1 - par);
                *A.ticket = 0u;
                __threadfence();
            }
        }
    }
}

// GetDeltaT + MinReduction over a state (initial dt, GPU/main_TSUNER.cu:147-148).
__global__ void __launch_bounds__(256) dt_partials_kernel(const double *__restrict__ V, long long pitch,
                                                          long long plane, Phys64 P, double *partials,
                                                          unsigned *ticket, double *scal) {
    __shared__ double sRed[8];
    __shared__ int sLast;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int gi = blockIdx.x * blockDim.x + threadIdx.x, gj = blockIdx.y * blockDim.y + threadIdx.y;
    double m = CUDART_INF;
    if (gi < P.npx && gj < P.npy) {
        long long g = (long long)gj * pitch + gi;
        double d = cfl_dt(P, V[g], V[plane + g], V[2 * plane + g]);
        if (!isnan(d)) m = d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) sRed[tid >> 5] = m;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < 8; w++) m = fmin(m, sRed[w]);
        const unsigned nb = gridDim.x * gridDim.y;
        partials[blockIdx.y * gridDim.x + blockIdx.x] = m;
        __threadfence();
        sLast = (atomicAdd(ticket, 1u) == nb - 1);
        if (sLast) {
            __threadfence();
            double mm = CUDART_INF;
            for (unsigned i = 0; i < nb; i++) mm = fmin(mm, __ldcg(partials + i));
            scal[1] = finalize_dt(mm, (long long)P.npx * P.npy);
            *ticket = 0u;
            __threadfence();
        }
    }
}

__global__ void fill_kernel(double *p, long long n, double v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// Per-run constants with the reference expressions (device pow()).
__global__ void consts_kernel(SimParams p, TsuConsts *k) {
    double nu = 1.002e-6;
    double s = p.R - 1.0;
    k->vs = sqrt((13.95 * nu / p.DS) * (13.95 * nu / p.DS) + 1.09 * s * kG * p.DS) - 13.95 * nu / p.DS;
    k->Rp = (p.DS * sqrt(s * kG * p.DS)) / nu;
    double a1, a2;
    if (k->Rp > 2.36) {
        a1 = 1;
        a2 = 0.6;
    } else {
        a1 = 0.586;
        a2 = 1.23;
    }
    k->A_er = a1 * pow(k->Rp, a2);
    k->sqrt_FR = sqrt(p.FR);
    k->VP = k->vs * (1 - p.porosity);
    k->K_dep = (1.64 + 0.4 * pow(p.DS / p.Dsg, 1.64));
    k->sqrt_OC = sqrt(p.OC);
    k->DS5 = 5 * p.DS;
}

// ------------------------------------------------------------------ host side
#define S64_INSTANCE(O, F, L) \
    template __global__ void stage64_kernel<O, F, L>(Stage64Args);
S64_INSTANCE(2, true, false)
S64_INSTANCE(2, false, true)
S64_INSTANCE(1, true, true)

cudaError_t stage64_prepare() {
    size_t sm = stage64_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(stage64_kernel<2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage64_kernel<2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage64_kernel<1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    return e;
}

dim3 stage64_grid(int npx, int npy) { return dim3((npx + TX - 1) / TX, (npy + TY - 1) / TY); }

cudaError_t stage64_launch(int order, int stage, const Stage64Args &a, cudaStream_t st) {
    dim3 g = stage64_grid(a.phys.npx, a.phys.npy);
    size_t sm = stage64_smem_bytes();
    if (order == 2 && stage == 0) stage64_kernel<2, true, false><<<g, NT, sm, st>>>(a);
    else if (order == 2) stage64_kernel<2, false, true><<<g, NT, sm, st>>>(a);
    else stage64_kernel<1, true, true><<<g, NT, sm, st>>>(a);
    return cudaGetLastError();
}

cudaError_t initial_dt_launch(const double *V, long long pitch, long long plane, const Phys64 &P, double *partials,
                              unsigned *ticket, double *scal, cudaStream_t st) {
    dim3 b(32, 8), g((P.npx + 31) / 32, (P.npy + 7) / 8);
    dt_partials_kernel<<<g, b, 0, st>>>(V, pitch, plane, P, partials, ticket, scal);
    return cudaGetLastError();
}

cudaError_t fill_launch(double *p, long long n, double v, cudaStream_t st) {
    fill_kernel<<<1184, 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t consts_launch(const SimParams &p, TsuConsts *k, cudaStream_t st) {
    consts_kernel<<<1, 1, 0, st>>>(p, k);
    return cudaGetLastError();
}

size_t partials_needed(int npx, int npy) {
    dim3 g = stage64_grid(npx, npy);
    size_t a = (size_t)g.x * g.y;
    size_t b = (size_t)((npx + 31) / 32) * ((npy + 7) / 8);
    return a > b ? a : b;
}

}  // namespace tsu
