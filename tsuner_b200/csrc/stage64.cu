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
// Phases 3 and 4 each have a single call site of the reconstruction and of
// the Riemann solver (boundary cases only select operands), which keeps the
// kernel body small enough for the instruction cache.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "physics64.cuh"
#include "async.cuh"
#include "stage64.h"

namespace tsu {

// A TX x TY tile processed by NTHR threads (NTHR >= TX*TY: the first TX*TY
// threads own a cell in the update; all of them share the halo loads, faces
// and edges).
template <int TX_, int TY_, int NTHR_ = TX_ * TY_>
struct Tile {
    static constexpr int TX = TX_, TY = TY_, NT = NTHR_;
    static_assert(NTHR_ >= TX_ * TY_ && NTHR_ % 32 == 0 && NTHR_ <= 1024, "threads per tile");
    static constexpr int LX = TX + 4, LY = TY + 4, PS = LX * LY;  // loaded tile, 2-cell halo
    static constexpr int FXW = TX + 2, FYH = TY + 2;               // faces incl. one halo cell
    static constexpr int kSV = 5 * PS, kSUC = 3 * PS, kFlux = 20 * TY * TX;
    static constexpr int kRegA = (kSV + kSUC) > kFlux ? (kSV + kSUC) : kFlux;
    static constexpr int kFx = 10 * TY * FXW, kFy = 10 * FYH * TX, kDeta = 2 * TY * TX, kRed = NT / 32;
    static constexpr int kDoubles = kRegA + kFx + kFy + kDeta + kRed;
    // the 1-byte mask: rows of MLX = TX + 32 cells starting 16 left of the
    // tile (a 16-byte aligned TMA origin for bytes), 128-byte aligned
    static constexpr int MHX = 16, MLX = TX + 2 * MHX, MPS = MLX * LY;
    static constexpr size_t kMaskOff = (sizeof(double) * kDoubles + 127) / 128 * 128;
    // the owned cells' U^n (5 planes) and running extrema (3 planes), [8][TY][TX],
    // staged by TMA in the second RK stage (OWN == 2), 128-byte aligned
    static constexpr size_t kOwnOff = (kMaskOff + MPS + 127) / 128 * 128;
    static constexpr size_t kOwnBytes = 8 * TX * TY * sizeof(double);
    // + 128: the base is rounded up to 128 bytes (TMA destination)
    static constexpr size_t smem(bool staged_own = false) {
        return (staged_own ? kOwnOff + kOwnBytes : kMaskOff + MPS + 16) + 128;
    }
};

__device__ __forceinline__ int wrap_clamp(int g, int n, bool periodic) {
    if (periodic) {
        g %= n;
        return g < 0 ? g + n : g;
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

// MUSCL reconstruction of one cell along one direction, GPU/Reconstructor.cu
// :124-194 (x) / :207-271 (y).  c/l/r index the centre and its two
// neighbours in the smem tile (plane stride PS).  Returns the two faces
// (minus side, plus side) before the state filter and the hydrostatic slope
// deta.
template <int PS>
__device__ __forceinline__ void reconstruct_dir(const double *sV, const double *sUC, int c, int l, int r,
                                                State5 &fm, State5 &fp, double &deta) {
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
}

__device__ __forceinline__ void filter5(State5 &s) { positivity_filter(s.h, s.qx, s.qy, s.hc); }

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

// RK0: MUSCL-Hancock (RK == 0 of the reference): one stage per step
// (FIRST = LAST = true), the state ping-pongs between bufA and bufB like the
// order-1 form, and bufK holds the unfiltered working state Vk that the
// reference carries from step to step (GPU/Volume_kernel.cu:283-299).
// OWN: where the second RK stage keeps U^n of the owned cell and its running
// extrema between tile start and the update.  0: U^n loaded into registers
// at tile start (held through the face and edge phases), extrema loaded in
// the update; 1: both requested into L2 at tile start and loaded in the
// update; 2: interior tiles stage both into shared memory with TMA boxes
// issued at tile start (they land during the face and edge phases), other
// tiles as 1.
template <int TX, int TY, int NTHR, int MINB, int ORDER, bool FIRST, bool LAST, bool RK0 = false, int OWN = 0>
__global__ void __launch_bounds__(NTHR, MINB) stage64_kernel(const __grid_constant__ Stage64Args A) {
    static_assert(!RK0 || (FIRST && LAST), "MUSCL-Hancock is a single stage");
    constexpr bool PINGPONG = (ORDER == 1) || RK0;
    constexpr bool LATE = (OWN >= 1);
    using T = Tile<TX, TY, NTHR>;
    constexpr int NT = T::NT, LX = T::LX, LY = T::LY, PS = T::PS, FXW = T::FXW, FYH = T::FYH;
    constexpr int MHX = T::MHX, MLX = T::MLX;
    extern __shared__ __align__(16) double smem_raw[];
    double *smem = smem_align<128>(smem_raw);
    __shared__ uint64_t sBar;     // the tile's TMA load
    __shared__ uint64_t sBarOwn;  // OWN == 2: the owned cells' U^n and extrema
    const Phys64 &P = A.phys;
    double *sV = smem;                  // [5][LY][LX]
    double *sUC = smem + T::kSV;        // [3][LY][LX]  (ux, uy, c)
    double *sFlux = smem;               // [4][5][TY][TX]  aliases sV/sUC (dead by then)
    double *sFx = smem + T::kRegA;      // [2][5][TY][FXW]
    double *sFy = sFx + T::kFx;         // [2][5][FYH][TX]
    double *sDeta = sFy + T::kFy;       // [2][TY][TX]
    double *sRed = sDeta + T::kDeta;    // [NT/32]
    unsigned char *sM = reinterpret_cast<unsigned char *>(smem) + T::kMaskOff;  // [LY][MLX], tile at column MHX
    __shared__ int sLast;

    const double t = A.scal[SC_T];
    if (!(t < A.scal[SC_TEND])) return;  // run_until predicate (uniform)
    const double dt = A.scal[SC_DT];

    const int npx = P.npx, npy = P.npy;
    const bool periodic = (P.wbc == 2);
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const long long pitch = A.pitch, plane = A.plane;

    const double *Vin;
    const double *V0;
    double *Vout;
    int par = 0;
    if (!PINGPONG) {
        Vin = FIRST ? A.bufA : A.bufB;
        V0 = A.bufA;
        Vout = FIRST ? A.bufB : A.bufA;
    } else {
        par = (int)A.scal[SC_PAR];
        Vin = par ? A.bufB : A.bufA;
        V0 = Vin;
        Vout = par ? A.bufA : A.bufB;
    }

    // tile and halo inside the stored rows (the owned rows and a slab's ghost
    // rows), not periodic: no clamping, and every edge of the tile is an
    // interior edge
    const bool inner =
        !periodic && x0 >= 2 && y0 - 2 >= -P.gs && x0 + TX + 2 <= npx && y0 + TY + 2 <= npy + P.gn;

    // ---- phase 1: tile + halo -> smem.  Interior tiles: one TMA box of the
    // 5 state planes (x0 - 2 doubles = a multiple of 16 bytes) and one of the
    // mask (from x0 - 16); boundary tiles (clamped or wrapped halo) with
    // ordinary loads.
    const bool use_tma = inner && A.tma;
    // the owned cells of an interior tile lie inside the stored rows: the
    // boxes at (x0, y0) are in bounds, x0 * 8 bytes a multiple of 256
    const bool own_tma = (OWN == 2) && !FIRST && use_tma;
    constexpr int TC = TX * TY;
    double *sOwn = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(smem) + T::kOwnOff);
    if (use_tma) {
        if (tid == 0) {
            mbar_init(&sBar, 1);
            if (own_tma) mbar_init(&sBarOwn, 1);
            mbar_init_fence();
            mbar_expect_tx(&sBar, 5 * PS * sizeof(double) + T::MPS);
            // the tensor maps start at the first stored row (a slab's lowest ghost row)
            tma_load_3d(sV, (Vin == A.bufB) ? &A.tmB : &A.tmA, x0 - 2, y0 - 2 + P.gs, 0, &sBar);
            tma_load_2d(sM, &A.tmM, x0 - MHX, y0 - 2 + P.gs, &sBar);
            if (own_tma) {
                mbar_expect_tx(&sBarOwn, (LAST ? 8 : 5) * TC * sizeof(double));
                tma_load_3d(sOwn, &A.tmO, x0, y0 + P.gs, 0, &sBarOwn);
                if (LAST) {
#pragma unroll
                    for (int f = 0; f < 3; f++) tma_load_2d(sOwn + (5 + f) * TC, &A.tmE[f], x0, y0 + P.gs, &sBarOwn);
                }
            }
        }
    } else {
        for (int idx = tid; idx < PS; idx += NT) {
            const int ly = idx / LX, lx = idx - ly * LX;
            int gx = x0 + lx - 2, gy = y0 + ly - 2;
            if (!inner) {
                gx = wrap_clamp(gx, npx, periodic);
                // rows outside the stored ones: the grid's own boundary (a
                // slab stores ghost rows wherever it has a neighbour)
                if (gy < -P.gs || gy >= npy + P.gn) gy = wrap_clamp(gy, npy, periodic);
            }
            const long long g = (long long)gy * pitch + gx;
#pragma unroll
            for (int f = 0; f < 5; f++) sV[f * PS + idx] = Vin[f * plane + g];
            sM[ly * MLX + lx + (MHX - 2)] = A.mask[g];
        }
    }
    const bool cell_thread = tid < TX * TY;  // owns a cell in the update
    const int tx = cell_thread ? tid % TX : 0, ty = cell_thread ? tid / TX : 0;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool own = cell_thread && (gi < npx) && (gj < npy);
    const long long gown = (long long)(own ? gj : 0) * pitch + (own ? gi : 0);
    double v0[5];
    if (!FIRST && !own_tma) {  // U^n of the owned cell (friction, erosion, RK combine)
#pragma unroll
        for (int f = 0; f < 5; f++) {
            if (LATE) prefetch_l2(V0 + f * plane + gown);
            else v0[f] = V0[f * plane + gown];
        }
    }
    if (LATE && LAST && own && !own_tma) {
        prefetch_l2(A.hmax + gown);
        prefetch_l2(A.bmin + gown);
        prefetch_l2(A.eta_max + gown);
    }
    __syncthreads();
    if (use_tma) {  // every thread sees the box land (bounded wait)
        const bool ok = mbar_wait_first(&sBar, 0);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                A.scal[SC_ERR] = 1.0;
                mbar_wait(&sBar, 0);
                if (own_tma) mbar_wait(&sBarOwn, 0);
            }
            return;
        }
    }

    const int cidx = (ty + 2) * LX + (tx + 2);
    double vc[5];
#pragma unroll
    for (int f = 0; f < 5; f++) vc[f] = sV[f * PS + cidx];
    if (FIRST) {
#pragma unroll
        for (int f = 0; f < 5; f++) v0[f] = vc[f];
    }

    // ---- phase 2: per-cell velocity and concentration
    if (ORDER == 2) {
        for (int idx = tid; idx < PS; idx += NT) {
            double h = sV[idx];
            double ux, uy;
            velocity(h, sV[PS + idx], sV[2 * PS + idx], ux, uy);
            sUC[idx] = ux;
            sUC[PS + idx] = uy;
            sUC[2 * PS + idx] = ddiv(sV[4 * PS + idx], h + kEpsilon);
        }
        __syncthreads();
    }

    // ---- phase 3: faces (one reconstruction call site)
    constexpr int NXI = FXW * TY, NYI = TX * FYH;
    if (RK0 && ORDER == 2) {
        // MUSCL-Hancock: the predictor needs all four faces of a cell, so an
        // item is a cell -- the tile, then its halo columns -1 / TX (x faces
        // kept) and halo rows -1 / TY (y faces kept)
        constexpr int NC = TX * TY + 2 * TY + 2 * TX;
        for (int item = tid; item < NC; item += NT) {
            int lx, ly;
            if (item < TX * TY) {
                ly = item / TX;
                lx = item - ly * TX;
            } else if (item < TX * TY + 2 * TY) {
                const int k = item - TX * TY;
                ly = k >> 1;
                lx = (k & 1) ? TX : -1;
            } else {
                const int k = item - TX * TY - 2 * TY;
                lx = k >> 1;
                ly = (k & 1) ? TY : -1;
            }
            const int c = (ly + 2) * LX + (lx + 2);
            State5 L, R, D, U;
            double detx, dety;
            reconstruct_dir<PS>(sV, sUC, c, c - 1, c + 1, L, R, detx);
            reconstruct_dir<PS>(sV, sUC, c, c - LX, c + LX, D, U, dety);
            hancock_predictor(P, dt, sV[c], detx, dety, L, R, D, U);
            filter5(L);
            filter5(R);
            filter5(U);
            filter5(D);
            if (ly >= 0 && ly < TY) {
                double *dst = sFx + ly * FXW + (lx + 1);
                put5(dst, TY * FXW, L);
                put5(dst + 5 * TY * FXW, TY * FXW, R);
            }
            if (lx >= 0 && lx < TX) {
                double *dst = sFy + (ly + 1) * TX + lx;
                put5(dst, FYH * TX, D);
                put5(dst + 5 * FYH * TX, FYH * TX, U);
            }
            if (lx >= 0 && lx < TX && ly >= 0 && ly < TY) {
                sDeta[ly * TX + lx] = detx;
                sDeta[TY * TX + ly * TX + lx] = dety;
            }
        }
    }
    for (int item = tid; item < ((RK0 && ORDER == 2) ? 0 : NXI + NYI); item += NT) {
        int c, step, fstride, side, didx = -1;
        double *dst;
        if (item < NXI) {
            int r = item / FXW, cx = item - r * FXW;  // tile col cx-1
            c = (r + 2) * LX + (cx + 1);
            step = 1;
            dst = sFx + r * FXW + cx;
            fstride = TY * FXW;
            side = 5 * TY * FXW;
            int tc = cx - 1;
            if (tc >= 0 && tc < TX) didx = r * TX + tc;
        } else {
            int it = item - NXI;
            int ry = it / TX, cc = it - ry * TX;  // tile row ry-1
            c = (ry + 1) * LX + (cc + 2);
            step = LX;
            dst = sFy + ry * TX + cc;
            fstride = FYH * TX;
            side = 5 * FYH * TX;
            int tr = ry - 1;
            if (tr >= 0 && tr < TY) didx = TY * TX + tr * TX + cc;
        }
        State5 fm, fp;
        if (ORDER == 2) {
            double deta;
            if (P.dry_skip && sV[c] == 0.0 && sV[c - step] == 0.0 && sV[c + step] == 0.0) {
                // a dry stencil: every slope is avg(0, 0) = 0, so both faces
                // are (0, q_i, 0, H_i, 0 * c) before the filter and (0, 0, 0,
                // H_i, 0) after it (zeros up to their sign), and deta = 0
                fm.h = fm.qx = fm.qy = fm.hc = 0.0;
                fm.H = sV[3 * PS + c];
                fp = fm;
                deta = 0.0;
            } else {
                reconstruct_dir<PS>(sV, sUC, c, c - step, c + step, fm, fp, deta);
                filter5(fm);  // GPU/Reconstructor.cu:344-348
                filter5(fp);
            }
            if (didx >= 0) sDeta[didx] = deta;
        } else {  // first order: faces are the cell values (GPU/Reconstructor.cu:99-107)
            fm = get5(sV + c, PS);
            fp = fm;
        }
        put5(dst, fstride, fm);
        put5(dst + side, fstride, fp);
    }
    __syncthreads();

    // ---- phase 4: edges (each once per tile, one Riemann call site)
    const bool series_on = !inner && P.read_files && (t < A.tCC[A.timeCC - 2]);
    constexpr int NV = (TX + 1) * TY, NH = TX * (TY + 1);
    constexpr int FS = TY * TX;  // flux plane stride; planes FL, FR, FD, FU
    for (int item = tid; item < NV + NH; item += NT) {
        State5 a, b;
        int nx, ny, fixed, seg = 0;
        bool bnd = false, seam = false, vert;
        double *outM = nullptr, *outP = nullptr;
        if (inner) {  // interior edges only (uniform per tile): no bounds or boundary cases
            if (item < NV) {
                vert = true;
                nx = 1;
                ny = 0;
                const int r = item / (TX + 1), e = item - r * (TX + 1);
                a = get5(sFx + (5 * TY + r) * FXW + e, TY * FXW);
                b = get5(sFx + r * FXW + (e + 1), TY * FXW);
                fixed = (int)sM[(r + 2) * MLX + e + 1 + (MHX - 2)] * (int)sM[(r + 2) * MLX + e + 2 + (MHX - 2)];
                if (e >= 1) outM = sFlux + 1 * 5 * FS + r * TX + (e - 1);
                if (e < TX) outP = sFlux + 0 * 5 * FS + r * TX + e;
            } else {
                vert = false;
                nx = 0;
                ny = 1;
                const int it = item - NV;
                const int e = it / TX, c = it - e * TX;
                a = get5(sFy + (5 * FYH + e) * TX + c, FYH * TX);
                b = get5(sFy + (e + 1) * TX + c, FYH * TX);
                fixed = (int)sM[(e + 1) * MLX + c + 2 + (MHX - 2)] * (int)sM[(e + 2) * MLX + c + 2 + (MHX - 2)];
                if (e >= 1) outM = sFlux + 3 * 5 * FS + (e - 1) * TX + c;
                if (e < TY) outP = sFlux + 2 * 5 * FS + e * TX + c;
            }
        } else if (item < NV) {
            vert = true;
            const int r = item / (TX + 1), e = item - r * (TX + 1);
            const int ex = x0 + e, ey = y0 + r;
            if (ey >= npy || ex > npx) continue;
            const int ly = r + 2;
            // R face of tile col e-1 is sFx col e; L face of tile col e is col e+1
            const double *Rf = sFx + (5 * TY + r) * FXW + e;
            const double *Lf = sFx + r * FXW + (e + 1);
            nx = 1;
            ny = 0;
            const int J = P.j0 + ey;  // the global row (boundary-series segments)
            if (periodic && (ex == 0 || ex == npx)) {  // seam: GPU/VolumeSolver.cu:262-275,289-298
                a = get5(Rf, TY * FXW);
                b = get5(Lf, TY * FXW);
                fixed = sM[ly * MLX + e + 1 + (MHX - 2)];
                seam = true;
                seg = npx + J;
                if (e >= 1) outM = sFlux + 1 * 5 * FS + r * TX + (e - 1);
                if (e < TX) outP = sFlux + 0 * 5 * FS + r * TX + e;
            } else if (ex == 0) {  // west: GPU/VolumeSolver.cu:233-258
                a = get5(Lf, TY * FXW);
                nx = -1;
                fixed = sM[ly * MLX + e + 2 + (MHX - 2)];
                bnd = true;
                seg = 2 * npx + P.ny_glob + J;
                outM = sFlux + 0 * 5 * FS + r * TX + e;
            } else if (ex == npx) {  // east: GPU/VolumeSolver.cu:276-298
                a = get5(Rf, TY * FXW);
                fixed = sM[ly * MLX + e + 1 + (MHX - 2)];
                bnd = true;
                seg = npx + J;
                outM = sFlux + 1 * 5 * FS + r * TX + (e - 1);
            } else {  // interior: GPU/VolumeSolver.cu:300-314
                a = get5(Rf, TY * FXW);
                b = get5(Lf, TY * FXW);
                fixed = (int)sM[ly * MLX + e + 1 + (MHX - 2)] * (int)sM[ly * MLX + e + 2 + (MHX - 2)];
                if (e >= 1) outM = sFlux + 1 * 5 * FS + r * TX + (e - 1);
                if (e < TX) outP = sFlux + 0 * 5 * FS + r * TX + e;
            }
        } else {
            vert = false;
            const int it = item - NV;
            const int e = it / TX, c = it - e * TX;
            const int ex = x0 + c, ey = y0 + e;
            if (ex >= npx || ey > npy) continue;
            // U face of tile row e-1 is sFy row e; D face of tile row e is row e+1
            const double *Uf = sFy + (5 * FYH + e) * TX + c;
            const double *Df = sFy + (e + 1) * TX + c;
            nx = 0;
            ny = 1;
            // the grid's own south / north boundary (a slab's other edges are
            // interior edges, their far side in the ghost rows)
            const int J = P.j0 + ey;
            const bool south = (J == 0), north = (J == P.ny_glob);
            if (periodic && (south || north)) {  // seam: GPU/VolumeSolver.cu:352-367,378-387
                a = get5(Uf, FYH * TX);
                b = get5(Df, FYH * TX);
                fixed = sM[(e + 1) * MLX + c + 2 + (MHX - 2)];
                seam = true;
                seg = npx + P.ny_glob + ex;
                if (e >= 1) outM = sFlux + 3 * 5 * FS + (e - 1) * TX + c;
                if (e < TY) outP = sFlux + 2 * 5 * FS + e * TX + c;
            } else if (south) {  // south: GPU/VolumeSolver.cu:324-349
                a = get5(Df, FYH * TX);
                ny = -1;
                fixed = sM[(e + 2) * MLX + c + 2 + (MHX - 2)];
                bnd = true;
                seg = ex;
                outM = sFlux + 2 * 5 * FS + e * TX + c;
            } else if (north) {  // north: GPU/VolumeSolver.cu:352-387
                a = get5(Uf, FYH * TX);
                fixed = sM[(e + 1) * MLX + c + 2 + (MHX - 2)];
                bnd = true;
                seg = npx + P.ny_glob + ex;
                outM = sFlux + 3 * 5 * FS + (e - 1) * TX + c;
            } else {  // interior: GPU/VolumeSolver.cu:389-403
                a = get5(Uf, FYH * TX);
                b = get5(Df, FYH * TX);
                fixed = (int)sM[(e + 1) * MLX + c + 2 + (MHX - 2)] * (int)sM[(e + 2) * MLX + c + 2 + (MHX - 2)];
                if (e >= 1) outM = sFlux + 3 * 5 * FS + (e - 1) * TX + c;
                if (e < TY) outP = sFlux + 2 * 5 * FS + e * TX + c;
            }
        }
        if (bnd) {  // ghost = copy, wall mirror of the normal momentum
            b = a;
            if (P.wbc == 1) {
                if (vert) b.qx = -a.qx;
                else b.qy = -a.qy;
            }
        }
        if ((bnd || seam) && P.read_files) {  // CC series while active, then wall
            if (series_on) series_state(A.CC, A.tCC, t, npx, P.ny_glob, seg, b);
            else if (vert) b.qx = -a.qx;
            else b.qy = -a.qy;
        }
        double Dm[5], Dp[5];
        edge_flux(P, a, b, nx, ny, fixed, Dm, Dp);
        if (outM) put5a(outM, FS, Dm);
        if (outP) put5a(outP, FS, Dp);
    }
    __syncthreads();

    if (own_tma) {  // the owned cells' U^n and extrema have landed (bounded wait)
        const bool ok = mbar_wait_first(&sBarOwn, 0);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                A.scal[SC_ERR] = 1.0;
                mbar_wait(&sBarOwn, 0);
            }
            return;
        }
    }

    // ---- phase 5: cell update
    double dtcell = CUDART_INF;
    bool bad = false;  // last stage: the new state of the owned cell is not finite
    const int cell = ty * TX + tx;
    if (own) {
        if (LATE && !FIRST) {
#pragma unroll
            for (int f = 0; f < 5; f++) v0[f] = own_tma ? sOwn[f * TC + cell] : V0[f * plane + gown];
        }
        double vk[5];  // the reference's Vk: this stage's input, or MUSCL-Hancock's carried working state
#pragma unroll
        for (int f = 0; f < 5; f++) vk[f] = RK0 ? A.bufK[f * plane + gown] : vc[f];
        if (ORDER == 2) {  // pressure source, GPU/Reconstructor.cu:197,274
            const double dtax = dt * P.inv_dx, dtay = dt * P.inv_dy;
            vk[1] -= dtax * kG * vc[0] * sDeta[ty * TX + tx];
            vk[2] -= dtay * kG * vc[0] * sDeta[TY * TX + ty * TX + tx];
        }
        // friction (GPU/Reconstructor.cu:33-55) and erosion/deposition
        // (:57-88) from U^n; one velocity evaluation serves both.
        {
            double ux, uy;
            velocity(v0[0], v0[1], v0[2], ux, uy);
            double modu = dsqrt(ux * ux + uy * uy);
            if (P.manning) {  // GPU/Reconstructor.cu:47-50 as written (multiplies)
                const double cm = dt * P.FR * P.FR * modu / pow(v0[0], 4.0 / 3.0);
                vk[1] *= cm;
                vk[2] *= cm;
            } else {
                double cf = ddiv(dt * P.FR * modu, v0[0] + kEpsilon);
                vk[1] = ddiv(vk[1], 1.0 + cf);
                vk[2] = ddiv(vk[2], 1.0 + cf);
            }
            double c = ddiv(v0[4], v0[0] + P.eps_h);
            double Z = ddiv(P.k.A_er * (modu * P.k.sqrt_FR), P.k.vs);
            double Z5 = Z * Z * Z * Z * Z;
            double Es = ddiv(1.3e-7 * Z5, 1 + 4.3e-7 * Z5);
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
#pragma unroll
        for (int f = 0; f < 5; f++) {
            double FL = sFlux[(0 * 5 + f) * FS + cell], FR = sFlux[(1 * 5 + f) * FS + cell];
            double FD = sFlux[(2 * 5 + f) * FS + cell], FU = sFlux[(3 * 5 + f) * FS + cell];
            vk[f] -= invx * (FL + FR) + invy * (FD + FU);
        }
        // RK combine + filter, GPU/Volume_kernel.cu:244-281; MUSCL-Hancock
        // filters Vk itself and keeps the unfiltered Vk (:283-299)
        double h, qx, qy, z, hc;
        if (RK0) {
            h = vk[0];
            qx = vk[1];
            qy = vk[2];
            z = vk[3];
            hc = vk[4];
#pragma unroll
            for (int f = 0; f < 5; f++) A.bufK[f * plane + gown] = vk[f];
        } else {
            const int k = (ORDER == 2 && !FIRST) ? 1 : 0;
            const double coef0 = 0.0 * (double)(k == 0) + 0.5 * (double)(k == 1);
            const double coef1 = 1.0 - coef0;
            h = coef0 * v0[0] + coef1 * vk[0];
            qx = coef0 * v0[1] + coef1 * vk[1];
            qy = coef0 * v0[2] + coef1 * vk[2];
            z = coef0 * v0[3] + coef1 * vk[3];
            hc = coef0 * v0[4] + coef1 * vk[4];
        }
        positivity_filter(h, qx, qy, hc);
        Vout[gown] = h;
        Vout[plane + gown] = qx;
        Vout[2 * plane + gown] = qy;
        Vout[3 * plane + gown] = z;
        Vout[4 * plane + gown] = hc;
        if (LAST) {
            const double eps_h = P.eps_h;
            if (own_tma) {
                if (h > eps_h) A.hmax[gown] = fmax(sOwn[5 * TC + cell], h);
                A.bmin[gown] = fmax(sOwn[6 * TC + cell], z);
                if (h > eps_h) A.eta_max[gown] = fmax(sOwn[7 * TC + cell], h - z);
            } else {
                if (h > eps_h) A.hmax[gown] = fmax(A.hmax[gown], h);
                A.bmin[gown] = fmax(A.bmin[gown], z);
                if (h > eps_h) A.eta_max[gown] = fmax(A.eta_max[gown], h - z);
            }
            double d = cfl_dt(P, h, qx, qy);
            if (!isnan(d)) dtcell = d;
            bad = !(finite64(h) && finite64(qx) && finite64(qy) && finite64(z) && finite64(hc));
        }
    }

    if (LAST) {
        // a NaN / Inf anywhere in the new state is reported to the host (the
        // values themselves are stored unchanged, as the reference would)
        if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) A.scal[SC_NAN] = 1.0;
        // CTA minimum with warp shuffles; the last CTA to finish reduces the
        // partials, advances t and publishes the next dt
        // (GPU/main_TSUNER.cu:185,190-192).
        double m = dtcell;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((tid & 31) == 0) sRed[tid >> 5] = m;
        __syncthreads();
        if (tid < 32) {
            m = (tid < T::kRed) ? sRed[tid] : CUDART_INF;
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
            __syncthreads();
            if ((tid & 31) == 0) sRed[tid >> 5] = mm;
            __syncthreads();
            if (tid == 0) {
                for (int w = 0; w < T::kRed; w++) mm = fmin(mm, sRed[w]);
                A.scal[SC_T] = t + dt;
                A.scal[SC_DT] = finalize_dt(mm, (long long)npx * P.ny_glob);
                A.scal[SC_STEPS] += 1.0;
                if (PINGPONG) A.scal[SC_PAR] = (double)(1 - par);
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
    bool bad = false;
    if (gi < P.npx && gj < P.npy) {
        long long g = (long long)gj * pitch + gi;
        double d = cfl_dt(P, V[g], V[plane + g], V[2 * plane + g]);
        if (!isnan(d)) m = d;
        bad = !(finite64(V[g]) && finite64(V[plane + g]) && finite64(V[2 * plane + g]) &&
                finite64(V[3 * plane + g]) && finite64(V[4 * plane + g]));
    }
    if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) scal[SC_NAN] = 1.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) sRed[tid >> 5] = m;
    __syncthreads();
    const unsigned nb = gridDim.x * gridDim.y;
    if (tid == 0) {
        for (int w = 1; w < 8; w++) m = fmin(m, sRed[w]);
        partials[blockIdx.y * gridDim.x + blockIdx.x] = m;
        __threadfence();
        sLast = (atomicAdd(ticket, 1u) == nb - 1);
    }
    __syncthreads();
    if (sLast) {
        __threadfence();
        double mm = CUDART_INF;
        for (unsigned i = tid; i < nb; i += 256) mm = fmin(mm, __ldcg(partials + i));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mm = fmin(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        __syncthreads();
        if ((tid & 31) == 0) sRed[tid >> 5] = mm;
        __syncthreads();
        if (tid == 0) {
            for (int w = 0; w < 8; w++) mm = fmin(mm, sRed[w]);
            scal[SC_DT] = finalize_dt(mm, (long long)P.npx * P.ny_glob);
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
static_assert(kDefaultWaitNs == kWaitNs, "one default wait limit");

cudaError_t set_wait_limit_stage64(unsigned long long ns) {
    return cudaMemcpyToSymbol(g_wait_limit_ns, &ns, sizeof(ns));
}

EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn f = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return f;
}

namespace {

struct Variant {
    int tx, ty, nthr, own;
    size_t smem;
    // order2 stage0, order2 stage1, order1, MUSCL-Hancock order2, MUSCL-Hancock order1
    void (*k[5])(Stage64Args);
};

template <int TX, int TY, int MINB, int NTHR = TX * TY, int OWN = 0>
Variant make_variant() {
    Variant v;
    v.tx = TX;
    v.ty = TY;
    v.nthr = NTHR;
    v.own = OWN;
    v.smem = Tile<TX, TY, NTHR>::smem(OWN == 2);
    v.k[0] = stage64_kernel<TX, TY, NTHR, MINB, 2, true, false, false, OWN>;
    v.k[1] = stage64_kernel<TX, TY, NTHR, MINB, 2, false, true, false, OWN>;
    v.k[2] = stage64_kernel<TX, TY, NTHR, MINB, 1, true, true, false, OWN>;
    v.k[3] = stage64_kernel<TX, TY, NTHR, MINB, 2, true, true, true, OWN>;
    v.k[4] = stage64_kernel<TX, TY, NTHR, MINB, 1, true, true, true, OWN>;
    return v;
}

const Variant &variant() {
    static Variant v = [] {
        const char *e = std::getenv("TSU_TILE64");
        if (e && !std::strcmp(e, "16x16")) return make_variant<16, 16, 2>();
        if (e && !std::strcmp(e, "32x16")) return make_variant<32, 16, 1>();
        if (e && !std::strcmp(e, "16x8")) return make_variant<16, 8, 4>();
        if (e && !std::strcmp(e, "32x4")) return make_variant<32, 4, 4>();
        if (e && !std::strcmp(e, "32x8t256")) return make_variant<32, 8, 2, 256>();
        if (e && !std::strcmp(e, "32x8t288")) return make_variant<32, 8, 2, 288>();
        if (e && !std::strcmp(e, "32x8t352")) return make_variant<32, 8, 2, 352>();
        if (e && !std::strcmp(e, "32x8t384")) return make_variant<32, 8, 2, 384>();
        if (e && !std::strcmp(e, "32x8t320reg")) return make_variant<32, 8, 2, 320, 0>();
        if (e && !std::strcmp(e, "32x8t320late")) return make_variant<32, 8, 2, 320, 1>();
        // default: 32 x 8 tile, 320 threads, 2 CTAs per SM (shared memory
        // allows 2; 20 warps per SM at 92-96 registers, no spills), the
        // second stage's U^n and extrema staged by TMA (OWN = 2, 107 KB of
        // shared memory per CTA).  Measured at 4096^2: 256 threads 2161, 288
        // 2308, 320 2514, 352 2365, 384 2331 Mcell-steps/s; with 320 threads
        // OWN = 0 / 1 / 2: 2533 / 2566 / 2585 (one box, 100 steps).  Every
        // choice is value-identical.
        return make_variant<32, 8, 2, 320, 2>();
    }();
    return v;
}

}  // namespace

size_t stage64_smem_bytes() { return variant().smem; }

cudaError_t stage64_prepare() {
    const Variant &v = variant();
    for (int i = 0; i < 5; i++) {
        cudaError_t e = cudaFuncSetAttribute(v.k[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

bool stage64_tma_maps(const double *bufA, const double *bufB, const unsigned char *mask, const double *const ext[3],
                      long long pitch, long long plane, int npx, int npy, CUtensorMap *tmA, CUtensorMap *tmB,
                      CUtensorMap *tmM, CUtensorMap *tmO, CUtensorMap tmE[3]) {
    EncodeTiledFn f = tensor_map_encoder();
    const Variant &v = variant();
    if (!f || npx < v.tx + 4 || npy < v.ty + 4) return false;
    if (reinterpret_cast<uintptr_t>(bufA) % 16 || reinterpret_cast<uintptr_t>(bufB) % 16 ||
        reinterpret_cast<uintptr_t>(mask) % 16 || pitch % 16)
        return false;
    for (int k = 0; k < 3; k++)
        if (reinterpret_cast<uintptr_t>(ext[k]) % 16) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)npx, (cuuint64_t)npy, 5};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(double), (cuuint64_t)plane * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)(v.tx + 4), (cuuint32_t)(v.ty + 4), 5};
    const cuuint32_t es[3] = {1, 1, 1};
    const double *bufs[2] = {bufA, bufB};
    CUtensorMap *maps[2] = {tmA, tmB};
    for (int k = 0; k < 2; k++)
        if (f(maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(bufs[k]), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    const cuuint64_t mdims[2] = {(cuuint64_t)npx, (cuuint64_t)npy};
    const cuuint64_t mstrides[1] = {(cuuint64_t)pitch};
    const cuuint32_t mbox[2] = {(cuuint32_t)(v.tx + 32), (cuuint32_t)(v.ty + 4)};  // Tile::MLX, LY
    if (f(tmM, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<unsigned char *>(mask), mdims, mstrides, mbox, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const cuuint32_t obox[3] = {(cuuint32_t)v.tx, (cuuint32_t)v.ty, 5};
    if (f(tmO, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(bufA), dims, strides, obox, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    for (int k = 0; k < 3; k++)
        if (f(&tmE[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(ext[k]), dims, strides, obox, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    return true;
}

dim3 stage64_grid(int npx, int npy) {
    const Variant &v = variant();
    return dim3((npx + v.tx - 1) / v.tx, (npy + v.ty - 1) / v.ty);
}

cudaError_t stage64_launch(int order, int stage, const Stage64Args &a, cudaStream_t st) {
    const Variant &v = variant();
    dim3 g = stage64_grid(a.phys.npx, a.phys.npy);
    int which = (order == 2) ? (stage == 0 ? 0 : 1) : 2;
    if (a.phys.rk == 0) which = (order == 2) ? 3 : 4;  // MUSCL-Hancock: one stage
    v.k[which]<<<g, v.nthr, v.smem, st>>>(a);
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
    // enough for every tile shape and for the 32x8 initial-dt grid
    size_t a = (size_t)((npx + 15) / 16) * ((npy + 3) / 4);
    size_t b = (size_t)((npx + 31) / 32) * ((npy + 7) / 8);
    return a > b ? a : b;
}

}  // namespace tsu
