// stage32.cu -- FP32 precision form: one fused kernel per RK stage, for a
// single grid (stage32_kernel) and for a batched ensemble of grids of uneven
// size in one persistent launch (ens32_kernel).
//
// Same pipeline as stage64.cu (tile + 2-cell halo in shared memory, faces,
// each edge once, cell update, on-device dt/extrema), on the FP32 state
// planes (z = eta - eta0, H, qx, qy, hc) with the FP64 islands of
// physics32.cuh.  The last stage also accumulates the FP64 global sums of
// water volume sum(h) and sediment volume sum(H + hc) (per-CTA partials,
// reduced by the last CTA of the grid in a fixed order: deterministic).
// Algorithmic bytes per cell-step: 5 planes x 4 B read+write per stage
// (stage 2 also reads U^n) = 100 B, mask 2 B, extrema 3 x 8 B = 126 B.
#include <cuda_runtime.h>

#include <cstdlib>

#include "async.cuh"
#include "physics32.cuh"
#include "stage32.h"

namespace tsu {

// Tile of TX x TY cells with a 2-cell halo.  In shared memory a row holds
// the HX = 4 cells left of the tile (so that a row starts at x0 - 4, a
// 16-byte aligned TMA coordinate for floats), the tile and 4 cells right of
// it; only the 2 halo cells on each side (LXC = TX + 4 columns) are used.
template <int TX_, int TY_>
struct T32 {
    static constexpr int TX = TX_, TY = TY_, NT = TX * TY;
    static constexpr int HX = 4, LXC = TX + 4, LX = TX + 2 * HX, LY = TY + 4, PS = LX * LY, PSC = LXC * LY;
    static constexpr int FXW = TX + 2, FYH = TY + 2;
    // per loaded cell: z, H, qx, qy, hc (loaded) + h, ux, uy, c (derived)
    static constexpr int kSV = 9 * PS, kFlux = 20 * TY * TX;
    static constexpr int kRegA = kSV > kFlux ? kSV : kFlux;
    static constexpr int kFx = 12 * TY * FXW, kFy = 12 * FYH * TX;  // 2 faces x 6 floats
    static constexpr int kDeta = 2 * TY * TX, kWarps = NT / 32;
    static constexpr int kFloats = kRegA + kFx + kFy + kDeta;
    // the 1-byte mask: rows of MLX = TX + 32 cells starting 16 left of the
    // tile (a 16-byte aligned TMA origin for bytes), 128-byte aligned
    static constexpr int MHX = 16, MLX = TX + 2 * MHX, MPS = MLX * LY;
    static constexpr size_t kMaskOff = (sizeof(float) * kFloats + sizeof(double) * 3 * kWarps + 127) / 128 * 128;
    // + 128: the base is rounded up to 128 bytes (TMA destination)
    static constexpr size_t smem() { return kMaskOff + MPS + 64 + 128; }
};

__device__ __forceinline__ int wrap_clamp32(int g, int n, bool periodic) {
    if (periodic) {
        g %= n;
        return g < 0 ? g + n : g;
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

// A face in shared memory: three planes of pairs (h, z), (u, v), (H, c),
// `stride` pairs apart; 8-byte accesses, consecutive items in consecutive
// pairs (no bank conflicts).
__device__ __forceinline__ void put_face(float2 *base, int stride, const Face32 &f) {
    base[0] = make_float2(f.h, f.z);
    base[stride] = make_float2(f.u, f.v);
    base[2 * stride] = make_float2(f.H, f.c);
}
__device__ __forceinline__ Face32 get_face(const float2 *base, int stride) {
    Face32 f;
    const float2 a = base[0], b = base[stride], c = base[2 * stride];
    f.h = a.x;
    f.z = a.y;
    f.u = b.x;
    f.v = b.y;
    f.H = c.x;
    f.c = c.y;
    return f;
}

// smem cell planes: 0 z, 1 H, 2 qx, 3 qy, 4 hc, 5 h, 6 ux, 7 uy, 8 c
template <int PS>
__device__ __forceinline__ void recon32(const Phys32 &P, const float *s, int c, int l, int r, Face32 &fm, Face32 &fp,
                                        float &deta) {
    const float hi = s[5 * PS + c], hl = s[5 * PS + l], hr = s[5 * PS + r];
    const float zi = s[c], zl = s[l], zr = s[r];
    const float Hi = s[PS + c], Hl = s[PS + l], Hr = s[PS + r];
    if (P.dry_skip && hi == 0.f && hl == 0.f && hr == 0.f) {
        // a dry stencil: every slope is 0, both faces are dry faces of bed
        // H_i (what filter32 makes of them) and deta = 0
        fm.h = fm.u = fm.v = fm.c = 0.f;
        fm.H = Hi;
        fm.z = dry_z(Hi, P.eta0);
        fp = fm;
        deta = 0.f;
        return;
    }
    float dh = limiter32(hi - hl, hr - hi);
    if (0.5f * fabsf(dh) > hi) dh = copysignf(2.f * hi, dh);
    // hydrostatic eta slope (GPU/Reconstructor.cu:157-162): differences of
    // max(eta + min(H), 0); exact z differences when both terms are clearly
    // wet, FP64 otherwise
    float dl, dr;
    {
        const float Hm = fminf(Hl, Hi), Kf = P.eta0f + Hm;
        if (zi + Kf > kWetMarginf && zl + Kf > kWetMarginf) {
            dl = zi - zl;
        } else {
            const double K = P.eta0 + (double)Hm;
            dl = (float)(fmax((double)zi + K, 0.0) - fmax((double)zl + K, 0.0));
        }
    }
    {
        const float Hm = fminf(Hr, Hi), Kf = P.eta0f + Hm;
        if (zr + Kf > kWetMarginf && zi + Kf > kWetMarginf) {
            dr = zr - zi;
        } else {
            const double K = P.eta0 + (double)Hm;
            dr = (float)(fmax((double)zr + K, 0.0) - fmax((double)zi + K, 0.0));
        }
    }
    deta = limiter32(dl, dr);
    const float dz = dh - deta;
    fm.h = hi - 0.5f * dh;
    fp.h = hi + 0.5f * dh;
    fm.H = Hi - 0.5f * dz;
    fp.H = Hi + 0.5f * dz;
    fm.z = zi - 0.5f * deta;
    fp.z = zi + 0.5f * deta;
    const float uix = s[6 * PS + c], uiy = s[7 * PS + c];
    float du = limiter32(uix - s[6 * PS + l], s[6 * PS + r] - uix);
    float dq = hi * du + uix * dh;
    const float qxm = s[2 * PS + c] - 0.5f * dq, qxp = s[2 * PS + c] + 0.5f * dq;
    du = limiter32(uiy - s[7 * PS + l], s[7 * PS + r] - uiy);
    dq = hi * du + uiy * dh;
    const float qym = s[3 * PS + c] - 0.5f * dq, qyp = s[3 * PS + c] + 0.5f * dq;
    const float ci = s[8 * PS + c];
    du = limiter32(ci - s[8 * PS + l], s[8 * PS + r] - ci);
    // face load (ci -+ dc/2) h_face: its concentration is ci -+ dc/2
    filter32(fm, qxm, qym, ci - 0.5f * du, P.eta0);
    filter32(fp, qxp, qyp, ci + 0.5f * du, P.eta0);
}

// One RK stage on tile (bx, by) of grid A.  blin / nb: linear index of the
// tile and number of tiles of this grid (for the end-of-step reduction).
// P: the grid's physical parameters (A.phys, or the ensemble's shared
// parameters with this member's grid fields).
// tm: TMA descriptors of the state buffers (single grid), or null (ensemble).
template <int TX, int TY, int ORDER, bool FIRST, bool LAST>
__device__ __forceinline__ void stage32_tile(const Stage32Args &A, const Phys32 &P, const Tma32 *tm, int bx, int by,
                                             unsigned blin, unsigned nb, float *smem_raw) {
    using T = T32<TX, TY>;
    constexpr int NT = T::NT, LX = T::LX, PS = T::PS, FXW = T::FXW, FYH = T::FYH, kWarps = T::kWarps;
    constexpr int HX = T::HX, LXC = T::LXC, PSC = T::PSC, MHX = T::MHX, MLX = T::MLX;
    float *smem32 = smem_align<128>(smem_raw);
    __shared__ uint64_t sBar;  // the tile's TMA load
    float *sV = smem32;
    // edge fluxes per cell side (4 directions): (f0, f1) and (f2, f3) as
    // float2 planes, f4 as a float plane; aliases the cell planes (dead by then)
    float2 *sFA = reinterpret_cast<float2 *>(smem32);  // [2][4][TY * TX]
    float *sFS = smem32 + 16 * TY * TX;                 // [4][TY * TX]
    float *sFx = smem32 + T::kRegA;
    float *sFy = sFx + T::kFx;
    // faces: [2 sides][3 pair planes][rows][columns] of float2
    float2 *sFx2 = reinterpret_cast<float2 *>(sFx), *sFy2 = reinterpret_cast<float2 *>(sFy);
    static_assert(T::kRegA % 2 == 0 && T::kFx % 2 == 0, "8-byte aligned face planes");
    float *sDeta = sFy + T::kFy;
    double *sRed = reinterpret_cast<double *>(sDeta + T::kDeta);  // [3][kWarps]
    unsigned char *sM = reinterpret_cast<unsigned char *>(smem32) + T::kMaskOff;
    __shared__ int sLast;

    // Global memory is accessed through explicit global-space loads and
    // stores: in the ensemble the buffer pointers come from a descriptor in
    // shared memory, and generic accesses through them are slower.
    const double t = __ldcg(A.scal + SC_T);
    if (!(t < __ldcg(A.scal + SC_TEND))) return;  // run_until predicate (uniform per grid)
    const double dtd = __ldcg(A.scal + SC_DT);
    const float dt = (float)dtd;
    const int npx = P.npx, npy = P.npy;
    const bool periodic = (P.wbc == 2);
    const int tid = threadIdx.x;
    const int x0 = bx * TX, y0 = by * TY;
    const long long pitch = A.pitch, plane = A.plane;
    const double eta0 = P.eta0;

    const float *Vin;
    const float *V0;
    float *Vout;
    int par = 0;
    if (ORDER == 2) {
        Vin = FIRST ? A.bufA : A.bufB;
        V0 = A.bufA;
        Vout = FIRST ? A.bufB : A.bufA;
    } else {
        par = (int)__ldcg(A.scal + SC_PAR);
        Vin = par ? A.bufB : A.bufA;
        V0 = Vin;
        Vout = par ? A.bufA : A.bufB;
    }

    // tile and halo inside the grid, not periodic: no clamping, and every
    // edge of the tile is an interior edge
    const bool inner = !periodic && x0 >= 2 && y0 >= 2 && x0 + TX + 2 <= npx && y0 + TY + 2 <= npy;

    // ---- phase 1: load z, H, qx, qy, hc (+mask) with a 2-cell halo.  With
    // descriptors, a tile whose 4-cell x-halo lies inside the grid stages the
    // 5 planes with one TMA box (origin x0 - 4: a multiple of 16 bytes); the
    // mask and the other tiles use ordinary loads of the needed cells.
    const bool use_tma =
        tm && tm->on && !periodic && x0 >= HX && y0 >= 2 && x0 + TX + HX <= npx && y0 + TY + 2 <= npy;
    if (use_tma && tid == 0) {
        mbar_init(&sBar, 1);
        mbar_init_fence();
        mbar_expect_tx(&sBar, 5 * PS * sizeof(float) + T::MPS);
        tma_load_3d(sV, (Vin == A.bufB) ? &tm->b : &tm->a, x0 - HX, y0 - 2, 0, &sBar);
        tma_load_2d(sM, &tm->m, x0 - MHX, y0 - 2, &sBar);
    }
    if (!use_tma) {
        for (int k = tid; k < PSC; k += NT) {
            const int ly = k / LXC, lxc = k - ly * LXC;
            const int idx = ly * LX + lxc + (HX - 2);
            int gx = x0 + lxc - 2, gy = y0 + ly - 2;
            if (!inner) {
                gx = wrap_clamp32(gx, npx, periodic);
                gy = wrap_clamp32(gy, npy, periodic);
            }
            const long long g = (long long)gy * pitch + gx;
#pragma unroll
            for (int f = 0; f < 5; f++) sV[f * PS + idx] = __ldg(Vin + f * plane + g);
            sM[ly * MLX + lxc + (MHX - 2)] = __ldg(A.mask + g);
        }
    }
    const int tx = tid % TX, ty = tid / TX;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool own = (gi < npx) && (gj < npy);
    const long long gown = (long long)(own ? gj : 0) * pitch + (own ? gi : 0);
    // U^n of the owned cell (second stage) and its running extrema are read
    // in the update; here they are only requested into L2, so that no
    // registers are held across the face and edge phases
    if (!FIRST) {
#pragma unroll
        for (int f = 0; f < 5; f++) prefetch_l2(V0 + f * plane + gown);
    }
    if (LAST && own) {
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
            }
            return;
        }
    }
    const int cidx = (ty + 2) * LX + (tx + HX);
    float vc[5];
#pragma unroll
    for (int f = 0; f < 5; f++) vc[f] = sV[f * PS + cidx];


    // ---- phase 2: depth, velocity, concentration per cell
    for (int k = tid; k < PSC; k += NT) {
        const int ly = k / LXC;
        const int idx = ly * LX + (k - ly * LXC) + (HX - 2);
        const float zz = sV[idx], HH = sV[PS + idx];
        const float hs = zz + (P.eta0f + HH);  // FP32 when clearly wet, FP64 near dryness
        const float h = (hs > kWetMarginf) ? hs : (float)depth64(zz, HH, eta0);
        float ux, uy, m;
        const float rh = (h > 0.f) ? rcp32(h) : 0.f;
        velocity32r(h, rh, sV[2 * PS + idx], sV[3 * PS + idx], ux, uy, m);
        sV[5 * PS + idx] = h;
        sV[6 * PS + idx] = ux;
        sV[7 * PS + idx] = uy;
        sV[8 * PS + idx] = (h > 0.f) ? fmaxf(sV[4 * PS + idx] * rh, 0.f) : 0.f;
    }
    __syncthreads();
    const float hcell = sV[5 * PS + cidx];

    // ---- phase 3: faces.  A thread's items: the x faces of its own cell,
    // its y faces, and (the first NFR threads) one fringe item: the x faces
    // of halo column -1 or TX, or the y faces of halo row -1 or TY.  One
    // call site of the reconstruction serves every item.
    constexpr int NFRX = 2 * TY, NFR = 2 * TY + 2 * TX;
    static_assert(NFR <= NT, "one fringe face item per thread at most");
    const int nk3 = (tid < NFR) ? 3 : 2;
#pragma unroll 1
    for (int k = 0; k < nk3; k++) {
        bool xdir;
        int lx, ly;
        if (k < 2) {
            xdir = (k == 0);
            lx = tx;
            ly = ty;
        } else if (tid < NFRX) {
            xdir = true;
            ly = tid >> 1;
            lx = (tid & 1) ? TX : -1;
        } else {
            const int j = tid - NFRX;
            xdir = false;
            lx = j >> 1;
            ly = (j & 1) ? TY : -1;
        }
        const int c = (ly + 2) * LX + (lx + HX);
        const int step = xdir ? 1 : LX;
        float2 *dst;
        int fstride, side, didx = -1;
        if (xdir) {
            dst = sFx2 + ly * FXW + (lx + 1);
            fstride = TY * FXW;
            side = 3 * TY * FXW;
            if (k == 0) didx = ty * TX + tx;
        } else {
            dst = sFy2 + (ly + 1) * TX + lx;
            fstride = FYH * TX;
            side = 3 * FYH * TX;
            if (k == 1) didx = TY * TX + ty * TX + tx;
        }
        Face32 fm, fp;
        if (ORDER == 2) {
            float deta;
            recon32<PS>(P, sV, c, c - step, c + step, fm, fp, deta);
            if (didx >= 0) sDeta[didx] = deta;
        } else {
            fm.h = sV[5 * PS + c];
            fm.z = sV[c];
            fm.H = sV[PS + c];
            fm.u = sV[6 * PS + c];
            fm.v = sV[7 * PS + c];
            fm.c = sV[8 * PS + c];
            fp = fm;
        }
        put_face(dst, fstride, fm);
        put_face(dst + side, fstride, fp);
    }
    __syncthreads();

    // ---- phase 4: edges.  One call site of the edge flux serves every kind
    // of edge, so the arithmetic (and its contraction into FMAs) of an edge
    // does not depend on which tile, tile shape or schedule computes it.
    constexpr int FS = TY * TX;
    const bool series_on = !inner && P.read_files && (t < __ldg(A.tCC + (A.timeCC - 2)));
    // A thread's items: the vertical edge east of its own cell, the
    // horizontal edge north of it, and (the first TX + TY threads) one fringe
    // edge: the west edge of row `tid` or the south edge of column tid - TY.
    constexpr int NFE = TX + TY;
    static_assert(NFE <= NT, "one fringe edge per thread at most");
    const int nk4 = (tid < NFE) ? 3 : 2;
#pragma unroll 1
    for (int k = 0; k < nk4; k++) {
        Face32 a, b;
        int sgnn = 1, fixed, seg = 0;
        bool bnd = false, seam = false;
        // vertical edge e (0..TX) of row r, or horizontal edge e (0..TY) of column c
        bool vert;
        int r, e, c;
        if (k == 0) {
            vert = true;
            r = ty;
            e = tx + 1;
            c = 0;
        } else if (k == 1) {
            vert = false;
            r = 0;
            e = ty + 1;
            c = tx;
        } else if (tid < TY) {
            vert = true;
            r = tid;
            e = 0;
            c = 0;
        } else {
            vert = false;
            r = 0;
            e = 0;
            c = tid - TY;
        }
        int outM = -1, outP = -1;  // flux slots: direction * FS + cell
        if (inner) {  // interior edges only (uniform per tile): no bounds or boundary cases
            if (vert) {
                a = get_face(sFx2 + (3 * TY + r) * FXW + e, TY * FXW);
                b = get_face(sFx2 + r * FXW + (e + 1), TY * FXW);
                fixed = (int)sM[(r + 2) * MLX + e + MHX - 1] * (int)sM[(r + 2) * MLX + e + MHX];
                if (e >= 1) outM = 1 * FS + r * TX + (e - 1);
                if (e < TX) outP = 0 * FS + r * TX + e;
            } else {
                a = get_face(sFy2 + (3 * FYH + e) * TX + c, FYH * TX);
                b = get_face(sFy2 + (e + 1) * TX + c, FYH * TX);
                fixed = (int)sM[(e + 1) * MLX + c + MHX] * (int)sM[(e + 2) * MLX + c + MHX];
                if (e >= 1) outM = 3 * FS + (e - 1) * TX + c;
                if (e < TY) outP = 2 * FS + e * TX + c;
            }
        } else if (vert) {
            const int ex = x0 + e, ey = y0 + r;
            if (ey >= npy || ex > npx) continue;
            const int ly = r + 2;
            const float2 *Rf = sFx2 + (3 * TY + r) * FXW + e;
            const float2 *Lf = sFx2 + r * FXW + (e + 1);
            if (periodic && (ex == 0 || ex == npx)) {
                a = get_face(Rf, TY * FXW);
                b = get_face(Lf, TY * FXW);
                fixed = sM[ly * MLX + e + MHX - 1];
                seam = true;
                seg = npx + ey;
                if (e >= 1) outM = 1 * FS + r * TX + (e - 1);
                if (e < TX) outP = 0 * FS + r * TX + e;
            } else if (ex == 0) {
                a = get_face(Lf, TY * FXW);
                sgnn = -1;
                fixed = sM[ly * MLX + e + MHX];
                bnd = true;
                seg = 2 * npx + npy + ey;
                outM = 0 * FS + r * TX + e;
            } else if (ex == npx) {
                a = get_face(Rf, TY * FXW);
                fixed = sM[ly * MLX + e + MHX - 1];
                bnd = true;
                seg = npx + ey;
                outM = 1 * FS + r * TX + (e - 1);
            } else {
                a = get_face(Rf, TY * FXW);
                b = get_face(Lf, TY * FXW);
                fixed = (int)sM[ly * MLX + e + MHX - 1] * (int)sM[ly * MLX + e + MHX];
                if (e >= 1) outM = 1 * FS + r * TX + (e - 1);
                if (e < TX) outP = 0 * FS + r * TX + e;
            }
        } else {
            const int ex = x0 + c, ey = y0 + e;
            if (ex >= npx || ey > npy) continue;
            const float2 *Uf = sFy2 + (3 * FYH + e) * TX + c;
            const float2 *Df = sFy2 + (e + 1) * TX + c;
            if (periodic && (ey == 0 || ey == npy)) {
                a = get_face(Uf, FYH * TX);
                b = get_face(Df, FYH * TX);
                fixed = sM[(e + 1) * MLX + c + MHX];
                seam = true;
                seg = npx + npy + ex;
                if (e >= 1) outM = 3 * FS + (e - 1) * TX + c;
                if (e < TY) outP = 2 * FS + e * TX + c;
            } else if (ey == 0) {
                a = get_face(Df, FYH * TX);
                sgnn = -1;
                fixed = sM[(e + 2) * MLX + c + MHX];
                bnd = true;
                seg = ex;
                outM = 2 * FS + e * TX + c;
            } else if (ey == npy) {
                a = get_face(Uf, FYH * TX);
                fixed = sM[(e + 1) * MLX + c + MHX];
                bnd = true;
                seg = npx + npy + ex;
                outM = 3 * FS + (e - 1) * TX + c;
            } else {
                a = get_face(Uf, FYH * TX);
                b = get_face(Df, FYH * TX);
                fixed = (int)sM[(e + 1) * MLX + c + MHX] * (int)sM[(e + 2) * MLX + c + MHX];
                if (e >= 1) outM = 3 * FS + (e - 1) * TX + c;
                if (e < TY) outP = 2 * FS + e * TX + c;
            }
        }
        if (bnd) {
            b = a;
            if (P.wbc == 1) {
                if (vert) b.u = -a.u;
                else b.v = -a.v;
            }
        }
        if ((bnd || seam) && P.read_files) {
            if (series_on) {  // GPU/VolumeSolver.cu:172-203 in FP64, then to the FP32 face
                State5 g;
                series_state(A.CC, A.tCC, t, npx, npy, seg, g);
                b.H = (float)g.H;
                b.h = (float)fmax(g.h, 0.0);
                b.z = (g.h > 0.0) ? (float)(g.h - g.H - eta0) : dry_z(b.H, eta0);
                float m;
                velocity32(b.h, (float)g.qx, (float)g.qy, b.u, b.v, m);
                b.c = 0.f;
            } else if (vert) {
                b.u = -a.u;
            } else {
                b.v = -a.v;
            }
        }
        // rotate to the edge normal: x edges n = (sgnn, 0), y edges n = (0, sgnn)
        const float una = vert ? sgnn * a.u : sgnn * a.v;
        const float uta = vert ? sgnn * a.v : -sgnn * a.u;
        const float unb = vert ? sgnn * b.u : sgnn * b.v;
        const float utb = vert ? sgnn * b.v : -sgnn * b.u;
        float Dm[5], Dp[5];
        edge32(P, a, una, uta, b, unb, utb, fixed, Dm, Dp);
        // back to x/y: x edges (nx = sgnn, ny = 0), y edges (nx = 0, ny = sgnn)
        const float m1 = vert ? sgnn * Dm[1] : -sgnn * Dm[2];
        const float m2 = vert ? sgnn * Dm[2] : sgnn * Dm[1];
        const float p1 = vert ? sgnn * Dp[1] : -sgnn * Dp[2];
        const float p2 = vert ? sgnn * Dp[2] : sgnn * Dp[1];
        if (outM >= 0) {
            sFA[outM] = make_float2(Dm[0], m1);
            sFA[4 * FS + outM] = make_float2(m2, Dm[3]);
            sFS[outM] = Dm[4];
        }
        if (outP >= 0) {
            sFA[outP] = make_float2(Dp[0], p1);
            sFA[4 * FS + outP] = make_float2(p2, Dp[3]);
            sFS[outP] = Dp[4];
        }
    }
    __syncthreads();

    // ---- phase 5: update (state: z, H, qx, qy, hc)
    float dtcell = CUDART_INF_F;
    double mass = 0.0, sed = 0.0;
    bool bad = false;  // last stage: the new state of the owned cell is not finite
    if (own) {
        float v0[5];
#pragma unroll
        for (int f = 0; f < 5; f++) v0[f] = FIRST ? vc[f] : __ldcg(V0 + f * plane + gown);
        float ex_h = 0.f, ex_b = 0.f, ex_e = 0.f;
        if (LAST) {
            ex_h = __ldcg(A.hmax + gown);
            ex_b = __ldcg(A.bmin + gown);
            ex_e = __ldcg(A.eta_max + gown);
        }
        float z = vc[0], H = vc[1], qx = vc[2], qy = vc[3], hc = vc[4];
        if (ORDER == 2) {
            qx -= dt * P.inv_dx * kGf * hcell * sDeta[ty * TX + tx];
            qy -= dt * P.inv_dy * kGf * hcell * sDeta[TY * TX + ty * TX + tx];
        }
        {  // friction + erosion/deposition from U^n (in the first stage U^n is
           // this stage's input, whose depth phase 2 already formed)
            const float h0 = FIRST ? hcell : (float)depth64(v0[0], v0[1], eta0);
            float ux, uy, modu;
            const float r0 = (h0 > 0.f) ? rcp32(h0) : 0.f;
            velocity32r(h0, r0, v0[2], v0[3], ux, uy, modu);
            const float cf = (h0 > 0.f) ? dt * P.FR * modu * r0 : 0.f;
            const float rf = rcp32(1.f + cf);
            qx *= rf;
            qy *= rf;
            const float c = (h0 + P.eps_h > 0.f) ? v0[4] * rcp32(h0 + P.eps_h) : 0.f;
            const float Z = P.A_er * modu * P.sqrt_FR * P.inv_vs;
            const float Z5 = Z * Z * Z * Z * Z;
            float Fe = P.VP * (1.3e-7f * Z5) * rcp32(1.f + 4.3e-7f * Z5);
            Fe = fminf(fmaxf(Fe, 0.f), 0.1f);
            float Fd = fminf(fmaxf(P.vs * P.K_dep * c, 0.f), 0.1f);
            const float phi = (Fe - Fd) * (float)P.suspension;
            H -= dt * phi;
            hc += dt * phi;
            z += dt * phi;  // z = h - H - eta0 and H decreased by dt*phi
        }
        const float invx = dt * P.inv_dx, invy = dt * P.inv_dy;
        const int cell = ty * TX + tx;
        float fl[4][5];  // the four sides' fluxes of this cell
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const float2 a = sFA[d * FS + cell], b = sFA[(4 + d) * FS + cell];
            fl[d][0] = a.x;
            fl[d][1] = a.y;
            fl[d][2] = b.x;
            fl[d][3] = b.y;
            fl[d][4] = sFS[d * FS + cell];
        }
        float dv[5];
#pragma unroll
        for (int f = 0; f < 5; f++)
            dv[f] = invx * (fl[0][f] + fl[1][f]) + invy * (fl[2][f] + fl[3][f]);
        z -= dv[0] - dv[3];
        qx -= dv[1];
        qy -= dv[2];
        H -= dv[3];
        hc -= dv[4];
        if (ORDER == 2 && !FIRST) {  // RK2 average with U^n (linear in z)
            z = 0.5f * (v0[0] + z);
            H = 0.5f * (v0[1] + H);
            qx = 0.5f * (v0[2] + qx);
            qy = 0.5f * (v0[3] + qy);
            hc = 0.5f * (v0[4] + hc);
        }
        const double hd = (double)z + eta0 + (double)H;
        float h, uxf = 0.f, uyf = 0.f;
        if (!(hd > 0.0)) {
            h = 0.f;
            z = dry_z(H, eta0);
            qx = qy = hc = 0.f;
        } else {
            h = (float)hd;
            float m;
            const float rh = rcp32(h);  // h > 0 here
            velocity32r(h, rh, qx, qy, uxf, uyf, m);
            const float c = fmaxf(hc * rh, 0.f);
            qx = h * uxf;
            qy = h * uyf;
            hc = h * c;
        }
        __stcg(Vout + gown, z);
        __stcg(Vout + plane + gown, H);
        __stcg(Vout + 2 * plane + gown, qx);
        __stcg(Vout + 3 * plane + gown, qy);
        __stcg(Vout + 4 * plane + gown, hc);
        if (LAST) {
            if (h > P.eps_h) {
                __stcg(A.hmax + gown, fmaxf(ex_h, h));
                __stcg(A.eta_max + gown, fmaxf(ex_e, (float)((double)z + eta0)));
            }
            __stcg(A.bmin + gown, fmaxf(ex_b, H));
            const float d = cfl_dt32v(P, h, uxf, uyf);
            if (!isnan(d)) dtcell = d;
            mass = fmax(hd, 0.0);
            sed = (double)H + (double)hc;
            bad = !(finite32(z) && finite32(H) && finite32(qx) && finite32(qy) && finite32(hc));
        }
    }

    if (LAST) {
        // a NaN / Inf anywhere in the new state is reported to the host
        if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) A.scal[SC_NAN] = 1.0;
        // dt: the minimum of non-negative floats (or +inf) is the minimum of
        // their bit patterns, one warp reduction instruction
        const unsigned mb = __reduce_min_sync(0xffffffffu, __float_as_uint(dtcell));
        // FP64 water / sediment sums: per-thread values through shared memory
        // (the face buffers are no longer needed), summed by warp 0 in a
        // fixed order (strided per lane, then a fixed shuffle tree)
        static_assert(T::kRegA % 2 == 0 && T::kFx >= 4 * NT, "sum buffer inside the face buffer");
        double *sSum = reinterpret_cast<double *>(sFx);
        sSum[tid] = mass;
        sSum[NT + tid] = sed;
        if ((tid & 31) == 0) sRed[tid >> 5] = (double)__uint_as_float(mb);
        __syncthreads();
        if (tid < 32) {
            double ms = 0.0, sd = 0.0;
            for (int k = tid; k < NT; k += 32) {
                ms += sSum[k];
                sd += sSum[NT + k];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ms += __shfl_xor_sync(0xffffffffu, ms, o);
                sd += __shfl_xor_sync(0xffffffffu, sd, o);
            }
            if (tid == 0) {
                double mm = sRed[0];
                for (int w = 1; w < kWarps; w++) mm = fmin(mm, sRed[w]);
                __stcg(A.partials + blin, mm);
                __stcg(A.partials + nb + blin, ms);
                __stcg(A.partials + 2 * nb + blin, sd);
                __threadfence();
                sLast = (atomicAdd(A.ticket, 1u) == nb - 1);
            }
        }
        __syncthreads();
        if (sLast) {
            __threadfence();
            // every thread owns a fixed strided subset and the tree below has a
            // fixed shape, so the FP64 sums do not depend on CTA timing
            double mm = CUDART_INF, ms = 0.0, sd = 0.0;
            for (unsigned i = tid; i < nb; i += NT) {
                mm = fmin(mm, __ldcg(A.partials + i));
                ms += __ldcg(A.partials + nb + i);
                sd += __ldcg(A.partials + 2 * nb + i);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mm = fmin(mm, __shfl_xor_sync(0xffffffffu, mm, o));
                ms += __shfl_xor_sync(0xffffffffu, ms, o);
                sd += __shfl_xor_sync(0xffffffffu, sd, o);
            }
            __syncthreads();
            if ((tid & 31) == 0) {
                sRed[tid >> 5] = mm;
                sRed[kWarps + (tid >> 5)] = ms;
                sRed[2 * kWarps + (tid >> 5)] = sd;
            }
            __syncthreads();
            if (tid == 0) {
                mm = sRed[0];
                ms = sRed[kWarps];
                sd = sRed[2 * kWarps];
                for (int w = 1; w < kWarps; w++) {
                    mm = fmin(mm, sRed[w]);
                    ms += sRed[kWarps + w];
                    sd += sRed[2 * kWarps + w];
                }
                A.scal[SC_T] = t + dtd;
                A.scal[SC_DT] = finalize_dt(mm, (long long)npx * npy);
                A.scal[SC_STEPS] += 1.0;
                A.scal[SC_MASS] = ms;
                A.scal[SC_SED] = sd;
                if (ORDER == 1) A.scal[SC_PAR] = (double)(1 - par);
                *A.ticket = 0u;
                __threadfence();
            }
        }
    }
}

// ---- single grid: one CTA per tile
template <int TX, int TY, int MINB, int ORDER, bool FIRST, bool LAST>
__global__ void __launch_bounds__(TX *TY, MINB)
    stage32_kernel(const __grid_constant__ Stage32Args A, const __grid_constant__ Tma32 M) {
    extern __shared__ __align__(16) float smem32[];
    stage32_tile<TX, TY, ORDER, FIRST, LAST>(A, A.phys, &M, blockIdx.x, blockIdx.y,
                                             blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, smem32);
}

// ---- ensemble: persistent CTAs walking the tile list of all members
// (static stride or a dynamic work counter); each member keeps its own
// time, dt (segmented min-reduction by the member's last CTA), extrema and
// sums.  The member descriptor (buffers) is staged in shared memory per
// tile; the physical parameters shared by all members come in as a kernel
// parameter (constant-bank operands in the flux arithmetic) and only the
// grid fields (size, spacing, still-water level, boundary switches) are
// taken from the member.
template <int TX, int TY, int MINB, int ORDER, bool FIRST, bool LAST>
__global__ void __launch_bounds__(TX *TY, MINB) ens32_kernel(EnsArgs E, Phys32 common) {
    extern __shared__ __align__(16) float smem32[];
    __shared__ Stage32Args sG;
    __shared__ unsigned sTile;
    unsigned tile = blockIdx.x;
    if (E.dynamic) {
        if (threadIdx.x == 0) sTile = atomicAdd(E.work, 1u);
        __syncthreads();
        tile = sTile;
    }
    while (tile < E.ntiles) {
        const int m = E.tile_member[tile];
        // the member's descriptor, one 8-byte word per thread (a copy by one
        // thread is a chain of dependent loads every tile waits for)
        static_assert(sizeof(Stage32Args) % 8 == 0 && sizeof(Stage32Args) / 8 <= TX * TY, "descriptor copy");
        if (threadIdx.x < sizeof(Stage32Args) / 8)
            reinterpret_cast<unsigned long long *>(&sG)[threadIdx.x] =
                __ldg(reinterpret_cast<const unsigned long long *>(&E.members[m].g) + threadIdx.x);
        __syncthreads();
        const unsigned lt = tile - E.members[m].tile0;
        const int ntx = E.members[m].ntx;
        Phys32 P = common;
        P.eta0 = sG.phys.eta0;
        P.eta0f = sG.phys.eta0f;
        P.dx = sG.phys.dx;
        P.dy = sG.phys.dy;
        P.inv_dx = sG.phys.inv_dx;
        P.inv_dy = sG.phys.inv_dy;
        P.npx = sG.phys.npx;
        P.npy = sG.phys.npy;
        P.wbc = sG.phys.wbc;
        P.read_files = sG.phys.read_files;
        stage32_tile<TX, TY, ORDER, FIRST, LAST>(sG, P, E.tmas ? E.tmas + m : nullptr, lt % ntx, lt / ntx, lt,
                                                 E.members[m].ntiles, smem32);
        __syncthreads();
        if (E.dynamic) {
            if (threadIdx.x == 0) sTile = atomicAdd(E.work, 1u);
            __syncthreads();
            tile = sTile;
            __syncthreads();
        } else {
            tile += gridDim.x;
        }
    }
}

__global__ void reset_work_kernel(unsigned *w) { *w = 0u; }

// FP64 host planes (device copy) -> FP32 state; and back.
__global__ void to32_kernel(const double *__restrict__ V64, long long pitch, long long plane, int npx, int npy,
                            double eta0, float *__restrict__ V32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= npx || j >= npy) return;
    const long long g = (long long)j * pitch + i;
    const double h = V64[g], H = V64[3 * plane + g];
    const float Hf = (float)H;
    V32[plane + g] = Hf;
    if (!(h <= 0.0)) {  // wet, or a NaN depth (kept, so that tsu_reset reports it)
        V32[g] = (float)(h - (double)Hf - eta0);
        V32[2 * plane + g] = (float)V64[plane + g];
        V32[3 * plane + g] = (float)V64[2 * plane + g];
        V32[4 * plane + g] = (float)V64[4 * plane + g];
    } else {
        V32[g] = dry_z(Hf, eta0);
        V32[2 * plane + g] = 0.f;
        V32[3 * plane + g] = 0.f;
        V32[4 * plane + g] = 0.f;
    }
}

__global__ void to64_kernel(const float *__restrict__ V32, long long pitch, long long plane, int npx, int npy,
                            double eta0, double *__restrict__ V64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= npx || j >= npy) return;
    const long long g = (long long)j * pitch + i;
    const float z = V32[g], H = V32[plane + g];
    V64[g] = depth64(z, H, eta0);
    V64[plane + g] = V32[2 * plane + g];
    V64[2 * plane + g] = V32[3 * plane + g];
    V64[3 * plane + g] = H;
    V64[4 * plane + g] = V32[4 * plane + g];
}

__global__ void widen_kernel(const float *__restrict__ a, double *__restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void fill32_kernel(float *p, long long n, float v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// initial dt on the FP32 state, same finalisation as the reference reduction
__global__ void __launch_bounds__(256) dt32_kernel(const float *__restrict__ V, long long pitch, long long plane,
                                                   Phys32 P, double *partials, unsigned *ticket, double *scal) {
    __shared__ double sRed[8];
    __shared__ int sLast;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int gi = blockIdx.x * blockDim.x + threadIdx.x, gj = blockIdx.y * blockDim.y + threadIdx.y;
    double m = CUDART_INF;
    bool bad = false;
    if (gi < P.npx && gj < P.npy) {
        long long g = (long long)gj * pitch + gi;
        float h = (float)depth64(V[g], V[plane + g], P.eta0);
        float d = cfl_dt32(P, h, V[2 * plane + g], V[3 * plane + g]);
        if (!isnan(d)) m = d;
        bad = !(finite32(V[g]) && finite32(V[plane + g]) && finite32(V[2 * plane + g]) &&
                finite32(V[3 * plane + g]) && finite32(V[4 * plane + g]));
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
            scal[SC_DT] = finalize_dt(mm, (long long)P.npx * P.npy);
            *ticket = 0u;
            __threadfence();
        }
    }
}

// ------------------------------------------------------------------ host side
cudaError_t set_wait_limit_stage32(unsigned long long ns) {
    return cudaMemcpyToSymbol(g_wait_limit_ns, &ns, sizeof(ns));
}

namespace {

struct Variant32 {
    int tx, ty, minb;
    size_t smem;
    void (*k[3])(Stage32Args, Tma32);
    void (*e[3])(EnsArgs, Phys32);
};

template <int TX, int TY, int MINB>
Variant32 make_variant32() {
    Variant32 v;
    v.tx = TX;
    v.ty = TY;
    v.minb = MINB;
    v.smem = T32<TX, TY>::smem();
    v.k[0] = stage32_kernel<TX, TY, MINB, 2, true, false>;
    v.k[1] = stage32_kernel<TX, TY, MINB, 2, false, true>;
    v.k[2] = stage32_kernel<TX, TY, MINB, 1, true, true>;
    v.e[0] = ens32_kernel<TX, TY, MINB, 2, true, false>;
    v.e[1] = ens32_kernel<TX, TY, MINB, 2, false, true>;
    v.e[2] = ens32_kernel<TX, TY, MINB, 1, true, true>;
    return v;
}

// tile W x H / minimum resident CTAs per SM (register budget)
const Variant32 *variants32(int *n) {
    static Variant32 v[9] = {make_variant32<32, 8, 2>(),  make_variant32<16, 16, 2>(), make_variant32<32, 16, 1>(),
                             make_variant32<64, 4, 2>(),  make_variant32<32, 8, 3>(),  make_variant32<16, 16, 3>(),
                             make_variant32<32, 8, 4>(),  make_variant32<32, 16, 2>(), make_variant32<16, 16, 4>()};
    if (n) *n = 9;
    return v;
}

// single-grid variant: TSU_TILE32 = index into variants32; default 32x8
// with 4 resident CTAs per SM (measured fastest at 4096^2: 32 warps per SM
// hide the fixed-latency dependencies of the flux arithmetic, 16 warps did
// not; 32x8 8579 vs 16x16 8429 Mcell-steps/s with the current code)
constexpr int kSingleDefault = 6;
int single_variant() {
    static int k = [] {
        int n;
        variants32(&n);
        const char *e = std::getenv("TSU_TILE32");
        const int i = e ? std::atoi(e) : kSingleDefault;
        return (i >= 0 && i < n) ? i : kSingleDefault;
    }();
    return k;
}

int which(int order, int stage) { return (order == 2) ? (stage == 0 ? 0 : 1) : 2; }

}  // namespace

bool stage32_tma_maps(int variant, const float *bufA, const float *bufB, const unsigned char *mask, long long pitch,
                      long long plane, int npx, int npy, Tma32 *out) {
    EncodeTiledFn f = tensor_map_encoder();
    int nv;
    variants32(&nv);
    if (variant < 0) variant = single_variant();
    if (variant >= nv) return false;
    const Variant32 &v = variants32(nullptr)[variant];
    const int lx = v.tx + 8, ly = v.ty + 4;  // T32<TX, TY>::LX, LY
    const int mlx = v.tx + 32;               // T32<TX, TY>::MLX
    if (!f || npx < lx || npy < ly) return false;
    if (reinterpret_cast<uintptr_t>(bufA) % 16 || reinterpret_cast<uintptr_t>(bufB) % 16 ||
        reinterpret_cast<uintptr_t>(mask) % 16 || pitch % 16)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)npx, (cuuint64_t)npy, 5};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(float), (cuuint64_t)plane * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)lx, (cuuint32_t)ly, 5};
    const cuuint32_t es[3] = {1, 1, 1};
    const float *bufs[2] = {bufA, bufB};
    CUtensorMap *maps[2] = {&out->a, &out->b};
    for (int k = 0; k < 2; k++)
        if (f(maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(bufs[k]), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    const cuuint64_t mdims[2] = {(cuuint64_t)npx, (cuuint64_t)npy};
    const cuuint64_t mstrides[1] = {(cuuint64_t)pitch};
    const cuuint32_t mbox[2] = {(cuuint32_t)mlx, (cuuint32_t)ly};
    if (f(&out->m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<unsigned char *>(mask), mdims, mstrides, mbox, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    return true;
}

bool phys32_shared(const Phys32 &a, const Phys32 &b) {
    Phys32 x = a, y = b;
    for (Phys32 *q : {&x, &y}) {  // clear the per-member grid fields
        q->eta0 = 0.0;
        q->eta0f = q->dx = q->dy = q->inv_dx = q->inv_dy = 0.f;
        q->npx = q->npy = q->wbc = q->read_files = 0;
    }
    return x.FR == y.FR && x.eps_h == y.eps_h && x.Opar == y.Opar && x.OC == y.OC && x.Q == y.Q && x.HQB == y.HQB &&
           x.porosity == y.porosity && x.CFL == y.CFL && x.vs == y.vs && x.A_er == y.A_er && x.sqrt_FR == y.sqrt_FR &&
           x.VP == y.VP && x.K_dep == y.K_dep && x.sqrt_OC == y.sqrt_OC && x.DS5 == y.DS5 && x.inv_vs == y.inv_vs &&
           x.order == y.order && x.bedload == y.bedload && x.suspension == y.suspension &&
           x.bedload_law == y.bedload_law && x.grass_ag == y.grass_ag;
}

int stage32_num_tiles() {
    int n;
    variants32(&n);
    return n;
}

void stage32_tile_shape(int variant, int *tx, int *ty, int *minb) {
    const Variant32 &v = variants32(nullptr)[variant];
    *tx = v.tx;
    *ty = v.ty;
    *minb = v.minb;
}

size_t stage32_smem_bytes() { return variants32(nullptr)[single_variant()].smem; }

cudaError_t stage32_prepare() {
    int n;
    const Variant32 *v = variants32(&n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < 3; i++) {
            cudaError_t e = cudaFuncSetAttribute(v[j].k[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v[j].smem);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(v[j].e[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v[j].smem);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

dim3 stage32_grid(int npx, int npy) {
    const Variant32 &v = variants32(nullptr)[single_variant()];
    return dim3((npx + v.tx - 1) / v.tx, (npy + v.ty - 1) / v.ty);
}

cudaError_t stage32_launch(int order, int stage, const Stage32Args &a, const Tma32 &tm, cudaStream_t st) {
    const Variant32 &v = variants32(nullptr)[single_variant()];
    dim3 g = stage32_grid(a.phys.npx, a.phys.npy);
    v.k[which(order, stage)]<<<g, v.tx * v.ty, v.smem, st>>>(a, tm);
    return cudaGetLastError();
}

cudaError_t ens32_launch(int variant, int order, int stage, const EnsArgs &e, const Phys32 &common, int ctas,
                         cudaStream_t st) {
    const Variant32 &v = variants32(nullptr)[variant];
    if (e.dynamic) reset_work_kernel<<<1, 1, 0, st>>>(e.work);
    v.e[which(order, stage)]<<<ctas, v.tx * v.ty, v.smem, st>>>(e, common);
    return cudaGetLastError();
}

int ens32_max_ctas_per_sm(int variant) {
    const Variant32 &v = variants32(nullptr)[variant];
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, v.e[1], v.tx * v.ty, v.smem);
    return n;
}

cudaError_t to32_launch(const double *V64, long long pitch, long long plane, int npx, int npy, double eta0, float *V32,
                        cudaStream_t st) {
    dim3 b(256), g((npx + 255) / 256, npy);
    to32_kernel<<<g, b, 0, st>>>(V64, pitch, plane, npx, npy, eta0, V32);
    return cudaGetLastError();
}

cudaError_t to64_launch(const float *V32, long long pitch, long long plane, int npx, int npy, double eta0, double *V64,
                        cudaStream_t st) {
    dim3 b(256), g((npx + 255) / 256, npy);
    to64_kernel<<<g, b, 0, st>>>(V32, pitch, plane, npx, npy, eta0, V64);
    return cudaGetLastError();
}

cudaError_t widen_launch(const float *a, double *b, long long n, cudaStream_t st) {
    widen_kernel<<<1184, 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

cudaError_t fill32_launch(float *p, long long n, float v, cudaStream_t st) {
    fill32_kernel<<<1184, 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t initial_dt32_launch(const float *V, long long pitch, long long plane, const Phys32 &P, double *partials,
                                unsigned *ticket, double *scal, cudaStream_t st) {
    dim3 b(32, 8), g((P.npx + 31) / 32, (P.npy + 7) / 8);
    dt32_kernel<<<g, b, 0, st>>>(V, pitch, plane, P, partials, ticket, scal);
    return cudaGetLastError();
}

}  // namespace tsu
