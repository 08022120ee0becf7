// physics32.cuh -- point physics of the FP32 precision form.
//
// The scheme is the reference's (MUSCL faces, hydrostatic reconstruction,
// HLL-type fluctuations with the bedload flux, friction, erosion/deposition,
// RK2) evaluated in FP32 with FP64 kept where the stability of a shallow-
// water solver in single precision needs it:
//   * the free surface is carried as z = eta - eta0, an FP32 deviation from
//     the FP64 still-water level eta0, so lake at rest is exact (z == 0) and
//     eta differences are differences of small numbers;
//   * depths h = z + eta0 + H and the hydrostatic reconstruction
//     max(eta + min(H_l, H_r), 0) at edges (GPU/VolumeSolver.cu:37-40) are
//     evaluated in FP64, so wet/dry decisions at fronts are not decided by
//     FP32 rounding of eta0 + H;
//   * a dry cell stores z rounded toward -infinity, so its depth is exactly 0;
//   * time, dt and the global water/sediment sums stay FP64.
// Everything else uses single-precision arithmetic with hardware
// reciprocal / square-root approximations (the unit is built with
// -use_fast_math).
#pragma once
#include <math_constants.h>

#include "physics64.cuh"

namespace tsu {

constexpr float kGf = 9.81f;
constexpr float kEpsf = 1e-6f;   // velocity cutoff EPS (Sim_parameters.hxx:35)
constexpr float kVmaxf = 10.0f;  // VMAX (Sim_parameters.hxx:36)

// Depth margin above which an FP32 sum z + (eta0 + H) cannot change sign by
// rounding (FP32 relative error ~6e-8 on |eta0 + H| < 1e5 m).
constexpr float kWetMarginf = 1e-2f;

struct Phys32 {
    double eta0;  // still-water level (FP64)
    float eta0f;  // the same rounded to FP32 (only used beyond kWetMarginf)
    float FR, eps_h, Opar, OC, Q, HQB, porosity, CFL, dx, dy, inv_dx, inv_dy;
    float vs, A_er, sqrt_FR, VP, K_dep, sqrt_OC, DS5, inv_vs;
    int npx, npy;
    int order, wbc, bedload, suspension, read_files, bedload_law;
    float grass_ag;
    int dry_skip;  // as Phys64::dry_skip (edge32)
};

// x is neither NaN nor an infinity (exponent field not all ones)
__device__ __forceinline__ bool finite32(float x) { return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u; }

// Reciprocal: the hardware approximation (at most 2 ulp for |x| in
// [2^-126, 2^126]) refined by one Newton-Raphson step for 1/x,
// r1 = r0 + r0 (1 - x r0), as two fused multiply-adds.  Every argument here
// is a normal float (depths and speeds above a positive threshold), so the
// special-case handling of the correctly rounded __frcp_rn is not needed.
__device__ __forceinline__ float rcp32(float x) {
    const float r0 = __fdividef(1.0f, x);
    return __fmaf_rn(r0, __fmaf_rn(-x, r0, 1.0f), r0);
}

// Depth from the stored surface deviation (FP64 island), and the stored
// deviation of a dry cell (rounded down so that z + eta0 + H <= 0 exactly).
__device__ __forceinline__ double depth64(float z, float H, double eta0) {
    return fmax((double)z + eta0 + (double)H, 0.0);
}
__device__ __forceinline__ float dry_z(float H, double eta0) { return __double2float_rd(-((double)H + eta0)); }

// u_calculator (GPU/SedFlux.cuh:26-36) in FP32, given r = 1/h (read only
// when h >= EPS), so that a caller that also divides by h computes the
// reciprocal once.
__device__ __forceinline__ void velocity32r(float h, float r, float qx, float qy, float &ux, float &uy,
                                            float &modu) {
    if (h >= kEpsf) {
        ux = qx * r;
        uy = qy * r;
        float m2 = ux * ux + uy * uy;
        if (m2 > kVmaxf * kVmaxf) {
            float s = kVmaxf * rsqrtf(m2);
            ux *= s;
            uy *= s;
            modu = kVmaxf;
        } else {
            modu = sqrtf(m2);
        }
    } else {
        ux = uy = 0.f;
        modu = 0.f;
    }
}

__device__ __forceinline__ void velocity32(float h, float qx, float qy, float &ux, float &uy, float &modu) {
    velocity32r(h, h >= kEpsf ? rcp32(h) : 0.f, qx, qy, ux, uy, modu);
}

// avg (GPU/Reconstructor.cu:19-31): (a|b| + b|a|)/(|a|+|b|) equals
// 2ab/(a+b) when a and b have the same sign and 0 otherwise.
__device__ __forceinline__ float limiter32(float a, float b) {
    float p = a * b;
    return (p > 0.f) ? __fdividef(2.f * p, a + b) : 0.f;
}

// A reconstructed face after the state filter: depth, surface deviation,
// (clamped) velocity, bed, concentration.  The edge flux works on velocity
// and concentration, so they are kept instead of discharge and load.
struct Face32 {
    float h, z, u, v, H, c;
};

// state_filter (GPU/SedFlux.cuh:103-117) of a face with discharges qx, qy and
// concentration cf (load / depth); a clipped face becomes a dry face (z from
// its bed).
__device__ __forceinline__ void filter32(Face32 &f, float qx, float qy, float cf, double eta0) {
    if (!(f.h > 0.f)) {
        f.h = 0.f;
        f.u = f.v = 0.f;
        f.c = 0.f;
        f.z = dry_z(f.H, eta0);
        return;
    }
    float m;
    velocity32(f.h, qx, qy, f.u, f.v, m);
    f.c = fmaxf(cf, 0.f);
}

// bedload (GPU/SedFlux.cuh:150-168) / Grass law.
__device__ __forceinline__ float bedload32(const Phys32 &P, float h, float ux, float modu) {
    if (P.bedload_law == 1) return -(P.grass_ag * ux * modu * modu / (1.f - P.porosity));
    float O = P.Opar * modu * modu;
    if (O <= P.OC || h <= P.HQB || h <= P.DS5) return 0.f;
    float K1 = 17.f * ux * rcp32(modu);
    return -(K1 * P.Q * (O - P.OC) * fmaxf(sqrtf(O) - P.sqrt_OC, 0.f));
}

// One edge (RiemannSolver_Vols, GPU/VolumeSolver.cu:19-126) in the rotated
// frame.  a leaves along the normal, b is entered.  Normal-frame velocities:
// un = n.u, ut = n x u (the faces' filtered velocities, so the division of
// the reference's u_calculator is not repeated here).  Outputs Dm (into a),
// Dp (into b) in the normal frame (components h, qn, qt, H, hc).
__device__ __forceinline__ void edge32(const Phys32 &P, const Face32 &a, float u0, float v0, const Face32 &b,
                                       float u1, float v1, int fixed, float Dm[5], float Dp[5]) {
    // both faces dry: zero fluctuations (the FP64 edge_flux gives the reason)
    if (P.dry_skip && a.h == 0.f && b.h == 0.f) {
#pragma unroll
        for (int i = 0; i < 5; i++) Dm[i] = Dp[i] = 0.f;
        return;
    }
    const float c0 = a.c, c1 = b.c;
    // hydrostatic reconstruction h* = max(eta + min(H_a, H_b), 0), eta = z + eta0:
    // on an edge that is wet by a clear margin on both sides the depths are
    // formed in FP32 and their difference is the exact difference of the
    // surface deviations; otherwise (fronts) both are evaluated in FP64.
    const float Hm = fminf(a.H, b.H);
    const float Kf = P.eta0f + Hm;
    float h0, h1, deta;
    if (a.z + Kf > kWetMarginf && b.z + Kf > kWetMarginf) {
        h0 = a.z + Kf;
        h1 = b.z + Kf;
        deta = b.z - a.z;
    } else {
        const double K = P.eta0 + (double)Hm;
        const double h0d = fmax((double)a.z + K, 0.0), h1d = fmax((double)b.z + K, 0.0);
        h0 = (float)h0d;
        h1 = (float)h1d;
        deta = (float)(h1d - h0d);
    }
    float F0[5], F1[5];
    F0[0] = h0 * u0;
    F0[1] = F0[0] * u0;
    F0[2] = F0[0] * v0;
    F0[4] = h0 * c0 * u0;
    F1[0] = h1 * u1;
    F1[1] = F1[0] * u1;
    F1[2] = F1[0] * v1;
    F1[4] = h1 * c1 * u1;
    if (fixed && P.bedload) {
        F0[3] = bedload32(P, h0, u0, sqrtf(u0 * u0 + v0 * v0));
        F1[3] = bedload32(P, h1, u1, sqrtf(u1 * u1 + v1 * v1));
    } else {
        F0[3] = F1[3] = 0.f;
    }
    const float s0 = sqrtf(h0), s1 = sqrtf(h1);
    const float hm = 0.5f * (h0 + h1);
    const float ss = s0 + s1;
    const float um = (ss > 0.f) ? (s0 * u0 + s1 * u1) * rcp32(ss) : CUDART_NAN_F;
    const float sg = 3.1320919526731650f;  // sqrt(9.81)
    float SL = u0 - sg * s0, SR = u1 + sg * s1;
    const float cm = sqrtf(kGf * hm);
    SL = fminf(SL, um - cm);
    SR = fmaxf(SR, um + cm);
    float a0, a1;
    const float dS = SR - SL;
    if (dS > 1e-30f) {
        const float r = rcp32(dS);
        a0 = (SR * fabsf(SL) - SL * fabsf(SR)) * r;
        a1 = (fabsf(SR) - fabsf(SL)) * r;
    } else {
        a0 = fmaxf(fabsf(SL), fabsf(SR));
        a1 = 0.f;
    }
    float df[5], DU[5];
#pragma unroll
    for (int i = 0; i < 5; i++) df[i] = F1[i] - F0[i];
    df[1] += kGf * hm * deta;
    DU[0] = deta;
    DU[1] = u1 * h1 - u0 * h0;
    DU[2] = v1 * h1 - v0 * h0;
    DU[3] = b.H - a.H;
    DU[4] = h1 * c1 - h0 * c0;
    // upwinding of the bed component (GPU/VolumeSolver.cu:100-120)
    const float dz = b.H - a.H;
    const int s0i = (dz > 0.f) - (dz < 0.f);
    int s1i = (df[3] > 0.f) - (df[3] < 0.f);
    const int s2i = (a1 > 0.f) - (a1 < 0.f);
    s1i = s0i ? s1i * s0i : 0;
    float vis[5];
#pragma unroll
    for (int i = 0; i < 5; i++) vis[i] = a0 * DU[i] + a1 * df[i];
    vis[3] = (s2i == s1i) ? a1 * df[3] : -a1 * df[3];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        Dm[i] = 0.5f * (df[i] - vis[i]) + F0[i];
        Dp[i] = 0.5f * (df[i] + vis[i]) - F1[i];
    }
}

// GetDeltaT per cell (GPU/Volume_kernel.cu:28-41) in FP32.
__device__ __forceinline__ float cfl_dt32(const Phys32 &P, float h, float qx, float qy) {
    float ux, uy, m;
    velocity32(h, qx, qy, ux, uy, m);
    float cg = sqrtf(kGf * h);
    float lx = fabsf(ux) + cg, ly = fabsf(uy) + cg;
    return P.CFL * 0.5f * fminf(P.dx / lx, P.dy / ly);
}

// The same from the velocity of the filtered state (the update has it).
__device__ __forceinline__ float cfl_dt32v(const Phys32 &P, float h, float ux, float uy) {
    float cg = sqrtf(kGf * h);
    float lx = fabsf(ux) + cg, ly = fabsf(uy) + cg;
    return P.CFL * 0.5f * fminf(P.dx / lx, P.dy / ly);
}

}  // namespace tsu
