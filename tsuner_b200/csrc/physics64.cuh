// physics64.cuh -- FP64 point physics of the TSUNER scheme, evaluated in the
// reference's exact operation order so that the fused kernels reproduce the
// reference CUDA build bit for bit (both are compiled with -fmad=false, and
// double division and sqrt are IEEE round-to-nearest on the device).
//
// What differs from the reference is WHERE things are computed, not how:
// per-run constants (settling velocity, pow() terms, sqrt(FR), sqrt(OC)) are
// evaluated once per run with the reference expressions (TsuConsts), cell
// velocities are evaluated once per cell instead of five times, and face
// states / edge fluxes never leave shared memory.
#pragma once
#include <math_constants.h>

#include <cfloat>
#include <cstdint>

#include "tsuner_b200.h"

namespace tsu {

constexpr double kG = 9.81;              // Sim_parameters.hxx:34
constexpr double kEpsilon = DBL_EPSILON; // Sim_parameters.hxx:28
constexpr double kEps = 1e-6;            // Sim_parameters.hxx:35
constexpr double kVmax = 10.0;           // Sim_parameters.hxx:36

// Scalar parameters the stage kernels need, packed once per run.
struct Phys64 {
    double FR, eps_h, Opar, OC, Q, HQB, porosity, CFL, dx, dy, inv_dx, inv_dy;
    TsuConsts k;
    int npx, npy;
    int order, wbc, bedload, suspension, read_files, bedload_law;
    double grass_ag;
    int rk, manning;
    // Row slab of a decomposed grid: npy is the number of rows this solver
    // owns, starting at global row j0 of a grid of ny_glob rows; gs / gn
    // ghost rows (0 or 2) below / above the owned rows are stored in the
    // state and mask planes and filled by the halo exchange.  A whole grid
    // has ny_glob = npy, j0 = 0, gs = gn = 0.
    int ny_glob, j0, gs, gn;
    // 1: an edge whose two faces are both dry returns zero fluctuations
    // without evaluating the Riemann solver (see edge_flux)
    int dry_skip;
};

// IEEE quotient and square root with the zero cases answered directly:
// (+-0)/b for finite non-zero b is a zero with the XOR of the signs, and
// sqrt(+-0) = +-0.  Value-identical to `/` and sqrt(); still water and dry
// land make such operands the common case of this scheme.
__device__ __forceinline__ double ddiv(double a, double b) {
    if (a == 0.0 && b != 0.0 && isfinite(b)) return (signbit(a) != signbit(b)) ? -0.0 : 0.0;
    return a / b;
}
__device__ __forceinline__ double dsqrt(double x) { return (x == 0.0) ? x : sqrt(x); }
// As ddiv, also answering a non-zero, non-NaN numerator over a zero divisor
// (an infinity with the XOR of the signs).
__device__ __forceinline__ double ddiv_inf(double a, double b) {
    if (b == 0.0 && a != 0.0 && !isnan(a)) return (signbit(a) != signbit(b)) ? -CUDART_INF : CUDART_INF;
    return ddiv(a, b);
}

// x is neither NaN nor an infinity (exponent field not all ones), with
// integer instructions only (the FP64 pipe is the stage kernels' bottleneck)
__device__ __forceinline__ bool finite64(double x) { return (__double2hiint(x) & 0x7ff00000) != 0x7ff00000; }

// SGN (Sim_parameters.hxx:29)
__device__ __forceinline__ int sgn(double x) { return (fabs(x) < kEpsilon) ? 0 : ((x) > 0) ? 1 : -1; }

// u_calculator_double (GPU/SedFlux.cuh:39-49).  `modb` receives the modulus
// of the returned velocity exactly as bedload() recomputes it
// (GPU/SedFlux.cuh:157): when no clamping happened it is the same expression
// on the same operands, so it is reused instead of a second sqrt.
// A dry state (h < EPS) gives u = (q / (h + EPSILON)) * 0, i.e. a zero with
// the sign of q; that is produced directly when the operands are finite and
// h + EPSILON > 0, which is value-identical and skips two divisions.
__device__ __forceinline__ void velocity(double h, double qx, double qy, double &ux, double &uy, double &modb) {
    double d = h + kEpsilon;
    if (!(h >= kEps) && d > 0.0 && !isnan(qx) && !isnan(qy)) {
        ux = copysign(0.0, qx);
        uy = copysign(0.0, qy);
        modb = 0.0;
        return;
    }
    double u = ddiv(qx, d) * (double)(h >= kEps);
    double v = ddiv(qy, d) * (double)(h >= kEps);
    double modu = dsqrt(u * u + v * v);
    if (modu > kVmax) {
        u = u / modu * kVmax;
        v = v / modu * kVmax;
        modb = dsqrt(u * u + v * v);
    } else {
        modb = modu;
    }
    ux = u;
    uy = v;
}
__device__ __forceinline__ void velocity(double h, double qx, double qy, double &ux, double &uy) {
    double m;
    velocity(h, qx, qy, ux, uy, m);
}

// avg, the van-Leer-type limiter (GPU/Reconstructor.cu:19-31).  When the
// numerator is a (signed) zero -- slopes of opposite sign or a zero slope --
// the quotient equals the numerator, so the division is skipped.
__device__ __forceinline__ double limiter(double a, double b) {
    double aa = fabs(a), bb = fabs(b);
    double den = aa + bb;
    if (!(den > kEpsilon)) return 0.0;
    double num = a * bb + b * aa;
    if (num == 0.0) return num;
    return num / den;
}

// state_filter_double (GPU/SedFlux.cuh:118-132)
__device__ __forceinline__ void positivity_filter(double &h, double &qx, double &qy, double &hc) {
    h = h * (double)(h > 0.0);
    double c = ddiv(hc, h + kEpsilon);
    c = c * (double)(c > 0.0);
    double ux, uy;
    velocity(h, qx, qy, ux, uy);
    qx = h * ux;
    qy = h * uy;
    hc = h * c;
}

struct State5 {
    double h, qx, qy, H, hc;
};

// bedload (GPU/SedFlux.cuh:150-168), or the Grass law when selected; modu
// is |u| as bedload() computes it.  The Ashida-Michiue product
// K1*Q*max(O-OC,0)*max(sqrt(O)-sqrt(OC),0)*(h>HQB)*(h>5DS) has the sign of
// u (K1 = 17u/(|u|+eps), every other factor >= +0), so whenever one factor
// vanishes it is a zero with the sign of u and the return value -qb is
// -copysign(0, u): that case skips the division and the sqrt.
__device__ __forceinline__ double bedload_flux(const Phys64 &P, double h, double ux, double modu) {
    if (P.bedload_law == 1) return -ddiv(P.grass_ag * ux * modu * modu, 1.0 - P.porosity);
    double O = P.Opar * modu * modu;
    if (!isnan(O) && (O <= P.OC || h <= P.HQB || h <= P.k.DS5)) return -copysign(0.0, ux);
    double K1 = ddiv(17.0 * ux, modu + kEpsilon);
    double qb = K1 * P.Q * fmax(O - P.OC, 0.0) * fmax(dsqrt(O) - P.k.sqrt_OC, 0.0) *
                (double)(h > P.HQB) * (double)(h > P.k.DS5);
    return -qb;
}

// Cflux (GPU/SedFlux.cuh:171-179).  With the bedload switched off or a fixed
// bed, F[3] = bedload * 0 is a zero with the sign of the bedload, i.e.
// -copysign(0, u) (NaN when |u| is NaN); produced without evaluating it.
__device__ __forceinline__ void phys_flux(const Phys64 &P, double h, double ux, double modu, double hc,
                                          int fixed, double uy, double F[5]) {
    F[0] = h * ux;
    F[1] = F[0] * ux;
    F[2] = F[0] * uy;
    if (fixed != 0 && P.bedload != 0) F[3] = bedload_flux(P, h, ux, modu) * (double)fixed * (double)P.bedload;
    else F[3] = isnan(modu) ? modu : -copysign(0.0, ux);
    F[4] = hc * ux;
}

// One edge: RiemannSolver_Vols (GPU/VolumeSolver.cu:19-126) with the
// rotation back of :129-152.  `a` is the state on the side the normal leaves
// (index 0 in the reference), `b` the state it enters.  Dm is the
// fluctuation into side a, Dp into side b, both in x/y components.
__device__ __forceinline__ void edge_flux(const Phys64 &P, const State5 &a, const State5 &b, int nx, int ny,
                                          int fixed, double Dm[5], double Dp[5]) {
    // Both faces dry (h == 0 exactly, which also excludes NaN): every
    // velocity, flux and depth below is a zero, the hydrostatic depths are
    // max(-H + min(H_a, H_b), 0) = 0, both wave speeds are 0, so a0 = a1 = 0
    // and all ten fluctuations evaluate to zeros.  They are returned as +0
    // (the full evaluation can give -0 for some; a zero's sign does not
    // reach any non-zero value of this scheme).  Dry land makes this the
    // common edge of a coastal grid.
    if (P.dry_skip && a.h == 0.0 && b.h == 0.0) {
#pragma unroll
        for (int i = 0; i < 5; i++) Dm[i] = Dp[i] = 0.0;
        return;
    }
    const double dnx = (double)nx, dny = (double)ny;
    double qlx = a.qx * dnx + a.qy * dny;
    double qly = a.qy * dnx - a.qx * dny;
    double qrx = b.qx * dnx + b.qy * dny;
    double qry = b.qy * dnx - b.qx * dny;
    double u0x, u0y, u1x, u1y, m0, m1;
    velocity(a.h, qlx, qly, u0x, u0y, m0);
    velocity(b.h, qrx, qry, u1x, u1y, m1);
    double c0 = ddiv(a.hc, a.h + kEpsilon);
    double c1 = ddiv(b.hc, b.h + kEpsilon);

    // hydrostatic reconstruction (:37-40)
    double zmH = fmin(a.H, b.H);
    double h0 = fmax(a.h - a.H + zmH, 0.0);
    double h1 = fmax(b.h - b.H + zmH, 0.0);
    double q0x = u0x * h0, q0y = u0y * h0;
    double q1x = u1x * h1, q1y = u1y * h1;
    double hc0 = h0 * c0, hc1 = h1 * c1;
    double deta = h1 - h0;

    double F0[5], F1[5];
    phys_flux(P, h0, u0x, m0, hc0, fixed, u0y, F0);
    phys_flux(P, h1, u1x, m1, hc1, fixed, u1y, F1);

    // Roe average + wave-speed bounds (GPU/SedFlux.cuh:181-199)
    double hm = 0.5 * (h0 + h1);
    double s0q = dsqrt(h0), s1q = dsqrt(h1);
    double umx = ddiv(s0q * u0x + s1q * u1x, s0q + s1q);
    double SL = u0x - dsqrt(kG * h0);
    double SR = u1x + dsqrt(kG * h1);
    double cm = dsqrt(kG * hm);
    SL = fmin(SL, umx - cm);
    SR = fmax(SR, umx + cm);

    double a0, a1;
    if (SR - SL > kEpsilon) {
        a0 = ddiv(SR * fabs(SL) - SL * fabs(SR), SR - SL);
        a1 = ddiv(fabs(SR) - fabs(SL), SR - SL);
    } else {
        a0 = fmax(fabs(SL), fabs(SR));
        a1 = 0.0;
    }

    double df[5], DU[5];
#pragma unroll
    for (int i = 0; i < 5; i++) df[i] = F1[i] - F0[i];
    df[1] += kG * hm * deta;
    DU[0] = h1 - h0;
    DU[1] = q1x - q0x;
    DU[2] = q1y - q0y;
    DU[3] = b.H - a.H;
    DU[4] = hc1 - hc0;
    double s0 = sgn(b.H - a.H);
    double s1 = sgn(df[3]);
    double s2 = sgn(a1);
    if (fabs(s0) > kEpsilon) s1 = s1 * s0;  // s0 is +-1: s1/s0 == s1*s0 exactly
    else s1 = 0.0;
    double vis[5];
#pragma unroll
    for (int i = 0; i < 5; i++) vis[i] = a0 * DU[i] + a1 * df[i];
    if (s2 == s1) vis[3] = a1 * df[3];
    else vis[3] = -a1 * df[3];
    double m[5], p[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        m[i] = 0.5 * (df[i] - vis[i]) + F0[i];
        p[i] = 0.5 * (df[i] + vis[i]) - F1[i];
    }
    Dm[0] = m[0];
    Dm[1] = (dnx * m[1] - dny * m[2]);
    Dm[2] = (dny * m[1] + dnx * m[2]);
    Dm[3] = m[3];
    Dm[4] = m[4];
    Dp[0] = p[0];
    Dp[1] = (dnx * p[1] - dny * p[2]);
    Dp[2] = (dny * p[1] + dnx * p[2]);
    Dp[3] = p[3];
    Dp[4] = p[4];
}

// MUSCL-Hancock half-step predictor (RK == 0, GPU/Reconstructor.cu:280-342)
// on a cell's four faces before the state filter: L/R along x, D/U along y.
// hi is the cell's depth, detx/dety its hydrostatic slopes (the pressure
// terms Tpx/Tpy of :199-201,276-278).  The face velocities are taken once,
// before any face is updated, and each update reads the faces as the
// previous ones left them -- the order of the reference.  Its bedload terms
// use bedload() directly (no mask, no BEDLOAD switch), as the reference does.
__device__ __forceinline__ void hancock_predictor(const Phys64 &P, double dt, double hi, double detx, double dety,
                                                  State5 &L, State5 &R, State5 &D, State5 &U) {
    const double Tpx = kG * hi * detx;
    const double Tpy = kG * hi * dety;
    double uRx, uRy, mR, uLx, uLy, mL, uUx, uUy, mU, uDx, uDy, mD;
    velocity(R.h, R.qx, R.qy, uRx, uRy, mR);
    velocity(L.h, L.qx, L.qy, uLx, uLy, mL);
    velocity(U.h, U.qx, U.qy, uUx, uUy, mU);
    velocity(D.h, D.qx, D.qy, uDx, uDy, mD);
    const double hdt = 0.5 * dt;
    double qhx = (R.qx - L.qx) * P.inv_dx;
    double qhy = (U.qy - D.qy) * P.inv_dy;
    double up = hdt * (qhx + qhy);
    L.h -= up;
    R.h -= up;
    D.h -= up;
    U.h -= up;
    qhx = (R.qx * uRx - L.qx * uLx) * P.inv_dx;
    qhy = (U.qx * uUy - D.qx * uDy) * P.inv_dy;
    up = hdt * (qhx + qhy);
    L.qx -= up;
    R.qx -= up;
    D.qx -= up;
    U.qx -= up;
    qhx = (R.qx * uRy - L.qx * uLy) * P.inv_dx;
    qhy = (U.qy * uUy - D.qy * uDy) * P.inv_dy;
    up = hdt * (qhx + qhy);
    L.qy -= up;
    R.qy -= up;
    D.qy -= up;
    U.qy -= up;
    qhx = (bedload_flux(P, R.h, uRx, mR) - bedload_flux(P, L.h, uLx, mL)) * P.inv_dx;
    qhy = (bedload_flux(P, U.h, uUx, mU) - bedload_flux(P, D.h, uDx, mD)) * P.inv_dy;
    up = hdt * (qhx + qhy);
    L.H -= up;
    R.H -= up;
    D.H -= up;
    U.H -= up;
    qhx = (R.hc * uRx - L.hc * uLx) * P.inv_dx;
    qhy = (U.hc * uUy - D.hc * uDy) * P.inv_dy;
    up = hdt * (qhx + qhy);
    L.hc -= up;
    R.hc -= up;
    D.hc -= up;
    U.hc -= up;
    up = hdt * P.inv_dx * Tpx;
    L.qx -= up;
    U.qx -= up;
    D.qx -= up;
    R.qx -= up;
    up = hdt * P.inv_dy * Tpy;
    L.qy -= up;
    U.qy -= up;
    D.qy -= up;
    R.qy -= up;
}

// interpolate_time (GPU/VolumeSolver.cu:172-203): boundary state from the
// CC series at segment `seg`; replaces h, H, qx, qy and zeroes hc.
__device__ __forceinline__ void series_state(const double *__restrict__ CC, const double *__restrict__ tCC,
                                             double t, int npx, int npy, int seg, State5 &g) {
    double dt = tCC[1] - tCC[0];
    int it = int((t - tCC[0]) / dt);
    it *= (it > 0);
    int tp = it + 1;
    long long nseg4 = (long long)(2 * npx + 2 * npy) * 4;
    long long posCC = it * nseg4 + (long long)seg * 4;
    long long posCCp = tp * nseg4 + (long long)seg * 4;
    double m = (CC[posCCp] - CC[posCC]) / dt;
    double b = CC[posCC] - m * tCC[it];
    double h1 = m * t + b;
    m = (CC[posCCp + 3] - CC[posCC + 3]) / dt;
    b = CC[posCC + 3] - m * tCC[it];
    double zb1 = m * t + b;
    h1 += zb1;
    m = (CC[posCCp + 1] - CC[posCC + 1]) / dt;
    b = CC[posCC + 1] - m * tCC[it];
    double qx = m * t + b;
    qx *= h1;
    m = (CC[posCCp + 2] - CC[posCC + 2]) / dt;
    b = CC[posCC + 2] - m * tCC[it];
    double qy = m * t + b;
    qy *= h1;
    g.h = h1;
    g.H = zb1;
    g.qx = qx;
    g.qy = qy;
    g.hc = 0.0;
}

// GetDeltaT per cell (GPU/Volume_kernel.cu:28-41)
__device__ __forceinline__ double cfl_dt(const Phys64 &P, double h, double qx, double qy) {
    double ux, uy;
    velocity(h, qx, qy, ux, uy);
    double cg = dsqrt(kG * h);
    double lx = fabs(ux) + cg;
    double ly = fabs(uy) + cg;
    return P.CFL * 0.5 * fmin(ddiv_inf(P.dx, lx), ddiv_inf(P.dy, ly));
}

}  // namespace tsu
