/*
 * oracle.c -- CPU restatement of the TSUNER finite-volume shallow-water +
 * Exner step (MUSCL reconstruction -> HLL-type edge fluxes with bedload ->
 * RK2 volume update -> CFL min-reduction).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library; the product path never
 * does.  It is the parity checker for the CUDA kernels and the timed CPU
 * baseline (the reference itself has no CPU solver).
 *
 * It follows the reference line by line, in the same operation order, and
 * keeps the reference's three-pass structure (reconstructor -> VolumeSolver
 * -> states_updater) with full face and flux arrays, so each function maps
 * onto one reference kernel.  Built with -O2 -ffp-contract=off so that every
 * expression rounds exactly as on the device (the reference is built with
 * -fmad=false, GPU/makefile:10).  Parity is pinned by running the reference's
 * own CUDA build (oracle/_ref) on the same inputs on a B200 and by the golden
 * fixtures under tests/golden/ produced that way.
 *
 * The only library function whose results may differ from the device is
 * pow(), used for two per-run constants; orc_* calls therefore accept the
 * device-evaluated constants (TsuConsts) and fall back to libm when given
 * NULL.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/tsuner_b200.h"

#define G_ 9.81              /* Sim_parameters.hxx:34 */
#define EPSILON_ DBL_EPSILON /* Sim_parameters.hxx:28 */
#define EPS_ 1e-6            /* Sim_parameters.hxx:35 */
#define VMAX_ 10.0           /* Sim_parameters.hxx:36 */

/* CUDA's double min()/max() (PTX min.f64/max.f64): a NaN operand yields the
 * other operand; otherwise the smaller/larger value. */
static inline double dmin(double a, double b)
{
    if (isnan(a)) return b;
    if (isnan(b)) return a;
    if (a == 0.0 && b == 0.0) return signbit(a) ? a : b; /* -0 < +0 */
    return (b < a) ? b : a;
}
static inline double dmax(double a, double b)
{
    if (isnan(a)) return b;
    if (isnan(b)) return a;
    if (a == 0.0 && b == 0.0) return signbit(a) ? b : a;
    return (b > a) ? b : a;
}

/* SGN, Sim_parameters.hxx:29 */
static inline int sgn(double x) { return (fabs(x) < EPSILON_) ? 0 : ((x) > 0) ? 1 : -1; }

/* u_calculator / u_calculator_double, GPU/SedFlux.cuh:26-49 */
static inline void vel(double h, double qx, double qy, double *ux, double *uy)
{
    double u = qx / (h + EPSILON_) * (double)(h >= EPS_);
    double v = qy / (h + EPSILON_) * (double)(h >= EPS_);
    double modu = sqrt(u * u + v * v);
    if (modu > VMAX_) {
        u = u / modu * VMAX_;
        v = v / modu * VMAX_;
    }
    *ux = u;
    *uy = v;
}

/* avg, GPU/Reconstructor.cu:19-31 */
static inline double avg(double a, double b)
{
    double aa = fabs(a), bb = fabs(b);
    if ((aa + bb) > EPSILON_) return (a * bb + b * aa) / (aa + bb);
    return 0.0;
}

/* state_filter / state_filter_double, GPU/SedFlux.cuh:103-132 */
static inline void filt(double *h, double *qx, double *qy, double *hc)
{
    double ux, uy, c;
    *h = *h * (double)(*h > 0.0);
    c = *hc / (*h + EPSILON_);
    c = c * (double)(c > 0.0);
    vel(*h, *qx, *qy, &ux, &uy);
    *qx = *h * ux;
    *qy = *h * uy;
    *hc = *h * c;
}

/* Per-run constants, GPU/Reconstructor.cu:64-77 and GPU/SedFlux.cuh:51-99,
 * 150-168; libm pow() stands in for the device pow() here. */
void orc_consts(const SimParams *p, TsuConsts *k)
{
    double nu = 1.002e-6;
    double s = p->R - 1.0;
    k->vs = sqrt((13.95 * nu / p->DS) * (13.95 * nu / p->DS) + 1.09 * s * G_ * p->DS) - 13.95 * nu / p->DS;
    k->Rp = (p->DS * sqrt(s * G_ * p->DS)) / nu;
    double a1, a2;
    if (k->Rp > 2.36) { a1 = 1; a2 = 0.6; } else { a1 = 0.586; a2 = 1.23; }
    k->A_er = a1 * pow(k->Rp, a2);
    k->sqrt_FR = sqrt(p->FR);
    k->VP = k->vs * (1 - p->porosity);
    k->K_dep = (1.64 + 0.4 * pow(p->DS / p->Dsg, 1.64));
    k->sqrt_OC = sqrt(p->OC);
    k->DS5 = 5 * p->DS;
}

typedef struct {
    SimParams p;
    TsuSwitches sw;
    TsuConsts k;
} Ctx;

/* bedload, GPU/SedFlux.cuh:150-168 (+ the optional Grass law, which has no
 * reference counterpart) */
static inline double bedload(const Ctx *C, double h, double ux, double uy)
{
    double u = ux;
    double modu = sqrt(ux * ux + uy * uy);
    if (C->sw.bedload_law == 1) {
        return -(C->sw.grass_ag * u * modu * modu / (1.0 - C->p.porosity));
    }
    double O = C->p.Opar * modu * modu;
    double K1 = 17.0 * u / (modu + EPSILON_);
    double qb = K1 * C->p.Q * dmax(O - C->p.OC, 0.0) * dmax(sqrt(O) - C->k.sqrt_OC, 0.0) *
                (double)(h > C->p.HQB) * (double)(h > C->k.DS5);
    return -qb;
}

/* Cflux, GPU/SedFlux.cuh:171-179 */
static inline void cflux(const Ctx *C, double h, double ux, double uy, double hc, double *F, int fixed)
{
    F[0] = h * ux;
    F[1] = F[0] * ux;
    F[2] = F[0] * uy;
    F[3] = bedload(C, h, ux, uy) * (double)fixed * (double)C->sw.bedload;
    F[4] = hc * ux;
}

/* RiemannSolver_Vols, GPU/VolumeSolver.cu:19-126: returns the one-sided
 * fluctuations Dm (into the `0` side) and Dp (into the `1` side), both
 * rotated back to x/y components (GPU/VolumeSolver.cu:129-152). */
static void riemann(const Ctx *C, double hhl, double zb0, double qlx, double qly, double hcl,
                    double hhr, double zb1, double qrx, double qry, double hcr, int nx, int ny,
                    int fixed, double Dmo[5], double Dpo[5])
{
    double qlnx = qlx * nx + qly * ny;
    double qlny = qly * nx - qlx * ny;
    double qrnx = qrx * nx + qry * ny;
    double qrny = qry * nx - qrx * ny;
    double u0x, u0y, u1x, u1y;
    vel(hhl, qlnx, qlny, &u0x, &u0y);
    vel(hhr, qrnx, qrny, &u1x, &u1y);
    double c0 = hcl / (hhl + EPSILON_);
    double c1 = hcr / (hhr + EPSILON_);

    double zmH = dmin(zb0, zb1);
    double h0 = dmax(hhl - zb0 + zmH, 0.0);
    double h1 = dmax(hhr - zb1 + zmH, 0.0);
    double q0x = u0x * h0, q0y = u0y * h0;
    double q1x = u1x * h1, q1y = u1y * h1;
    double hc0 = h0 * c0, hc1 = h1 * c1;
    double deta = h1 - h0;

    double F0[5], F1[5];
    cflux(C, h0, u0x, u0y, hc0, F0, fixed);
    cflux(C, h1, u1x, u1y, hc1, F1, fixed);

    /* roe_average, GPU/SedFlux.cuh:181-189 */
    double hm = 0.5 * (h0 + h1);
    double umx = (sqrt(h0) * u0x + sqrt(h1) * u1x) / (sqrt(h0) + sqrt(h1));

    /* calc_eigen_aprox0, GPU/SedFlux.cuh:192-199 */
    double SL = u0x - sqrt(G_ * h0);
    double SR = u1x + sqrt(G_ * h1);
    double cm = sqrt(G_ * hm);
    SL = dmin(SL, umx - cm);
    SR = dmax(SR, umx + cm);

    double a0, a1;
    if (SR - SL > EPSILON_) {
        a0 = (SR * fabs(SL) - SL * fabs(SR)) / (SR - SL);
        a1 = (fabs(SR) - fabs(SL)) / (SR - SL);
    } else {
        a0 = dmax(fabs(SL), fabs(SR));
        a1 = 0.0;
    }

    double df[5], vis[5], DU[5];
    for (int i = 0; i < 5; i++) df[i] = F1[i] - F0[i];
    df[1] += G_ * hm * deta;
    DU[0] = h1 - h0;
    DU[1] = q1x - q0x;
    DU[2] = q1y - q0y;
    DU[3] = zb1 - zb0;
    DU[4] = hc1 - hc0;
    double s0 = sgn(zb1 - zb0);
    double s1 = sgn(df[3]);
    double s2 = sgn(a1);
    if (fabs(s0) > EPSILON_) s1 = s1 / s0;
    else s1 = 0.0;
    for (int i = 0; i < 5; i++) vis[i] = a0 * DU[i] + a1 * df[i];
    if (s2 == s1) vis[3] = a1 * df[3];
    else vis[3] = -a1 * df[3];
    double Dm[5], Dp[5];
    for (int i = 0; i < 5; i++) {
        Dm[i] = 0.5 * (df[i] - vis[i]) + F0[i];
        Dp[i] = 0.5 * (df[i] + vis[i]) - F1[i];
    }
    Dmo[0] = Dm[0];
    Dmo[1] = (nx * Dm[1] - ny * Dm[2]);
    Dmo[2] = (ny * Dm[1] + nx * Dm[2]);
    Dmo[3] = Dm[3];
    Dmo[4] = Dm[4];
    Dpo[0] = Dp[0];
    Dpo[1] = (nx * Dp[1] - ny * Dp[2]);
    Dpo[2] = (ny * Dp[1] + nx * Dp[2]);
    Dpo[3] = Dp[3];
    Dpo[4] = Dp[4];
}

/* interpolate_time, GPU/VolumeSolver.cu:172-203 */
static void interp_time(const double *CC, const double *tCC, double t, int npx, int npy, int pos,
                        double *h1, double *zb1, double *q1x, double *q1y, double *hc1)
{
    double dt = tCC[1] - tCC[0];
    int it = (int)((t - tCC[0]) / dt);
    it *= (it > 0);
    int tp = it + 1;
    long posCC = (long)it * (2 * npx + 2 * npy) * 4 + (long)pos * 4;
    long posCCp = (long)tp * (2 * npx + 2 * npy) * 4 + (long)pos * 4;
    double m = (CC[posCCp] - CC[posCC]) / dt;
    double b = CC[posCC] - m * tCC[it];
    *h1 = m * t + b;
    m = (CC[posCCp + 3] - CC[posCC + 3]) / dt;
    b = CC[posCC + 3] - m * tCC[it];
    *zb1 = m * t + b;
    *h1 += *zb1;
    m = (CC[posCCp + 1] - CC[posCC + 1]) / dt;
    b = CC[posCC + 1] - m * tCC[it];
    *q1x = m * t + b;
    *q1x *= *h1;
    m = (CC[posCCp + 2] - CC[posCC + 2]) / dt;
    b = CC[posCC + 2] - m * tCC[it];
    *q1y = m * t + b;
    *q1y *= *h1;
    *hc1 = 0.0;
}

/* Arrays of stored rows.  A whole grid stores its ny rows.  A row slab of
 * a decomposed grid (not a reference feature: the reference runs one grid on
 * one GPU) owns global rows [j0, j1) and also stores gs / gn ghost rows below
 * / above them, copies of its neighbours' edge rows: stored row r is global
 * row j0 - gs + r, where rows below 0 or from ny up stand for the wrapped
 * rows of a periodic grid.  Every array is [5][stored rows][npx]. */
typedef struct {
    long nvol;                         /* cells per stored plane */
    double *V, *V0, *Vk;               /* 5*nvol each */
    double *rL, *rR, *rD, *rU;         /* 5*nvol each */
    double *FL, *FR, *FD, *FU;         /* 5*nvol each */
    double *dtv;                       /* nvol */
    int j0, j1, gs, gn, ny;            /* owned rows, ghost rows, global rows */
} Bufs;

static inline long rowpos(const Bufs *B, int npx, int j) { return (long)(j - (B->j0 - B->gs)) * npx; }

/* reconstructor, GPU/Reconstructor.cu:90-356 including friction (:33-55)
 * and erosion_deposition (:57-88).  Faces are built for the owned rows and,
 * in a slab, for the ghost row next to them (the far side of the slab's
 * edge); the working state Vk changes only in owned rows. */
static void reconstruct(const Ctx *C, Bufs *B, double dT, double inv_dx, double inv_dy)
{
    const SimParams *p = &C->p;
    const int npx = p->npx, ny = B->ny;
    const long nvol = B->nvol;
    double *V = B->V, *Vk = B->Vk, *V0 = B->V0;
    double *rL = B->rL, *rR = B->rR, *rD = B->rD, *rU = B->rU;
    const int periodic = (C->sw.wbc == 2);
    const int jr0 = B->j0 - (B->gs ? 1 : 0), jr1 = B->j1 + (B->gn ? 1 : 0);
#pragma omp parallel for schedule(static)
    for (int j = jr0; j < jr1; j++) {
        const int owned = (j >= B->j0 && j < B->j1);
        for (int i = 0; i < npx; i++) {
            long pos = rowpos(B, npx, j) + i;
            if (C->sw.order == 1) {
                for (int f = 0; f < 5; f++)
                    rL[f * nvol + pos] = rR[f * nvol + pos] = rU[f * nvol + pos] = rD[f * nvol + pos] = V[f * nvol + pos];
            } else {
                double uix, uiy, ulx, uly, urx, ury;
                double hi = V[pos];
                double Hi = V[3 * nvol + pos];
                double ci = V[4 * nvol + pos] / (hi + EPSILON_);
                /* x direction (:124-197) */
                int im = i - 1 * (i > 0), ip = i + 1 * (i < npx - 1);
                if (periodic) {
                    if (i == 0) im = npx - 1;
                    if (i == npx - 1) ip = 0;
                }
                long pl = rowpos(B, npx, j) + im, pr = rowpos(B, npx, j) + ip;
                double hl = V[pl], Hl = V[3 * nvol + pl], cl = V[4 * nvol + pl] / (hl + EPSILON_);
                double hr = V[pr], Hr = V[3 * nvol + pr], cr = V[4 * nvol + pr] / (hr + EPSILON_);
                double dta = dT * inv_dx;
                double dl = hi - hl, dr = hr - hi;
                double dh = avg(dl, dr);
                if (0.5 * fabs(dh) > hi) dh = 2.0 * hi * sgn(dh);
                rL[pos] = hi - 0.5 * dh;
                rR[pos] = hi + 0.5 * dh;
                double zm = dmin(Hl, Hi);
                dl = dmax(hi - Hi + zm, 0.0) - dmax(hl - Hl + zm, 0.0);
                zm = dmin(Hr, Hi);
                dr = dmax(hr - Hr + zm, 0.0) - dmax(hi - Hi + zm, 0.0);
                double deta = avg(dl, dr);
                double dz = dh - deta;
                rL[3 * nvol + pos] = Hi - 0.5 * dz;
                rR[3 * nvol + pos] = Hi + 0.5 * dz;
                vel(hi, V[1 * nvol + pos], V[2 * nvol + pos], &uix, &uiy);
                vel(hl, V[1 * nvol + pl], V[2 * nvol + pl], &ulx, &uly);
                vel(hr, V[1 * nvol + pr], V[2 * nvol + pr], &urx, &ury);
                dl = uix - ulx; dr = urx - uix;
                double du = avg(dl, dr);
                double dq = hi * du + uix * dh;
                rL[1 * nvol + pos] = V[1 * nvol + pos] - 0.5 * dq;
                rR[1 * nvol + pos] = V[1 * nvol + pos] + 0.5 * dq;
                dl = uiy - uly; dr = ury - uiy;
                du = avg(dl, dr);
                dq = hi * du + uiy * dh;
                rL[2 * nvol + pos] = V[2 * nvol + pos] - 0.5 * dq;
                rR[2 * nvol + pos] = V[2 * nvol + pos] + 0.5 * dq;
                dl = ci - cl; dr = cr - ci;
                du = avg(dl, dr);
                rL[4 * nvol + pos] = (ci - 0.5 * du) * rL[pos];
                rR[4 * nvol + pos] = (ci + 0.5 * du) * rR[pos];
                if (owned) Vk[1 * nvol + pos] -= dta * G_ * hi * deta;
                const double Tpx = G_ * hi * deta; /* :199-201, used by RK == 0 */

                /* y direction (:207-274): the stored neighbour row where there
                 * is one (a slab's ghost rows), else the reference's clamp or
                 * periodic wrap at the grid's own edge */
                int jm, jp;
                if (j - 1 >= B->j0 - B->gs) {
                    jm = j - 1;
                } else {
                    jm = j - 1 * (j > 0);
                    if (periodic && j == 0) jm = ny - 1;
                }
                if (j + 1 < B->j1 + B->gn) {
                    jp = j + 1;
                } else {
                    jp = j + 1 * (j < ny - 1);
                    if (periodic && j == ny - 1) jp = 0;
                }
                pl = rowpos(B, npx, jm) + i;
                pr = rowpos(B, npx, jp) + i;
                hl = V[pl]; Hl = V[3 * nvol + pl]; cl = V[4 * nvol + pl] / (hl + EPSILON_);
                hr = V[pr]; Hr = V[3 * nvol + pr]; cr = V[4 * nvol + pr] / (hr + EPSILON_);
                dta = dT * inv_dy;
                dl = hi - hl; dr = hr - hi;
                dh = avg(dl, dr);
                if (0.5 * fabs(dh) > hi) dh = 2.0 * hi * sgn(dh);
                rD[pos] = hi - 0.5 * dh;
                rU[pos] = hi + 0.5 * dh;
                zm = dmin(Hl, Hi);
                dl = dmax(hi - Hi + zm, 0.0) - dmax(hl - Hl + zm, 0.0);
                zm = dmin(Hr, Hi);
                dr = dmax(hr - Hr + zm, 0.0) - dmax(hi - Hi + zm, 0.0);
                deta = avg(dl, dr);
                dz = dh - deta;
                rD[3 * nvol + pos] = Hi - 0.5 * dz;
                rU[3 * nvol + pos] = Hi + 0.5 * dz;
                vel(hl, V[1 * nvol + pl], V[2 * nvol + pl], &ulx, &uly);
                vel(hr, V[1 * nvol + pr], V[2 * nvol + pr], &urx, &ury);
                dl = uix - ulx; dr = urx - uix;
                du = avg(dl, dr);
                dq = hi * du + uix * dh;
                rD[1 * nvol + pos] = V[1 * nvol + pos] - 0.5 * dq;
                rU[1 * nvol + pos] = V[1 * nvol + pos] + 0.5 * dq;
                dl = uiy - uly; dr = ury - uiy;
                du = avg(dl, dr);
                dq = hi * du + uiy * dh;
                rD[2 * nvol + pos] = V[2 * nvol + pos] - 0.5 * dq;
                rU[2 * nvol + pos] = V[2 * nvol + pos] + 0.5 * dq;
                dl = ci - cl; dr = cr - ci;
                du = avg(dl, dr);
                rD[4 * nvol + pos] = (ci - 0.5 * du) * rD[pos];
                rU[4 * nvol + pos] = (ci + 0.5 * du) * rU[pos];
                if (owned) Vk[2 * nvol + pos] -= dta * G_ * hi * deta;
                const double Tpy = G_ * hi * deta; /* :276-278 */

                if (C->sw.rk == 0) {
                    /* MUSCL-Hancock half-step predictor on the four unfiltered
                     * faces, :280-342 (velocities from the faces before it) */
                    double uRx, uRy, uLx, uLy, uUx, uUy, uDx, uDy;
                    const long q1 = nvol + pos, q2 = 2 * nvol + pos, q3 = 3 * nvol + pos, q4 = 4 * nvol + pos;
                    vel(rR[pos], rR[q1], rR[q2], &uRx, &uRy);
                    vel(rL[pos], rL[q1], rL[q2], &uLx, &uLy);
                    vel(rU[pos], rU[q1], rU[q2], &uUx, &uUy);
                    vel(rD[pos], rD[q1], rD[q2], &uDx, &uDy);
                    double qhx = (rR[q1] - rL[q1]) * inv_dx;
                    double qhy = (rU[q2] - rD[q2]) * inv_dy;
                    double up = 0.5 * dT * (qhx + qhy);
                    rL[pos] -= up; rR[pos] -= up; rD[pos] -= up; rU[pos] -= up;
                    qhx = (rR[q1] * uRx - rL[q1] * uLx) * inv_dx;
                    qhy = (rU[q1] * uUy - rD[q1] * uDy) * inv_dy;
                    up = 0.5 * dT * (qhx + qhy);
                    rL[q1] -= up; rR[q1] -= up; rD[q1] -= up; rU[q1] -= up;
                    qhx = (rR[q1] * uRy - rL[q1] * uLy) * inv_dx;
                    qhy = (rU[q2] * uUy - rD[q2] * uDy) * inv_dy;
                    up = 0.5 * dT * (qhx + qhy);
                    rL[q2] -= up; rR[q2] -= up; rD[q2] -= up; rU[q2] -= up;
                    qhx = (bedload(C, rR[pos], uRx, uRy) - bedload(C, rL[pos], uLx, uLy)) * inv_dx;
                    qhy = (bedload(C, rU[pos], uUx, uUy) - bedload(C, rD[pos], uDx, uDy)) * inv_dy;
                    up = 0.5 * dT * (qhx + qhy);
                    rL[q3] -= up; rR[q3] -= up; rD[q3] -= up; rU[q3] -= up;
                    qhx = (rR[q4] * uRx - rL[q4] * uLx) * inv_dx;
                    qhy = (rU[q4] * uUy - rD[q4] * uDy) * inv_dy;
                    up = 0.5 * dT * (qhx + qhy);
                    rL[q4] -= up; rR[q4] -= up; rD[q4] -= up; rU[q4] -= up;
                    up = 0.5 * dT * inv_dx * Tpx;
                    rL[q1] -= up; rU[q1] -= up; rD[q1] -= up; rR[q1] -= up;
                    up = 0.5 * dT * inv_dy * Tpy;
                    rL[q2] -= up; rU[q2] -= up; rD[q2] -= up; rR[q2] -= up;
                }

                /* filters (:344-348) */
                filt(&rL[pos], &rL[1 * nvol + pos], &rL[2 * nvol + pos], &rL[4 * nvol + pos]);
                filt(&rR[pos], &rR[1 * nvol + pos], &rR[2 * nvol + pos], &rR[4 * nvol + pos]);
                filt(&rU[pos], &rU[1 * nvol + pos], &rU[2 * nvol + pos], &rU[4 * nvol + pos]);
                filt(&rD[pos], &rD[1 * nvol + pos], &rD[2 * nvol + pos], &rD[4 * nvol + pos]);
            }
            /* friction, :33-55: Chezy (Manning == 0) or the reference's
             * unfinished Manning branch (:47-50), which multiplies by c */
            if (owned) {
                double h = V0[pos], ux, uy;
                vel(h, V0[1 * nvol + pos], V0[2 * nvol + pos], &ux, &uy);
                double modu = sqrt(ux * ux + uy * uy);
                double c = dT * p->FR * modu / (h + EPSILON_);
                if (C->sw.manning) {
                    c = dT * p->FR * p->FR * modu / (pow(h, 4.0 / 3.0));
                    Vk[1 * nvol + pos] *= c;
                    Vk[2 * nvol + pos] *= c;
                } else {
                    Vk[1 * nvol + pos] /= (1.0 + c);
                    Vk[2 * nvol + pos] /= (1.0 + c);
                }
            }
            /* erosion_deposition, :57-88, calculate_erosion/deposition SedFlux.cuh:51-99 */
            if (owned) {
                double h = V0[pos], ux, uy;
                double c = V0[4 * nvol + pos] / (h + p->epsilon_h);
                vel(h, V0[1 * nvol + pos], V0[2 * nvol + pos], &ux, &uy);
                double modu = sqrt(ux * ux + uy * uy);
                double Z = C->k.A_er * (modu * C->k.sqrt_FR) / C->k.vs;
                double Z5 = Z * Z * Z * Z * Z;
                double Es = (1.3e-7 * Z5) / (1 + 4.3e-7 * Z5);
                double Fe = C->k.VP * Es;
                if (Fe > 0.1) Fe = 0.1;
                Fe = Fe * (double)(Fe > 0.0);
                double Cb = C->k.K_dep * c;
                double Fd = C->k.vs * Cb;
                if (Fd > 0.1) Fd = 0.1;
                Fd = Fd * (double)(Fd > 0.0);
                double phi = (Fe - Fd) * (double)C->sw.suspension;
                Vk[3 * nvol + pos] -= dT * phi;
                Vk[4 * nvol + pos] += dT * phi;
            }
        }
    }
}

static inline void put(double *F, long nvol, long pos, const double D[5])
{
    for (int f = 0; f < 5; f++) F[f * nvol + pos] = D[f];
}

/* Boundary ghost of GPU/VolumeSolver.cu:233-255 etc.: wall mirror (WBC==1),
 * then the CC series while t < tCC[timeCC-2], else a wall mirror. */
static void ghost(const Ctx *C, const double *CC, const double *tCC, unsigned long timeCC, double t,
                  int seg, int normal_is_x, double q0x, double q0y, double *h1, double *zb1,
                  double *q1x, double *q1y, double *hc1)
{
    if (C->sw.wbc == 1) {
        if (normal_is_x) *q1x = -q0x; else *q1y = -q0y;
    }
    if (C->sw.read_files) {
        if (t < tCC[timeCC - 2]) {
            interp_time(CC, tCC, t, C->p.npx, C->p.npy, seg, h1, zb1, q1x, q1y, hc1);
        } else {
            if (normal_is_x) *q1x = -q0x; else *q1y = -q0y;
        }
    }
}

/* VolumeSolver, GPU/VolumeSolver.cu:217-408.  In a slab the edges of the
 * owned rows are evaluated: the horizontal edge between an owned row and a
 * ghost row is an interior edge (or, at a periodic grid's south / north
 * edge, the periodic seam of :352-367,378-387), and only the owned side's
 * fluctuation is used. */
static void volume_solver(const Ctx *C, Bufs *B, const int *fixH, double t, const double *CC,
                          const double *tCC, unsigned long timeCC)
{
    const int npx = C->p.npx, npy = C->p.npy;
    const long nvol = B->nvol;
    const double *rL = B->rL, *rR = B->rR, *rD = B->rD, *rU = B->rU;
    double *FL = B->FL, *FR = B->FR, *FD = B->FD, *FU = B->FU;
    const int periodic = (C->sw.wbc == 2);
#pragma omp parallel for schedule(static)
    for (int j = B->j0; j <= B->j1; j++) {
        for (int i = 0; i <= npx; i++) {
            double Dm[5], Dp[5];
            double h0, h1, zb0, zb1, hc0, hc1, q0x, q0y, q1x, q1y;
            if (j < B->j1) { /* vertical edges (:228-317) */
                long pos0 = i - 1 + rowpos(B, npx, j), pos1 = i + rowpos(B, npx, j);
                if (i == 0) {
                    if (!periodic) {
                        pos0 = pos1;
                        h1 = h0 = rL[pos0]; q1x = q0x = rL[nvol + pos0]; q1y = q0y = rL[2 * nvol + pos0];
                        zb1 = zb0 = rL[3 * nvol + pos0]; hc1 = hc0 = rL[4 * nvol + pos0];
                        ghost(C, CC, tCC, timeCC, t, 2 * npx + npy + j, 1, q0x, q0y, &h1, &zb1, &q1x, &q1y, &hc1);
                        riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, -1, 0, fixH[pos0], Dm, Dp);
                        put(FL, nvol, pos0, Dm);
                    }
                } else if (i == npx) {
                    h0 = rR[pos0]; q0x = rR[nvol + pos0]; q0y = rR[2 * nvol + pos0];
                    zb0 = rR[3 * nvol + pos0]; hc0 = rR[4 * nvol + pos0];
                    if (periodic) {
                        pos1 = rowpos(B, npx, j);
                        h1 = rL[pos1]; q1x = rL[nvol + pos1]; q1y = rL[2 * nvol + pos1];
                        zb1 = rL[3 * nvol + pos1]; hc1 = rL[4 * nvol + pos1];
                        if (C->sw.read_files) {
                            if (t < tCC[timeCC - 2])
                                interp_time(CC, tCC, t, npx, npy, npx + j, &h1, &zb1, &q1x, &q1y, &hc1);
                            else q1x = -q0x;
                        }
                    } else {
                        h1 = h0; q1x = q0x; q1y = q0y; zb1 = zb0; hc1 = hc0;
                        ghost(C, CC, tCC, timeCC, t, npx + j, 1, q0x, q0y, &h1, &zb1, &q1x, &q1y, &hc1);
                    }
                    riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 1, 0, fixH[pos0], Dm, Dp);
                    put(FR, nvol, pos0, Dm);
                    if (periodic) put(FL, nvol, pos1, Dp);
                } else {
                    h0 = rR[pos0]; q0x = rR[nvol + pos0]; q0y = rR[2 * nvol + pos0];
                    zb0 = rR[3 * nvol + pos0]; hc0 = rR[4 * nvol + pos0];
                    h1 = rL[pos1]; q1x = rL[nvol + pos1]; q1y = rL[2 * nvol + pos1];
                    zb1 = rL[3 * nvol + pos1]; hc1 = rL[4 * nvol + pos1];
                    riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 1, 0, fixH[pos0] * fixH[pos1], Dm, Dp);
                    put(FR, nvol, pos0, Dm);
                    put(FL, nvol, pos1, Dp);
                }
            }
            if (i < npx) { /* horizontal edges (:319-406) */
                long pos0 = i + rowpos(B, npx, j - 1), pos1 = i + rowpos(B, npx, j);
                if (j == 0 && B->gs == 0) {
                    if (!periodic) {
                        pos0 = pos1;
                        h1 = h0 = rD[pos0]; q1x = q0x = rD[nvol + pos0]; q1y = q0y = rD[2 * nvol + pos0];
                        zb1 = zb0 = rD[3 * nvol + pos0]; hc1 = hc0 = rD[4 * nvol + pos0];
                        ghost(C, CC, tCC, timeCC, t, i, 0, q0x, q0y, &h1, &zb1, &q1x, &q1y, &hc1);
                        riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 0, -1, fixH[pos0], Dm, Dp);
                        put(FD, nvol, pos0, Dm);
                    }
                } else if (j == npy && B->gn == 0) {
                    h0 = rU[pos0]; q0x = rU[nvol + pos0]; q0y = rU[2 * nvol + pos0];
                    zb0 = rU[3 * nvol + pos0]; hc0 = rU[4 * nvol + pos0];
                    if (periodic) {
                        pos1 = i + rowpos(B, npx, 0);
                        h1 = rD[pos1]; q1x = rD[nvol + pos1]; q1y = rD[2 * nvol + pos1];
                        zb1 = rD[3 * nvol + pos1]; hc1 = rD[4 * nvol + pos1];
                        if (C->sw.read_files) {
                            if (t < tCC[timeCC - 2])
                                interp_time(CC, tCC, t, npx, npy, npx + npy + i, &h1, &zb1, &q1x, &q1y, &hc1);
                            else q1y = -q0y;
                        }
                    } else {
                        h1 = h0; q1x = q0x; q1y = q0y; zb1 = zb0; hc1 = hc0;
                        ghost(C, CC, tCC, timeCC, t, npx + npy + i, 0, q0x, q0y, &h1, &zb1, &q1x, &q1y, &hc1);
                    }
                    riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 0, 1, fixH[pos0], Dm, Dp);
                    put(FU, nvol, pos0, Dm);
                    if (periodic) put(FD, nvol, pos1, Dp);
                } else if (periodic && (j == 0 || j == npy)) {
                    /* a slab's side of the periodic seam: the wrapped row is
                     * its ghost row; the same edge as the j == npy case above */
                    h0 = rU[pos0]; q0x = rU[nvol + pos0]; q0y = rU[2 * nvol + pos0];
                    zb0 = rU[3 * nvol + pos0]; hc0 = rU[4 * nvol + pos0];
                    h1 = rD[pos1]; q1x = rD[nvol + pos1]; q1y = rD[2 * nvol + pos1];
                    zb1 = rD[3 * nvol + pos1]; hc1 = rD[4 * nvol + pos1];
                    if (C->sw.read_files) {
                        if (t < tCC[timeCC - 2])
                            interp_time(CC, tCC, t, npx, npy, npx + npy + i, &h1, &zb1, &q1x, &q1y, &hc1);
                        else q1y = -q0y;
                    }
                    riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 0, 1, fixH[pos0], Dm, Dp);
                    put(FU, nvol, pos0, Dm);
                    put(FD, nvol, pos1, Dp);
                } else {
                    h0 = rU[pos0]; q0x = rU[nvol + pos0]; q0y = rU[2 * nvol + pos0];
                    zb0 = rU[3 * nvol + pos0]; hc0 = rU[4 * nvol + pos0];
                    h1 = rD[pos1]; q1x = rD[nvol + pos1]; q1y = rD[2 * nvol + pos1];
                    zb1 = rD[3 * nvol + pos1]; hc1 = rD[4 * nvol + pos1];
                    riemann(C, h0, zb0, q0x, q0y, hc0, h1, zb1, q1x, q1y, hc1, 0, 1, fixH[pos0] * fixH[pos1], Dm, Dp);
                    put(FU, nvol, pos0, Dm);
                    put(FD, nvol, pos1, Dp);
                }
            }
        }
    }
}

/* states_updater, GPU/Volume_kernel.cu:180-299: RK == 1 (:244-282) or
 * RK == 0 (:283-299: V and V0 get the filtered state, Vk keeps the
 * unfiltered one and carries it into the next step) */
static void update(const Ctx *C, Bufs *B, int k, double invx, double invy)
{
    const long nvol = B->nvol;
    const int npx = C->p.npx, nown = B->j1 - B->j0;
    double *Vk = B->Vk, *V0 = B->V0, *V = B->V;
    const double *FL = B->FL, *FR = B->FR, *FD = B->FD, *FU = B->FU;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)nown * npx; c++) { /* the owned cells */
        const long pos = rowpos(B, npx, B->j0 + (int)(c / npx)) + c % npx;
        for (int f = 0; f < 5; f++) {
            long q = f * nvol + pos;
            Vk[q] -= invx * (FL[q] + FR[q]) + invy * (FD[q] + FU[q]);
        }
        if (C->sw.rk == 0) {
            double h = Vk[pos], qx = Vk[nvol + pos], qy = Vk[2 * nvol + pos], hc = Vk[4 * nvol + pos];
            filt(&h, &qx, &qy, &hc);
            double out[5] = {h, qx, qy, Vk[3 * nvol + pos], hc};
            for (int f = 0; f < 5; f++) V[f * nvol + pos] = V0[f * nvol + pos] = out[f];
            continue;
        }
        double coef0 = 0.0 * (double)(k == 0) + 0.5 * (double)(k == 1);
        double coef1 = 1.0 - coef0;
        double h = coef0 * V0[pos] + coef1 * Vk[pos];
        double qx = coef0 * V0[nvol + pos] + coef1 * Vk[nvol + pos];
        double qy = coef0 * V0[2 * nvol + pos] + coef1 * Vk[2 * nvol + pos];
        double z = coef0 * V0[3 * nvol + pos] + coef1 * Vk[3 * nvol + pos];
        double hc = coef0 * V0[4 * nvol + pos] + coef1 * Vk[4 * nvol + pos];
        filt(&h, &qx, &qy, &hc);
        double out[5] = {h, qx, qy, z, hc};
        for (int f = 0; f < 5; f++) {
            Vk[f * nvol + pos] = out[f];
            V[f * nvol + pos] = out[f];
            if (k == C->sw.order - 1) V0[f * nvol + pos] = out[f];
        }
    }
}

/* GetDeltaT (GPU/Volume_kernel.cu:19-43) + MinReduction<double>
 * (GPU/Reduction_kernel_min.cu:155-196): for n > 4096 every device compare is
 * fminf on doubles, so the result is the float-rounded minimum; for n <= 4096
 * an exact host minimum.  Both are capped by the 1e30 start value. */
static double get_dt(const Ctx *C, const double *V, const Bufs *B)
{
    const SimParams *p = &C->p;
    const long nvol = B->nvol;
    const int npx = p->npx, nown = B->j1 - B->j0;
    double m = INFINITY;
    int any = 0;
#pragma omp parallel
    {
        double lm = INFINITY;
        int la = 0;
#pragma omp for schedule(static)
        for (long c = 0; c < (long)nown * npx; c++) { /* the owned cells */
            const long pos = rowpos(B, npx, B->j0 + (int)(c / npx)) + c % npx;
            double ux, uy;
            double h = V[pos];
            vel(h, V[nvol + pos], V[2 * nvol + pos], &ux, &uy);
            double cg = sqrt(G_ * h);
            double lx = fabs(ux) + cg;
            double ly = fabs(uy) + cg;
            double dt = p->CFL * 0.5 * dmin(p->dx / lx, p->dy / ly);
            if (!isnan(dt)) { lm = (la ? dmin(lm, dt) : dt); la = 1; }
        }
#pragma omp critical
        {
            if (la) { m = (any ? dmin(m, lm) : lm); any = 1; }
        }
    }
    if (!any) return 1e30;
    /* the rounding follows the whole grid's cell count (a slab's minimum is
     * rounded as the grid's would be; rounding is monotonic, so the minimum
     * over slabs of their rounded minima is the grid's) */
    if ((long)npx * B->ny > 4096) m = (double)(float)m;
    if (!(m < 1e30)) m = 1e30;
    return m;
}

double orc_initial_dt(const SimParams *p, const TsuSwitches *sw, const double *V, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Ctx C;
    C.p = *p;
    C.sw = *sw;
    orc_consts(p, &C.k);
    Bufs B;
    memset(&B, 0, sizeof(B));
    B.nvol = (long)p->npx * p->npy;
    B.j0 = 0;
    B.j1 = B.ny = p->npy;
    return get_dt(&C, V, &B);
}

/*
 * Runs the reference time loop (GPU/main_TSUNER.cu:142-197) on the host.
 * V: 5*nvol SoA state, in/out.  hmax/bmin/eta_max: running extrema, in/out
 * (bmin holds the running max of H; init with orc_init_extrema).  *t and *dt
 * are the simulated time and the next step's dt, in/out (*dt < 0 on entry:
 * compute the initial dt first).  nsteps >= 0 runs exactly that many steps,
 * nsteps < 0 runs while t < t_end.  kin: device-evaluated constants, or NULL
 * for libm ones.  Vk_io: the unfiltered working state that MUSCL-Hancock
 * (RK == 0) carries from step to step, in/out (NULL: it starts equal to V,
 * as at the start of the reference run, GPU/main_TSUNER.cu:113-115).
 * Returns the number of steps taken, or -1 on allocation failure / -2 on an
 * invalid boundary series.
 */
long orc_run(const SimParams *p, const TsuSwitches *sw, const TsuConsts *kin, double *V,
             const int *fixH, const double *CC, const double *tCC, unsigned long timeCC,
             double *hmax, double *bmin, double *eta_max, double *t, double *dt, long nsteps,
             double t_end, int nthreads, double *Vk_io)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Ctx C;
    C.p = *p;
    C.sw = *sw;
    if (kin) C.k = *kin;
    else orc_consts(p, &C.k);
    if (sw->read_files && timeCC < 2) return -2;
    Bufs B;
    B.nvol = (long)p->npx * p->npy;
    B.j0 = 0;
    B.j1 = B.ny = p->npy;
    B.gs = B.gn = 0;
    size_t n5 = (size_t)5 * B.nvol;
    double *mem = (double *)malloc(sizeof(double) * (n5 * 10 + B.nvol));
    if (!mem) return -1;
    B.V = V;
    B.V0 = mem;
    B.Vk = mem + n5;
    B.rL = mem + 2 * n5; B.rR = mem + 3 * n5; B.rD = mem + 4 * n5; B.rU = mem + 5 * n5;
    B.FL = mem + 6 * n5; B.FR = mem + 7 * n5; B.FD = mem + 8 * n5; B.FU = mem + 9 * n5;
    B.dtv = mem + 10 * n5;
    memset(B.FL, 0, sizeof(double) * n5 * 4);
    memcpy(B.V0, V, sizeof(double) * n5);
    memcpy(B.Vk, Vk_io ? Vk_io : V, sizeof(double) * n5);
    double inv_dx = 1.0 / p->dx, inv_dy = 1.0 / p->dy;
    double dT = *dt;
    if (dT < 0) dT = get_dt(&C, V, &B);
    double ct = *t;
    long it = 0;
    /* GPU/main_TSUNER.cu:169-174: `order` RK stages, or one MUSCL-Hancock stage */
    const int nstages = (sw->rk == 0) ? 1 : sw->order;
    while (nsteps >= 0 ? it < nsteps : ct < t_end) {
        for (int k = 0; k < nstages; k++) {
            reconstruct(&C, &B, dT, inv_dx, inv_dy);
            volume_solver(&C, &B, fixH, ct, CC, tCC, timeCC);
            update(&C, &B, k, dT * inv_dx, dT * inv_dy);
        }
        ct += dT;
        /* hmax/bmin/eta_max_calculator, GPU/Volume_kernel.cu:79-110 */
        if (hmax || bmin || eta_max) {
            const double eps_h = p->epsilon_h;
            const long nvol = B.nvol;
#pragma omp parallel for schedule(static)
            for (long pos = 0; pos < nvol; pos++) {
                double h = V[pos], H = V[3 * nvol + pos];
                if (hmax && h > eps_h) hmax[pos] = dmax(hmax[pos], h);
                if (bmin) bmin[pos] = dmax(bmin[pos], H);
                if (eta_max && h > eps_h) eta_max[pos] = dmax(eta_max[pos], h - H);
            }
        }
        dT = get_dt(&C, V, &B);
        it++;
    }
    *t = ct;
    *dt = dT;
    if (Vk_io) memcpy(Vk_io, B.Vk, sizeof(double) * n5);
    free(mem);
    return it;
}

/* ---- row slabs of a decomposed grid (the multi-GPU form; no reference
 * counterpart).  p is the WHOLE grid; the slab owns global rows [j0, j1) and
 * stores gs / gn ghost rows below / above them, so every array is
 * [5][gs + (j1 - j0) + gn][npx] (fixH [stored rows][npx]).  The caller fills
 * the ghost rows of V (the state the stage reads) and of fixH from the
 * neighbouring slabs before each stage. */
static void slab_bufs(const SimParams *p, int j0, int j1, int gs, int gn, Bufs *B)
{
    memset(B, 0, sizeof(*B));
    B->j0 = j0;
    B->j1 = j1;
    B->gs = gs;
    B->gn = gn;
    B->ny = p->npy;
    B->nvol = (long)p->npx * (gs + (j1 - j0) + gn);
}

/* Stage k of a step (GPU/main_TSUNER.cu:169-183: reconstructor,
 * VolumeSolver, states_updater) for the owned rows at time t with step dT.
 * V, V0, Vk are the reference's three state arrays for the stored rows.
 * Returns 0, or -1 on allocation failure. */
int orc_slab_stage(const SimParams *p, const TsuSwitches *sw, const TsuConsts *kin, int j0, int j1, int gs, int gn,
                   int k, double *V, double *V0, double *Vk, const int *fixH, const double *CC, const double *tCC,
                   unsigned long timeCC, double t, double dT, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Ctx C;
    C.p = *p;
    C.sw = *sw;
    if (kin) C.k = *kin;
    else orc_consts(p, &C.k);
    Bufs B;
    slab_bufs(p, j0, j1, gs, gn, &B);
    const size_t n5 = (size_t)5 * B.nvol;
    double *mem = (double *)calloc(n5 * 8, sizeof(double));
    if (!mem) return -1;
    B.V = V;
    B.V0 = V0;
    B.Vk = Vk;
    B.rL = mem; B.rR = mem + n5; B.rD = mem + 2 * n5; B.rU = mem + 3 * n5;
    B.FL = mem + 4 * n5; B.FR = mem + 5 * n5; B.FD = mem + 6 * n5; B.FU = mem + 7 * n5;
    const double inv_dx = 1.0 / p->dx, inv_dy = 1.0 / p->dy;
    reconstruct(&C, &B, dT, inv_dx, inv_dy);
    volume_solver(&C, &B, fixH, t, CC, tCC, timeCC);
    update(&C, &B, k, dT * inv_dx, dT * inv_dy);
    free(mem);
    return 0;
}

/* GetDeltaT + MinReduction over the owned rows, rounded as for the whole
 * grid: the minimum over all slabs of these values is the grid's dt. */
double orc_slab_dt(const SimParams *p, const TsuSwitches *sw, int j0, int j1, int gs, int gn, const double *V)
{
    Ctx C;
    C.p = *p;
    C.sw = *sw;
    orc_consts(p, &C.k);
    Bufs B;
    slab_bufs(p, j0, j1, gs, gn, &B);
    return get_dt(&C, V, &B);
}

/* hmax / bmin / eta_max_calculator (GPU/Volume_kernel.cu:79-110) on the owned
 * rows; the extrema arrays are [stored rows][npx] like V's planes. */
void orc_slab_extrema(const SimParams *p, int j0, int j1, int gs, int gn, const double *V, double *hmax,
                      double *bmin, double *eta_max)
{
    Bufs B;
    slab_bufs(p, j0, j1, gs, gn, &B);
    const long nvol = B.nvol;
    const int npx = p->npx;
    for (int j = j0; j < j1; j++)
        for (int i = 0; i < npx; i++) {
            const long pos = rowpos(&B, npx, j) + i;
            const double h = V[pos], H = V[3 * nvol + pos];
            if (h > p->epsilon_h) hmax[pos] = dmax(hmax[pos], h);
            bmin[pos] = dmax(bmin[pos], H);
            if (h > p->epsilon_h) eta_max[pos] = dmax(eta_max[pos], h - H);
        }
}

/* set_inicializacion*, GPU/Volume_kernel.cu:112-137 */
void orc_init_extrema(long nvol, double *hmax, double *bmin, double *eta_max)
{
    for (long i = 0; i < nvol; i++) {
        if (hmax) hmax[i] = -1e30;
        if (bmin) bmin[i] = -1e30;
        if (eta_max) eta_max[i] = -1e30;
    }
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
