// amhd_physics.cuh -- per-cell and per-face device physics of the MHD step.
//
// Real = double reproduces the reference's float64 arithmetic operation by
// operation (the translation unit that instantiates it is built with
// -fmad=false, so no contraction changes a rounding); Real = float is the
// bulk of the fp32 path (built with contraction on).
//
// Formula order follows the reference routines cited on each function, which
// is what makes float64 results bit-identical to the reference's.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "aeromhd.h"

namespace amhd {

constexpr int NV = 10;
constexpr int NG = 2;
enum { RHO = 0, MX = 1, MY = 2, MZ = 3, BX = 4, BY = 5, BZ = 6, EN = 7, PSI = 8, RHOC = 9 };
enum { IVX = 1, IVY = 2, IVZ = 3, IPR = 7, ICLR = 9 };
constexpr double FLOOR_RHO = 1e-12;  // config.py:40
constexpr double FLOOR_PR = 1e-12;   // config.py:41

// numpy.maximum / numpy.minimum semantics (a NaN operand propagates)
template <typename R>
__device__ __forceinline__ R np_max(R a, R b) { return (a != a || a >= b) ? a : b; }
template <typename R>
__device__ __forceinline__ R np_min(R a, R b) { return (a != a || a <= b) ? a : b; }

// ---------------------------------------------------------------------------
// MUSCL slope (physics.py:325-328: van Leer harmonic mean; minmod optional)
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R limited_slope(R wm, R w0, R wp, int limiter)
{
    R dm = w0 - wm, dp = wp - w0;
    if (limiter == AMHD_LIMITER_MINMOD) {
        R ab = dm * dp;
        return (ab > R(0)) ? (fabs(dm) < fabs(dp) ? dm : dp) : R(0);
    }
    R ab = dm * dp;
    return (ab > R(0)) ? R(2.0) * ab / (dm + dp + R(1e-30)) : R(0);
}

// One face: cells a..a+3 along the normal -> (WL, WR) as physics.py:329-334
template <typename R>
__device__ __forceinline__ void muscl_pair(R w0, R w1, R w2, R w3, int limiter, R &l, R &r)
{
    l = w1 + R(0.5) * limited_slope(w0, w1, w2, limiter);
    r = w2 - R(0.5) * limited_slope(w1, w2, w3, limiter);
}

// ---------------------------------------------------------------------------
// HLLD (physics.py:43-276) -- one x-normal face, primitive input states in
// the slot order of config.py:19-22.  Floors as physics.py:63-70.
// ---------------------------------------------------------------------------
template <typename R>
struct Side {
    R rho, vx, vy, vz, by, bz, p, psi, c;
    R pt, e, vb, dS, rs, sq, vys, vzs, bys, bzs, es, vbs;
};

template <typename R>
__device__ __forceinline__ R fast_speed(const Side<R> &s, R gamma, R bx2)
{
    // physics.py:93-102
    R bm2 = bx2 + s.by * s.by + s.bz * s.bz;
    R a2 = gamma * s.p / s.rho;
    R tmp = a2 + bm2 / s.rho;
    R disc = tmp * tmp - R(4.0) * a2 * bx2 / s.rho;
    if (disc < R(0)) disc = R(0);
    return sqrt(fmax(R(0.5) * (tmp + sqrt(disc)), R(0)));
}

template <typename R>
__device__ __forceinline__ void star_prep(Side<R> &s, R S, R SM, R ptS, R bxf, R bx2, R eps_rel, R floor_rho)
{
    // physics.py:122-154 for one side
    R dsm = S - SM;
    if (fabs(dsm) < R(1e-14)) dsm = R(1e-14);
    s.rs = fmax(s.rho * s.dS / dsm, floor_rho);
    s.sq = sqrt(s.rs);
    R dn = s.rho * s.dS * dsm - bx2;
    if (fabs(dn) < eps_rel) dn = (dn >= R(0)) ? eps_rel : -eps_rel;
    s.vys = s.vy - bxf * s.by * (SM - s.vx) / dn;
    s.vzs = s.vz - bxf * s.bz * (SM - s.vx) / dn;
    s.bys = s.by * (s.rho * s.dS * s.dS - bx2) / dn;
    s.bzs = s.bz * (s.rho * s.dS * s.dS - bx2) / dn;
    s.vbs = SM * bxf + s.vys * s.bys + s.vzs * s.bzs;
    s.es = ((S - s.vx) * s.e - s.pt * s.vx + ptS * SM + bxf * (s.vb - s.vbs)) / dsm;
    // keep S - SM for the caller's region selection (unused otherwise)
    s.dS = s.dS;
}

// side flux (physics.py:202-211, identical to the supersonic branches :178-198)
template <typename R>
__device__ __forceinline__ void side_flux(const Side<R> &s, R bxf, R bx2, R psif, R ch, R f[NV])
{
    f[0] = s.rho * s.vx;
    f[1] = s.rho * s.vx * s.vx + s.pt - bx2;
    f[2] = s.rho * s.vy * s.vx - bxf * s.by;
    f[3] = s.rho * s.vz * s.vx - bxf * s.bz;
    f[4] = (ch > R(0)) ? psif : R(0);
    f[5] = s.by * s.vx - bxf * s.vy;
    f[6] = s.bz * s.vx - bxf * s.vz;
    f[7] = (s.e + s.pt) * s.vx - bxf * s.vb;
    f[8] = (ch > R(0)) ? bxf * ch * ch : R(0);
    f[9] = s.rho * s.c * s.vx;
}

// f: flux; returns the face's signal speed max(|SL|, |SR|) (physics.py:108)
template <typename R>
__device__ __forceinline__ R hlld_flux(const R wl[NV], const R wr[NV], R gamma, R ch, R f[NV])
{
    const R floor_rho = R(FLOOR_RHO), floor_pr = R(FLOOR_PR);
    const R gm1 = gamma - R(1.0);
    Side<R> L, Rt;
    L.rho = wl[0]; if (L.rho < floor_rho) L.rho = floor_rho;
    Rt.rho = wr[0]; if (Rt.rho < floor_rho) Rt.rho = floor_rho;
    L.vx = wl[1]; L.vy = wl[2]; L.vz = wl[3];
    Rt.vx = wr[1]; Rt.vy = wr[2]; Rt.vz = wr[3];
    R bxl = wl[4], bxr = wr[4];
    L.by = wl[5]; L.bz = wl[6]; Rt.by = wr[5]; Rt.bz = wr[6];
    L.p = wl[7]; if (L.p < floor_pr) L.p = floor_pr;
    Rt.p = wr[7]; if (Rt.p < floor_pr) Rt.p = floor_pr;
    L.psi = wl[8]; Rt.psi = wr[8];
    L.c = wl[9]; Rt.c = wr[9];

    // Dedner face values, physics.py:74-82
    R bxf, psif;
    if (ch > R(0)) {
        bxf = R(0.5) * (bxl + bxr) - R(0.5) / ch * (Rt.psi - L.psi);
        psif = R(0.5) * (L.psi + Rt.psi) - R(0.5) * ch * (bxr - bxl);
    } else {
        bxf = R(0.5) * (bxl + bxr);
        psif = R(0);
    }
    R bx2 = bxf * bxf;
    R bmL2 = bx2 + L.by * L.by + L.bz * L.bz;
    R bmR2 = bx2 + Rt.by * Rt.by + Rt.bz * Rt.bz;
    L.pt = L.p + R(0.5) * bmL2;
    Rt.pt = Rt.p + R(0.5) * bmR2;

    // outer speeds with the GLM speed folded in, physics.py:104-108
    R cfL = fast_speed(L, gamma, bx2), cfR = fast_speed(Rt, gamma, bx2);
    R SL = fmin(L.vx - cfL, Rt.vx - cfR);
    R SR = fmax(L.vx + cfL, Rt.vx + cfR);
    if (ch > R(0)) { SL = fmin(SL, -ch); SR = fmax(SR, ch); }
    R smax = fmax(fabs(SL), fabs(SR));

    // contact speed, physics.py:111-120
    L.dS = SL - L.vx;
    Rt.dS = SR - Rt.vx;
    R den = Rt.dS * Rt.rho - L.dS * L.rho;
    if (fabs(den) < R(1e-14)) den = (den >= R(0)) ? R(1e-14) : R(-1e-14);
    R SM = (Rt.dS * Rt.rho * Rt.vx - L.dS * L.rho * L.vx - Rt.pt + L.pt) / den;
    if (SM < SL + R(1e-14)) SM = SL + R(1e-14);
    if (SM > SR - R(1e-14)) SM = SR - R(1e-14);
    R ptS = L.pt + L.rho * L.dS * (SM - L.vx);

    if (SL >= R(0)) {  // physics.py:177-187
        L.vb = L.vx * bxf + L.vy * L.by + L.vz * L.bz;
        L.e = L.p / gm1 + R(0.5) * L.rho * (L.vx * L.vx + L.vy * L.vy + L.vz * L.vz) + R(0.5) * bmL2;
        side_flux(L, bxf, bx2, psif, ch, f);
        return smax;
    }
    if (SR <= R(0)) {  // physics.py:188-198
        Rt.vb = Rt.vx * bxf + Rt.vy * Rt.by + Rt.vz * Rt.bz;
        Rt.e = Rt.p / gm1 + R(0.5) * Rt.rho * (Rt.vx * Rt.vx + Rt.vy * Rt.vy + Rt.vz * Rt.vz) + R(0.5) * bmR2;
        side_flux(Rt, bxf, bx2, psif, ch, f);
        return smax;
    }

    // star states, physics.py:122-154
    L.vb = L.vx * bxf + L.vy * L.by + L.vz * L.bz;
    Rt.vb = Rt.vx * bxf + Rt.vy * Rt.by + Rt.vz * Rt.bz;
    L.e = L.p / gm1 + R(0.5) * L.rho * (L.vx * L.vx + L.vy * L.vy + L.vz * L.vz) + R(0.5) * bmL2;
    Rt.e = Rt.p / gm1 + R(0.5) * Rt.rho * (Rt.vx * Rt.vx + Rt.vy * Rt.vy + Rt.vz * Rt.vz) + R(0.5) * bmR2;
    R eps_rel = R(1e-8) * fmax(fabs(ptS), R(1.0));
    star_prep(L, SL, SM, ptS, bxf, bx2, eps_rel, floor_rho);
    star_prep(Rt, SR, SM, ptS, bxf, bx2, eps_rel, floor_rho);

    // Alfven waves and the double-star state, physics.py:156-172
    R sbx = (bxf >= R(0)) ? R(1.0) : R(-1.0);
    R SAL = SM - fabs(bxf) / fmax(L.sq, R(1e-14));
    R SAR = SM + fabs(bxf) / fmax(Rt.sq, R(1e-14));
    if (SAL < SL) SAL = SL;
    if (SAL > SM) SAL = SM;
    if (SAR < SM) SAR = SM;
    if (SAR > SR) SAR = SR;

    // region of x/t = 0: SAL>=0 -> FLS, SM>=0 -> FLDS, SAR>=0 -> FRDS, else FRS
    const bool left = (SAL >= R(0)) || (SM >= R(0));
    const bool dstar = left ? !(SAL >= R(0)) : (SAR >= R(0));
    const Side<R> &K = left ? L : Rt;
    const R S = left ? SL : SR;
    const R SA = left ? SAL : SAR;

    R fk[NV];
    side_flux(K, bxf, bx2, psif, ch, fk);
    // star minus outer conserved state (physics.py:213-220)
    R du[NV];
    du[0] = K.rs - K.rho;
    du[1] = K.rs * SM - K.rho * K.vx;
    du[2] = K.rs * K.vys - K.rho * K.vy;
    du[3] = K.rs * K.vzs - K.rho * K.vz;
    du[4] = bxf - bxf;
    du[5] = K.bys - K.by;
    du[6] = K.bzs - K.bz;
    du[7] = K.es - K.e;
    du[8] = psif - K.psi;
    du[9] = K.rs * K.c - K.rho * K.c;
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = fk[v] + S * du[v];
    if (dstar) {
        R dds = fmax(L.sq + Rt.sq, R(1e-14));
        R vyds = (L.sq * L.vys + Rt.sq * Rt.vys + (Rt.bys - L.bys) * sbx) / dds;
        R vzds = (L.sq * L.vzs + Rt.sq * Rt.vzs + (Rt.bzs - L.bzs) * sbx) / dds;
        R byds = (L.sq * Rt.bys + Rt.sq * L.bys + L.sq * Rt.sq * (Rt.vys - L.vys) * sbx) / dds;
        R bzds = (L.sq * Rt.bzs + Rt.sq * L.bzs + L.sq * Rt.sq * (Rt.vzs - L.vzs) * sbx) / dds;
        R vbds = SM * bxf + vyds * byds + vzds * bzds;
        R eds = left ? (L.es - L.sq * (L.vbs - vbds) * sbx) : (Rt.es + Rt.sq * (Rt.vbs - vbds) * sbx);
        // double-star minus star (physics.py:244-253)
        R dd[NV];
        dd[0] = K.rs - K.rs;
        dd[1] = K.rs * SM - K.rs * SM;
        dd[2] = K.rs * vyds - K.rs * K.vys;
        dd[3] = K.rs * vzds - K.rs * K.vzs;
        dd[4] = bxf - bxf;
        dd[5] = byds - K.bys;
        dd[6] = bzds - K.bzs;
        dd[7] = eds - K.es;
        dd[8] = psif - psif;
        dd[9] = K.rs * K.c - K.rs * K.c;
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = f[v] + SA * dd[v];
    }
    if (ch > R(0)) {
        f[4] = psif;
        f[8] = ch * ch * bxf;
    }
    return smax;
}

// swap the normal and first transverse components (physics.py:373-379)
template <typename R>
__device__ __forceinline__ void rot_xy(R w[NV])
{
    R t = w[1]; w[1] = w[2]; w[2] = t;
    t = w[4]; w[4] = w[5]; w[5] = t;
}

// ---------------------------------------------------------------------------
// cons -> prim of one cell (physics.py:284-301).  For float the pressure is
// recovered in double from the stored values (the cancellation-prone step).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cons_to_prim_cell(const double u[NV], double gamma, double w[NV])
{
    double rho = np_max(u[RHO], FLOOR_RHO);
    double ri = 1.0 / rho;
    double vx = u[MX] * ri, vy = u[MY] * ri, vz = u[MZ] * ri;
    double ke = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    double me = 0.5 * (u[BX] * u[BX] + u[BY] * u[BY] + u[BZ] * u[BZ]);
    w[0] = rho; w[1] = vx; w[2] = vy; w[3] = vz;
    w[4] = u[BX]; w[5] = u[BY]; w[6] = u[BZ];
    w[7] = np_max((gamma - 1.0) * (u[EN] - ke - me), FLOOR_PR);
    w[8] = u[PSI];
    w[9] = u[RHOC] * ri;
}

__device__ __forceinline__ void cons_to_prim_cell(const float u[NV], double gamma, float w[NV])
{
    float rho = np_max(u[RHO], float(FLOOR_RHO));
    float ri = 1.0f / rho;
    w[0] = rho; w[1] = u[MX] * ri; w[2] = u[MY] * ri; w[3] = u[MZ] * ri;
    w[4] = u[BX]; w[5] = u[BY]; w[6] = u[BZ];
    w[8] = u[PSI];
    w[9] = u[RHOC] * ri;
    // float64 recovery: p = (gamma-1) (E - |m|^2 / (2 rho) - |B|^2 / 2)
    double rd = (double)rho;
    double m2 = (double)u[MX] * u[MX] + (double)u[MY] * u[MY] + (double)u[MZ] * u[MZ];
    double b2 = (double)u[BX] * u[BX] + (double)u[BY] * u[BY] + (double)u[BZ] * u[BZ];
    double p = (gamma - 1.0) * ((double)u[EN] - 0.5 * m2 / rd - 0.5 * b2);
    w[7] = (float)np_max(p, FLOOR_PR);
}

// CFL quantities of one stored cell (compute_dt, solver.py:209-214), in double:
// q[0] = cf^2 (max of cf is sqrt of max cf^2), q[1] = |vx|+|vy|, q[2] = |vx|, q[3] = |vy|
template <typename R>
__device__ __forceinline__ void cfl_quantities(const R u[NV], double gamma, double q[4])
{
    double ud[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ud[v] = (double)u[v];
    double w[NV];
    cons_to_prim_cell(ud, gamma, w);
    double b2 = w[4] * w[4] + w[5] * w[5] + w[6] * w[6];
    q[0] = gamma * w[7] / w[0] + b2 / w[0];
    q[2] = fabs(w[1]);
    q[3] = fabs(w[2]);
    q[1] = q[2] + q[3];
}

// same from a primitive cell (compute_dt(W), solver.py:209-214)
__device__ __forceinline__ void cfl_quantities_prim(const double w[NV], double gamma, double q[4])
{
    double rho = np_max(w[0], FLOOR_RHO);
    double p = np_max(w[7], FLOOR_PR);
    double b2 = w[4] * w[4] + w[5] * w[5] + w[6] * w[6];
    q[0] = gamma * p / rho + b2 / rho;
    q[2] = fabs(w[1]);
    q[3] = fabs(w[2]);
    q[1] = q[2] + q[3];
}

// ---------------------------------------------------------------------------
// ghost cells (apply_bc, solver.py:158-197).  After the reference's apply_bc
// every ghost holds the value of one interior cell: per axis,
//   periodic:      g < NG -> g + n;    g >= NG + n -> g - n
//   extrapolation: g < NG -> NG;       g >= NG + n -> NG + n - 1
// (characteristic == extrapolation once psi is zeroed), and psi is zero in
// x-ghost rows whenever the x boundary is not periodic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ghost_source(int g, int n, int bc)
{
    if (g < NG) return bc == AMHD_BC_PERIODIC ? g + n : NG;
    if (g >= NG + n) return bc == AMHD_BC_PERIODIC ? g - n : NG + n - 1;
    return g;
}

// the ghost indices whose source is interior index i (at most 4)
__device__ __forceinline__ int ghost_targets(int i, int n, int bc, int g[4])
{
    int k = 0;
    if (bc == AMHD_BC_PERIODIC) {
        if (i >= n && i - n < NG) g[k++] = i - n;
        if (i < 2 * NG) g[k++] = i + n;
    } else {
        if (i == NG) { g[k++] = 0; g[k++] = 1; }
        if (i == NG + n - 1) { g[k++] = n + NG; g[k++] = n + NG + 1; }
    }
    return k;
}

// bit pattern of a non-negative double (or NaN) ordered as an unsigned integer
__device__ __forceinline__ unsigned long long ord_bits(double x)
{
    return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b)
{
    return a > b ? a : b;
}

}  // namespace amhd
