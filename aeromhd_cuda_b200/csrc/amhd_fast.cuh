// amhd_fast.cuh -- float32 device physics tuned for throughput.
//
// The float32 path of the fused stage kernel computes the same scheme as the
// float64 path (van Leer / minmod MUSCL, HLLD of physics.py:43-276, GLM,
// cons->prim with float64 pressure recovery) but arranges the arithmetic for
// the SM: one reciprocal per denominator reused by every quotient, hardware
// approximate reciprocal / square root (rcp.approx, sqrt.approx, rsqrt.approx:
// <= 2 ulp), and a float64 reciprocal obtained from the float one by one
// Newton step (relative error ~1e-14) instead of an IEEE float64 divide.
// Its results are checked against the float64 oracle (relative L1 <= 1e-5).
#pragma once
#include <cuda_runtime.h>

#include "amhd_physics.cuh"

namespace amhd {
namespace fast {

__device__ __forceinline__ float rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// float64 reciprocal of a positive float: float estimate + one Newton step
__device__ __forceinline__ double rcp64(float x)
{
    const double xd = (double)x;
    double r = (double)rcp(x);
    return r * fma(-xd, r, 2.0);
}

// van Leer (2ab/(a+b) when ab > 0) or minmod slope of the middle of three values
__device__ __forceinline__ float slope(float wm, float w0, float wp, int limiter)
{
    const float dm = w0 - wm, dp = wp - w0;
    const float ab = dm * dp;
    if (limiter == AMHD_LIMITER_MINMOD) return (ab > 0.f) ? (fabsf(dm) < fabsf(dp) ? dm : dp) : 0.f;
    // 2ab / den as ab / (den / 2): halving is exact, so is the factor 2 it saves
    return (ab > 0.f) ? ab * rcp(fmaf(0.5f, dm + dp, 0.5e-30f)) : 0.f;
}

// the same for two independent values at once, on the packed float32x2 path of
// sm_100 (one FFMA2/FADD2/FMUL2 per pair; per component the scalar arithmetic)
__device__ __forceinline__ float2 slope2(float2 wm, float2 w0, float2 wp, int limiter)
{
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 dm = __ffma2_rn(wm, m1, w0), dp = __ffma2_rn(w0, m1, wp);
    const float2 ab = __fmul2_rn(dm, dp);
    if (limiter == AMHD_LIMITER_MINMOD)
        return make_float2((ab.x > 0.f) ? (fabsf(dm.x) < fabsf(dp.x) ? dm.x : dp.x) : 0.f,
                           (ab.y > 0.f) ? (fabsf(dm.y) < fabsf(dp.y) ? dm.y : dp.y) : 0.f);
    // 2ab / den as ab / (den / 2): halving is exact, so is the factor 2 it saves
    const float2 hden = __ffma2_rn(make_float2(0.5f, 0.5f), __fadd2_rn(dm, dp), make_float2(0.5e-30f, 0.5e-30f));
    const float2 q = __fmul2_rn(ab, make_float2(rcp(hden.x), rcp(hden.y)));
    return make_float2(ab.x > 0.f ? q.x : 0.f, ab.y > 0.f ? q.y : 0.f);
}

// conserved -> primitive with the pressure recovered in float64
__device__ __forceinline__ void cons_to_prim(const float u[NV], double gamma, float w[NV])
{
    const float rho = fmaxf(u[RHO], float(FLOOR_RHO));
    const double ri_d = rcp64(rho);
    const float ri = (float)ri_d;
    w[0] = rho;
    w[1] = u[MX] * ri;
    w[2] = u[MY] * ri;
    w[3] = u[MZ] * ri;
    w[4] = u[BX];
    w[5] = u[BY];
    w[6] = u[BZ];
    w[8] = u[PSI];
    w[9] = u[RHOC] * ri;
    const double m2 = (double)u[MX] * u[MX] + (double)u[MY] * u[MY] + (double)u[MZ] * u[MZ];
    const double b2 = (double)u[BX] * u[BX] + (double)u[BY] * u[BY] + (double)u[BZ] * u[BZ];
    const double p = (gamma - 1.0) * ((double)u[EN] - 0.5 * m2 * ri_d - 0.5 * b2);
    w[7] = (float)fmax(p, FLOOR_PR);
}

// CFL quantities of a stored float cell, in float64: cf^2, |vx|+|vy|, |vx|, |vy|
__device__ __forceinline__ void cfl_quantities(const float u[NV], double gamma, double q[4])
{
    const float rho = fmaxf(u[RHO], float(FLOOR_RHO));
    const double ri = rcp64(rho);
    const double mx = u[MX], my = u[MY], mz = u[MZ];
    const double m2 = mx * mx + my * my + mz * mz;
    const double b2 = (double)u[BX] * u[BX] + (double)u[BY] * u[BY] + (double)u[BZ] * u[BZ];
    const double p = fmax((gamma - 1.0) * ((double)u[EN] - 0.5 * m2 * ri - 0.5 * b2), FLOOR_PR);
    q[0] = (gamma * p + b2) * ri;
    q[2] = fabs(mx * ri);
    q[3] = fabs(my * ri);
    q[1] = q[2] + q[3];
}

struct FSide {
    float rho, ir, vx, vy, vz, by, bz, p, psi, c;
    float bm2, pt, e, vb;
    float dS, idsm, rs, isq, sq, vys, vzs, bys, bzs, es, vbs;
};

__device__ __forceinline__ void load_side(FSide &s, const float w[NV], float bxf2)
{
    s.rho = fmaxf(w[0], float(FLOOR_RHO));
    s.ir = rcp(s.rho);
    s.vx = w[1];
    s.vy = w[2];
    s.vz = w[3];
    s.by = w[5];
    s.bz = w[6];
    s.p = fmaxf(w[7], float(FLOOR_PR));
    s.psi = w[8];
    s.c = w[9];
    s.bm2 = bxf2 + s.by * s.by + s.bz * s.bz;
    s.pt = s.p + 0.5f * s.bm2;
}

// bx2_4 = 4 Bx^2 of the face, shared by both sides
__device__ __forceinline__ float fast_speed(const FSide &s, float gamma, float bx2_4)
{
    const float a2 = gamma * s.p * s.ir;
    const float tmp = a2 + s.bm2 * s.ir;
    const float disc = fmaxf(tmp * tmp - a2 * bx2_4 * s.ir, 0.f);
    return sqrt_(fmaxf(0.5f * (tmp + sqrt_(disc)), 0.f));
}

__device__ __forceinline__ void side_flux(const FSide &s, float bxf, float bx2, float psif, float ch, bool glm,
                                          float f[NV])
{
    const float mx = s.rho * s.vx;
    f[0] = mx;
    f[1] = mx * s.vx + s.pt - bx2;
    f[2] = mx * s.vy - bxf * s.by;
    f[3] = mx * s.vz - bxf * s.bz;
    f[4] = glm ? psif : 0.f;
    f[5] = s.by * s.vx - bxf * s.vy;
    f[6] = s.bz * s.vx - bxf * s.vz;
    f[7] = (s.e + s.pt) * s.vx - bxf * s.vb;
    f[8] = glm ? bxf * ch * ch : 0.f;
    f[9] = mx * s.c;
}

// star-state transverse quantities of one side (physics.py:122-146), reciprocals shared
__device__ __forceinline__ void star(FSide &s, float S, float SM, float bxf, float bx2, float eps_rel)
{
    float dsm = S - SM;
    if (fabsf(dsm) < 1e-14f) dsm = 1e-14f;
    s.idsm = rcp(dsm);
    s.rs = fmaxf(s.rho * s.dS * s.idsm, float(FLOOR_RHO));
    s.isq = rsqrt(s.rs);
    s.sq = s.rs * s.isq;
    const float rds = s.rho * s.dS;
    float dn = rds * dsm - bx2;
    if (fabsf(dn) < eps_rel) dn = (dn >= 0.f) ? eps_rel : -eps_rel;
    const float idn = rcp(dn);
    const float tv = bxf * (SM - s.vx) * idn;
    s.vys = s.vy - s.by * tv;
    s.vzs = s.vz - s.bz * tv;
    const float tb = (rds * s.dS - bx2) * idn;
    s.bys = s.by * tb;
    s.bzs = s.bz * tb;
}

// total energy, v.B and their star values (physics.py:146-154): only the side
// whose fan holds x/t = 0 needs them
__device__ __forceinline__ void side_energy(FSide &s, float bxf, float igm1)
{
    s.vb = s.vx * bxf + s.vy * s.by + s.vz * s.bz;
    s.e = s.p * igm1 + 0.5f * s.rho * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz) + 0.5f * s.bm2;
}
__device__ __forceinline__ void star_energy(FSide &s, float S, float SM, float ptS, float bxf)
{
    s.vbs = SM * bxf + s.vys * s.bys + s.vzs * s.bzs;
    s.es = ((S - s.vx) * s.e - s.pt * s.vx + ptS * SM + bxf * (s.vb - s.vbs)) * s.idsm;
}

// HLLD flux through an x-normal face (physics.py:43-276), float32.  glm: ch > 0
// (a caller that knows it passes the constant, which removes the ch = 0 code
// and the supersonic branch: with GLM the outer speeds bracket -ch .. ch)
__device__ __forceinline__ void hlld(const float wl[NV], const float wr[NV], float gamma, float igm1, float ch,
                                     float half_ich, float f[NV], bool glm)
{
    float bxf, psif;
    if (glm) {
        bxf = 0.5f * (wl[4] + wr[4]) - half_ich * (wr[8] - wl[8]);
        psif = 0.5f * (wl[8] + wr[8]) - 0.5f * ch * (wr[4] - wl[4]);
    } else {
        bxf = 0.5f * (wl[4] + wr[4]);
        psif = 0.f;
    }
    const float bx2 = bxf * bxf;
    FSide L, R;
    load_side(L, wl, bx2);
    load_side(R, wr, bx2);
    const float bx2_4 = 4.f * bx2;
    const float cfL = fast_speed(L, gamma, bx2_4), cfR = fast_speed(R, gamma, bx2_4);
    float SL = fminf(L.vx - cfL, R.vx - cfR);
    float SR = fmaxf(L.vx + cfL, R.vx + cfR);
    if (glm) {
        SL = fminf(SL, -ch);
        SR = fmaxf(SR, ch);
    }
    L.dS = SL - L.vx;
    R.dS = SR - R.vx;
    const float rdl = L.dS * L.rho, rdr = R.dS * R.rho;
    float den = rdr - rdl;
    if (fabsf(den) < 1e-14f) den = (den >= 0.f) ? 1e-14f : -1e-14f;
    float SM = (rdr * R.vx - rdl * L.vx - R.pt + L.pt) * rcp(den);
    if (SM < SL + 1e-14f) SM = SL + 1e-14f;
    if (SM > SR - 1e-14f) SM = SR - 1e-14f;
    const float ptS = L.pt + rdl * (SM - L.vx);

    if (!glm && (SL >= 0.f || SR <= 0.f)) {  // supersonic: the upwind side's flux (only without GLM)
        FSide U = SL >= 0.f ? L : R;  // a copy: writing through a runtime-chosen reference would put L and R in local memory
        side_energy(U, bxf, igm1);
        side_flux(U, bxf, bx2, psif, ch, glm, f);
        return;
    }
    const float eps_rel = 1e-8f * fmaxf(fabsf(ptS), 1.f);
    star(L, SL, SM, bxf, bx2, eps_rel);
    star(R, SR, SM, bxf, bx2, eps_rel);
    const float abx = fabsf(bxf);
    float SAL = SM - abx * fminf(L.isq, 1e14f);
    float SAR = SM + abx * fminf(R.isq, 1e14f);
    SAL = fminf(fmaxf(SAL, SL), SM);
    SAR = fminf(fmaxf(SAR, SM), SR);

    const bool left = (SAL >= 0.f) || (SM >= 0.f);
    const bool dstar = left ? !(SAL >= 0.f) : (SAR >= 0.f);
    FSide K = left ? L : R;  // a copy (see above)
    const float S = left ? SL : SR;
    side_energy(K, bxf, igm1);
    star_energy(K, S, SM, ptS, bxf);
    side_flux(K, bxf, bx2, psif, ch, glm, f);
    // + S (U* - U)
    f[0] += S * (K.rs - K.rho);
    f[1] += S * (K.rs * SM - K.rho * K.vx);
    f[2] += S * (K.rs * K.vys - K.rho * K.vy);
    f[3] += S * (K.rs * K.vzs - K.rho * K.vz);
    f[5] += S * (K.bys - K.by);
    f[6] += S * (K.bzs - K.bz);
    f[7] += S * (K.es - K.e);
    f[8] += S * (psif - K.psi);
    f[9] += S * (K.rs - K.rho) * K.c;
    if (dstar) {
        const float sbx = (bxf >= 0.f) ? 1.f : -1.f;
        const float idds = rcp(fmaxf(L.sq + R.sq, 1e-14f));
        const float vyds = (L.sq * L.vys + R.sq * R.vys + (R.bys - L.bys) * sbx) * idds;
        const float vzds = (L.sq * L.vzs + R.sq * R.vzs + (R.bzs - L.bzs) * sbx) * idds;
        const float sqq = L.sq * R.sq * sbx;
        const float byds = (L.sq * R.bys + R.sq * L.bys + sqq * (R.vys - L.vys)) * idds;
        const float bzds = (L.sq * R.bzs + R.sq * L.bzs + sqq * (R.vzs - L.vzs)) * idds;
        const float vbds = SM * bxf + vyds * byds + vzds * bzds;
        const float eds = left ? (K.es - K.sq * (K.vbs - vbds) * sbx) : (K.es + K.sq * (K.vbs - vbds) * sbx);
        const float SA = left ? SAL : SAR;
        // + SA (U** - U*)
        f[2] += SA * K.rs * (vyds - K.vys);
        f[3] += SA * K.rs * (vzds - K.vzs);
        f[5] += SA * (byds - K.bys);
        f[6] += SA * (bzds - K.bzs);
        f[7] += SA * (eds - K.es);
    }
    if (glm) {
        f[4] = psif;
        f[8] = ch * ch * bxf;
    }
}

}  // namespace fast
}  // namespace amhd
