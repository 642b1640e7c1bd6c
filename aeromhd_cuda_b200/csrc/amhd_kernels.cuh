// amhd_kernels.cuh -- CUDA kernels of the MHD hot path, templated on the real
// type.  Included by amhd_f64.cu (Real = double, -fmad=false) and amhd_f32.cu
// (Real = float).  Host-side launchers are declared in amhd_launch.h.
//
// One RK stage is one fused kernel: stage input -> primitives (float64
// pressure recovery), MUSCL + HLLD on every x and y face, flux divergence +
// Powell source, the SSP-RK3 combination with the step's base state, the
// passive-scalar clamp, psi damping (last stage) and on the last stage the CFL
// reduction of the new state for the next dt.  Two kernels implement it with
// the same per-cell functions (update_cell_d, face_flux / hlld):
//   march_stage_kernel (default) -- one warp walks a 28-column strip row by
//     row, rows staged with cp.async, x-slopes and x-face fluxes carried from
//     row to row, y neighbours by warp shuffles, no CTA barriers;
//   rk_stage_kernel -- one CTA per 8..16 x 32 tile staged (TMA) with its halo
//     in shared memory, boundary cells pushing their values into the ghosts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "aeromhd.h"
#include "amhd_launch.h"
#include "amhd_fast.cuh"
#include "amhd_physics.cuh"
#include "amhd_tma.cuh"

#include <type_traits>

namespace amhd {

constexpr int TY = 32;           // tile width along y (the contiguous axis): one warp
constexpr int HW = TY + 2 * NG;  // halo width along y

template <typename R>
struct Vec;
template <>
struct Vec<float> {
    using T = float4;
    static constexpr int N = 4;
};
template <>
struct Vec<double> {
    using T = double2;
    static constexpr int N = 2;
};

template <typename R>
constexpr bool kFast = std::is_same<R, float>::value;  // float32: slope pre-pass + fast HLLD

template <typename R, int TX>
struct TileSmem {
    alignas(128) R w[NV][TX + 2 * NG][HW];  // tile + halo: TMA lands conserved, converted in place
    // limited slopes (float32 path only): x-slopes of halo rows 1..TX+2 over the
    // tile's columns, y-slopes of the tile's rows over halo columns 1..TY+2
    R sx[kFast<R> ? NV : 1][kFast<R> ? TX + 2 : 1][TY];
    R sy[kFast<R> ? NV : 1][kFast<R> ? TX : 1][TY + 2];
    R fx[NV][TX + 1][TY];          // x-face fluxes (face a: between tile rows a-1 and a)
    R fy[NV][TX][TY + 1];          // y-face fluxes
    unsigned long long red[4][32]; // per-warp dt partials
    uint64_t mbar;                 // TMA completion barrier
    int nonfinite;
    int tma_ok;
};

// Programmatic dependent launch (sm_90 and later): pdl_trigger lets the next
// kernel of the stream be scheduled onto SMs this grid frees, pdl_wait blocks
// until the previous kernel has completed and its writes are visible.  For a
// kernel launched without the programmatic-serialization attribute both have
// nothing to do (stream order already holds).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ const amhd_instance &inst_of(const StageParams &p, int tile, int &inst_idx)
{
    if (p.inst != nullptr) {
        inst_idx = p.tile_inst[tile];
        return p.inst[inst_idx];
    }
    inst_idx = 0;
    return p.one;
}

// ---------------------------------------------------------------------------
// fused RK stage; STAGE 1..3 (solver.py:319-329), STAGE 0 = compute_rhs (R out)
// ---------------------------------------------------------------------------
// does interior index i (of n) feed a ghost cell? (see ghost_targets)
__device__ __forceinline__ bool feeds_ghosts(int i, int n, int bc)
{
    return bc == AMHD_BC_PERIODIC ? (i < 2 * NG || i >= n) : (i == NG || i == NG + n - 1);
}

// Copy boundary cell (i, j) of U, which this thread has just written, into
// every ghost cell that copies it (apply_bc, solver.py:158-197; psi is zero in
// the x-ghost rows of a non-periodic x boundary).  Few cells take this path;
// it stays out of line so that its registers do not weigh on the caller.
template <typename R>
__device__ __noinline__ void push_ghosts(const amhd_grid g, R *U, int i, int j)
{
    int gx[4], gy[4];
    const int nxg = ghost_targets(i, g.nx, g.bc_x, gx);
    const int nyg = ghost_targets(j, g.ny, g.bc_y, gy);
    const bool zero_psi_x = g.bc_x != AMHD_BC_PERIODIC;
    const int64_t vs = g.var_stride;
    const int pitch = g.pitch;
    for (int v = 0; v < NV; ++v) {
        const R val = U[v * vs + (int64_t)i * pitch + j];
        for (int m = 0; m < nyg; ++m) U[v * vs + (int64_t)i * pitch + gy[m]] = val;
        const R ox = (v == PSI && zero_psi_x) ? R(0) : val;
        for (int n = 0; n < nxg; ++n) {
            U[v * vs + (int64_t)gx[n] * pitch + j] = ox;
            for (int m = 0; m < nyg; ++m) U[v * vs + (int64_t)gx[n] * pitch + gy[m]] = ox;
        }
    }
}

// cell values the Powell source needs (solver.py:242-266): Bx at i, i-1, i+1;
// By at j, j-1, j+1; v and Bz at the cell
template <typename R>
struct PowellIn {
    R bxc, bxm, bxp, byc, bym, byp, vx, vy, vz, bzc;
};

// Everything after the face fluxes for one interior cell (i, j): flux divergence,
// Powell source, SSP-RK3 combination (solver.py:319-329), scalar clamp
// (solver.py:199-204), psi damping (:331-333), CFL quantities of the new state
// (stage 3, max-accumulated into q), then the cell and every ghost cell that
// copies it (apply_bc, solver.py:158-197).  STAGE 0 writes the right-hand side
// instead.  dfx / dfy: flux differences (face +1/2 minus face -1/2) in x and
// y; powell_in() gives the Powell inputs; base_at(v) / in_at(v) the cell's
// value of U0 / of the stage input in plane v.  Without PUSH the caller fills
// the ghost cells afterwards (march_bc_fill_kernel).
// cell_values computes the new values (out; the compensated low part in lo_new)
// without storing them; update_cell_d stores them as well.
template <typename R, int STAGE, bool COMP = false, typename PowellFn, typename BaseFn, typename InFn>
__device__ __forceinline__ void cell_values(const StageParams &p, const amhd_grid &g, int i, int j, const R dfx[NV],
                                            const R dfy[NV], PowellFn powell_in, BaseFn base_at, InFn in_at,
                                            double dt, double ch, double decay, unsigned long long q[4], bool &bad,
                                            const R *ulo, R out[NV], R lo_new[NV])
{
    static_assert(!COMP || (STAGE == 3 && kFast<R>), "compensation is for the last float32 stage");
    R rhs[NV];
    const R dx = R(g.dx), dy = R(g.dy);
    if constexpr (kFast<R>) {
        const float idx = float(1.0 / g.dx), idy = float(1.0 / g.dy);
        const float2 nix = make_float2(-idx, -idx), niy = make_float2(-idy, -idy);
#pragma unroll
        for (int v = 0; v < NV; v += 2) {
            const float2 r = __ffma2_rn(make_float2(dfy[v], dfy[v + 1]), niy,
                                        __fmul2_rn(make_float2(dfx[v], dfx[v + 1]), nix));
            rhs[v] = r.x;
            rhs[v + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R r0 = R(0);
            r0 -= dfx[v] / dx;
            r0 -= dfy[v] / dy;
            rhs[v] = r0;
        }
    }
    if (g.powell) {
        // _compute_powell_source, solver.py:242-266 (centred face-average divB)
        const PowellIn<R> pw = powell_in();
        R divb;
        if constexpr (kFast<R>)  // float32: reciprocal spacings instead of two divisions
            divb = (R(0.5) * (pw.bxc + pw.bxp) - R(0.5) * (pw.bxm + pw.bxc)) * float(1.0 / g.dx) +
                   (R(0.5) * (pw.byc + pw.byp) - R(0.5) * (pw.bym + pw.byc)) * float(1.0 / g.dy);
        else
            divb = (R(0.5) * (pw.bxc + pw.bxp) - R(0.5) * (pw.bxm + pw.bxc)) / dx +
                   (R(0.5) * (pw.byc + pw.byp) - R(0.5) * (pw.bym + pw.byc)) / dy;
        R vb = pw.vx * pw.bxc + pw.vy * pw.byc + pw.vz * pw.bzc;
        rhs[MX] += -divb * pw.bxc;
        rhs[MY] += -divb * pw.byc;
        rhs[MZ] += -divb * pw.bzc;
        rhs[BX] += -divb * pw.vx;
        rhs[BY] += -divb * pw.vy;
        rhs[BZ] += -divb * pw.vz;
        rhs[EN] += -divb * vb;
        rhs[RHO] += R(0);  // the reference adds a zero source to these slots too
        rhs[PSI] += R(0);
        rhs[RHOC] += R(0);
    }
    if (STAGE == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] = rhs[v];
    } else {
        const R dtr = R(dt);
        if constexpr (kFast<R>) {
            // pairs of variables on the packed float32x2 path; stages 2, 3 in the
            // increment form U0 + w ((U* - U0) + dt R): in float32 the weights 1/3
            // and 2/3 round to a sum of 1 + 3e-8, which as a weighted average would
            // scale the state every step (a mass drift); U* - U0 is exact
            const float w = STAGE == 2 ? 0.25f : float(2.0 / 3.0);
            const float2 dt2 = make_float2(dtr, dtr), w2 = make_float2(w, w), m1 = make_float2(-1.f, -1.f);
#pragma unroll
            for (int v = 0; v < NV; v += 2) {
                const float2 b0 = make_float2(base_at(v), base_at(v + 1));
                const float2 r = make_float2(rhs[v], rhs[v + 1]);
                float2 o;
                if (STAGE == 1) {
                    o = __ffma2_rn(dt2, r, b0);
                } else {
                    const float2 us = make_float2(in_at(v), in_at(v + 1));
                    if constexpr (COMP) {
                        // compensated: U = hi + lo; the increment w((U2 - hi) + dt R) is
                        // the true one (U2 was formed from hi), added to hi + lo as
                        // lo + inc, then TwoSum(hi, lo + inc) splits the result into the
                        // stored float32 and its exact rounding error, the new lo
                        const float2 inc = __fmul2_rn(w2, __ffma2_rn(dt2, r, __ffma2_rn(b0, m1, us)));
                        const float2 lo = make_float2(ulo[v * g.var_stride + (int64_t)i * g.pitch + j],
                                                      ulo[(v + 1) * g.var_stride + (int64_t)i * g.pitch + j]);
                        const float2 t = __fadd2_rn(lo, inc);
                        o = __fadd2_rn(b0, t);
                        const float2 bb = __ffma2_rn(b0, m1, o);                 // o - hi
                        const float2 ea = __ffma2_rn(__ffma2_rn(bb, m1, o), m1, b0);  // hi - (o - bb)
                        const float2 eb = __ffma2_rn(bb, m1, t);                 // t - bb
                        const float2 e = __fadd2_rn(ea, eb);
                        lo_new[v] = e.x;
                        lo_new[v + 1] = e.y;
                    } else {
                        o = __ffma2_rn(w2, __ffma2_rn(dt2, r, __ffma2_rn(b0, m1, us)), b0);
                    }
                }
                out[v] = o.x;
                out[v + 1] = o.y;
            }
        } else
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R b0 = base_at(v);
            if (STAGE == 1) {
                out[v] = b0 + dtr * rhs[v];
            } else {
                R us = in_at(v);
                if constexpr (kFast<R>) {
                    // increment form of the same combination: in float32 the weights
                    // 1/3 and 2/3 round to a sum of 1 + 3e-8, which as a weighted
                    // average would scale the state every step (a mass drift);
                    // U0 + w ((U* - U0) + dt R) has no such bias (U* - U0 is exact)
                    const float w = STAGE == 2 ? 0.25f : float(2.0 / 3.0);
                    out[v] = b0 + w * ((us - b0) + dtr * rhs[v]);
                } else {
                    if (STAGE == 2)
                        out[v] = R(0.75) * b0 + R(0.25) * (us + dtr * rhs[v]);
                    else
                        out[v] = R(1.0 / 3.0) * b0 + R(2.0 / 3.0) * (us + dtr * rhs[v]);
                }
            }
        }
        // enforce_scalar_bounds, solver.py:199-204
        R rho = np_max(out[RHO], R(FLOOR_RHO));
        R cc;
        if constexpr (kFast<R>)
            cc = np_min(np_max(out[RHOC] * fast::rcp(rho), R(0)), R(1));
        else
            cc = np_min(np_max(out[RHOC] / rho, R(0)), R(1));
        const R rhoc_before = out[RHOC];
        out[RHOC] = rho * cc;
        if (STAGE == 3) {
            if (ch > 0.0) out[PSI] *= R(decay);  // solver.py:331-333
            if constexpr (COMP) {
                if (out[RHOC] != rhoc_before) lo_new[RHOC] = R(0);  // clamped: the stored value is the state
                if (ch > 0.0) lo_new[PSI] *= R(decay);
            }
            if (p.fuse_dt) {
                double qd[4];
                if constexpr (kFast<R>)
                    fast::cfl_quantities(out, g.gamma, qd);
                else
                    cfl_quantities(out, g.gamma, qd);
#pragma unroll
                for (int k = 0; k < 4; ++k) q[k] = umax64(q[k], ord_bits(qd[k]));
            }
            if constexpr (kFast<R>) {
                // x * 0 is NaN exactly when x is not finite: one test for the cell
                float2 z = make_float2(0.f, 0.f);
#pragma unroll
                for (int v = 0; v < NV; v += 2) z = __ffma2_rn(make_float2(out[v], out[v + 1]), make_float2(0.f, 0.f), z);
                bad |= !(z.x == 0.f && z.y == 0.f);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) bad |= !isfinite((double)out[v]);
            }
        }
    }
}

template <typename R, int STAGE, bool PUSH = true, bool COMP = false, typename PowellFn, typename BaseFn,
          typename InFn>
__device__ __forceinline__ void update_cell_d(const StageParams &p, const amhd_grid &g, R *uout, int i, int j,
                                              const R dfx[NV], const R dfy[NV], PowellFn powell_in, BaseFn base_at,
                                              InFn in_at, double dt, double ch, double decay, unsigned long long q[4],
                                              bool &bad, R *ulo = nullptr)
{
    const int64_t vs = g.var_stride;
    const int64_t gi = (int64_t)i * g.pitch + j;
    R out[NV];
    R lo_new[NV];  // compensated stage 3 only: the new low part of the base state
    cell_values<R, STAGE, COMP>(p, g, i, j, dfx, dfy, powell_in, base_at, in_at, dt, ch, decay, q, bad, ulo, out,
                                lo_new);
    // write the cell, then every ghost that copies it (apply_bc, solver.py:158-197)
#pragma unroll
    for (int v = 0; v < NV; ++v) uout[v * vs + gi] = out[v];
    if constexpr (COMP) {
#pragma unroll
        for (int v = 0; v < NV; ++v) ulo[v * vs + gi] = lo_new[v];
    }
    if (PUSH && STAGE != 0 && (feeds_ghosts(i, g.nx, g.bc_x) || feeds_ghosts(j, g.ny, g.bc_y)))
        push_ghosts(g, uout, i, j);
}

// the same from the four face fluxes
template <typename R, int STAGE, typename PowellFn, typename BaseFn, typename InFn>
__device__ __forceinline__ void update_cell(const StageParams &p, const amhd_grid &g, R *uout, int i, int j,
                                            const R fxl[NV], const R fxr[NV], const R fyl[NV], const R fyr[NV],
                                            PowellFn powell_in, BaseFn base_at, InFn in_at, double dt, double ch,
                                            double decay, unsigned long long q[4], bool &bad)
{
    R dfx[NV], dfy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        dfx[v] = fxr[v] - fxl[v];
        dfy[v] = fyr[v] - fyl[v];
    }
    update_cell_d<R, STAGE>(p, g, uout, i, j, dfx, dfy, powell_in, base_at, in_at, dt, ch, decay, q, bad);
}

// returns false when the CTA must stop (a TMA transfer did not complete)
template <typename R, int TX, int STAGE>
__device__ __forceinline__ bool rk_stage_tile(const StageParams &p, TileSmem<R, TX> &sm, int tile, uint32_t &phase)
{
    constexpr int NT = TX * TY;  // threads per block: one per tile cell
    constexpr int VN = Vec<R>::N;
    constexpr int HROWS = TX + 2 * NG;
    using VT = typename Vec<R>::T;

    int ii;
    const amhd_instance &in = inst_of(p, tile, ii);
    const amhd_grid g = in.grid;
    amhd_control *ctl = p.ctl ? p.ctl + ii : nullptr;

    double dt = p.dt, ch = p.ch, decay = p.decay;
    if (p.use_ctl) {
        if (!ctl->active) return true;
        dt = ctl->dt;
        ch = ctl->ch;
        decay = ctl->decay;
    }
    const int local = tile - in.first_tile;
    const int ty = local % in.tiles_y, tx = local / in.tiles_y;
    const int i0 = NG + tx * TX, j0 = NG + ty * TY;  // first interior cell of the tile
    const int64_t vs = g.var_stride;
    const int pitch = g.pitch;
    const R *uin = reinterpret_cast<const R *>(p.uin) + in.offset;
    const R *u0 = reinterpret_cast<const R *>(p.u0) + in.offset;
    R *uout = reinterpret_cast<R *>(p.uout) + in.offset;
    const int t = threadIdx.x;

    // ---- phase A: tile + halo -> primitives in shared memory --------------
    // the padded layout keeps every halo row/column of every tile in bounds
    constexpr int QPR = HW / VN;  // vectors per halo row
    if (p.use_tma) {
        if (t == 0) {
            const CUtensorMap *map = p.inst ? &p.tmaps[3 * ii + p.in_buf] : &p.tmap;
            tma::fence_proxy_async();
            tma::arrive_expect_tx(&sm.mbar, (uint32_t)sizeof(sm.w));
            tma::load_3d(&sm.w[0][0][0], map, j0 - NG, i0 - NG, 0, &sm.mbar);
            sm.tma_ok = tma::wait(&sm.mbar, phase);
        }
        phase ^= 1u;
        __syncthreads();
        if (!sm.tma_ok) {
            if (t == 0) {
                if (ctl != nullptr) atomicOr(&ctl->flags, AMHD_FLAG_TIMEOUT);
                tma::wait(&sm.mbar, phase ^ 1u);  // give the copy in flight a second bounded chance to land
            }
            return false;
        }
    }
    for (int q = t; q < HROWS * QPR; q += NT) {
        const int r = q / QPR, c = (q % QPR) * VN;
        R u[VN][NV];
        if (p.use_tma) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                VT x = *reinterpret_cast<const VT *>(&sm.w[v][r][c]);
                const R *xs = reinterpret_cast<const R *>(&x);
#pragma unroll
                for (int k = 0; k < VN; ++k) u[k][v] = xs[k];
            }
        } else {
            const int64_t gi = (int64_t)(i0 - NG + r) * pitch + (j0 - NG + c);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                VT x = __ldg(reinterpret_cast<const VT *>(uin + v * vs + gi));
                const R *xs = reinterpret_cast<const R *>(&x);
#pragma unroll
                for (int k = 0; k < VN; ++k) u[k][v] = xs[k];
            }
        }
        R wq[NV][VN];
#pragma unroll
        for (int k = 0; k < VN; ++k) {
            R w[NV];
            if constexpr (kFast<R>)
                fast::cons_to_prim(u[k], g.gamma, w);
            else
                cons_to_prim_cell(u[k], g.gamma, w);
#pragma unroll
            for (int v = 0; v < NV; ++v) wq[v][k] = w[v];
        }
        // one 16-byte shared store per plane (rows are 16-byte aligned: HW * sizeof(R) % 16 == 0)
#pragma unroll
        for (int v = 0; v < NV; ++v) *reinterpret_cast<VT *>(&sm.w[v][r][c]) = *reinterpret_cast<const VT *>(wq[v]);
    }
    __syncthreads();

    if constexpr (kFast<R>) {
        // ---- phase A2 (float32): limited slopes, once per cell and direction.
        // Work in 32-lane tasks that each stay on one shared-memory row:
        // TX+2 rows of x-slopes, TX rows of y-slopes (columns 1..32), and one
        // task for the last two y-slope columns of every row.
        constexpr int NTASK = (TX + 2) + TX + 1;
        const int lane = t & 31;
        for (int task = t >> 5; task < NTASK; task += NT / 32) {
            if (task < TX + 2) {
                const int r = task + 1, c = lane + NG;
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    sm.sx[v][r - 1][lane] = fast::slope(sm.w[v][r - 1][c], sm.w[v][r][c], sm.w[v][r + 1][c],
                                                        g.limiter);
            } else {
                int r, k;
                if (task < 2 * TX + 2) {
                    r = task - (TX + 2) + NG;
                    k = lane + 1;
                } else {
                    if (lane >= 2 * TX) continue;
                    r = (lane >> 1) + NG;
                    k = TY + 1 + (lane & 1);
                }
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    sm.sy[v][r - NG][k - 1] = fast::slope(sm.w[v][r][k - 1], sm.w[v][r][k], sm.w[v][r][k + 1],
                                                          g.limiter);
            }
        }
        __syncthreads();
    }

    // ---- phase B: MUSCL + HLLD on all faces of the tile -------------------
    const R gam = R(g.gamma), chr = R(ch);
    const int lim = g.limiter;
    constexpr int NFX = (TX + 1) * TY;
    constexpr int NFY = TX * (TY + 1);
    // one HLLD call site for x and y faces (y faces in the rotated slot order
    // rho, vy, vx, vz, By, Bx, Bz, p, psi, C of physics.py:376-379)
    constexpr int rot[NV] = {0, 2, 1, 3, 5, 4, 6, 7, 8, 9};
    const float igm1 = 1.0f / float(g.gamma - 1.0), half_ich = ch > 0.0 ? float(0.5 / ch) : 0.f;
    // 32-lane tasks on one row each: TX+1 rows of x faces, TX rows of y faces
    // (columns 0..31), one task for the last y face (column 32) of every row
    constexpr int NFTASK = (TX + 1) + TX + 1;
    static_assert(NFX + NFY == 32 * (2 * TX + 1) + TX, "face count");
    for (int f = t; f < 32 * NFTASK; f += NT) {
        const int task = f >> 5, lane = f & 31;
        if (task == NFTASK - 1 && lane >= TX) continue;
        R wl[NV], wr[NV], fl[NV];
        const bool xf = task <= TX;
        const int a = xf ? task : (task < NFTASK - 1 ? task - (TX + 1) : lane);
        const int c = xf ? lane : (task < NFTASK - 1 ? lane : TY);
        if constexpr (kFast<R>) {
            if (xf) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    wl[v] = sm.w[v][a + 1][c + NG] + 0.5f * sm.sx[v][a][c];
                    wr[v] = sm.w[v][a + 2][c + NG] - 0.5f * sm.sx[v][a + 1][c];
                }
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    wl[v] = sm.w[rot[v]][a + NG][c + 1] + 0.5f * sm.sy[rot[v]][a][c];
                    wr[v] = sm.w[rot[v]][a + NG][c + 2] - 0.5f * sm.sy[rot[v]][a][c + 1];
                }
            }
            fast::hlld(wl, wr, gam, igm1, chr, half_ich, fl, chr > 0.f);
        } else {
            if (xf) {
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    muscl_pair(sm.w[v][a][c + NG], sm.w[v][a + 1][c + NG], sm.w[v][a + 2][c + NG],
                               sm.w[v][a + 3][c + NG], lim, wl[v], wr[v]);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    muscl_pair(sm.w[rot[v]][a + NG][c], sm.w[rot[v]][a + NG][c + 1], sm.w[rot[v]][a + NG][c + 2],
                               sm.w[rot[v]][a + NG][c + 3], lim, wl[v], wr[v]);
            }
            // floors of physics.py:331-334 (slot 7 is p in both orders)
            wl[RHO] = np_max(wl[RHO], R(FLOOR_RHO));
            wr[RHO] = np_max(wr[RHO], R(FLOOR_RHO));
            wl[IPR] = np_max(wl[IPR], R(FLOOR_PR));
            wr[IPR] = np_max(wr[IPR], R(FLOOR_PR));
            hlld_flux(wl, wr, gam, chr, fl);
        }
        if (xf) {
#pragma unroll
            for (int v = 0; v < NV; ++v) sm.fx[v][a][c] = fl[v];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) sm.fy[rot[v]][a][c] = fl[v];
        }
    }
    __syncthreads();

    // ---- phase C: divergence, Powell, RK combine, clamp, BC push ----------
    const int a = t / TY, c = t % TY;  // tile cell
    const int i = i0 + a, j = j0 + c;   // storage index
    const bool valid = (i < NG + g.nx) && (j < NG + g.ny);
    unsigned long long q[4] = {0ull, 0ull, 0ull, 0ull};
    bool bad = false;
    if (valid) {
        R fxl[NV], fxr[NV], fyl[NV], fyr[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            fxl[v] = sm.fx[v][a][c];
            fxr[v] = sm.fx[v][a + 1][c];
            fyl[v] = sm.fy[v][a][c];
            fyr[v] = sm.fy[v][a][c + 1];
        }
        const int hr = a + NG, hc = c + NG;
        auto pw = [&]() {
            return PowellIn<R>{sm.w[BX][hr][hc],  sm.w[BX][hr - 1][hc], sm.w[BX][hr + 1][hc], sm.w[BY][hr][hc],
                               sm.w[BY][hr][hc - 1], sm.w[BY][hr][hc + 1], sm.w[IVX][hr][hc], sm.w[IVY][hr][hc],
                               sm.w[IVZ][hr][hc], sm.w[BZ][hr][hc]};
        };
        const int64_t gi = (int64_t)i * pitch + j;
        auto base_at = [&](int v) { return u0[v * vs + gi]; };
        auto in_at = [&](int v) { return uin[v * vs + gi]; };
        update_cell<R, STAGE>(p, g, uout, i, j, fxl, fxr, fyl, fyr, pw, base_at, in_at, dt, ch, decay, q, bad);
    }
    if (STAGE == 3) {
        // block reduction of the CFL maxima and of the non-finite flag
        const int lane = t & 31, warp = t >> 5;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            for (int o = 16; o > 0; o >>= 1) q[k] = umax64(q[k], __shfl_xor_sync(0xffffffffu, q[k], o));
        const unsigned any_bad = __any_sync(0xffffffffu, bad);
        if (t == 0) sm.nonfinite = 0;
        __syncthreads();
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k) sm.red[k][warp] = q[k];
            if (any_bad) sm.nonfinite = 1;
        }
        __syncthreads();
        if (t == 0 && ctl != nullptr) {
            if (p.fuse_dt) {
                for (int k = 0; k < 4; ++k) {
                    unsigned long long m = 0ull;
                    for (int w = 0; w < NT / 32; ++w) m = umax64(m, sm.red[k][w]);
                    atomicMax(reinterpret_cast<unsigned long long *>(&ctl->red[k]), m);
                }
            }
            if (sm.nonfinite) atomicOr(&ctl->flags, AMHD_FLAG_NONFINITE);
        }
    }
    return true;
}

// resident CTAs per SM the register budget is shaped for (float32 path)
template <typename R, int TX>
constexpr int kMinBlocks = kFast<R> ? (TX == 4 ? 6 : (TX == 8 ? 3 : 1)) : 1;

template <typename R, int TX, int STAGE>
__global__ void __launch_bounds__(TX * TY, (kMinBlocks<R, TX>)) rk_stage_kernel(const __grid_constant__ StageParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileSmem<R, TX> &sm = *reinterpret_cast<TileSmem<R, TX> *>(smem_raw);
    uint32_t phase = 0;
    if (p.use_tma) {
        if (threadIdx.x == 0) tma::mbar_init(&sm.mbar, 1);
        __syncthreads();
    }
    for (int pos = blockIdx.x; pos < p.n_tiles; pos += gridDim.x) {
        const int tile = p.tile_order ? p.tile_order[pos] : pos;
        if (!rk_stage_tile<R, TX, STAGE>(p, sm, tile, phase)) return;
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// ---------------------------------------------------------------------------
// warp-marching RK stage.  One warp owns a work item of kMarchCols interior
// columns x march_rows rows; lane l holds column (first - 2 + l), so the 32
// lanes cover the item's columns plus a 2-column halo on each side.  The warp
// walks the rows in x order: each row of the input state is fetched once
// (cp.async, one row ahead) and converted to primitives once, the x-slope and
// the flux through the face below the current row are carried from the
// previous row, and y-neighbours come from the adjacent lanes (warp shuffles).
// No CTA barrier: the warps of a CTA run independently.  The per-cell
// arithmetic is the tiled kernel's (same functions, same operation order), so
// float64 results are identical to it.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void to_prim(const R u[NV], double gamma, R w[NV])
{
    if constexpr (kFast<R>)
        fast::cons_to_prim(u, gamma, w);
    else
        cons_to_prim_cell(u, gamma, w);
}

template <typename R>
__device__ __forceinline__ R cell_slope(R wm, R w0, R wp, int limiter)
{
    if constexpr (kFast<R>)
        return fast::slope(wm, w0, wp, limiter);
    else
        return limited_slope(wm, w0, wp, limiter);
}

// HLLD flux of one face from its reconstructed states (slot order of an x face);
// glm: chr > 0 (see fast::hlld)
template <typename R>
__device__ __forceinline__ void face_flux(R wl[NV], R wr[NV], R gam, float igm1, R chr, float half_ich, R f[NV],
                                          bool glm)
{
    if constexpr (kFast<R>) {
        fast::hlld(wl, wr, gam, igm1, chr, half_ich, f, glm);
    } else {
        // floors of physics.py:331-334 (slot 7 is p in both orders)
        wl[RHO] = np_max(wl[RHO], R(FLOOR_RHO));
        wr[RHO] = np_max(wr[RHO], R(FLOOR_RHO));
        wl[IPR] = np_max(wl[IPR], R(FLOOR_PR));
        wr[IPR] = np_max(wr[IPR], R(FLOOR_PR));
        hlld_flux(wl, wr, gam, chr, f);
    }
}

// per-warp shared memory of the marching kernel.  A row holds the 10 planes of
// 32 lanes as [pair][lane][2]: variables 2k and 2k+1 of one lane side by side,
// so that a lane moves a pair with one 8-byte (float) or 16-byte (double)
// access and a warp's access covers 256 / 512 contiguous bytes (conflict-free).
// Every row but fy is private to its lane.
template <typename R>
using MarchRow = R[NV / 2][32][2];
// one row of the 10 planes as a TMA box {32 columns, 1 row, 10 planes} lands: plane-major
template <typename R>
using MarchPlanes = R[NV][32];

// TMA: the staged rows are plane-major boxes written by the tensor-memory
// accelerator (one copy per row for the whole warp, completion on an mbarrier
// per slot); otherwise pair-interleaved rows that each lane fills with cp.async
template <typename R, bool TMA>
struct MarchSmem;
template <typename R>
struct MarchSmem<R, false> {
    MarchRow<R> raw[3];  // conserved stage-input rows i .. i+2 (cp.async), row r in slot r % 3
    MarchRow<R> base;    // U0 of row i when U0 is not the stage input
    MarchRow<R> sx;      // limited x-slope of the current row
    MarchRow<R> fx;      // flux through the x face below the current row
    MarchRow<R> fy;      // flux through each lane's left y face of the current row (read by the lane on the left)
};
template <typename R>
struct __align__(128) MarchSmem<R, true> {
    MarchPlanes<R> raw[3];  // conserved stage-input rows i .. i+2 (TMA), row r in slot r % 3
    MarchPlanes<R> base;    // U0 of row i when U0 is not the stage input (TMA)
    MarchRow<R> sx;
    MarchRow<R> fx;
    MarchRow<R> fy;
    uint64_t bar[4];        // completion of raw[0..2] and base
};

template <typename R>
struct Pair;
template <>
struct Pair<float> {
    using T = float2;
};
template <>
struct Pair<double> {
    using T = double2;
};

// the 10 values of one lane's column of a row, pairwise
template <typename R>
__device__ __forceinline__ void row_load(const MarchRow<R> &r, int lane, R u[NV])
{
#pragma unroll
    for (int k = 0; k < NV / 2; ++k) {
        const typename Pair<R>::T t = *reinterpret_cast<const typename Pair<R>::T *>(&r[k][lane][0]);
        u[2 * k] = t.x;
        u[2 * k + 1] = t.y;
    }
}
template <typename R>
__device__ __forceinline__ void row_store(MarchRow<R> &r, int lane, const R u[NV])
{
#pragma unroll
    for (int k = 0; k < NV / 2; ++k) {
        typename Pair<R>::T t;
        t.x = u[2 * k];
        t.y = u[2 * k + 1];
        *reinterpret_cast<typename Pair<R>::T *>(&r[k][lane][0]) = t;
    }
}

template <typename R>
__device__ __forceinline__ typename Pair<R>::T pair_load(const MarchRow<R> &r, int k, int lane)
{
    return *reinterpret_cast<const typename Pair<R>::T *>(&r[k][lane][0]);
}
template <typename R>
__device__ __forceinline__ void pair_store(MarchRow<R> &r, int k, int lane, R a, R b)
{
    typename Pair<R>::T t;
    t.x = a;
    t.y = b;
    *reinterpret_cast<typename Pair<R>::T *>(&r[k][lane][0]) = t;
}

// asynchronous copy of one row of the state (this lane's column) into shared memory
template <typename R>
__device__ __forceinline__ void fetch_row(MarchRow<R> &dst, const R *u, int64_t vs, int64_t gi, int lane)
{
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const uint32_t d = (uint32_t)__cvta_generic_to_shared(&dst[v >> 1][lane][v & 1]);
        if constexpr (sizeof(R) == 4)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(u + v * vs + gi) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(u + v * vs + gi) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void fetch_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One work item: rows [ib, ie) of a 28-column strip.  SPEC: the item runs the
// van Leer limiter with GLM on (ch > 0), known at compile time -- the walk the
// solver's loop takes; otherwise both are read at run time.
template <typename R, int STAGE, bool SPEC, bool TMA, bool COMP>
__device__ __forceinline__ bool march_walk(const StageParams &p, MarchSmem<R, TMA> &ms, const amhd_instance &in,
                                           int ii, const amhd_grid &g, int item, int lane, double dt, double ch,
                                           double decay, unsigned long long q[4], bool &bad, uint32_t &phase)
{
    // Item -> column strip, row chunk and this lane's column.  A plain item is one
    // chunk of one strip across the warp's 32 lanes (28 columns updated).  With
    // in.pack = P > 1 the items of the last strip, whose leftover columns (with
    // their 2-column halo on each side) fit 32/P lanes, put P segments of 32/P
    // lanes side by side, segment s walking chunk P m + s; all segments of an
    // item have as many rows (the short last chunk has an item of its own).
    // The packed items come first, the plain ones chunk-major after them.  A pack
    // value other than the rule's (march_pack) is taken as none.
    const int local = item - in.first_tile;
    const int P = (TMA || in.pack <= 1 || in.pack != march_pack(g.ny)) ? 1 : in.pack;
    const int plain_strips = P > 1 ? in.tiles_y - 1 : in.tiles_y;
    const int full_chunks = g.nx / p.march_rows;
    const int n_full_packed = P > 1 ? (full_chunks + P - 1) / P : 0;
    const int n_packed = P > 1 ? n_full_packed + (full_chunks * p.march_rows < g.nx ? 1 : 0) : 0;
    int strip, chunk, n_rows, lane_c = lane, seg_w = 32;
    bool seg_live = true;
    if (local >= n_packed) {
        strip = (local - n_packed) % plain_strips;
        chunk = (local - n_packed) / plain_strips;
        n_rows = min(p.march_rows, g.nx - chunk * p.march_rows);
    } else {
        const int m = local;
        const int seg = P == 4 ? lane >> 3 : lane >> 4;
        seg_w = P == 4 ? 8 : 16;
        lane_c = lane - seg * seg_w;
        strip = in.tiles_y - 1;
        if (m < n_full_packed) {
            chunk = m * P + seg;
            seg_live = chunk < full_chunks;
            if (!seg_live) chunk = m * P;  // walks the first segment's rows, stores nothing
            n_rows = p.march_rows;
        } else {
            chunk = full_chunks;
            seg_live = seg == 0;
            n_rows = g.nx - full_chunks * p.march_rows;
        }
    }
    if (n_rows <= 0) return true;  // an item past the instance's last (a work list that counts too many)
    const int j = kMarchCols * strip + lane_c;  // storage column of this lane (first interior column - 2 + lane_c)
    // ghost cells of the input: as stored, or (pull) taken from the interior cells
    // they copy (apply_bc, solver.py:158-197; psi zero in non-periodic x ghosts)
    const bool pull = p.pull_ghosts != 0;
    const int jl = pull ? ghost_source(min(j, NG + g.ny + 1), g.ny, g.bc_y)
                        : min(j, g.pitch - 1);  // lanes past the padded row load a cell they do not use
    const bool zero_psi = pull && g.bc_x != AMHD_BC_PERIODIC;
    auto src_row = [&](int r) { return pull ? ghost_source(r, g.nx, g.bc_x) : r; };
    auto ghost_psi = [&](int r, R u[NV]) {
        if (zero_psi && (r < NG || r >= NG + g.nx)) u[PSI] = R(0);
    };
    const int ib = NG + chunk * p.march_rows;  // first row of this lane's chunk
    const int64_t vs = g.var_stride;
    const int pitch = g.pitch;
    const R *uin = reinterpret_cast<const R *>(p.uin) + in.offset;
    const R *u0 = reinterpret_cast<const R *>(p.u0) + in.offset;
    R *uout = reinterpret_cast<R *>(p.uout) + in.offset;
    R *ulo = COMP ? reinterpret_cast<R *>(p.ulo) + in.offset : nullptr;
    // the segment's two lanes on each side are its halo
    const bool out_lane = seg_live && lane_c >= NG && lane_c < seg_w - NG && j < NG + g.ny;
    // U0 comes from its own buffer unless it is the stage input (stage 1 of a step)
    const bool own_base = STAGE >= 1 && p.u0 != p.uin;

    // ---- row staging: per-lane cp.async into pair rows, or one TMA box per row
    const int x0 = j - lane;  // column of lane 0 (28 x strip: 16-byte aligned for 4- and 8-byte values)
    const CUtensorMap *map_in = nullptr, *map_base = nullptr;
    if constexpr (TMA) {
        map_in = p.inst ? &p.tmaps[3 * ii + p.in_buf] : &p.tmap;
        map_base = p.inst ? &p.tmaps[3 * ii] : &p.tmap_base;
    }
    uint32_t pending = 0;  // TMA: slots (bits 0-2) and the base row (bit 3) with a copy in flight
    bool gave_up = false;
    auto fetch_in = [&](int slot, int r) {
        if constexpr (TMA) {
            __syncwarp();  // every lane is done reading the slot
            if (lane == 0) {
                tma::fence_proxy_async();
                tma::arrive_expect_tx(&ms.bar[slot], (uint32_t)sizeof(MarchPlanes<R>));
                tma::load_3d(&ms.raw[slot][0][0], map_in, x0, src_row(r), 0, &ms.bar[slot]);
            }
            pending |= 1u << slot;
        } else {
            fetch_row(ms.raw[slot], uin, vs, (int64_t)src_row(r) * pitch + jl, lane);
        }
    };
    auto fetch_base = [&](int r) {
        if constexpr (TMA) {
            __syncwarp();
            if (lane == 0) {
                tma::fence_proxy_async();
                tma::arrive_expect_tx(&ms.bar[3], (uint32_t)sizeof(MarchPlanes<R>));
                tma::load_3d(&ms.base[0][0], map_base, x0, r, 0, &ms.bar[3]);
            }
            pending |= 8u;
        } else {
            fetch_row(ms.base, u0, vs, (int64_t)r * pitch + jl, lane);
        }
    };
    // wait for the copies of the slots in `mask` (TMA) or for every copy (cp.async)
    auto wait_rows = [&](uint32_t mask) {
        if constexpr (TMA) {
            mask &= pending;
            for (int k = 0; k < 4; ++k)
                if (mask >> k & 1u) {
                    if (tma::wait(&ms.bar[k], phase >> k & 1u)) {
                        phase ^= 1u << k;
                        pending &= ~(1u << k);
                    } else {
                        gave_up = true;  // still in flight: the abort path waits for it once more
                    }
                }
        } else {
            fetch_wait();
        }
    };
    // this lane's column of an input row; in TMA boxes the ghost columns hold what
    // is stored, so a lane whose column is a ghost the row pulls reads its source
    const bool fix_col = TMA && pull && (j < NG || j >= NG + g.ny) && j < NG + g.ny + NG;
    auto load_in = [&](int slot, int r, R u[NV]) {
        if constexpr (TMA) {
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = ms.raw[slot][v][lane];
            if (fix_col) {
                const R *src = uin + (int64_t)src_row(r) * pitch + jl;
#pragma unroll
                for (int v = 0; v < NV; ++v) u[v] = src[v * vs];
            }
        } else {
            row_load(ms.raw[slot], lane, u);
        }
    };
    auto load_cell = [&](int slot, R u[NV]) {  // interior cells: as staged
        if constexpr (TMA) {
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = ms.raw[slot][v][lane];
        } else {
            row_load(ms.raw[slot], lane, u);
        }
    };
    auto load_base = [&](R u[NV]) {
        if constexpr (TMA) {
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = ms.base[v][lane];
        } else {
            row_load(ms.base, lane, u);
        }
    };

    const R gam = R(g.gamma), chr = R(ch);
    const int lim = SPEC ? AMHD_LIMITER_VANLEER : g.limiter;
    const bool glm = SPEC || chr > R(0);
    const float igm1 = 1.0f / float(g.gamma - 1.0), half_ich = ch > 0.0 ? float(0.5 / ch) : 0.f;
    constexpr int rot[NV] = {0, 2, 1, 3, 5, 4, 6, 7, 8, 9};

    // Rows ib-2 .. ib are fetched up front and row ib+1 behind them.  The walk
    // starts one row early: iteration ib-1 only computes the flux through face
    // ib-1/2 (no y faces, no update), so the x-face code is not repeated in a
    // prologue.  Input row ib-2+k lives in slot k % 3 (the same slot in every
    // segment of an item); each iteration fetches the input row three ahead and
    // the next row of U0 once it is done with the slots they replace, and waits
    // for them just before the x faces.
    int s0 = 0;  // slot of row i (ib-2 here)
    constexpr int s1i = 1, s2i = 2;
    fetch_in(s0, ib - 2);
    fetch_in(s1i, ib - 1);
    fetch_in(s2i, ib);
    wait_rows(7u);
    R w0[NV], w1[NV], bxm = R(0);
    {
        R u[NV], wa[NV];
        load_in(s0, ib - 2, u);
        ghost_psi(ib - 2, u);
        to_prim(u, g.gamma, wa);
        fetch_in(s0, ib + 1);  // row ib-2 is converted
        load_in(s1i, ib - 1, u);
        ghost_psi(ib - 1, u);
        to_prim(u, g.gamma, w0);
        load_in(s2i, ib, u);
        to_prim(u, g.gamma, w1);
#pragma unroll
        for (int v = 0; v < NV; ++v) wa[v] = cell_slope(wa[v], w0[v], w1[v], lim);
        row_store(ms.sx, lane, wa);  // slope of row ib-1
    }
    s0 = s1i;  // slot of row ib-1

    for (int r = -1; r < n_rows; ++r) {
        const int i = ib + r;       // row of this lane's chunk
        const bool full = r >= 0;  // warp-uniform: iteration ib-1 only prepares face ib-1/2
        const int s2 = s0 == 0 ? 2 : s0 - 1;  // slot of row i+2 (== (i + 2) % 3)
        __syncwarp();  // the left neighbour has read ms.fy of row i-1
        R bym = R(0), byp = R(0);
        if (full) {
            // y: slope of this lane's cell of row i from its lane neighbours, and
            // the flux through the face on the cell's left (rotated slot order of
            // physics.py:376-379); the right face is the next lane's left face
            R wl[NV], wr[NV], f[NV];
            if constexpr (kFast<R>) {
                R ll[NV];  // states on each variable's left face, from the lane on the left
#pragma unroll
                for (int v = 0; v < NV; v += 2) {
                    // pairs in the stored slot order (as the x-slopes pair them);
                    // the rotation to the y-face order is a renaming below
                    const float2 c = make_float2(w0[v], w0[v + 1]);
                    const float2 m = make_float2(__shfl_up_sync(0xffffffffu, c.x, 1),
                                                 __shfl_up_sync(0xffffffffu, c.y, 1));
                    const float2 q = make_float2(__shfl_down_sync(0xffffffffu, c.x, 1),
                                                 __shfl_down_sync(0xffffffffu, c.y, 1));
                    const float2 sy = fast::slope2(m, c, q, lim);
                    const float2 r = __ffma2_rn(make_float2(-0.5f, -0.5f), sy, c);
                    const float2 l = __ffma2_rn(make_float2(0.5f, 0.5f), sy, c);
                    f[v] = r.x;
                    f[v + 1] = r.y;
                    ll[v] = __shfl_up_sync(0xffffffffu, l.x, 1);
                    ll[v + 1] = __shfl_up_sync(0xffffffffu, l.y, 1);
                    if (v + 1 == BY) {
                        bym = m.y;
                        byp = q.y;
                    }
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    wr[k] = f[rot[k]];
                    wl[k] = ll[rot[k]];
                }
            } else {
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const int v = rot[k];
                    const R wm = __shfl_up_sync(0xffffffffu, w0[v], 1);
                    const R wp = __shfl_down_sync(0xffffffffu, w0[v], 1);
                    const R sy = cell_slope(wm, w0[v], wp, lim);
                    wr[k] = w0[v] - R(0.5) * sy;
                    wl[k] = __shfl_up_sync(0xffffffffu, w0[v] + R(0.5) * sy, 1);
                    if (v == BY) {
                        bym = wm;
                        byp = wp;
                    }
                }
            }
            face_flux(wl, wr, gam, igm1, chr, half_ich, f, glm);
#pragma unroll
            for (int k = 0; k < NV; ++k) wl[rot[k]] = f[k];  // back to the unrotated slot order
            row_store(ms.fy, lane, wl);
        }
        // x: primitives of row i+2, slope of row i+1, flux through face i+1/2 and
        // the x-flux difference of row i
        wait_rows((1u << s2) | 8u);  // input row i+2 and U0 of row i have landed
        if (TMA && __any_sync(0xffffffffu, gave_up)) {
            // a copy never completed: give the others in flight a bounded chance to
            // land (the shared rows must not be written after the CTA leaves), then stop
            wait_rows(15u);
            return false;
        }
        R w2[NV], dfx[NV];
        {
            R u[NV], wl[NV], wr[NV], f[NV];
            load_in(s2, i + 2, u);
            ghost_psi(i + 2, u);
            to_prim(u, g.gamma, w2);
            if constexpr (kFast<R>) {
                // pairs of variables on the packed float32x2 path
#pragma unroll
                for (int v = 0; v < NV; v += 2) {
                    const float2 a = make_float2(w0[v], w0[v + 1]), b = make_float2(w1[v], w1[v + 1]);
                    const float2 s1 = fast::slope2(a, b, make_float2(w2[v], w2[v + 1]), lim);
                    const float2 l = __ffma2_rn(make_float2(0.5f, 0.5f), pair_load(ms.sx, v >> 1, lane), a);
                    const float2 r = __ffma2_rn(make_float2(-0.5f, -0.5f), s1, b);
                    wl[v] = l.x;
                    wl[v + 1] = l.y;
                    wr[v] = r.x;
                    wr[v + 1] = r.y;
                    pair_store(ms.sx, v >> 1, lane, s1.x, s1.y);
                }
            } else {
                R sx[NV];
                row_load(ms.sx, lane, sx);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const R s1 = cell_slope(w0[v], w1[v], w2[v], lim);
                    wl[v] = w0[v] + R(0.5) * sx[v];
                    wr[v] = w1[v] - R(0.5) * s1;
                    sx[v] = s1;
                }
                row_store(ms.sx, lane, sx);
            }
            face_flux(wl, wr, gam, igm1, chr, half_ich, f, glm);
#pragma unroll
            for (int k = 0; k < NV / 2; ++k) {
                const typename Pair<R>::T o = pair_load(ms.fx, k, lane);
                if constexpr (kFast<R>) {
                    const float2 d = __ffma2_rn(o, make_float2(-1.f, -1.f), make_float2(f[2 * k], f[2 * k + 1]));
                    dfx[2 * k] = d.x;
                    dfx[2 * k + 1] = d.y;
                } else {
                    dfx[2 * k] = f[2 * k] - o.x;
                    dfx[2 * k + 1] = f[2 * k + 1] - o.y;
                }
                pair_store(ms.fx, k, lane, f[2 * k], f[2 * k + 1]);
            }
        }
        if (full) {
            __syncwarp();  // every lane's y-face flux of row i is in ms.fy
            if (out_lane) {
                R dfy[NV];
#pragma unroll
                for (int k = 0; k < NV / 2; ++k) {  // output lanes stop at 29
                    const typename Pair<R>::T a = pair_load(ms.fy, k, lane + 1), b = pair_load(ms.fy, k, lane);
                    if constexpr (kFast<R>) {
                        const float2 d = __ffma2_rn(b, make_float2(-1.f, -1.f), a);  // a - b, one rounding
                        dfy[2 * k] = d.x;
                        dfy[2 * k + 1] = d.y;
                    } else {
                        dfy[2 * k] = a.x - b.x;
                        dfy[2 * k + 1] = a.y - b.y;
                    }
                }
                auto pw = [&]() {
                    return PowellIn<R>{w0[BX], bxm, w1[BX], w0[BY], bym, byp, w0[IVX], w0[IVY], w0[IVZ], w0[BZ]};
                };
                R us[NV], ub[NV];
                load_cell(s0, us);
                if (own_base)
                    load_base(ub);
                else
                    load_cell(s0, ub);
                auto in_at = [&](int v) { return us[v]; };
                auto base_at = [&](int v) { return ub[v]; };
                update_cell_d<R, STAGE, false, COMP>(p, g, uout, i, j, dfx, dfy, pw, base_at, in_at, dt, ch, decay, q,
                                                     bad, ulo);
            }
        }
        // rows done with: input row i (slot s0) -> row i+3; U0 of row i -> row i+1
        if (r + 1 < n_rows) {
            fetch_in(s0, i + 3);
            if (own_base) fetch_base(i + 1);
        }
        s0 = s0 == 2 ? 0 : s0 + 1;
        bxm = w0[BX];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            w0[v] = w1[v];
            w1[v] = w2[v];
        }
    }
    __syncwarp();  // the next item reuses the shared rows
    return true;
}

// false when a row copy never completed (TMA): the warp then stops
template <typename R, int STAGE, bool TMA, bool COMP>
__device__ __forceinline__ bool march_item(const StageParams &p, MarchSmem<R, TMA> &ms, int item, int lane,
                                           unsigned long long q[4], bool &bad, amhd_control *&ctl_out,
                                           uint32_t &phase)
{
    int ii;
    const amhd_instance &in = inst_of(p, item, ii);
    const amhd_grid g = in.grid;
    amhd_control *ctl = p.ctl ? p.ctl + ii : nullptr;
    ctl_out = ctl;
    double dt = p.dt, ch = p.ch, decay = p.decay;
    if (p.use_ctl) {
        if (!ctl->active) return true;
        dt = ctl->dt;
        ch = ctl->ch;
        decay = ctl->decay;
    }
    bool ok;
    if (g.limiter == AMHD_LIMITER_VANLEER && R(ch) > R(0))
        ok = march_walk<R, STAGE, true, TMA, COMP>(p, ms, in, ii, g, item, lane, dt, ch, decay, q, bad, phase);
    else
        ok = march_walk<R, STAGE, false, TMA, COMP>(p, ms, in, ii, g, item, lane, dt, ch, decay, q, bad, phase);
    if (!ok && lane == 0 && ctl != nullptr) atomicOr(&ctl->flags, AMHD_FLAG_TIMEOUT);
    return ok;
}

// resident CTAs of kMarchThreads per SM the register budget is shaped for:
// float32 4 (128 registers, no spills; 5 CTAs at 96 registers spilled and ran
// 5 % slower), float64 2
template <typename R, int STAGE>
constexpr int kMarchMinBlocks = kFast<R> ? 4 : 2;

// The work loop of a marching kernel's warp: take items (from the queue or the
// static split), run each (run_item(item, q, bad, ctl) returns false when the
// warp must stop), reduce each item's CFL maxima and non-finite flag into its
// instance's control block (last stage), and reset the queue at the end.
template <int STAGE, typename ItemFn>
__device__ __forceinline__ void march_items(const StageParams &p, int lane, ItemFn run_item)
{
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int n_warps = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    // work positions: from the queue (each warp takes the next free position when it
    // is done with its item, so uneven items leave no warp idle while work remains),
    // or the static split w, w + n_warps, ...
    auto next_pos = [&](int prev) {
        if (p.queue == nullptr) return prev < 0 ? warp : prev + n_warps;
        int t = 0;
        if (lane == 0) t = atomicAdd(&p.queue[0], 1);
        return __shfl_sync(0xffffffffu, t, 0);
    };
    for (int pos = next_pos(-1); pos < p.n_tiles; pos = next_pos(pos)) {
        const int item = p.tile_order ? p.tile_order[pos] : pos;
        unsigned long long q[4] = {0ull, 0ull, 0ull, 0ull};
        bool bad = false;
        amhd_control *ctl = nullptr;
        if (!run_item(item, q, bad, ctl)) break;
        if (STAGE == 3 && ctl != nullptr) {
            // warp reduction of the CFL maxima and of the non-finite flag of the item
#pragma unroll
            for (int k = 0; k < 4; ++k)
                for (int o = 16; o > 0; o >>= 1) q[k] = umax64(q[k], __shfl_xor_sync(0xffffffffu, q[k], o));
            const unsigned any_bad = __any_sync(0xffffffffu, bad);
            if (lane == 0) {
                if (p.fuse_dt)
                    for (int k = 0; k < 4; ++k)
                        if (q[k]) atomicMax(reinterpret_cast<unsigned long long *>(&ctl->red[k]), q[k]);
                if (any_bad) atomicOr(&ctl->flags, AMHD_FLAG_NONFINITE);
            }
        }
    }
    if (p.queue != nullptr && lane == 0) {
        // every warp has drawn a position past the end before it counts itself out, so
        // the last one out may reset the queue for the next launch of the stream
        if (atomicAdd(&p.queue[1], 1) == n_warps - 1) {
            atomicExch(&p.queue[0], 0);
            atomicExch(&p.queue[1], 0);
        }
    }
}

template <typename R, int STAGE, bool TMA, bool COMP = false>
__global__ void __launch_bounds__(kMarchThreads, (kMarchMinBlocks<R, STAGE>)) march_stage_kernel(
    const __grid_constant__ StageParams p)
{
    extern __shared__ __align__(128) unsigned char march_smem[];
    // run loop: the next launch may take SM slots as this grid drains; nothing
    // of the previous launch (stage input, controls) is read before it is done
    pdl_trigger();
    pdl_wait();
    MarchSmem<R, TMA> &ms = reinterpret_cast<MarchSmem<R, TMA> *>(march_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    uint32_t phase = 0;  // TMA: parity of the next completion of each of the warp's 4 barriers
    if constexpr (TMA) {
        if (lane < 4) tma::mbar_init(&ms.bar[lane], 1);
        __syncwarp();
    }
    march_items<STAGE>(p, lane, [&](int item, unsigned long long q[4], bool &bad, amhd_control *&ctl) {
        return march_item<R, STAGE, TMA, COMP>(p, ms, item, lane, q, bad, ctl, phase);
    });
}

// ---------------------------------------------------------------------------
// ghost fill by pull (apply_bc, solver.py:158-197): every ghost takes its
// interior source, so one pass in any order reproduces the reference.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void fill_ghosts(const amhd_grid &g, R *U, int64_t first, int64_t step)
{
    const int nxt = g.nx + 2 * NG, nyt = g.ny + 2 * NG;
    const int64_t n_rows = 4LL * nyt;  // x-ghost rows, full length
    const int64_t n_total = n_rows + 4LL * g.nx;
    for (int64_t k = first; k < n_total; k += step) {
        int i, j;
        if (k < n_rows) {
            const int r = (int)(k / nyt);
            i = r < NG ? r : nxt - 2 * NG + r;
            j = (int)(k % nyt);
        } else {
            const int64_t h = k - n_rows;
            i = NG + (int)(h / 4);
            const int c = (int)(h % 4);
            j = c < NG ? c : nyt - 2 * NG + c;
        }
        const int si = ghost_source(i, g.nx, g.bc_x), sj = ghost_source(j, g.ny, g.bc_y);
        const bool xg = (i < NG) || (i >= NG + g.nx);
        for (int v = 0; v < NV; ++v) {
            R val = U[v * g.var_stride + (int64_t)si * g.pitch + sj];
            if (v == PSI && xg && g.bc_x != AMHD_BC_PERIODIC) val = R(0);
            U[v * g.var_stride + (int64_t)i * g.pitch + j] = val;
        }
    }
}

template <typename R>
__global__ void bc_fill_kernel(const amhd_grid g, R *U)
{
    fill_ghosts(g, U, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// ghost fill of a marching stage's output, every instance of the stage
// (blockIdx.y = instance); instances whose loop has stopped are skipped
template <typename R>
__global__ void march_bc_fill_kernel(const __grid_constant__ StageParams p)
{
    const int k = blockIdx.y;
    const amhd_instance &in = p.inst ? p.inst[k] : p.one;
    if (p.use_ctl && !p.ctl[k].active) return;
    fill_ghosts(in.grid, reinterpret_cast<R *>(p.uout) + in.offset, blockIdx.x * (int64_t)blockDim.x + threadIdx.x,
                (int64_t)gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// elementwise kernels over all cells (ghosts included)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void cons_to_prim_kernel(const Layout li, const R *U, const Layout lo, R *W, double gamma)
{
    const int64_t n = (int64_t)li.nxt * li.nyt;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / li.nyt), j = (int)(k % li.nyt);
        R u[NV], w[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) u[v] = U[v * li.var_stride + (int64_t)i * li.pitch + j];
        cons_to_prim_cell(u, gamma, w);
#pragma unroll
        for (int v = 0; v < NV; ++v) W[v * lo.var_stride + (int64_t)i * lo.pitch + j] = w[v];
    }
}

// prim_to_cons, physics.py:304-320 (double arithmetic for both precisions)
template <typename R>
__global__ void prim_to_cons_kernel(const Layout li, const R *W, const Layout lo, R *U, double gamma)
{
    const int64_t n = (int64_t)li.nxt * li.nyt;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / li.nyt), j = (int)(k % li.nyt);
        double w[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = (double)W[v * li.var_stride + (int64_t)i * li.pitch + j];
        double rho = np_max(w[0], FLOOR_RHO);
        double u[NV];
        u[RHO] = rho;
        u[MX] = rho * w[1];
        u[MY] = rho * w[2];
        u[MZ] = rho * w[3];
        u[BX] = w[4];
        u[BY] = w[5];
        u[BZ] = w[6];
        u[PSI] = w[8];
        u[RHOC] = rho * w[9];
        double ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
        double me = 0.5 * (w[4] * w[4] + w[5] * w[5] + w[6] * w[6]);
        u[EN] = w[7] / (gamma - 1.0) + ke + me;
#pragma unroll
        for (int v = 0; v < NV; ++v) U[v * lo.var_stride + (int64_t)i * lo.pitch + j] = (R)u[v];
    }
}

// enforce_scalar_bounds, solver.py:199-204
template <typename R>
__global__ void scalar_bounds_kernel(const Layout l, R *U)
{
    const int64_t n = (int64_t)l.nxt * l.nyt;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = (k / l.nyt) * l.pitch + (k % l.nyt);
        R rho = np_max(U[RHO * l.var_stride + c], R(FLOOR_RHO));
        R cc = np_min(np_max(U[RHOC * l.var_stride + c] / rho, R(0)), R(1));
        U[RHOC * l.var_stride + c] = rho * cc;
    }
}

// muscl_x / muscl_y, physics.py:323-350 -> contiguous [10][nf]
template <typename R>
__global__ void muscl_kernel(const Layout l, const R *W, int axis, int limiter, R *WL, R *WR)
{
    const int nfx = axis == 0 ? l.nxt - 3 : l.nxt, nfy = axis == 0 ? l.nyt : l.nyt - 3;
    const int64_t nf = (int64_t)nfx * nfy;
    const int64_t step = axis == 0 ? l.pitch : 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nf; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / nfy), j = (int)(k % nfy);
        const int64_t c0 = (int64_t)i * l.pitch + j;
        R wl[NV], wr[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const R *pv = W + v * l.var_stride + c0;
            muscl_pair(pv[0], pv[step], pv[2 * step], pv[3 * step], limiter, wl[v], wr[v]);
        }
        wl[RHO] = np_max(wl[RHO], R(FLOOR_RHO));
        wr[RHO] = np_max(wr[RHO], R(FLOOR_RHO));
        wl[IPR] = np_max(wl[IPR], R(FLOOR_PR));
        wr[IPR] = np_max(wr[IPR], R(FLOOR_PR));
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            WL[v * nf + k] = wl[v];
            WR[v * nf + k] = wr[v];
        }
    }
}

// hlld_flux_x / hlld_flux_y, physics.py:353-379
template <typename R>
__global__ void hlld_kernel(const R *WL, const R *WR, R *F, R *smax, int64_t n, int axis, R gamma, R ch)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        R wl[NV], wr[NV], f[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            wl[v] = WL[v * n + k];
            wr[v] = WR[v * n + k];
        }
        if (axis == 1) {
            rot_xy(wl);
            rot_xy(wr);
        }
        R s = hlld_flux(wl, wr, gamma, ch, f);
        if (axis == 1) rot_xy(f);
#pragma unroll
        for (int v = 0; v < NV; ++v) F[v * n + k] = f[v];
        if (smax) smax[k] = s;
    }
}

// _compute_powell_source, solver.py:242-266 from primitive W
template <typename R>
__global__ void powell_kernel(const Layout l, const R *W, R *S, R dx, R dy)
{
    const int64_t n = (int64_t)l.nxt * l.nyt;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / l.nyt), j = (int)(k % l.nyt);
        const int64_t c = (int64_t)i * l.pitch + j;
        R s[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = R(0);
        if (i >= 1 && i < l.nxt - 1 && j >= 1 && j < l.nyt - 1) {
            const R *bx = W + BX * l.var_stride, *by = W + BY * l.var_stride;
            R divb = (R(0.5) * (bx[c] + bx[c + l.pitch]) - R(0.5) * (bx[c - l.pitch] + bx[c])) / dx +
                     (R(0.5) * (by[c] + by[c + 1]) - R(0.5) * (by[c - 1] + by[c])) / dy;
            R vx = W[IVX * l.var_stride + c], vy = W[IVY * l.var_stride + c], vz = W[IVZ * l.var_stride + c];
            R b0 = bx[c], b1 = by[c], b2 = W[BZ * l.var_stride + c];
            R vb = vx * b0 + vy * b1 + vz * b2;
            s[MX] = -divb * b0;
            s[MY] = -divb * b1;
            s[MZ] = -divb * b2;
            s[BX] = -divb * vx;
            s[BY] = -divb * vy;
            s[BZ] = -divb * vz;
            s[EN] = -divb * vb;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) S[v * l.var_stride + c] = s[v];
    }
}

// ---------------------------------------------------------------------------
// CFL reduction over all cells (compute_dt, solver.py:206-223) into ctl->red.
// from_prim: W (primitive) instead of U (conserved).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void dt_reduce_kernel(const Layout l, const R *A, int from_prim, double gamma, amhd_control *ctl)
{
    const int64_t n = (int64_t)l.nxt * l.nyt;
    unsigned long long q[4] = {0ull, 0ull, 0ull, 0ull};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = (k / l.nyt) * l.pitch + (k % l.nyt);
        double qd[4];
        if (from_prim) {
            double w[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) w[v] = (double)A[v * l.var_stride + c];
            cfl_quantities_prim(w, gamma, qd);
        } else {
            R u[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = A[v * l.var_stride + c];
            // float32 state: the arithmetic of the stage kernels' fused reduction,
            // so that a run resumed from a stored state takes the same dt
            if constexpr (kFast<R>)
                fast::cfl_quantities(u, gamma, qd);
            else
                cfl_quantities(u, gamma, qd);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) q[m] = umax64(q[m], ord_bits(qd[m]));
    }
    __shared__ unsigned long long red[4][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 4; ++m)
        for (int o = 16; o > 0; o >>= 1) q[m] = umax64(q[m], __shfl_xor_sync(0xffffffffu, q[m], o));
    if (lane == 0)
        for (int m = 0; m < 4; ++m) red[m][warp] = q[m];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int m = 0; m < 4; ++m) {
            unsigned long long v = 0ull;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = umax64(v, red[m][w]);
            atomicMax(reinterpret_cast<unsigned long long *>(&ctl->red[m]), v);
        }
    }
}

// _compute_boundary_energy_flux, solver.py:225-240: one block sums both columns
template <typename R>
__device__ double boundary_flux_block(const amhd_grid &g, const R *U, int cut_x = 0)
{
    __shared__ double part[2][32];
    const int nyt = g.ny + 2 * NG;
    const int cols[2] = {NG, g.nx + NG - 1};
    double acc[2] = {0.0, 0.0};
    for (int s = 0; s < 2; ++s)
        for (int j = NG + threadIdx.x; j < nyt - NG && !(cut_x >> s & 1); j += blockDim.x) {
            const int64_t c = (int64_t)cols[s] * g.pitch + j;
            double u[NV], w[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = (double)U[v * g.var_stride + c];
            cons_to_prim_cell(u, g.gamma, w);
            double b2 = w[4] * w[4] + w[5] * w[5] + w[6] * w[6];
            double pt = w[7] + 0.5 * b2;
            double vb = w[1] * w[4] + w[2] * w[5] + w[3] * w[6];
            acc[s] += ((u[EN] + pt) * w[1] - w[4] * vb) * g.dy;
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s = 0; s < 2; ++s) {
        double a = acc[s];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) part[s][warp] = a;
    }
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t0 += part[0][w];
            t1 += part[1][w];
        }
        r = t0 - t1;
    }
    __syncthreads();
    return r;  // valid in thread 0
}

template <typename R>
__global__ void bflux_kernel(const amhd_grid g, const R *U, double *out)
{
    double r = boundary_flux_block(g, U);
    if (threadIdx.x == 0) *out = r;
}

template <typename R>
__global__ void bflux_accum_kernel(const amhd_grid g, const R *U, amhd_control *ctl, double dt)
{
    double r = boundary_flux_block(g, U);
    if (threadIdx.x == 0) ctl->e_bnd += r * dt;
}

// ---------------------------------------------------------------------------
// finalize: dt, ch and loop control from the reduced maxima.
//   advance = 0: before the first step (run(), solver.py:476-479)
//   advance = 1: after a step: t += dt, step += 1, then the next dt
//   set_only = 1: compute_dt API -- only dt_cfl / ch (no loop state touched)
// One block per instance (blockIdx.x), U / grid from the instance table.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void finalize_kernel(const amhd_instance *insts, const amhd_instance one, const R *Ubase,
                                amhd_control *ctls, int advance, int set_only)
{
    pdl_trigger();
    pdl_wait();  // the reduced maxima of the stage before
    const amhd_instance &in = insts ? insts[blockIdx.x] : one;
    const amhd_grid &g = in.grid;
    amhd_control *ctl = ctls + blockIdx.x;
    const R *U = Ubase ? Ubase + in.offset : nullptr;
    __shared__ int go;
    __shared__ double dt_next;
    if (threadIdx.x == 0) {
        go = 0;
        if (set_only || ctl->active || !advance) {
            if (advance && !set_only) {
                ctl->t += ctl->dt;  // solver.py:481-482
                ctl->last_dt = ctl->dt;
                ctl->step += 1;
                ctl->e_bnd += ctl->e_bnd_next;  // the step just taken (solver.py:316-317)
                ctl->e_bnd_next = 0.0;
            }
            // a step that wrote a non-finite value, or whose bounded wait gave up and
            // left tiles stale, ends the loop: the host reads the flag and raises
            const bool healthy = !(ctl->flags & (AMHD_FLAG_NONFINITE | AMHD_FLAG_TIMEOUT));
            const bool loop_on = set_only || (healthy && ctl->t < ctl->t_end && ctl->step < ctl->max_steps);
            if (loop_on) {
                // compute_dt, solver.py:213-223 (max cf = sqrt of max cf^2; max(cf, ch) == ch)
                double cf_max = sqrt(__longlong_as_double((long long)ctl->red[0]));
                double vabs = __longlong_as_double((long long)ctl->red[1]);
                double s = cf_max + vabs;
                double ch = (1.0 > s ? 1.0 : s) * 1.5;
                double sx = (__longlong_as_double((long long)ctl->red[2]) + ch) / g.dx;
                double sy = (__longlong_as_double((long long)ctl->red[3]) + ch) / g.dy;
                double smx = (sx != sx || sx >= sy) ? sx : sy;
                double dtc = (smx < 1e-14) ? g.cfl * (g.dx < g.dy ? g.dx : g.dy) : g.cfl / smx;
                ctl->ch = ch;
                ctl->dt_cfl = dtc;
                if (!set_only) {
                    double rem = ctl->t_end - ctl->t;
                    double dt = (rem < dtc) ? rem : dtc;  // solver.py:478
                    ctl->dt = dt;
                    if (dt <= 1e-16) {
                        ctl->active = 0;
                        ctl->flags |= AMHD_FLAG_DT_TINY;
                    } else {
                        ctl->active = 1;
                        // snapshot due after this step (solver.py:487-490): pause, the host resumes
                        if (advance && fabs(ctl->t - ctl->snap_t) < 1.5 * ctl->last_dt) {
                            ctl->active = 0;
                            ctl->flags |= AMHD_FLAG_PAUSED;
                        }
                        double m = g.dx < g.dy ? g.dx : g.dy;
                        ctl->decay = ch > 0 ? exp(-g.glm_alpha * ch * dt / m) : 1.0;
                        go = (g.bc_x != AMHD_BC_PERIODIC) && (U != nullptr);
                        dt_next = dt;
                    }
                }
            } else {
                ctl->active = 0;
            }
            for (int k = 0; k < 4; ++k) ctl->red[k] = 0ull;
        }
    }
    __syncthreads();
    if (go) {
        double bf = boundary_flux_block(g, U, in.cut_x);  // solver.py:316-317
        if (threadIdx.x == 0) ctl->e_bnd_next = bf * dt_next;  // counted once the step is taken
    }
}

// ---------------------------------------------------------------------------
// diagnostics (solver.py:335-444, conserved-quantity part) in float64
//   row pass: per interior x-row i, sum_j clip(C), sum_j rho, sum_j E,
//   sum_j rho w^2 and row maxima of |divB| and stagnation pressure; sum divB^2
// ---------------------------------------------------------------------------
// Colour-field diagnostics of solver.py:353-417 that look at the field again
// after the row sums: the clipped colour C = clip(rhoC / max(rho, floor), 0, 1)
// in double, as diag_rows_kernel computes it.
template <typename R>
__device__ __forceinline__ double clipped_colour(const amhd_grid &g, const R *U, int i, int j)
{
    const int64_t c = (int64_t)i * g.pitch + j;
    const double rho = np_max((double)U[RHO * g.var_stride + c], FLOOR_RHO);
    const double ri = 1.0 / rho;
    return fmin(fmax((double)U[RHOC * g.var_stride + c] * ri, 0.0), 1.0);
}

// numpy's pairwise summation of a short array (n <= 128: eight running sums
// combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), then the remainder in
// order; below 8 elements a plain loop), so that a sum the reference takes
// with numpy.sum comes out with the same bits
__device__ __forceinline__ double np_pairwise_sum(const double *a, int n)
{
    if (n < 8) {
        double res = 0.0;
        for (int k = 0; k < n; ++k) res += a[k];
        return res;
    }
    double r[8];
    for (int k = 0; k < 8; ++k) r[k] = a[k];
    int k = 8;
    for (; k < n - (n % 8); k += 8)
        for (int m = 0; m < 8; ++m) r[m] += a[k + m];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; k < n; ++k) res += a[k];
    return res;
}

// one block per interior row: sum over y of (C - Cbar)^2 with Cbar = csum[r] / ny
// (C_prime_sq of solver.py:360 times ny)
template <typename R>
__global__ void diag_colour_rows_kernel(const amhd_grid g, const R *U, const double *csum, double *cp2)
{
    const int r = blockIdx.x;
    const double cbar = csum[r] / g.ny;
    double s = 0.0;
    for (int jj = threadIdx.x; jj < g.ny; jj += blockDim.x) {
        const double d = clipped_colour(g, U, NG + r, NG + jj) - cbar;
        s += d * d;
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        cp2[r] = t;
    }
}

// One thread per interior column j: the interface position of solver.py:368-383
// -- |dC/dx| as numpy.gradient takes it along x (central differences inside,
// one-sided at the two ends), its first maximum over the column, and the
// |dC/dx|-weighted mean of x over up to 10 rows either side of it; NaN when the
// column's maximum is <= 1e-6, the window is empty or the weights sum to <= 1e-12.
template <typename R>
__global__ void diag_interface_kernel(const amhd_grid g, const R *U, double x0, double *pos)
{
    const int nx = g.nx;
    const double dx = g.dx;
    for (int jj = blockIdx.x * blockDim.x + threadIdx.x; jj < g.ny; jj += gridDim.x * blockDim.x) {
        const int j = NG + jj;
        auto grad = [&](int r) -> double {
            if (r == 0) return fabs((clipped_colour(g, U, NG + 1, j) - clipped_colour(g, U, NG, j)) / dx);
            if (r == nx - 1)
                return fabs((clipped_colour(g, U, NG + nx - 1, j) - clipped_colour(g, U, NG + nx - 2, j)) / dx);
            return fabs((clipped_colour(g, U, NG + r + 1, j) - clipped_colour(g, U, NG + r - 1, j)) / (2.0 * dx));
        };
        double best = -1.0;
        int ip = 0;
        for (int r = 0; r < nx; ++r) {
            const double d = grad(r);
            if (d > best) {
                best = d;
                ip = r;
            }
        }
        double out = __longlong_as_double(0x7ff8000000000000LL);  // NaN
        const int hw = min(10, min(ip, nx - ip - 1));
        if (best > 1e-6 && hw > 0) {
            double wgt[21], xw[21];
            const int n = 2 * hw + 1;
            for (int k = 0; k < n; ++k) {
                const int r = ip - hw + k;
                wgt[k] = grad(r);
                xw[k] = (x0 + ((double)r + 0.5) * dx) * wgt[k];
            }
            const double ws = np_pairwise_sum(wgt, n);
            if (ws > 1e-12) out = np_pairwise_sum(xw, n) / ws;
        }
        pos[jj] = out;
    }
}

template <typename R>
__global__ void diag_rows_kernel(const amhd_grid g, const R *U, double *rows)
{
    // one block per interior row
    const int r = blockIdx.x;
    const int i = NG + r;
    double s_c = 0, s_rho = 0, s_e = 0, s_div2 = 0, s_ens = 0, m_div = 0, m_stag = 0;
    const int nx = g.nx, ny = g.ny;
    for (int jj = threadIdx.x; jj < ny; jj += blockDim.x) {
        const int j = NG + jj;
        auto load = [&](int ii, int jx, double w[NV]) {
            double u[NV];
            const int64_t c = (int64_t)ii * g.pitch + jx;
#pragma unroll
            for (int v = 0; v < NV; ++v) u[v] = (double)U[v * g.var_stride + c];
            cons_to_prim_cell(u, g.gamma, w);
        };
        double w[NV];
        load(i, j, w);
        double cc = fmin(fmax(w[9], 0.0), 1.0);
        s_c += cc;
        s_rho += (double)U[RHO * g.var_stride + (int64_t)i * g.pitch + j];
        s_e += (double)U[EN * g.var_stride + (int64_t)i * g.pitch + j];
        double v2 = w[1] * w[1] + w[2] * w[2];
        double b2 = w[4] * w[4] + w[5] * w[5] + w[6] * w[6];
        m_stag = fmax(m_stag, w[7] + 0.5 * w[0] * v2 + 0.5 * b2);
        // divB on the interior minus its outer ring (solver.py:419-426)
        if (r >= 1 && r < nx - 1 && jj >= 1 && jj < ny - 1) {
            double wxp[NV], wxm[NV], wyp[NV], wym[NV];
            load(i + 1, j, wxp);
            load(i - 1, j, wxm);
            load(i, j + 1, wyp);
            load(i, j - 1, wym);
            double d = (0.5 * (w[4] + wxp[4]) - 0.5 * (wxm[4] + w[4])) / g.dx +
                       (0.5 * (w[5] + wyp[5]) - 0.5 * (wym[5] + w[5])) / g.dy;
            s_div2 += d * d;
            m_div = fmax(m_div, fabs(d));
        }
        // vorticity with numpy.gradient's one-sided ends on the interior (solver.py:399-402)
        {
            double vyp, vym, hx, vxp, vxm, hy;
            double t[NV];
            if (r == 0) { load(i + 1, j, t); vyp = t[2]; vym = w[2]; hx = g.dx; }
            else if (r == nx - 1) { load(i - 1, j, t); vyp = w[2]; vym = t[2]; hx = g.dx; }
            else { load(i + 1, j, t); vyp = t[2]; load(i - 1, j, t); vym = t[2]; hx = 2 * g.dx; }
            if (jj == 0) { load(i, j + 1, t); vxp = t[1]; vxm = w[1]; hy = g.dy; }
            else if (jj == ny - 1) { load(i, j - 1, t); vxp = w[1]; vxm = t[1]; hy = g.dy; }
            else { load(i, j + 1, t); vxp = t[1]; load(i, j - 1, t); vxm = t[1]; hy = 2 * g.dy; }
            double om = (vyp - vym) / hx - (vxp - vxm) / hy;
            s_ens += w[0] * om * om;
        }
    }
    __shared__ double red[7][32];
    double vals[7] = {s_c, s_rho, s_e, s_div2, s_ens, m_div, m_stag};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 7; ++k) {
        double a = vals[k];
        for (int o = 16; o > 0; o >>= 1) {
            double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = k < 5 ? a + b : fmax(a, b);
        }
        if (lane == 0) red[k][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double out[7];
        for (int k = 0; k < 7; ++k) {
            double a = red[k][0];
            for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) a = k < 5 ? a + red[k][w2] : fmax(a, red[k][w2]);
            out[k] = a;
        }
        for (int k = 0; k < 7; ++k) rows[(int64_t)k * nx + r] = out[k];
    }
}

// finish: trapezoid mixing width and global sums, single block
__global__ void diag_finish_kernel(const amhd_grid g, double x0, const double *rows, double *out);

}  // namespace amhd
