// amhd_launch_impl.cuh -- definitions of Launch<R>; included once per
// precision translation unit, which then instantiates Launch<R>.
#pragma once
#include <atomic>
#include <cstdint>
#include <cstring>
#include <utility>

#include "amhd_kernels.cuh"

namespace amhd {

// A set-up step that must run once per device (kernel function attributes such
// as the shared-memory opt-in are per device): one bit per device ordinal.
// Two threads may both run the step for the same device; it is idempotent.
struct PerDeviceOnce {
    std::atomic<uint64_t> done{0};
    template <typename F>
    cudaError_t run(F &&step)
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
        if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
        e = step();
        if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
        return e;
    }
};

static inline int elem_blocks(int64_t n, int threads = 256)
{
    int64_t b = (n + threads - 1) / threads;
    const int64_t cap = 148LL * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

template <typename R, bool TMA = false>
constexpr size_t kMarchSmem = sizeof(MarchSmem<R, TMA>) * (kMarchThreads / 32);

template <typename R>
size_t Launch<R>::stage_smem(int tile_x)
{
    if (is_march(tile_x)) return kMarchSmem<R, true> > kMarchSmem<R> ? kMarchSmem<R, true> : kMarchSmem<R>;
    switch (tile_x) {
    case 4: return sizeof(TileSmem<R, 4>);
    case 8: return sizeof(TileSmem<R, 8>);
    case 16: return sizeof(TileSmem<R, 16>);
    default: return 0;
    }
}

// shared-memory opt-in of one stage instantiation, set once per device
template <typename R, int TX, int ST>
static cudaError_t configure_t()
{
    static PerDeviceOnce once;
    return once.run([] {
        return cudaFuncSetAttribute(rk_stage_kernel<R, TX, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(TileSmem<R, TX>));
    });
}

template <typename R, int TX, int ST>
static cudaError_t launch_stage_t(const StageParams &p, int grid, cudaStream_t s)
{
    cudaError_t e = configure_t<R, TX, ST>();
    if (e != cudaSuccess) return e;
    rk_stage_kernel<R, TX, ST><<<grid, TX * TY, sizeof(TileSmem<R, TX>), s>>>(p);
    return cudaGetLastError();
}

template <typename R, int TX>
static cudaError_t configure_tx()
{
    cudaError_t e;
    if ((e = configure_t<R, TX, 0>()) != cudaSuccess) return e;
    if ((e = configure_t<R, TX, 1>()) != cudaSuccess) return e;
    if ((e = configure_t<R, TX, 2>()) != cudaSuccess) return e;
    return configure_t<R, TX, 3>();
}

template <typename R>
cudaError_t Launch<R>::configure()
{
    cudaError_t e;
    if ((e = configure_tx<R, 4>()) != cudaSuccess) return e;
    if ((e = configure_tx<R, 8>()) != cudaSuccess) return e;
    return configure_tx<R, 16>();
}

template <typename R, int TX>
static cudaError_t launch_stage_tx(int stage, const StageParams &p, int grid, cudaStream_t s)
{
    switch (stage) {
    case 0: return launch_stage_t<R, TX, 0>(p, grid, s);
    case 1: return launch_stage_t<R, TX, 1>(p, grid, s);
    case 2: return launch_stage_t<R, TX, 2>(p, grid, s);
    case 3: return launch_stage_t<R, TX, 3>(p, grid, s);
    default: return cudaErrorInvalidValue;
    }
}

// a launch that may start while the previous kernel of the stream drains
// (programmatic dependent launch; the kernel waits in pdl_wait before it reads
// anything the previous one wrote)
template <typename... KArgs, typename... Args>
static cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                    Args &&...args)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <typename R, int ST, bool TMA, bool COMP = false>
static cudaError_t launch_march_tt(const StageParams &p, int grid, cudaStream_t s)
{
    constexpr size_t smem = kMarchSmem<R, TMA>;
    static PerDeviceOnce once;  // shared-memory opt-in, once per device
    cudaError_t e = once.run([] {
        return cudaFuncSetAttribute(march_stage_kernel<R, ST, TMA, COMP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    if (e != cudaSuccess) return e;
    if (p.pdl)
        return launch_dependent(march_stage_kernel<R, ST, TMA, COMP>, dim3(grid), dim3(kMarchThreads), smem, s, p);
    march_stage_kernel<R, ST, TMA, COMP><<<grid, kMarchThreads, smem, s>>>(p);
    return cudaGetLastError();
}

// rows staged by TMA (p.use_tma: the tensor maps are in p) or by per-lane cp.async;
// the compensated last stage (p.ulo, float32) is built with cp.async rows only
template <typename R, int ST>
static cudaError_t launch_march_t(const StageParams &p, int grid, cudaStream_t s)
{
    if constexpr (ST == 3 && kFast<R>)
        if (p.ulo != nullptr) {
            if (p.use_tma) return cudaErrorNotSupported;
            return launch_march_tt<R, ST, false, true>(p, grid, s);
        }
    return p.use_tma ? launch_march_tt<R, ST, true>(p, grid, s) : launch_march_tt<R, ST, false>(p, grid, s);
}

template <typename R>
cudaError_t Launch<R>::stage(int stage, int tile_x, const StageParams &p, int grid, cudaStream_t s)
{
    if (p.n_tiles <= 0) return cudaSuccess;
    if (is_march(tile_x)) {
        // grid counts CTAs of kMarchThreads / 32 warps; one warp per work item at a time
        const int wpc = kMarchThreads / 32;
        const int need = (p.n_tiles + wpc - 1) / wpc;
        if (grid <= 0 || grid > need) grid = need;
        StageParams q = p;
        q.march_rows = -tile_x;
        cudaError_t e;
        switch (stage) {
        case 0: return launch_march_t<R, 0>(q, grid, s);
        case 1: e = launch_march_t<R, 1>(q, grid, s); break;
        case 2: e = launch_march_t<R, 2>(q, grid, s); break;
        case 3: e = launch_march_t<R, 3>(q, grid, s); break;
        default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        // the marching kernel leaves the ghost cells of its output to this pass
        // (not needed after stages 1 and 2 when the next stage pulls them, nor
        // after stage 3 when the loop fills U once after its last step)
        if (p.pull_ghosts && (stage < 3 || p.defer_fill)) return cudaSuccess;
        const int n_inst = p.inst ? p.n_inst : 1;
        if (n_inst <= 0) return cudaErrorInvalidValue;
        const int per = p.inst ? 8 : elem_blocks(4LL * (p.one.grid.ny + 2 * NG) + 4LL * p.one.grid.nx);
        march_bc_fill_kernel<R><<<dim3(per, n_inst), 256, 0, s>>>(q);
        return cudaGetLastError();
    }
    if (grid <= 0) grid = p.n_tiles;
    switch (tile_x) {
    case 4: return launch_stage_tx<R, 4>(stage, p, grid, s);
    case 8: return launch_stage_tx<R, 8>(stage, p, grid, s);
    case 16: return launch_stage_tx<R, 16>(stage, p, grid, s);
    default: return cudaErrorInvalidValue;
    }
}

template <typename R, int TX>
static int ctas_per_sm_t()
{
    int n = 0;
    const size_t smem = sizeof(TileSmem<R, TX>);
    configure_t<R, TX, 3>();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rk_stage_kernel<R, TX, 3>, TX * TY, smem) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

template <typename R>
int Launch<R>::stage_ctas_per_sm(int tile_x)
{
    if (is_march(tile_x)) {
        int n = 0;
        cudaFuncSetAttribute(march_stage_kernel<R, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMarchSmem<R>);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_stage_kernel<R, 3, false>, kMarchThreads,
                                                          kMarchSmem<R>) != cudaSuccess)
            return 1;
        return n > 0 ? n : 1;
    }
    switch (tile_x) {
    case 4: return ctas_per_sm_t<R, 4>();
    case 8: return ctas_per_sm_t<R, 8>();
    case 16: return ctas_per_sm_t<R, 16>();
    default: return 1;
    }
}

template <typename R>
cudaError_t Launch<R>::march_fill(const StageParams &p, cudaStream_t s)
{
    const int n_inst = p.inst ? p.n_inst : 1;
    if (n_inst <= 0) return cudaErrorInvalidValue;
    StageParams q = p;
    q.use_ctl = 0;  // every instance: one that stopped during the loop still has its last state to fill
    const int per = p.inst ? 8 : elem_blocks(4LL * (p.one.grid.ny + 2 * NG) + 4LL * p.one.grid.nx);
    march_bc_fill_kernel<R><<<dim3(per, n_inst), 256, 0, s>>>(q);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::bc_fill(const amhd_grid &g, R *U, cudaStream_t s)
{
    const int64_t n = 4LL * (g.ny + 2 * NG) + 4LL * g.nx;
    bc_fill_kernel<R><<<elem_blocks(n), 256, 0, s>>>(g, U);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::cons_to_prim(const Layout &li, const R *U, const Layout &lo, R *W, double gamma,
                                    cudaStream_t s)
{
    cons_to_prim_kernel<R><<<elem_blocks((int64_t)li.nxt * li.nyt), 256, 0, s>>>(li, U, lo, W, gamma);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::prim_to_cons(const Layout &li, const R *W, const Layout &lo, R *U, double gamma,
                                    cudaStream_t s)
{
    prim_to_cons_kernel<R><<<elem_blocks((int64_t)li.nxt * li.nyt), 256, 0, s>>>(li, W, lo, U, gamma);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::scalar_bounds(const Layout &l, R *U, cudaStream_t s)
{
    scalar_bounds_kernel<R><<<elem_blocks((int64_t)l.nxt * l.nyt), 256, 0, s>>>(l, U);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::muscl(const Layout &l, const R *W, int axis, int limiter, R *WL, R *WR, cudaStream_t s)
{
    const int64_t nf = axis == 0 ? (int64_t)(l.nxt - 3) * l.nyt : (int64_t)l.nxt * (l.nyt - 3);
    muscl_kernel<R><<<elem_blocks(nf), 256, 0, s>>>(l, W, axis, limiter, WL, WR);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::hlld(const R *WL, const R *WR, R *F, R *smax, int64_t n, int axis, double gamma, double ch,
                            cudaStream_t s)
{
    hlld_kernel<R><<<elem_blocks(n), 256, 0, s>>>(WL, WR, F, smax, n, axis, R(gamma), R(ch));
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::powell(const Layout &l, const R *W, R *S, double dx, double dy, cudaStream_t s)
{
    powell_kernel<R><<<elem_blocks((int64_t)l.nxt * l.nyt), 256, 0, s>>>(l, W, S, R(dx), R(dy));
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::dt_reduce(const Layout &l, const R *A, int from_prim, double gamma, amhd_control *ctl,
                                 cudaStream_t s)
{
    dt_reduce_kernel<R><<<elem_blocks((int64_t)l.nxt * l.nyt), 256, 0, s>>>(l, A, from_prim, gamma, ctl);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::finalize(const amhd_instance *insts, int n_inst, const amhd_instance &one, const R *U,
                                amhd_control *ctl, int advance, int set_only, cudaStream_t s, int pdl)
{
    if (pdl) return launch_dependent(finalize_kernel<R>, dim3(n_inst), dim3(256), 0, s, insts, one, U, ctl, advance, set_only);
    finalize_kernel<R><<<n_inst, 256, 0, s>>>(insts, one, U, ctl, advance, set_only);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::diag_colour(const amhd_grid &g, const R *U, double x0, const double *csum, double *cp2,
                                   double *pos, cudaStream_t s)
{
    diag_colour_rows_kernel<R><<<g.nx, 256, 0, s>>>(g, U, csum, cp2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    diag_interface_kernel<R><<<(g.ny + 127) / 128, 128, 0, s>>>(g, U, x0, pos);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::diag_rows(const amhd_grid &g, const R *U, double *rows, cudaStream_t s)
{
    diag_rows_kernel<R><<<g.nx, 256, 0, s>>>(g, U, rows);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::bflux(const amhd_grid &g, const R *U, double *out, cudaStream_t s)
{
    bflux_kernel<R><<<1, 256, 0, s>>>(g, U, out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Launch<R>::bflux_accum(const amhd_grid &g, const R *U, amhd_control *ctl, double dt, cudaStream_t s)
{
    bflux_accum_kernel<R><<<1, 256, 0, s>>>(g, U, ctl, dt);
    return cudaGetLastError();
}

}  // namespace amhd
