// amhd_capi.cu -- the extern "C" entry points of libaeromhd.so (include/aeromhd.h):
// argument checks, precision dispatch, and the launch sequences of the step,
// the device-side run loop and the ensemble.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "aeromhd.h"
#include "amhd_launch.h"
#include "amhd_tma.cuh"

using namespace amhd;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess) return fail(AMHD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e__)); \
    } while (0)

constexpr int kNG = 2;
constexpr int kTY = 32;

int g_tile_x = 0;  // 0: per precision (tile_of)
int g_ctas_per_sm = 0;
int g_use_tma = 1;
int g_march_pack = 1;  // single grids: the last strip's row chunks share warps (march_pack)

inline size_t elem_size(int dtype) { return dtype == AMHD_F32 ? 4 : 8; }

// stage-kernel geometry of a grid: the one set by amhd_set_tiling, else the
// marching kernel with 24 rows per item in float32 and 16 in float64 (the
// fastest measured at 2048 x 2048: float64 runs 2 CTAs per SM, where 16-row
// items fill whole waves)
inline int tile_of(const amhd_grid *g) { return g_tile_x ? g_tile_x : (g->dtype == AMHD_F32 ? -24 : -16); }

int check_grid(const amhd_grid *g)
{
    if (!g) return fail(AMHD_ERR_ARG, "grid is NULL");
    if (g->nx < 2 || g->ny < 2) return fail(AMHD_ERR_ARG, "grid must be at least 2x2 cells (got %dx%d)", g->nx, g->ny);
    if (g->dtype != AMHD_F32 && g->dtype != AMHD_F64) return fail(AMHD_ERR_ARG, "unknown dtype %d", g->dtype);
    if (g->pitch < g->ny + 2 * kNG) return fail(AMHD_ERR_ARG, "pitch %d < ny+4", g->pitch);
    if (g->var_stride < (int64_t)(g->nx + 2 * kNG) * g->pitch)
        return fail(AMHD_ERR_ARG, "var_stride %lld < (nx+4)*pitch", (long long)g->var_stride);
    if (!(g->dx > 0) || !(g->dy > 0)) return fail(AMHD_ERR_ARG, "dx, dy must be positive");
    if (!(g->gamma > 1)) return fail(AMHD_ERR_ARG, "gamma must exceed 1");
    if (g->bc_x < 0 || g->bc_x > 2 || g->bc_y < 0 || g->bc_y > 2) return fail(AMHD_ERR_ARG, "unknown boundary kind");
    if (g->limiter != AMHD_LIMITER_VANLEER && g->limiter != AMHD_LIMITER_MINMOD)
        return fail(AMHD_ERR_ARG, "unknown limiter %d", g->limiter);
    return AMHD_OK;
}

void padded_dims(int nx, int ny, int *pitch, int *rows)
{
    *pitch = kTY * ((ny + kTY - 1) / kTY) + 2 * kNG;
    *rows = 16 * ((nx + 15) / 16) + 2 * kNG;
}

int check_padded(const amhd_grid *g, const void *const *ptrs, int n)
{
    int pitch, rows;
    padded_dims(g->nx, g->ny, &pitch, &rows);
    const size_t es = elem_size(g->dtype);
    if (g->pitch < pitch) return fail(AMHD_ERR_ARG, "fused step needs pitch >= %d (got %d)", pitch, g->pitch);
    if (g->var_stride < (int64_t)rows * g->pitch)
        return fail(AMHD_ERR_ARG, "fused step needs var_stride >= %d * pitch", rows);
    if ((g->pitch * es) % 16 || (g->var_stride * es) % 16)
        return fail(AMHD_ERR_ARG, "pitch and var_stride must be multiples of 16 bytes");
    for (int k = 0; k < n; ++k) {
        if (!ptrs[k]) return fail(AMHD_ERR_ARG, "state pointer %d is NULL", k);
        if (reinterpret_cast<uintptr_t>(ptrs[k]) % 16) return fail(AMHD_ERR_ARG, "state pointer %d not 16-byte aligned", k);
    }
    return AMHD_OK;
}

Layout layout_of(const amhd_grid *g) { return Layout{g->nx + 2 * kNG, g->ny + 2 * kNG, g->pitch, g->var_stride}; }

amhd_instance single_instance(const amhd_grid *g, int tile_x)
{
    amhd_instance in;
    memset(&in, 0, sizeof in);
    in.grid = *g;
    in.offset = 0;
    in.first_tile = 0;
    if (is_march(tile_x)) {
        in.tiles_x = (g->nx - tile_x - 1) / -tile_x;
        in.tiles_y = (g->ny + kMarchCols - 1) / kMarchCols;
        // the last strip's chunks share warps unless the rows are staged by TMA
        in.pack = (g_march_pack && !(g_use_tma & 2)) ? march_pack(g->ny) : 1;
    } else {
        in.tiles_x = (g->nx + tile_x - 1) / tile_x;
        in.tiles_y = (g->ny + kTY - 1) / kTY;
    }
    return in;
}

// work items of a single-grid launch of this geometry
int n_items(const amhd_instance &in, int tile_x)
{
    return is_march(tile_x) ? march_item_count(in.grid.nx, in.grid.ny, -tile_x, in.pack) : in.tiles_x * in.tiles_y;
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int stage_grid(int dtype, int tile_x, int n_tiles, int ctas_per_sm)
{
    if (ctas_per_sm <= 0) return n_tiles;
    int per = ctas_per_sm;
    const int occ = dtype == AMHD_F64 ? Launch<double>::stage_ctas_per_sm(tile_x)
                                      : Launch<float>::stage_ctas_per_sm(tile_x);
    if (per > occ) per = occ;
    int grid = per * device_sm_count();
    return grid < n_tiles ? grid : n_tiles;
}

// stage input and base state: pointers, and their tensor maps when TMA staging
// is on for the kernel of this geometry (bit 0 of amhd_set_tma: tiled kernel,
// bit 1: marching kernel, which also stages the base state's rows)
void set_input(StageParams &p, const void *uin, const void *u0, const amhd_grid *g, int tile_x)
{
    p.uin = uin;
    p.u0 = u0;
    p.use_tma = 0;
    const int want = is_march(tile_x) ? (g_use_tma & 2) : (g_use_tma & 1);
    if (!want || encode_state_map(&p.tmap, uin, g->dtype, g->pitch, g->var_stride, tile_x) != 0) return;
    if (is_march(tile_x) && encode_state_map(&p.tmap_base, u0, g->dtype, g->pitch, g->var_stride, tile_x) != 0)
        return;
    p.use_tma = 1;
}

cudaError_t run_stage(int dtype, int stage, int tile_x, const StageParams &p, int grid, cudaStream_t s)
{
    return dtype == AMHD_F64 ? Launch<double>::stage(stage, tile_x, p, grid, s)
                             : Launch<float>::stage(stage, tile_x, p, grid, s);
}

cudaError_t run_bc_fill(const amhd_grid *g, void *U, cudaStream_t s)
{
    return g->dtype == AMHD_F64 ? Launch<double>::bc_fill(*g, static_cast<double *>(U), s)
                                : Launch<float>::bc_fill(*g, static_cast<float *>(U), s);
}

cudaError_t run_finalize(int dtype, const amhd_instance *insts, int n, const amhd_instance &one, const void *U,
                         amhd_control *ctl, int advance, int set_only, cudaStream_t s, int pdl = 0)
{
    return dtype == AMHD_F64
               ? Launch<double>::finalize(insts, n, one, static_cast<const double *>(U), ctl, advance, set_only, s, pdl)
               : Launch<float>::finalize(insts, n, one, static_cast<const float *>(U), ctl, advance, set_only, s, pdl);
}

cudaError_t run_dt_reduce(const amhd_grid *g, const void *A, int from_prim, amhd_control *ctl, cudaStream_t s)
{
    const Layout l = layout_of(g);
    return g->dtype == AMHD_F64
               ? Launch<double>::dt_reduce(l, static_cast<const double *>(A), from_prim, g->gamma, ctl, s)
               : Launch<float>::dt_reduce(l, static_cast<const float *>(A), from_prim, g->gamma, ctl, s);
}

// three fused stages of one step; dt/ch/decay from the host or from ctl
// One run-loop step.  defer_fill (marching kernel): U's ghost cells are not
// filled after stage 3 either -- the next step pulls them like those of U1 and
// U2 -- and the caller fills them after its last step (fill_after_loop).
int three_stages(const amhd_grid *g, const amhd_instance &one, const amhd_instance *insts, const int32_t *tile_inst,
                 int n_tiles, int tile_x, int grid, void *U, void *U1, void *U2, amhd_control *ctl, int use_ctl,
                 double dt, double ch, double decay, int fuse_dt, cudaStream_t s, const int32_t *tile_order = nullptr,
                 const CUtensorMap *tmaps = nullptr, int n_inst = 1, int defer_fill = 0, int32_t *queue = nullptr,
                 void *ulo = nullptr)
{
    StageParams p;
    memset(&p, 0, sizeof p);
    p.queue = is_march(tile_x) ? queue : nullptr;
    p.inst = insts;
    p.n_inst = n_inst;
    p.pull_ghosts = 1;  // the run loop: U1 and U2 are internal, their ghost cells are never stored
    p.defer_fill = defer_fill;
    p.pdl = defer_fill;  // the marching run loop: each launch overlaps the previous one's tail
    p.one = one;
    p.tile_inst = tile_inst;
    p.tile_order = tile_order;
    p.n_tiles = n_tiles;
    p.ctl = ctl;
    p.dt = dt;
    p.ch = ch;
    p.decay = decay;
    p.use_ctl = use_ctl;
    const int dtype = g->dtype;
    void *in[3] = {U, U1, U2};
    void *out[3] = {U1, U2, U};
    for (int st = 1; st <= 3; ++st) {
        if (insts) {  // ensemble: per-instance maps in device memory
            p.uin = in[st - 1];
            p.use_tma = tmaps != nullptr;
            p.tmaps = tmaps;
            p.in_buf = st - 1;
        } else {
            set_input(p, in[st - 1], U, g, tile_x);
        }
        p.u0 = U;
        p.uout = out[st - 1];
        p.ulo = (st == 3 && is_march(tile_x)) ? ulo : nullptr;
        p.fuse_dt = st == 3 ? fuse_dt : 0;
        CK(run_stage(dtype, st, tile_x, p, grid, s));
    }
    return AMHD_OK;
}

// the ghost cells of U after a run loop whose steps deferred them (every instance)
int fill_after_loop(int dtype, const amhd_instance &one, const amhd_instance *insts, int n_inst, void *U,
                    cudaStream_t s)
{
    StageParams p;
    memset(&p, 0, sizeof p);
    p.inst = insts;
    p.n_inst = n_inst;
    p.one = one;
    p.uout = U;
    CK(dtype == AMHD_F64 ? Launch<double>::march_fill(p, s) : Launch<float>::march_fill(p, s));
    return AMHD_OK;
}

int control_upload(amhd_control *ctl, double t, double t_end, int64_t step, int64_t max_steps, cudaStream_t s)
{
    amhd_control h;
    memset(&h, 0, sizeof h);
    h.t = t;
    h.t_end = t_end;
    h.step = step;
    h.max_steps = max_steps;
    h.active = 1;
    h.decay = 1.0;
    h.snap_t = __builtin_inf();
    // pageable source: the copy is staged before the call returns
    CK(cudaMemcpyAsync(ctl, &h, sizeof h, cudaMemcpyHostToDevice, s));
    return AMHD_OK;
}

// one thread waits on a CTA-local mbarrier that expects one arrival: after
// arriving itself (the wait must succeed) or with nothing arriving (the wait
// must give up after limit_ns); out = {gave up, microseconds waited}
__global__ void selftest_wait_kernel(int arrive, uint64_t limit_ns, int32_t *out)
{
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    amhd::tma::mbar_init(&bar, 1);
    if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(amhd::tma::smem_addr(&bar)) : "memory");
    const uint64_t t0 = amhd::tma::globaltimer_ns();
    const bool done = amhd::tma::wait_for(&bar, 0u, limit_ns, amhd::tma::kTmaWaitIters);
    const uint64_t us = (amhd::tma::globaltimer_ns() - t0) / 1000u;
    out[0] = done ? 0 : 1;
    out[1] = us > 0x7fffffffull ? 0x7fffffff : (int32_t)us;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    }
    return fn;
}

}  // namespace

namespace amhd {
int encode_state_map(CUtensorMap *map, const void *base, int dtype, int pitch, int64_t var_stride, int tile_x)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || !base) return -1;
    const size_t es = elem_size(dtype);
    const cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)(var_stride / pitch), 10};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * es, (cuuint64_t)var_stride * es};
    // tiled kernel: the tile and its halo; marching kernel: one row of a 32-lane strip
    const cuuint32_t box[3] = {(cuuint32_t)(is_march(tile_x) ? 32 : kTY + 2 * kNG),
                               (cuuint32_t)(is_march(tile_x) ? 1 : tile_x + 2 * kNG), 10};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dtype == AMHD_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                    const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}
}  // namespace amhd

#pragma GCC visibility push(default)
extern "C" {

const char *amhd_version(void) { return "aeromhd-b200 0.1.0 (sm_100a)"; }

const char *amhd_last_error(void) { return g_err.c_str(); }

int amhd_init(void)
{
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (n <= 0) return fail(AMHD_ERR_CUDA, "no CUDA device");
    CK(Launch<double>::configure());
    CK(Launch<float>::configure());
    return AMHD_OK;
}

size_t amhd_control_size(void) { return sizeof(amhd_control); }

int amhd_padded_layout(int32_t nx, int32_t ny, int32_t dtype, int32_t *pitch, int32_t *rows)
{
    if (nx < 2 || ny < 2) return fail(AMHD_ERR_ARG, "grid must be at least 2x2 cells");
    if (dtype != AMHD_F32 && dtype != AMHD_F64) return fail(AMHD_ERR_ARG, "unknown dtype %d", dtype);
    if (!pitch || !rows) return fail(AMHD_ERR_ARG, "NULL output");
    padded_dims(nx, ny, pitch, rows);
    return AMHD_OK;
}

int amhd_set_tiling(int32_t tile_x, int32_t ctas_per_sm)
{
    if (tile_x != 0 && !valid_geometry(tile_x))
        return fail(AMHD_ERR_ARG, "tile_x must be 0 (default), 4, 8, 16 or -1024..-4 (marching rows)");
    if (ctas_per_sm < 0 || ctas_per_sm > 32) return fail(AMHD_ERR_ARG, "ctas_per_sm out of range");
    g_tile_x = tile_x;
    g_ctas_per_sm = ctas_per_sm;
    return AMHD_OK;
}

int amhd_set_tma(int32_t mode)
{
    if (mode < 0 || mode > 3) return fail(AMHD_ERR_ARG, "TMA mode must be 0..3, got %d", mode);
    g_use_tma = mode;
    return AMHD_OK;
}

int amhd_march_pack(int32_t ny) { return ny > 0 ? march_pack(ny) : 1; }

int amhd_march_items(int32_t nx, int32_t ny, int32_t rows, int32_t pack)
{
    if (nx <= 0 || ny <= 0 || rows <= 0) return fail(AMHD_ERR_ARG, "nx, ny and rows must be positive");
    if (pack > 1 && pack != march_pack(ny))
        return fail(AMHD_ERR_ARG, "pack must be 0, 1 or amhd_march_pack(%d) = %d, got %d", ny, march_pack(ny), pack);
    return march_item_count(nx, ny, rows, pack);
}

int amhd_set_march_pack(int32_t on)
{
    if (on != 0 && on != 1) return fail(AMHD_ERR_ARG, "march pack switch must be 0 or 1, got %d", on);
    g_march_pack = on;
    return AMHD_OK;
}

int amhd_selftest_wait(int32_t arrive, int64_t limit_ns, int32_t *timed_out, int32_t *waited_us)
{
    if (limit_ns <= 0 || limit_ns > 2000000000LL || !timed_out || !waited_us)
        return fail(AMHD_ERR_ARG, "limit_ns must be in (0, 2e9] and the outputs non-NULL");
    int32_t *d = nullptr;
    CK(cudaMalloc(reinterpret_cast<void **>(&d), 2 * sizeof(int32_t)));
    selftest_wait_kernel<<<1, 32>>>(arrive ? 1 : 0, (uint64_t)limit_ns, d);
    cudaError_t e = cudaGetLastError();
    int32_t h[2] = {-1, -1};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(AMHD_ERR_CUDA, "selftest_wait: %s", cudaGetErrorString(e));
    *timed_out = h[0];
    *waited_us = h[1];
    return AMHD_OK;
}

int amhd_ensemble_tensormaps(const amhd_instance *inst_host, int32_t n_inst, int32_t dtype, int32_t tile_x,
                             const void *U, const void *U1, const void *U2, void *maps_host)
{
    if (!inst_host || n_inst <= 0 || !U || !U1 || !U2 || !maps_host) return fail(AMHD_ERR_ARG, "bad arguments");
    if (!valid_geometry(tile_x)) return fail(AMHD_ERR_ARG, "tile_x must be 4, 8, 16 or -1024..-4 (marching rows)");
    const size_t es = elem_size(dtype);
    CUtensorMap *maps = static_cast<CUtensorMap *>(maps_host);
    const void *bufs[3] = {U, U1, U2};
    for (int k = 0; k < n_inst; ++k) {
        const amhd_grid *g = &inst_host[k].grid;
        if (int e = check_grid(g)) return fail(e, "instance %d: %s", k, g_err.c_str());
        for (int b = 0; b < 3; ++b) {
            const char *base = static_cast<const char *>(bufs[b]) + (size_t)inst_host[k].offset * es;
            if (reinterpret_cast<uintptr_t>(base) % 16)
                return fail(AMHD_ERR_ARG, "instance %d state not 16-byte aligned", k);
            if (encode_state_map(&maps[3 * k + b], base, dtype, g->pitch, g->var_stride, tile_x) != 0)
                return fail(AMHD_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled failed for instance %d", k);
        }
    }
    return AMHD_OK;
}

int amhd_stage_info(int32_t dtype, int32_t tile_x, int32_t *smem_bytes, int32_t *ctas_per_sm, int32_t *sm_count)
{
    if (!valid_geometry(tile_x)) return fail(AMHD_ERR_ARG, "tile_x must be 4, 8, 16 or -1024..-4 (marching rows)");
    if (dtype != AMHD_F32 && dtype != AMHD_F64) return fail(AMHD_ERR_ARG, "unknown dtype %d", dtype);
    if (smem_bytes)
        *smem_bytes = (int32_t)(dtype == AMHD_F64 ? Launch<double>::stage_smem(tile_x) : Launch<float>::stage_smem(tile_x));
    if (ctas_per_sm)
        *ctas_per_sm = dtype == AMHD_F64 ? Launch<double>::stage_ctas_per_sm(tile_x)
                                         : Launch<float>::stage_ctas_per_sm(tile_x);
    if (sm_count) *sm_count = device_sm_count();
    return AMHD_OK;
}

int amhd_cons_to_prim(const amhd_grid *g, const void *U, void *W, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !W) return fail(AMHD_ERR_ARG, "NULL array");
    const Layout l = layout_of(g);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::cons_to_prim(l, static_cast<const double *>(U), l, static_cast<double *>(W), g->gamma, S(stream)));
    else
        CK(Launch<float>::cons_to_prim(l, static_cast<const float *>(U), l, static_cast<float *>(W), g->gamma, S(stream)));
    return AMHD_OK;
}

int amhd_prim_to_cons(const amhd_grid *g, const void *W, void *U, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !W) return fail(AMHD_ERR_ARG, "NULL array");
    const Layout l = layout_of(g);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::prim_to_cons(l, static_cast<const double *>(W), l, static_cast<double *>(U), g->gamma, S(stream)));
    else
        CK(Launch<float>::prim_to_cons(l, static_cast<const float *>(W), l, static_cast<float *>(U), g->gamma, S(stream)));
    return AMHD_OK;
}

int amhd_muscl(const amhd_grid *g, int32_t axis, const void *W, void *WL, void *WR, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (axis != 0 && axis != 1) return fail(AMHD_ERR_ARG, "axis must be 0 or 1");
    if (!W || !WL || !WR) return fail(AMHD_ERR_ARG, "NULL array");
    const Layout l = layout_of(g);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::muscl(l, static_cast<const double *>(W), axis, g->limiter, static_cast<double *>(WL),
                                 static_cast<double *>(WR), S(stream)));
    else
        CK(Launch<float>::muscl(l, static_cast<const float *>(W), axis, g->limiter, static_cast<float *>(WL),
                                static_cast<float *>(WR), S(stream)));
    return AMHD_OK;
}

int amhd_hlld_flux(int32_t axis, int32_t dtype, const void *WL, const void *WR, void *F, void *smax, int64_t n_faces,
                   double gamma, double ch, void *stream)
{
    if (axis != 0 && axis != 1) return fail(AMHD_ERR_ARG, "axis must be 0 or 1");
    if (dtype != AMHD_F32 && dtype != AMHD_F64) return fail(AMHD_ERR_ARG, "unknown dtype %d", dtype);
    if (n_faces < 0) return fail(AMHD_ERR_ARG, "n_faces < 0");
    if (n_faces == 0) return AMHD_OK;
    if (!WL || !WR || !F) return fail(AMHD_ERR_ARG, "NULL array");
    if (dtype == AMHD_F64)
        CK(Launch<double>::hlld(static_cast<const double *>(WL), static_cast<const double *>(WR), static_cast<double *>(F),
                                static_cast<double *>(smax), n_faces, axis, gamma, ch, S(stream)));
    else
        CK(Launch<float>::hlld(static_cast<const float *>(WL), static_cast<const float *>(WR), static_cast<float *>(F),
                               static_cast<float *>(smax), n_faces, axis, gamma, ch, S(stream)));
    return AMHD_OK;
}

int amhd_apply_bc(const amhd_grid *g, void *U, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U) return fail(AMHD_ERR_ARG, "NULL array");
    CK(run_bc_fill(g, U, S(stream)));
    return AMHD_OK;
}

int amhd_enforce_scalar_bounds(const amhd_grid *g, void *U, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U) return fail(AMHD_ERR_ARG, "NULL array");
    const Layout l = layout_of(g);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::scalar_bounds(l, static_cast<double *>(U), S(stream)));
    else
        CK(Launch<float>::scalar_bounds(l, static_cast<float *>(U), S(stream)));
    return AMHD_OK;
}

static int compute_dt_impl(const amhd_grid *g, const void *A, int from_prim, amhd_control *ctl, double *dt_host,
                           double *ch_host, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!A || !ctl) return fail(AMHD_ERR_ARG, "NULL array or control");
    cudaStream_t s = S(stream);
    CK(cudaMemsetAsync(&ctl->red[0], 0, sizeof(ctl->red), s));
    CK(run_dt_reduce(g, A, from_prim, ctl, s));
    const amhd_instance one = single_instance(g, 8);
    CK(run_finalize(g->dtype, nullptr, 1, one, nullptr, ctl, 0, 1, s));
    if (dt_host || ch_host) {
        double v[2];
        CK(cudaMemcpyAsync(&v[0], &ctl->dt_cfl, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&v[1], &ctl->ch, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (dt_host) *dt_host = v[0];
        if (ch_host) *ch_host = v[1];
    }
    return AMHD_OK;
}

int amhd_compute_dt(const amhd_grid *g, const void *W, amhd_control *ctl, double *dt_host, double *ch_host,
                    void *stream)
{
    return compute_dt_impl(g, W, 1, ctl, dt_host, ch_host, stream);
}

int amhd_compute_dt_cons(const amhd_grid *g, const void *U, amhd_control *ctl, double *dt_host, double *ch_host,
                         void *stream)
{
    return compute_dt_impl(g, U, 0, ctl, dt_host, ch_host, stream);
}

int amhd_boundary_energy_flux(const amhd_grid *g, const void *U, amhd_control *ctl, double *out_host, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !ctl || !out_host) return fail(AMHD_ERR_ARG, "NULL argument");
    if (g->bc_x == AMHD_BC_PERIODIC) {
        *out_host = 0.0;
        return AMHD_OK;
    }
    cudaStream_t s = S(stream);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::bflux(*g, static_cast<const double *>(U), &ctl->scratch, s));
    else
        CK(Launch<float>::bflux(*g, static_cast<const float *>(U), &ctl->scratch, s));
    CK(cudaMemcpyAsync(out_host, &ctl->scratch, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return AMHD_OK;
}

int amhd_powell_source(const amhd_grid *g, const void *W, void *Sout, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!W || !Sout) return fail(AMHD_ERR_ARG, "NULL array");
    const Layout l = layout_of(g);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::powell(l, static_cast<const double *>(W), static_cast<double *>(Sout), g->dx, g->dy, S(stream)));
    else
        CK(Launch<float>::powell(l, static_cast<const float *>(W), static_cast<float *>(Sout), g->dx, g->dy, S(stream)));
    return AMHD_OK;
}

int amhd_compute_rhs(const amhd_grid *g, void *U, void *R, double ch, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[2] = {U, R};
    if (int e = check_padded(g, ptrs, 2)) return e;
    cudaStream_t s = S(stream);
    CK(run_bc_fill(g, U, s));
    CK(cudaMemsetAsync(R, 0, (size_t)g->var_stride * 10 * elem_size(g->dtype), s));
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    StageParams p;
    memset(&p, 0, sizeof p);
    set_input(p, U, U, g, tx);
    p.uout = R;
    p.one = one;
    p.n_tiles = n_items(one, tx);
    p.ch = ch;
    CK(run_stage(g->dtype, 0, tx, p, stage_grid(g->dtype, tx, p.n_tiles, g_ctas_per_sm), s));
    return AMHD_OK;
}

int amhd_step_ssprk3(const amhd_grid *g, void *U, void *U1, void *U2, double dt, double ch, double decay,
                     amhd_control *ctl, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[3] = {U, U1, U2};
    if (int e = check_padded(g, ptrs, 3)) return e;
    cudaStream_t s = S(stream);
    if (ctl && g->bc_x != AMHD_BC_PERIODIC) {
        // _cumulative_boundary_energy += flux(U0) * dt (solver.py:316-317), on the device
        if (g->dtype == AMHD_F64)
            CK(Launch<double>::bflux_accum(*g, static_cast<const double *>(U), ctl, dt, s));
        else
            CK(Launch<float>::bflux_accum(*g, static_cast<const float *>(U), ctl, dt, s));
    }
    CK(run_bc_fill(g, U, s));  // compute_rhs(U0) fills U0's ghosts first (solver.py:276)
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    const int n_tiles = n_items(one, tx);
    return three_stages(g, one, nullptr, nullptr, n_tiles, tx, stage_grid(g->dtype, tx, n_tiles, g_ctas_per_sm), U,
                        U1, U2, ctl, 0, dt, ch, ch > 0 ? decay : 1.0, 0, s);
}

int amhd_rk_stage(const amhd_grid *g, int32_t stage, const void *Uin, const void *U0, void *Uout, double dt,
                  double ch, double decay, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (stage < 1 || stage > 3) return fail(AMHD_ERR_ARG, "stage must be 1, 2 or 3");
    const void *ptrs[3] = {Uin, U0, Uout};
    if (int e = check_padded(g, ptrs, 3)) return e;
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    StageParams p;
    memset(&p, 0, sizeof p);
    set_input(p, Uin, U0, g, tx);
    p.uout = Uout;
    p.one = one;
    p.n_tiles = n_items(one, tx);
    p.dt = dt;
    p.ch = ch;
    p.decay = ch > 0 ? decay : 1.0;
    CK(run_stage(g->dtype, stage, tx, p, stage_grid(g->dtype, tx, p.n_tiles, g_ctas_per_sm), S(stream)));
    return AMHD_OK;
}

int amhd_control_init(const amhd_grid *g, const void *U, amhd_control *ctl, double t, double t_end, int64_t step,
                      int64_t max_steps, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !ctl) return fail(AMHD_ERR_ARG, "NULL argument");
    cudaStream_t s = S(stream);
    if (int e = control_upload(ctl, t, t_end, step, max_steps, s)) return e;
    // dt from the state as the caller left it, ghosts included (solver.py:476-477)
    CK(run_dt_reduce(g, U, 0, ctl, s));
    const amhd_instance one = single_instance(g, 8);
    CK(run_finalize(g->dtype, nullptr, 1, one, U, ctl, 0, 0, s));
    CK(run_bc_fill(g, const_cast<void *>(U), s));
    return AMHD_OK;
}

int amhd_control_resume(amhd_control *ctl, int32_t n, double snap_t, void *stream)
{
    if (!ctl || n <= 0) return fail(AMHD_ERR_ARG, "bad control arguments");
    CK(launch_control_resume(ctl, n, snap_t, S(stream)));
    return AMHD_OK;
}

static int advance_impl(const amhd_grid *g, void *U, void *Ulo, void *U1, void *U2, amhd_control *ctl,
                        int32_t n_steps, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[4] = {U, U1, U2, Ulo};
    if (int e = check_padded(g, ptrs, Ulo ? 4 : 3)) return e;
    if (!ctl) return fail(AMHD_ERR_ARG, "NULL control");
    if (n_steps < 0) return fail(AMHD_ERR_ARG, "n_steps < 0");
    cudaStream_t s = S(stream);
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    const int n_tiles = n_items(one, tx);
    const int grid = stage_grid(g->dtype, tx, n_tiles, g_ctas_per_sm);
    const int defer = is_march(tx);
    // a persistent marching grid (fewer CTAs than items) draws its items from the
    // control block's work queue, so that no warp idles while items remain
    int32_t *queue = (is_march(tx) && grid * (kMarchThreads / 32) < n_tiles) ? ctl->queue : nullptr;
    for (int k = 0; k < n_steps; ++k) {
        if (int e = three_stages(g, one, nullptr, nullptr, n_tiles, tx, grid, U, U1, U2, ctl, 1, 0, 0, 1, 1, s,
                                 nullptr, nullptr, 1, defer, queue, Ulo))
            return e;
        CK(run_finalize(g->dtype, nullptr, 1, one, U, ctl, 1, 0, s, defer));
    }
    if (defer && n_steps > 0)
        if (int e = fill_after_loop(g->dtype, one, nullptr, 1, U, s)) return e;
    return AMHD_OK;
}

int amhd_advance(const amhd_grid *g, void *U, void *U1, void *U2, amhd_control *ctl, int32_t n_steps, void *stream)
{
    return advance_impl(g, U, nullptr, U1, U2, ctl, n_steps, stream);
}

int amhd_advance_compensated(const amhd_grid *g, void *U, void *U_lo, void *U1, void *U2, amhd_control *ctl,
                             int32_t n_steps, void *stream)
{
    if (!U_lo) return fail(AMHD_ERR_ARG, "NULL low part");
    if (g && g->dtype != AMHD_F32) return fail(AMHD_ERR_ARG, "the compensated loop is for float32 states");
    if (g && !is_march(tile_of(g))) return fail(AMHD_ERR_UNSUPPORTED, "the compensated loop needs the marching kernel");
    return advance_impl(g, U, U_lo, U1, U2, ctl, n_steps, stream);
}

int amhd_control_init_split(const amhd_grid *g, void *U, amhd_control *ctl, double t, double t_end, int64_t step,
                            int64_t max_steps, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !ctl) return fail(AMHD_ERR_ARG, "NULL argument");
    cudaStream_t s = S(stream);
    if (int e = control_upload(ctl, t, t_end, step, max_steps, s)) return e;
    CK(run_dt_reduce(g, U, 0, ctl, s));
    CK(run_bc_fill(g, U, s));
    return AMHD_OK;
}

int amhd_advance_stage(const amhd_grid *g, int32_t stage, void *U, void *U1, void *U2, amhd_control *ctl,
                       void *stream)
{
    if (int e = check_grid(g)) return e;
    if (stage < 1 || stage > 3) return fail(AMHD_ERR_ARG, "stage must be 1, 2 or 3");
    const void *ptrs[3] = {U, U1, U2};
    if (int e = check_padded(g, ptrs, 3)) return e;
    if (!ctl) return fail(AMHD_ERR_ARG, "NULL control");
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    StageParams p;
    memset(&p, 0, sizeof p);
    void *in[3] = {U, U1, U2};
    void *out[3] = {U1, U2, U};
    set_input(p, in[stage - 1], U, g, tx);
    p.uout = out[stage - 1];
    p.one = one;
    p.n_tiles = n_items(one, tx);
    p.ctl = ctl;
    p.use_ctl = 1;
    p.fuse_dt = stage == 3;
    CK(run_stage(g->dtype, stage, tx, p, stage_grid(g->dtype, tx, p.n_tiles, g_ctas_per_sm), S(stream)));
    return AMHD_OK;
}

int amhd_advance_finish(const amhd_grid *g, void *U, amhd_control *ctl, int32_t advance, int32_t cut_x,
                        void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !ctl) return fail(AMHD_ERR_ARG, "NULL argument");
    if (cut_x < 0 || cut_x > 3) return fail(AMHD_ERR_ARG, "cut_x must be a mask of bits 0 and 1, got %d", cut_x);
    amhd_instance one = single_instance(g, tile_of(g));
    one.cut_x = cut_x;
    CK(run_finalize(g->dtype, nullptr, 1, one, U, ctl, advance ? 1 : 0, 0, S(stream)));
    return AMHD_OK;
}

int amhd_advance_profile(const amhd_grid *g, void *U, void *U1, void *U2, amhd_control *ctl, int32_t n_steps,
                         double *ms_out, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[3] = {U, U1, U2};
    if (int e = check_padded(g, ptrs, 3)) return e;
    if (!ctl || !ms_out) return fail(AMHD_ERR_ARG, "NULL argument");
    if (n_steps <= 0) return fail(AMHD_ERR_ARG, "n_steps must be positive");
    cudaStream_t s = S(stream);
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    const int n_tiles = n_items(one, tx);
    const int grid = stage_grid(g->dtype, tx, n_tiles, g_ctas_per_sm);
    std::vector<cudaEvent_t> ev(4 * (size_t)n_steps + 1);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    int rc = AMHD_OK;
    StageParams p;
    memset(&p, 0, sizeof p);
    p.one = one;
    p.n_tiles = n_tiles;
    p.ctl = ctl;
    p.use_ctl = 1;
    p.pull_ghosts = 1;
    p.defer_fill = is_march(tx);  // as amhd_advance: U's ghost cells once, after the last step (timed)
    cudaError_t ce = cudaEventRecord(ev[0], s);
    for (int k = 0; k < n_steps && ce == cudaSuccess; ++k) {
        for (int st = 1; st <= 3 && ce == cudaSuccess; ++st) {
            set_input(p, st == 1 ? U : (st == 2 ? U1 : U2), U, g, tx);
            p.uout = st == 1 ? U1 : (st == 2 ? U2 : U);
            p.fuse_dt = st == 3;
            ce = run_stage(g->dtype, st, tx, p, grid, s);
            if (ce == cudaSuccess) ce = cudaEventRecord(ev[4 * k + st], s);
        }
        if (ce == cudaSuccess) ce = run_finalize(g->dtype, nullptr, 1, one, U, ctl, 1, 0, s);
        if (ce == cudaSuccess && p.defer_fill && k == n_steps - 1)
            ce = g->dtype == AMHD_F64 ? Launch<double>::march_fill(p, s) : Launch<float>::march_fill(p, s);
        if (ce == cudaSuccess) ce = cudaEventRecord(ev[4 * k + 4], s);
    }
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev.back());
    if (ce != cudaSuccess) {
        rc = fail(AMHD_ERR_CUDA, "amhd_advance_profile: %s", cudaGetErrorString(ce));
    } else {
        for (int q = 0; q < 5; ++q) ms_out[q] = 0.0;
        for (int k = 0; k < n_steps; ++k)
            for (int q = 0; q < 4; ++q) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[4 * k + q], ev[4 * k + q + 1]);
                ms_out[q] += ms;
            }
        float tot = 0.f;
        cudaEventElapsedTime(&tot, ev[0], ev.back());
        ms_out[4] = tot;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

int amhd_step_host(const amhd_grid *g, void *U_host, void *dev_U, void *dev_U1, void *dev_U2, amhd_control *ctl,
                   double t, double t_end, double *out_host, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[3] = {dev_U, dev_U1, dev_U2};
    if (int e = check_padded(g, ptrs, 3)) return e;
    if (!U_host || !ctl) return fail(AMHD_ERR_ARG, "NULL argument");
    cudaStream_t s = S(stream);
    const size_t es = elem_size(g->dtype);
    const int nxt = g->nx + 2 * kNG, nyt = g->ny + 2 * kNG;
    char *h = static_cast<char *>(U_host);
    char *d = static_cast<char *>(dev_U);
    // the device planes are the host array itself when no row or plane is padded
    const bool contiguous = g->pitch == nyt && g->var_stride == (int64_t)nxt * nyt;
    if (contiguous)
        CK(cudaMemcpyAsync(d, h, (size_t)10 * nxt * nyt * es, cudaMemcpyHostToDevice, s));
    else
        for (int v = 0; v < 10; ++v)
            CK(cudaMemcpy2DAsync(d + (size_t)v * g->var_stride * es, (size_t)g->pitch * es,
                                 h + (size_t)v * nxt * nyt * es, (size_t)nyt * es, (size_t)nyt * es, nxt,
                                 cudaMemcpyHostToDevice, s));
    // dt of this step from the uploaded state, ghosts as given (solver.py:476-479)
    if (int e = control_upload(ctl, t, t_end, 0, 1, s)) return e;
    CK(run_dt_reduce(g, dev_U, 0, ctl, s));
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    CK(run_finalize(g->dtype, nullptr, 1, one, dev_U, ctl, 0, 0, s));
    CK(run_bc_fill(g, dev_U, s));
    const int n_tiles = n_items(one, tx);
    if (int e = three_stages(g, one, nullptr, nullptr, n_tiles, tx, stage_grid(g->dtype, tx, n_tiles, g_ctas_per_sm),
                             dev_U, dev_U1, dev_U2, ctl, 1, 0, 0, 1, 0, s))
        return e;
    CK(run_finalize(g->dtype, nullptr, 1, one, dev_U, ctl, 1, 0, s));
    if (contiguous)
        CK(cudaMemcpyAsync(h, d, (size_t)10 * nxt * nyt * es, cudaMemcpyDeviceToHost, s));
    else
        for (int v = 0; v < 10; ++v)
            CK(cudaMemcpy2DAsync(h + (size_t)v * nxt * nyt * es, (size_t)nyt * es, d + (size_t)v * g->var_stride * es,
                                 (size_t)g->pitch * es, (size_t)nyt * es, nxt, cudaMemcpyDeviceToHost, s));
    amhd_control r;
    CK(cudaMemcpyAsync(&r, ctl, sizeof r, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (out_host) {
        out_host[0] = r.t;
        out_host[1] = r.last_dt;
        out_host[2] = r.ch;
        out_host[3] = r.e_bnd;
    }
    if (r.flags & AMHD_FLAG_TIMEOUT) return fail(AMHD_ERR_TIMEOUT, "a bounded device wait expired; tiles not updated");
    if (r.flags & AMHD_FLAG_NONFINITE) return fail(AMHD_ERR_NONFINITE, "non-finite value in the new state");
    return AMHD_OK;
}

// Copy streams and events of amhd_step_host_n, created once per device: one
// stream per direction (both PCIe directions busy at once), an event per piece
// (kHostPieces row ranges per plane) marking that a step's copy of that piece
// has reached the host.  Whole planes: 4 pieces per plane measured no better
// at 2048^2 (5.28 against 4.96 ms per step).
constexpr int kHostPieces = 1;
struct HostLoopStreams {
    std::mutex busy;  // one call at a time per device (the call is synchronous)
    bool ready = false;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t out[10 * kHostPieces] = {}, in_done = nullptr, step_done = nullptr, out_done = nullptr;
};

static HostLoopStreams *host_loop_streams()
{
    static std::mutex mu;
    static std::map<int, HostLoopStreams> cache;  // nodes never move: the entries stay valid
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    HostLoopStreams &h = cache[dev];
    if (h.ready) return &h;
    bool ok = cudaStreamCreateWithFlags(&h.h2d, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&h.d2h, cudaStreamNonBlocking) == cudaSuccess;
    for (int v = 0; v < 10 * kHostPieces && ok; ++v)
        ok = cudaEventCreateWithFlags(&h.out[v], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&h.in_done, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.step_done, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.out_done, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) return nullptr;
    h.ready = true;
    return &h;
}

int amhd_step_host_n(const amhd_grid *g, void *U_host, void *dev_U, void *dev_U1, void *dev_U2, amhd_control *ctl,
                     double t, double t_end, int32_t n_steps, double *out_host, void *stream)
{
    if (int e = check_grid(g)) return e;
    const void *ptrs[3] = {dev_U, dev_U1, dev_U2};
    if (int e = check_padded(g, ptrs, 3)) return e;
    if (!U_host || !ctl) return fail(AMHD_ERR_ARG, "NULL argument");
    if (n_steps < 1) return fail(AMHD_ERR_ARG, "n_steps < 1");
    HostLoopStreams *hs = host_loop_streams();
    if (!hs) return fail(AMHD_ERR_CUDA, "copy streams could not be created");
    std::lock_guard<std::mutex> busy(hs->busy);  // callers on other threads share the copy streams
    cudaStream_t s = S(stream);
    const size_t es = elem_size(g->dtype);
    const int nxt = g->nx + 2 * kNG, nyt = g->ny + 2 * kNG;
    char *h = static_cast<char *>(U_host);
    char *d = static_cast<char *>(dev_U);
    const bool contiguous = g->pitch == nyt;
    // piece q of plane v: rows [r0, r1) of the plane
    auto copy_piece = [&](int v, int q, bool to_device, cudaStream_t cs) -> cudaError_t {
        const int r0 = (int)((int64_t)nxt * q / kHostPieces), r1 = (int)((int64_t)nxt * (q + 1) / kHostPieces);
        if (r1 <= r0) return cudaSuccess;
        char *hp = h + ((size_t)v * nxt + r0) * nyt * es;
        char *dp = d + ((size_t)v * g->var_stride + (size_t)r0 * g->pitch) * es;
        if (contiguous)
            return to_device ? cudaMemcpyAsync(dp, hp, (size_t)(r1 - r0) * nyt * es, cudaMemcpyHostToDevice, cs)
                             : cudaMemcpyAsync(hp, dp, (size_t)(r1 - r0) * nyt * es, cudaMemcpyDeviceToHost, cs);
        return to_device ? cudaMemcpy2DAsync(dp, (size_t)g->pitch * es, hp, (size_t)nyt * es, (size_t)nyt * es,
                                             r1 - r0, cudaMemcpyHostToDevice, cs)
                         : cudaMemcpy2DAsync(hp, (size_t)nyt * es, dp, (size_t)g->pitch * es, (size_t)nyt * es,
                                             r1 - r0, cudaMemcpyDeviceToHost, cs);
    };
    const int tx = tile_of(g);
    const amhd_instance one = single_instance(g, tx);
    const int n_tiles = n_items(one, tx);
    const int grid = stage_grid(g->dtype, tx, n_tiles, g_ctas_per_sm);
    // the copy streams start after what the caller queued before this call
    CK(cudaEventRecord(hs->step_done, s));
    CK(cudaStreamWaitEvent(hs->h2d, hs->step_done, 0));
    if (int e = control_upload(ctl, t, t_end, 0, n_steps, s)) return e;
    for (int k = 0; k < n_steps; ++k) {
        // the inputs of step k, piece by piece, each as soon as step k-1's result
        // for that piece is back in U_host (the other direction is still busy
        // with the later pieces)
        for (int v = 0; v < 10; ++v)
            for (int q = 0; q < kHostPieces; ++q) {
                if (k > 0) CK(cudaStreamWaitEvent(hs->h2d, hs->out[v * kHostPieces + q], 0));
                CK(copy_piece(v, q, true, hs->h2d));
            }
        CK(cudaEventRecord(hs->in_done, hs->h2d));
        CK(cudaStreamWaitEvent(s, hs->in_done, 0));
        // as amhd_step_host: dt from the uploaded state, one SSP-RK3 step
        CK(run_dt_reduce(g, dev_U, 0, ctl, s));
        CK(run_finalize(g->dtype, nullptr, 1, one, dev_U, ctl, 0, 0, s));
        CK(run_bc_fill(g, dev_U, s));
        if (int e = three_stages(g, one, nullptr, nullptr, n_tiles, tx, grid, dev_U, dev_U1, dev_U2, ctl, 1, 0, 0, 1,
                                 0, s))
            return e;
        CK(run_finalize(g->dtype, nullptr, 1, one, dev_U, ctl, 1, 0, s));
        CK(cudaEventRecord(hs->step_done, s));
        CK(cudaStreamWaitEvent(hs->d2h, hs->step_done, 0));
        for (int v = 0; v < 10; ++v)
            for (int q = 0; q < kHostPieces; ++q) {
                CK(copy_piece(v, q, false, hs->d2h));
                CK(cudaEventRecord(hs->out[v * kHostPieces + q], hs->d2h));
            }
    }
    CK(cudaEventRecord(hs->out_done, hs->d2h));
    CK(cudaStreamWaitEvent(s, hs->out_done, 0));
    amhd_control r;
    CK(cudaMemcpyAsync(&r, ctl, sizeof r, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (out_host) {
        out_host[0] = r.t;
        out_host[1] = r.last_dt;
        out_host[2] = r.ch;
        out_host[3] = r.e_bnd;
    }
    if (r.flags & AMHD_FLAG_TIMEOUT) return fail(AMHD_ERR_TIMEOUT, "a bounded device wait expired; tiles not updated");
    if (r.flags & AMHD_FLAG_NONFINITE) return fail(AMHD_ERR_NONFINITE, "non-finite value in the new state");
    return AMHD_OK;
}

int amhd_diagnostics(const amhd_grid *g, const void *U, double x0, double *out_dev, double *rows_dev, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !out_dev || !rows_dev) return fail(AMHD_ERR_ARG, "NULL argument");
    cudaStream_t s = S(stream);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::diag_rows(*g, static_cast<const double *>(U), rows_dev, s));
    else
        CK(Launch<float>::diag_rows(*g, static_cast<const float *>(U), rows_dev, s));
    CK(launch_diag_finish(*g, x0, rows_dev, out_dev, s));
    return AMHD_OK;
}

int amhd_diagnostics_colour(const amhd_grid *g, const void *U, double x0, const double *rows_dev, double *cp2_dev,
                            double *pos_dev, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !rows_dev || !cp2_dev || !pos_dev) return fail(AMHD_ERR_ARG, "NULL argument");
    cudaStream_t s = S(stream);
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::diag_colour(*g, static_cast<const double *>(U), x0, rows_dev, cp2_dev, pos_dev, s));
    else
        CK(Launch<float>::diag_colour(*g, static_cast<const float *>(U), x0, rows_dev, cp2_dev, pos_dev, s));
    return AMHD_OK;
}

int amhd_ensemble_init(const amhd_instance *inst_host, const amhd_instance *inst_dev, int32_t n_inst, int32_t dtype,
                       void *U, amhd_control *ctl_dev, double t_end, int64_t max_steps, void *stream)
{
    if (!inst_host || !inst_dev || !U || !ctl_dev || n_inst <= 0) return fail(AMHD_ERR_ARG, "bad ensemble arguments");
    cudaStream_t s = S(stream);
    const size_t es = elem_size(dtype);
    std::vector<amhd_control> h(n_inst);
    memset(h.data(), 0, sizeof(amhd_control) * n_inst);
    for (int k = 0; k < n_inst; ++k) {
        h[k].t_end = t_end;
        h[k].max_steps = max_steps;
        h[k].active = 1;
        h[k].decay = 1.0;
        h[k].snap_t = __builtin_inf();
    }
    CK(cudaMemcpyAsync(ctl_dev, h.data(), sizeof(amhd_control) * n_inst, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // h goes out of scope
    for (int k = 0; k < n_inst; ++k) {
        const amhd_grid *g = &inst_host[k].grid;
        if (int e = check_grid(g)) return fail(e, "instance %d: %s", k, g_err.c_str());
        if (g->dtype != dtype) return fail(AMHD_ERR_ARG, "instance %d has a different dtype", k);
        void *Uk = static_cast<char *>(U) + (size_t)inst_host[k].offset * es;
        CK(run_dt_reduce(g, Uk, 0, ctl_dev + k, s));
    }
    amhd_instance dummy;
    memset(&dummy, 0, sizeof dummy);
    CK(run_finalize(dtype, inst_dev, n_inst, dummy, U, ctl_dev, 0, 0, s));
    for (int k = 0; k < n_inst; ++k) {
        void *Uk = static_cast<char *>(U) + (size_t)inst_host[k].offset * es;
        CK(run_bc_fill(&inst_host[k].grid, Uk, s));
    }
    return AMHD_OK;
}

int amhd_ensemble_continue(const amhd_instance *inst_host, const amhd_instance *inst_dev, int32_t n_inst,
                           int32_t dtype, void *U, amhd_control *ctl_dev, double t_end, void *stream)
{
    if (!inst_host || !inst_dev || !U || !ctl_dev || n_inst <= 0) return fail(AMHD_ERR_ARG, "bad ensemble arguments");
    cudaStream_t s = S(stream);
    const size_t es = elem_size(dtype);
    CK(launch_control_retarget(ctl_dev, n_inst, t_end, s));
    for (int k = 0; k < n_inst; ++k) {
        const amhd_grid *g = &inst_host[k].grid;
        if (int e = check_grid(g)) return fail(e, "instance %d: %s", k, g_err.c_str());
        void *Uk = static_cast<char *>(U) + (size_t)inst_host[k].offset * es;
        CK(run_dt_reduce(g, Uk, 0, ctl_dev + k, s));
    }
    amhd_instance dummy;
    memset(&dummy, 0, sizeof dummy);
    CK(run_finalize(dtype, inst_dev, n_inst, dummy, U, ctl_dev, 0, 0, s));
    return AMHD_OK;
}

int amhd_ensemble_advance(const amhd_instance *inst_dev, int32_t n_inst, const int32_t *tile_inst_dev,
                          const int32_t *tile_order_dev, int32_t n_tiles, int32_t dtype, int32_t tile_x, void *U,
                          void *U1, void *U2, amhd_control *ctl_dev, int32_t n_steps, int32_t ctas,
                          const void *tmaps_dev, int32_t *queue_dev, void *stream)
{
    if (!inst_dev || !tile_inst_dev || !U || !U1 || !U2 || !ctl_dev || n_inst <= 0 || n_tiles <= 0)
        return fail(AMHD_ERR_ARG, "bad ensemble arguments");
    if (dtype != AMHD_F32 && dtype != AMHD_F64) return fail(AMHD_ERR_ARG, "unknown dtype %d", dtype);
    if (!valid_geometry(tile_x)) return fail(AMHD_ERR_ARG, "tile_x must be 4, 8, 16 or -1024..-4 (marching rows)");
    cudaStream_t s = S(stream);
    int grid = ctas;
    if (grid <= 0) {
        const int occ = dtype == AMHD_F64 ? Launch<double>::stage_ctas_per_sm(tile_x)
                                          : Launch<float>::stage_ctas_per_sm(tile_x);
        grid = occ * device_sm_count();
    }
    if (grid > n_tiles) grid = n_tiles;
    amhd_grid gdt;
    memset(&gdt, 0, sizeof gdt);
    gdt.dtype = dtype;
    amhd_instance dummy;
    memset(&dummy, 0, sizeof dummy);
    const int defer = is_march(tile_x);
    for (int k = 0; k < n_steps; ++k) {
        if (int e = three_stages(&gdt, dummy, inst_dev, tile_inst_dev, n_tiles, tile_x, grid, U, U1, U2, ctl_dev, 1, 0,
                                 0, 1, 1, s, tile_order_dev, static_cast<const CUtensorMap *>(tmaps_dev), n_inst, defer,
                                 queue_dev))
            return e;
        CK(run_finalize(dtype, inst_dev, n_inst, dummy, U, ctl_dev, 1, 0, s, defer));
    }
    if (defer && n_steps > 0)
        if (int e = fill_after_loop(dtype, dummy, inst_dev, n_inst, U, s)) return e;
    return AMHD_OK;
}

}  // extern "C"
#pragma GCC visibility pop

// ---------------------------------------------------------------------------
// Diagnostics without any allocation by the caller or the library.
//
// The row pass of amhd_diagnostics needs 7 * nx doubles of scratch.  Here that
// scratch is a fixed file-scope device array: it is part of the module image,
// so every GPU that loads this library holds it (AMHD_NOALLOC_MAX_NX * 7 * 8
// bytes = 896 KiB) until the process exits, and no call ever allocates.
// In host code `g_noalloc_rows` only names a host-side shadow of the symbol,
// never a device address; the device address is looked up per device with
// cudaGetSymbolAddress, on the first call made while that device is current.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_rows[7 * AMHD_NOALLOC_MAX_NX];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

int noalloc_rows_ptr(double **out)
{
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(AMHD_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_rows);
        if (e != cudaSuccess || !p)
            return fail(AMHD_ERR_CUDA, "cudaGetSymbolAddress of the diagnostics scratch on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<double *>(g_noalloc_ptr[dev]);
    return AMHD_OK;
}
}  // namespace

#pragma GCC visibility push(default)
extern "C" int amhd_diagnostics_noalloc(const amhd_grid *g, const void *U, double x0, double *out_dev, void *stream)
{
    if (int e = check_grid(g)) return e;
    if (!U || !out_dev) return fail(AMHD_ERR_ARG, "NULL argument");
    if (g->nx > AMHD_NOALLOC_MAX_NX)
        return fail(AMHD_ERR_ARG, "amhd_diagnostics_noalloc: nx = %d exceeds the fixed scratch limit of %d rows", g->nx,
                    AMHD_NOALLOC_MAX_NX);
    double *rows = nullptr;
    if (int e = noalloc_rows_ptr(&rows)) return e;
    cudaStream_t s = S(stream);
    // every one of the 7 * nx scratch entries the finish kernel reads is written by
    // the row kernel of the same call, so nothing has to be cleared between calls
    if (g->dtype == AMHD_F64)
        CK(Launch<double>::diag_rows(*g, static_cast<const double *>(U), rows, s));
    else
        CK(Launch<float>::diag_rows(*g, static_cast<const float *>(U), rows, s));
    CK(launch_diag_finish(*g, x0, rows, out_dev, s));
    return AMHD_OK;
}
#pragma GCC visibility pop
