// amhd_launch.h -- host-side launch interface between the C ABI (amhd_capi.cu)
// and the per-precision kernel translation units (amhd_f64.cu, amhd_f32.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "aeromhd.h"

namespace amhd {

// arguments of one fused RK stage launch over a list of (instance, tile);
// passed by value as a __grid_constant__ kernel parameter (the tensor map
// must live there or in global memory for the TMA unit to read it)
struct StageParams {
    CUtensorMap tmap;              // single grid: tensor map of uin (when use_tma)
    CUtensorMap tmap_base;         // single grid, marching kernel: tensor map of u0 (when use_tma)
    const CUtensorMap *tmaps;      // ensemble: 3 maps per instance (U, U1, U2), device memory
    int32_t use_tma;               // stage the tile + halo with TMA
    int32_t in_buf;                // ensemble: which of the 3 maps is uin
    const void *uin;               // stage input state (stencil source)
    const void *u0;                // step base state U0
    void *uout;                    // stage output (may alias u0 on stage 3)
    const amhd_instance *inst;     // device instance table, or nullptr: use `one`
    amhd_instance one;             // the single instance when inst == nullptr
    const int32_t *tile_inst;      // device: instance of each tile (with inst)
    const int32_t *tile_order;     // device: tile taken at each work position, or nullptr
    int32_t n_tiles;
    amhd_control *ctl;             // per-instance controls (device) or nullptr
    double dt, ch, decay;          // host scalars when !use_ctl
    int32_t use_ctl;               // take dt / ch / decay / active from ctl
    int32_t fuse_dt;               // stage 3: accumulate the CFL reduction
    int32_t march_rows;            // warp-marching kernel: rows of one work item
    int32_t n_inst;                // instances in inst (ghost fill after a marching stage)
    int32_t pull_ghosts;           // marching kernel: read ghost cells from their interior sources,
                                   // so stages 1 and 2 need no ghost fill of their output
    int32_t defer_fill;            // with pull_ghosts: stage 3 leaves U's ghost cells too (the run
                                   // loop fills them once after its last step, Launch::march_fill)
    int32_t pdl;                   // marching kernel: launch as a programmatic dependent of the
                                   // previous kernel in the stream (run loop)
    void *ulo;                     // float32 stage 3 of the marching kernel: low part of the base
                                   // state (U = U_hi + U_lo, same layout as U), read and rewritten
                                   // so that the base state is accumulated compensated; nullptr: off
    int32_t *queue;                // marching kernel: device work queue {next position, warps
                                   // finished}, zero between launches; nullptr: warp w takes
                                   // positions w, w + warps, ... (static split)
};

// Work geometry of the stage kernels, passed around as one int "tile_x":
// 4, 8, 16 -- the tiled kernel (tile_x x 32 cells per CTA);
// -1024 .. -4 -- the warp-marching kernel, -tile_x rows x kMarchCols columns per warp.
constexpr int kMarchCols = 28;     // 32 lanes minus a 2-column halo on each side
constexpr int kMarchThreads = 128; // 4 independent warps per CTA
inline bool is_march(int tile_x) { return tile_x < 0; }
// row chunks of an instance's last column strip per work item: its ny mod 28
// leftover columns plus a 2-column halo each side in 8 lanes (4 chunks to a
// warp) or 16 lanes (2); 1 when the strip is full or wider than 12 columns
__host__ __device__ inline int march_pack(int ny)
{
    const int rem = ny % kMarchCols;
    return rem == 0 ? 1 : rem <= 4 ? 4 : rem <= 12 ? 2 : 1;
}
// work items of an nx x ny instance in chunks of `rows` rows with that packing
inline int march_item_count(int nx, int ny, int rows, int pack)
{
    const int chunks = (nx + rows - 1) / rows, strips = (ny + kMarchCols - 1) / kMarchCols;
    if (pack <= 1) return chunks * strips;
    const int full = nx / rows;
    return (strips - 1) * chunks + (full + pack - 1) / pack + (nx % rows ? 1 : 0);
}
inline bool valid_geometry(int tile_x)
{
    return tile_x == 4 || tile_x == 8 || tile_x == 16 || (tile_x <= -4 && tile_x >= -1024);
}

struct Layout {
    int32_t nxt, nyt, pitch;
    int64_t var_stride;
};

template <typename R>
struct Launch {
    static cudaError_t stage(int stage, int tile_x, const StageParams &p, int grid, cudaStream_t s);
    // ghost cells of p.uout for every instance of p, active or not (idempotent)
    static cudaError_t march_fill(const StageParams &p, cudaStream_t s);
    static size_t stage_smem(int tile_x);
    static cudaError_t configure();
    static int stage_ctas_per_sm(int tile_x);
    static cudaError_t bc_fill(const amhd_grid &g, R *U, cudaStream_t s);
    static cudaError_t cons_to_prim(const Layout &li, const R *U, const Layout &lo, R *W, double gamma,
                                    cudaStream_t s);
    static cudaError_t prim_to_cons(const Layout &li, const R *W, const Layout &lo, R *U, double gamma,
                                    cudaStream_t s);
    static cudaError_t scalar_bounds(const Layout &l, R *U, cudaStream_t s);
    static cudaError_t muscl(const Layout &l, const R *W, int axis, int limiter, R *WL, R *WR, cudaStream_t s);
    static cudaError_t hlld(const R *WL, const R *WR, R *F, R *smax, int64_t n, int axis, double gamma, double ch,
                            cudaStream_t s);
    static cudaError_t powell(const Layout &l, const R *W, R *S, double dx, double dy, cudaStream_t s);
    static cudaError_t dt_reduce(const Layout &l, const R *A, int from_prim, double gamma, amhd_control *ctl,
                                 cudaStream_t s);
    // pdl: launch as a programmatic dependent of the previous kernel (run loop)
    static cudaError_t finalize(const amhd_instance *insts, int n_inst, const amhd_instance &one, const R *U,
                                amhd_control *ctl, int advance, int set_only, cudaStream_t s, int pdl = 0);
    static cudaError_t diag_rows(const amhd_grid &g, const R *U, double *rows, cudaStream_t s);
    static cudaError_t diag_colour(const amhd_grid &g, const R *U, double x0, const double *csum, double *cp2,
                                   double *pos, cudaStream_t s);
    static cudaError_t bflux(const amhd_grid &g, const R *U, double *out, cudaStream_t s);
    static cudaError_t bflux_accum(const amhd_grid &g, const R *U, amhd_control *ctl, double dt, cudaStream_t s);
};

// tensor map of one state buffer for the boxes of a stage kernel geometry (0 on success):
// tiled kernel (tile_x > 0) [10 planes][tile_x + 4 rows][36 columns];
// marching kernel (tile_x < 0) [10 planes][1 row][32 columns]
int encode_state_map(CUtensorMap *map, const void *base, int dtype, int pitch, int64_t var_stride, int tile_x);

cudaError_t launch_control_resume(amhd_control *ctl, int n, double snap_t, cudaStream_t s);
cudaError_t launch_control_retarget(amhd_control *ctl, int n, double t_end, cudaStream_t s);
cudaError_t launch_diag_finish(const amhd_grid &g, double x0, const double *rows, double *out, cudaStream_t s);
int device_sm_count();

}  // namespace amhd
