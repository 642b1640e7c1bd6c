// amhd_f64.cu -- float64 instantiation of the kernels.  Built with
// -fmad=false: no multiply-add contraction, so every rounding matches the
// reference's float64 arithmetic (numpy / CuPy elementwise + its HLLD kernel).
#include "amhd_launch_impl.cuh"

namespace amhd {

template struct Launch<double>;

// trapezoid mixing width (solver.py:353-356) and the global sums / maxima
__global__ void diag_finish_kernel(const amhd_grid g, double x0, const double *rows, double *out)
{
    const int nx = g.nx;
    const double *s_c = rows, *s_rho = rows + nx, *s_e = rows + 2 * nx, *s_div2 = rows + 3 * nx,
                 *s_ens = rows + 4 * nx, *m_div = rows + 5 * nx, *m_stag = rows + 6 * nx;
    __shared__ double red[6][256];
    double a_rho = 0, a_e = 0, a_div2 = 0, a_ens = 0, a_mw = 0, a_mdiv = 0, a_stag = 0;
    const double inv_ny = 1.0 / g.ny;
    for (int r = threadIdx.x; r < nx; r += blockDim.x) {
        a_rho += s_rho[r];
        a_e += s_e[r];
        a_div2 += s_div2[r];
        a_ens += s_ens[r];
        a_mdiv = fmax(a_mdiv, m_div[r]);
        a_stag = fmax(a_stag, m_stag[r]);
        if (r + 1 < nx) {
            double c0 = s_c[r] * inv_ny, c1 = s_c[r + 1] * inv_ny;
            double xa = x0 + ((double)r + 0.5) * g.dx, xb = x0 + ((double)(r + 1) + 0.5) * g.dx;
            a_mw += (xb - xa) * (c0 * (1.0 - c0) + c1 * (1.0 - c1)) / 2.0;
        }
    }
    // fixed-order tree: reproducible from run to run
    red[0][threadIdx.x] = a_rho;
    red[1][threadIdx.x] = a_e;
    red[2][threadIdx.x] = a_div2;
    red[3][threadIdx.x] = a_ens;
    red[4][threadIdx.x] = a_mw;
    __shared__ double mx[2][256];
    mx[0][threadIdx.x] = a_mdiv;
    mx[1][threadIdx.x] = a_stag;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            for (int k = 0; k < 5; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + h];
            for (int k = 0; k < 2; ++k) mx[k][threadIdx.x] = fmax(mx[k][threadIdx.x], mx[k][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double ncell = (double)g.nx * (double)g.ny;
        out[0] = red[0][0] * g.dx * g.dy;
        out[1] = red[1][0] * g.dx * g.dy;
        out[2] = mx[0][0];
        out[3] = sqrt(red[2][0] / ncell);
        out[4] = red[4][0];
        out[5] = mx[1][0];
        out[6] = red[3][0] / ncell;
    }
}

cudaError_t launch_diag_finish(const amhd_grid &g, double x0, const double *rows, double *out, cudaStream_t s)
{
    diag_finish_kernel<<<1, 256, 0, s>>>(g, x0, rows, out);
    return cudaGetLastError();
}

__global__ void control_resume_kernel(amhd_control *ctl, int n, double snap_t)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (ctl[k].flags & AMHD_FLAG_PAUSED) {
        ctl[k].flags &= ~AMHD_FLAG_PAUSED;
        ctl[k].active = 1;
    }
    ctl[k].snap_t = snap_t;
}

cudaError_t launch_control_resume(amhd_control *ctl, int n, double snap_t, cudaStream_t s)
{
    control_resume_kernel<<<(n + 127) / 128, 128, 0, s>>>(ctl, n, snap_t);
    return cudaGetLastError();
}

__global__ void control_retarget_kernel(amhd_control *ctl, int n, double t_end)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    ctl[k].t_end = t_end;
    ctl[k].active = 1;
    ctl[k].flags &= ~(AMHD_FLAG_DT_TINY | AMHD_FLAG_PAUSED);
    for (int q = 0; q < 4; ++q) ctl[k].red[q] = 0ull;
}

cudaError_t launch_control_retarget(amhd_control *ctl, int n, double t_end, cudaStream_t s)
{
    control_retarget_kernel<<<(n + 127) / 128, 128, 0, s>>>(ctl, n, t_end);
    return cudaGetLastError();
}

int device_sm_count()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n;
}

}  // namespace amhd
