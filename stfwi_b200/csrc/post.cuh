// Per-iteration work around the gradient that stays on the device: the
// gradient post-processing of fwi/gradient.py:266-277 (Gaussian smoothing of
// fwi/loss.py:17-30, source taper, illumination / preconditioner multiply),
// the velocity feasibility projection of fwi/projections.py:67-117, and the
// two preconditioners built from the forward energy Ws (fwi/illumination.py:
// 38-47 and fwi/preconditioning.py:65-139).  All FP64, elementwise or
// separable; these are small (one pass over the physical grid).
#pragma once
#include <cuda_runtime.h>

namespace stfwi {

constexpr int POST_MAX_RADIUS = 64;   // Gaussian half-width limit: sigma <= 21

// one axis of the normalised Gaussian 'same' convolution with zero padding
// (the 2-D kernel of fwi/loss.py:17-30 is the outer product of this one, so
// the two passes give the same convolution)
__global__ void k_gauss_axis(int nz, int nx, int axis, int radius, const double *w, const double *in,
                             double *out)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz * nx) return;
    const int i = (int)(q / nx), j = (int)(q % nx);
    double s = 0.0;
    for (int k = -radius; k <= radius; ++k) {
        const int ii = axis == 0 ? i + k : i, jj = axis == 1 ? j + k : j;
        if (ii < 0 || ii >= nz || jj < 0 || jj >= nx) continue;
        s += w[k + radius] * in[(long long)ii * nx + jj];
    }
    out[q] = s;
}

__global__ void k_mul_planes(long long n, int planes, double *g, const double *a, const double *b)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    double f = 1.0;
    if (a) f *= a[q];
    if (b) f *= b[q];
    for (int p = 0; p < planes; ++p) g[(long long)p * n + q] *= f;
}

// fwi/projections.py:67-117 in FP64: Vp <= vp_cap (if given), Vs <= Vp / r
// with r = (1 + K_margin) 2/sqrt(3), then the floors on Vs and rho
__global__ void k_project_velocity(long long n, double *vs, double *vp, double *rho, double r, double vp_cap,
                                   int use_cap, double vs_floor, double rho_floor)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    double p = vp[q];
    if (use_cap) p = fmin(p, vp_cap);
    vp[q] = p;
    const double cap = p / r;
    vs[q] = fmax(fmin(vs[q], cap), vs_floor);
    rho[q] = fmax(rho[q], rho_floor);
}

// max over n values (one block; n is a physical grid, at most a few million)
__global__ void k_max_1block(long long n, const double *x, double *out)
{
    __shared__ double red[1024];
    double m = -INFINITY;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) m = fmax(m, x[q]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// crop the padded-grid energy rows [z0, z0 + nz_dom) x columns [pad, pad + nx_dom)
__global__ void k_crop(int nz_dom, int nx_dom, int nx, int z0, int pad, const double *Ws, double *out)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz_dom * nx_dom) return;
    const int i = (int)(q / nx_dom), j = (int)(q % nx_dom);
    out[q] = Ws[(long long)(i + z0) * nx + j + pad];
}

// fwi/illumination.py:45-47: H = 1 / (Ws + eps max Ws)
__global__ void k_illum_inverse(long long n, const double *Ws, const double *wmax, double eps, double *out)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    out[q] = 1.0 / (Ws[q] + eps * wmax[0]);
}

// fwi/preconditioning.py:119-138 on the padded grid: We = |sqrt(Ws) (asinh((l1
// - c)/y) - asinh((l0 - c)/y))|, y = max(|perp - perp0|, spacing)
__global__ void k_eprecond3_we(int nz, int nx, int z0, int pad, double dx, double dz, int horizontal,
                               double line_min, double line_max, double perp_pos, const double *Ws, double *We)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz * nx) return;
    const int i = (int)(q / nx), j = (int)(q % nx);
    const double cz = (i - z0) * dz, cx = (j - pad) * dx;
    const double c_perp = horizontal ? cz : cx, c_line = horizontal ? cx : cz, sp = horizontal ? dz : dx;
    const double y = fmax(fabs(c_perp - perp_pos), sp);
    const double w = sqrt(Ws[q]) * (asinh((line_max - c_line) / y) - asinh((line_min - c_line) / y));
    We[q] = fabs(w);
}

// We + eps max We, cropped, then 1 / We (the preconditioner before normalising)
__global__ void k_eprecond3_inv(int nz_dom, int nx_dom, int nx, int z0, int pad, const double *We,
                                const double *wmax, double eps, double *out)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz_dom * nx_dom) return;
    const int i = (int)(q / nx_dom), j = (int)(q % nx_dom);
    out[q] = 1.0 / (We[(long long)(i + z0) * nx + j + pad] + eps * wmax[0]);
}

__global__ void k_scale_by_inverse_max(long long n, double *x, const double *xmax)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    x[q] = x[q] / xmax[0];
}

}  // namespace stfwi
