// Table-driven, pair-arithmetic stencil kernels (sm_100a).
//
// Four kernels per time step pair: fwd_vel (U, V), fwd_str (the stresses,
// receivers, history), adj_a (P, Q) and adj_b (the strain adjoints and the
// gradient sums), each over every tile of every shot of the batch, with the
// tiling, TMA staging and per-term slice ranges of stencil_parts.cuh, and:
//  * tiles that touch an edge, a C-PML strip or the free surface evaluate
//    every stencil with per-column (x) and per-row (z) coefficient vectors
//    from shared memory, the reference's dropped high-order terms as zero
//    coefficients: one code path for all lanes of a warp instead of a masked
//    and an unmasked path side by side;
//  * interior tiles compute the z-stencils and the pointwise updates of a
//    thread's two columns as pairs (__ffma2_rn / __fmul2_rn: one paired FP32
//    instruction for both columns).
// A coefficient that is zero contributes fma(0, f, d) = d exactly, so the
// masked terms drop out as in the reference.
#pragma once
#include <type_traits>

#include "stencil_parts.cuh"

namespace stfwi {

// coefficient vectors of the masked stencils at index t of n (term k of the
// vector is c_k where the reference forms it, else 0)
template <int FD> __device__ __forceinline__ float cfk(int k) { return k <= FD / 2 ? cf<FD>(k) : 0.f; }

template <int FD, class Pred> __device__ __forceinline__ float4 cvec(Pred p)
{
    return make_float4(p(1) ? cfk<FD>(1) : 0.f, p(2) ? cfk<FD>(2) : 0.f, p(3) ? cfk<FD>(3) : 0.f,
                       p(4) ? cfk<FD>(4) : 0.f);
}
// D+ at t: f[t+k] - f[t-k+1]
template <int FD> __device__ __forceinline__ float4 cv_P(int t, int n)
{
    return cvec<FD>([&](int k) { return mP(t, k, n); });
}
// D- at t: f[t+k-1] - f[t-k]
template <int FD> __device__ __forceinline__ float4 cv_M(int t, int n)
{
    return cvec<FD>([&](int k) { return mM(t, k, n); });
}
// transposed D+ at t: + c_k f[t-k] (A) - c_k f[t+k-1] (B)
template <int FD> __device__ __forceinline__ float4 cv_tPA(int t, int n)
{
    return cvec<FD>([&](int k) { return mP(t - k, k, n); });
}
template <int FD> __device__ __forceinline__ float4 cv_tPB(int t, int n)
{
    return cvec<FD>([&](int k) { return mP(t + k - 1, k, n); });
}
// transposed D- at t below `lim`: + c_k f[t-k+1] (A) - c_k f[t+k] (B)
template <int FD> __device__ __forceinline__ float4 cv_tMA(int t, int n, int lim)
{
    return cvec<FD>([&](int k) { return mM(t - k + 1, k, n) && t - k + 1 < lim; });
}
template <int FD> __device__ __forceinline__ float4 cv_tMB(int t, int n, int lim)
{
    return cvec<FD>([&](int k) { return mM(t + k, k, n) && t + k < lim; });
}

__device__ __forceinline__ float v4k(const float4 &v, int k)
{
    return k == 1 ? v.x : k == 2 ? v.y : k == 3 ? v.z : v.w;
}
__device__ __forceinline__ float f2c(const float2 &v, int c) { return c == 0 ? v.x : v.y; }

// table-driven stencils on the x-neighbourhood a (column c of the pair)
template <int FD> __device__ __forceinline__ float a_dp_t(const float (&a)[10], int c, const float4 &v)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) d += v4k(v, k) * (a[4 + c + k] - a[5 + c - k]);
    return d;
}
template <int FD> __device__ __forceinline__ float a_dm_t(const float (&a)[10], int c, const float4 &v)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) d += v4k(v, k) * (a[3 + c + k] - a[4 + c - k]);
    return d;
}
template <int FD>
__device__ __forceinline__ float a_tdp_t(const float (&a)[10], int c, const float4 &A, const float4 &B)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        d += v4k(A, k) * a[4 + c - k];
        d -= v4k(B, k) * a[3 + c + k];
    }
    return d;
}
template <int FD>
__device__ __forceinline__ float a_tdm_t(const float (&a)[10], int c, const float4 &A, const float4 &B)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        d += v4k(A, k) * a[5 + c - k];
        d -= v4k(B, k) * a[4 + c + k];
    }
    return d;
}
// table-driven z stencils on the pair's window w (row r of the thread at w[r + K])
template <int FD, int W> __device__ __forceinline__ float w_dp_t(const float2 (&w)[W], int r, int c, const float4 &v)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) d += v4k(v, k) * (f2c(w[r + K + k], c) - f2c(w[r + K - k + 1], c));
    return d;
}
template <int FD, int W> __device__ __forceinline__ float w_dm_t(const float2 (&w)[W], int r, int c, const float4 &v)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) d += v4k(v, k) * (f2c(w[r + K + k - 1], c) - f2c(w[r + K - k], c));
    return d;
}
template <int FD, int W>
__device__ __forceinline__ float w_tdp_t(const float2 (&w)[W], int r, int c, const float4 &A, const float4 &B)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        d += v4k(A, k) * f2c(w[r + K - k], c);
        d -= v4k(B, k) * f2c(w[r + K + k - 1], c);
    }
    return d;
}
template <int FD, int W>
__device__ __forceinline__ float w_tdm_t(const float2 (&w)[W], int r, int c, const float4 &A, const float4 &B)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        d += v4k(A, k) * f2c(w[r + K - k + 1], c);
        d -= v4k(B, k) * f2c(w[r + K + k], c);
    }
    return d;
}

// paired FP32 arithmetic (both columns of a thread in one instruction)
__device__ __forceinline__ float2 dup2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, dup2(-1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// unmasked z stencils of the pair, paired
template <int FD, int W> __device__ __forceinline__ float2 w_dp2(const float2 (&w)[W], int r)
{
    constexpr int K = FD / 2;
    float2 d = mul2(dup2(cf<FD>(1)), sub2(w[r + K + 1], w[r + K]));
#pragma unroll
    for (int k = 2; k <= K; ++k) d = fma2(dup2(cf<FD>(k)), sub2(w[r + K + k], w[r + K - k + 1]), d);
    return d;
}
template <int FD, int W> __device__ __forceinline__ float2 w_dm2(const float2 (&w)[W], int r)
{
    constexpr int K = FD / 2;
    float2 d = mul2(dup2(cf<FD>(1)), sub2(w[r + K], w[r + K - 1]));
#pragma unroll
    for (int k = 2; k <= K; ++k) d = fma2(dup2(cf<FD>(k)), sub2(w[r + K + k - 1], w[r + K - k]), d);
    return d;
}
template <int FD, int W> __device__ __forceinline__ float2 w_tdp2(const float2 (&w)[W], int r)
{
    constexpr int K = FD / 2;
    float2 d = mul2(dup2(cf<FD>(1)), w[r + K - 1]);
    d = fma2(dup2(-cf<FD>(1)), w[r + K], d);
#pragma unroll
    for (int k = 2; k <= K; ++k) {
        d = fma2(dup2(cf<FD>(k)), w[r + K - k], d);
        d = fma2(dup2(-cf<FD>(k)), w[r + K + k - 1], d);
    }
    return d;
}
template <int FD, int W> __device__ __forceinline__ float2 w_tdm2(const float2 (&w)[W], int r)
{
    constexpr int K = FD / 2;
    float2 d = mul2(dup2(cf<FD>(1)), w[r + K]);
    d = fma2(dup2(-cf<FD>(1)), w[r + K + 1], d);
#pragma unroll
    for (int k = 2; k <= K; ++k) {
        d = fma2(dup2(cf<FD>(k)), w[r + K - k + 1], d);
        d = fma2(dup2(-cf<FD>(k)), w[r + K + k], d);
    }
    return d;
}

// z window of the pair as float2 rows
template <int W, int RPT>
__device__ __forceinline__ void zwin2p(float2 (&w)[W], const float *s, int ty, int tx)
{
#pragma unroll
    for (int m = 0; m < W; ++m) w[m] = *reinterpret_cast<const float2 *>(s + (ty * RPT + m) * SW4 + XO4 + 2 * tx);
}

// tile and shot group of this block, boundary tiles first: the blocks of
// every (boundary tile, shot group) pair are dispatched before the interior
// ones, so that the long blocks do not form the tail of the launch
__device__ __forceinline__ Ctx3 ctx5(const Geo &g, int spg, int tzh, int tiles_x, const int *order, int heavy)
{
    const int tiles = gridDim.x, groups = gridDim.y;
    const int b = blockIdx.y * tiles + blockIdx.x;
    int t = blockIdx.x, grp = blockIdx.y;
    if (order && heavy > 0 && heavy < tiles) {
        if (b < heavy * groups) {
            t = order[b % heavy];
            grp = b / heavy;
        } else {
            const int b2 = b - heavy * groups, light = tiles - heavy;
            t = order[heavy + b2 % light];
            grp = b2 / light;
        }
    }
    Ctx3 c;
    c.tile = t;
    c.j0 = (t % tiles_x) * TX4;
    c.i0 = (t / tiles_x) * tzh;
    c.s0 = (grp + g.goff) * spg;
    c.s1 = min(c.s0 + spg, g.nshot);
    return c;
}

// shared-memory plans of the table-driven kernels: the two-column layout
// followed by the coefficient tables (float4 per column of the tile for
// each x-stencil set, per row of the tile for each z-stencil set)
template <int FD, int R> struct L5 {
    using P4 = L4<FD, R>;
    static constexpr int CTA = 4 * (2 * TX4 + 2 * P4::A::TZH);                    // 2 x-sets, 2 z-sets
    static constexpr int CTB = 4 * (4 * TX4 + 4 * P4::A::TZH);                    // 4 x-sets, 4 z-sets (adj_a)
    static constexpr int CTBB = 4 * (4 * TX4 + 4 * P4::B::TZH);                   // 4 x-sets, 4 z-sets (adj_b)
    static constexpr int VEL = P4::VEL + CTA, STR = P4::STR + CTA;
    static constexpr int ADA = P4::ADA + CTB, ADB = P4::ADB + CTBB;
    static constexpr size_t bytes(int floats, int nbar) { return (size_t)floats * 4 + 8 * nbar; }
};

// ------------------------------------------------------------- forward: velocities

template <int FD, int RPT>
__global__ void __launch_bounds__(NTHR, STFWI_MINBLOCKS)
    st_fwd_vel(Geo g, Mat m, Shots sh, float *F, float *PX, float *PZ, int n, int spg, int tiles_x, int *status,
               const __grid_constant__ CUtensorMap tmS, const __grid_constant__ CUtensorMap tmUo)
{
    using T = G4<FD, RPT>;
    constexpr int K = T::K, SN = T::SN;
    constexpr int STG = L4<FD, RPT>::VEL_STAGE, OWNB = 2 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    // coefficient tables: x sets (D+ of sxx, D- of sxz), z sets (D- of sxz, D+ of szz)
    float4 *xt = reinterpret_cast<float4 *>(sm + L4<FD, RPT>::VEL);
    float4 *zt = xt + 2 * TX4;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L5<FD, RPT>::VEL);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx5(g, spg, T::TZH, tiles_x, g.tordA, g.theavyA);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 3 * SN * 4 + OWNB);
            tma_load_4d(sm + b * STG, &tmS, bar + b, c.j0 - XO4, c.i0 - K, F_EX, c.s0 + b);
            tma_load_4d(sm + b * STG + T::S3, &tmUo, bar + b, c.j0, c.i0, F_U, c.s0 + b);
        }
    }
    for (int t = tid; t < 2 * TX4; t += NTHR) {
        const int j = c.j0 + t % TX4;
        xt[t] = t < TX4 ? cv_P<FD>(j, g.nx) : cv_M<FD>(j, g.nx);
    }
    for (int t = tid; t < 2 * T::TZH; t += NTHR) {
        const int i = c.i0 + t % T::TZH;
        zt[t] = t < T::TZH ? cv_M<FD>(i, g.nz) : cv_P<FD>(i, g.nz);
    }
    __syncthreads();
    const int jb = c.j0 + 2 * tx;
    int xs[2];
    float bxv[2], axv[2], ikxv[2];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int j = jb + cc;
        xs[cc] = (j < g.nx) ? xstrip_index(g, j) : -1;
        bxv[cc] = xs[cc] >= 0 ? m.bx[j] : 0.f;
        axv[cc] = xs[cc] >= 0 ? m.ax[j] : 0.f;
        ikxv[cc] = xs[cc] >= 0 ? m.ikx[j] : 1.f;
    }
    // dt/dx B and dt/dz B of the thread's cells
    float2 bx2[RPT], bz2[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        float bc[2];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            bc[cc] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
        }
        bx2[r] = make_float2(g.dtdx * bc[0], g.dtdx * bc[1]);
        bz2[r] = make_float2(g.dtdz * bc[0], g.dtdz * bc[1]);
    }

    const bool plain = tile_plain4(g, c.i0, c.j0, T::TZH, T::M);
    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * STG;
        const float *own = S + T::S3;   // [U, V][TZH][TX4] of the tile's own cells
        float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, g.wait_polls))) {
            abort3(bar, it, nsh, status);
            return;
        }
        const float *sxx = S, *szz = S + SN, *sxz = S + 2 * SN;
        float2 wxz[T::W], wzz[T::W];
        zwin2p<T::W, RPT>(wxz, sxz, ty, tx);
        zwin2p<T::W, RPT>(wzz, szz, ty, tx);
        if (plain && !in_tile4(sh.sz[s], sh.sx[s], c.i0, c.j0, T::TZH)) {
            // interior tile without this shot's source: no guards, paired arithmetic
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                float ax[10], az[10];
                xrow(ax, sxx, q);
                xrow(az, sxz, q);
                const float2 u2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
                const float2 v2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
                const float2 dxx = make_float2(a_dp<FD, false>(ax, 0, 0, 0), a_dp<FD, false>(ax, 1, 0, 0));
                const float2 dxxz = make_float2(a_dm<FD, false>(az, 0, 0, 0), a_dm<FD, false>(az, 1, 0, 0));
                const float2 un = fma2(bz2[r], w_dm2<FD>(wxz, r), fma2(bx2[r], dxx, u2));
                const float2 vn = fma2(bz2[r], w_dp2<FD>(wzz, r), fma2(bx2[r], dxxz, v2));
                const long long o = (long long)i * g.P + jb;
                *reinterpret_cast<float2 *>(U + o) = un;
                *reinterpret_cast<float2 *>(V + o) = vn;
            }
        } else {
            const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
            float *pSXX = px_ptr(g, PX, s, PX_SXX), *pSXZx = px_ptr(g, PX, s, PX_SXZ);
            float *pSXZz = pz_ptr(g, PZ, s, PZ_SXZ), *pSZZ = pz_ptr(g, PZ, s, PZ_SZZ);
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                float ax[10], az[10];
                xrow(ax, sxx, q);
                xrow(az, sxz, q);
                const int zs = zstrip_index(g, i);
                // this row's C-PML memories, requested before the stencils
                float pxo[2][2] = {{0.f, 0.f}, {0.f, 0.f}}, pzo[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
                float zb = 0.f, za = 0.f, zik = 1.f;
                if (i < g.nz - 1) {
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        const int j = jb + cc;
                        if (j < 1 || j >= g.nx - 1) continue;
                        if (xs[cc] >= 0) {
                            const int px = i * g.xs_n + xs[cc];
                            pxo[cc][0] = pSXX[px];
                            pxo[cc][1] = pSXZx[px];
                        }
                        if (zs >= 0) {
                            const int pz = zs * g.P + j;
                            pzo[cc][0] = pSXZz[pz];
                            pzo[cc][1] = pSZZ[pz];
                        }
                    }
                    if (zs >= 0) { zb = m.bz[i]; za = m.az[i]; zik = m.ikz[i]; }
                }
                const float2 u2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
                const float2 v2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
                const float u[2] = {u2.x, u2.y}, v[2] = {v2.x, v2.y};
                const float4 czm = zt[ty * RPT + r], czp = zt[T::TZH + ty * RPT + r];
                float un[2], vn[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc;
                    un[cc] = u[cc];
                    vn[cc] = v[cc];
                    if (i >= g.nz - 1 || j < 1 || j >= g.nx - 1) continue;
                    float dxx = a_dp_t<FD>(ax, cc, xt[2 * tx + cc]);
                    float dxxz = a_dm_t<FD>(az, cc, xt[TX4 + 2 * tx + cc]);
                    float dzxz = (g.fs && i == 0) ? 2.f * cf<FD>(1) * f2c(wxz[r + K], cc) : w_dm_t<FD>(wxz, r, cc, czm);
                    float dzz = w_dp_t<FD>(wzz, r, cc, czp);
                    if (xs[cc] >= 0) {
                        const int px = i * g.xs_n + xs[cc];
                        dxx = pml_fwd_pre(dxx, bxv[cc], axv[cc], ikxv[cc], pxo[cc][0], pSXX + px);
                        dxxz = pml_fwd_pre(dxxz, bxv[cc], axv[cc], ikxv[cc], pxo[cc][1], pSXZx + px);
                    }
                    if (zs >= 0) {
                        const int pz = zs * g.P + j;
                        dzxz = pml_fwd_pre(dzxz, zb, za, zik, pzo[cc][0], pSXZz + pz);
                        dzz = pml_fwd_pre(dzz, zb, za, zik, pzo[cc][1], pSZZ + pz);
                    }
                    const float bxc = cc ? bx2[r].y : bx2[r].x, bzc = cc ? bz2[r].y : bz2[r].x;
                    un[cc] = u[cc] + bxc * dxx + bzc * dzxz;
                    float vv = v[cc] + bxc * dxxz + bzc * dzz;
                    if (stype == 0 && i == ssz && j == ssx) vv = vv + sh.fcoef[s] * sh.wav[(long long)s * g.nt + n];
                    vn[cc] = vv;
                }
                // cells outside the update region keep their value (column 0, nx-1, row nz-1)
                if (i < g.nz - 1 && jb < g.nx) {
                    const long long o = (long long)i * g.P + jb;
                    if (jb + 1 < g.nx) {
                        *reinterpret_cast<float2 *>(U + o) = make_float2(un[0], un[1]);
                        *reinterpret_cast<float2 *>(V + o) = make_float2(vn[0], vn[1]);
                    } else {
                        U[o] = un[0];
                        V[o] = vn[0];
                    }
                }
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4 + OWNB);
            tma_load_4d(S, &tmS, bar + (it & 1), c.j0 - XO4, c.i0 - K, F_EX, s + 2);
            tma_load_4d(S + T::S3, &tmUo, bar + (it & 1), c.j0, c.i0, F_U, s + 2);
        }
    }
}

// ------------------------------------------------------------- forward: stresses

template <int FD, int RPT, bool ENERGY>
__global__ void __launch_bounds__(NTHR, STFWI_MINBLOCKS)
    st_fwd_str(Geo g, Mat m, Shots sh, Recv rv, float *F, float *PX, float *PZ, int n, int spg, int tiles_x,
               FwdOut out, const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmSo)
{
    using T = G4<FD, RPT>;
    constexpr int K = T::K, SN = T::SN;
    constexpr int STG = L4<FD, RPT>::STR_STAGE, OWNB = 3 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    // coefficient tables: x sets (D- of U, D+ of V), z sets (D- of V, D+ of U)
    float4 *xt = reinterpret_cast<float4 *>(sm + L4<FD, RPT>::STR);
    float4 *zt = xt + 2 * TX4;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L5<FD, RPT>::STR);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx5(g, spg, T::TZH, tiles_x, g.tordA, g.theavyA);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 2 * SN * 4 + OWNB);
            tma_load_4d(sm + b * STG, &tmV, bar + b, c.j0 - XO4, c.i0 - K, F_U, c.s0 + b);
            tma_load_4d(sm + b * STG + T::S2, &tmSo, bar + b, c.j0, c.i0, F_EX, c.s0 + b);
        }
    }
    for (int t = tid; t < 2 * TX4; t += NTHR) {
        const int j = c.j0 + t % TX4;
        xt[t] = t < TX4 ? cv_M<FD>(j, g.nx) : cv_P<FD>(j, g.nx);
    }
    for (int t = tid; t < 2 * T::TZH; t += NTHR) {
        const int i = c.i0 + t % T::TZH;
        zt[t] = t < T::TZH ? cv_M<FD>(i, g.nz) : cv_P<FD>(i, g.nz);
    }
    __syncthreads();
    const int jb = c.j0 + 2 * tx;
    int xs[2];
    float bxv[2], axv[2], ikxv[2], Lr0[2];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int j = jb + cc;
        xs[cc] = (j < g.nx) ? xstrip_index(g, j) : -1;
        bxv[cc] = xs[cc] >= 0 ? m.bx[j] : 0.f;
        axv[cc] = xs[cc] >= 0 ? m.ax[j] : 0.f;
        ikxv[cc] = xs[cc] >= 0 ? m.ikx[j] : 1.f;
        Lr0[cc] = (g.fs && j < g.nx) ? m.Lr[j] : 0.f;
    }
    float2 ml2m[RPT], ml[RPT], mm2[RPT];
    constexpr int RG = ENERGY ? RPT : 1;
    double eacc[RG][2];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        float a[2], b[2], d[2];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            a[cc] = ok ? m.L2M[o] : 0.f;
            b[cc] = ok ? m.L[o] : 0.f;
            d[cc] = ok ? 2.f * m.M[o] : 0.f;
            if (r < RG) eacc[r][cc] = 0.0;
        }
        ml2m[r] = make_float2(a[0], a[1]);
        ml[r] = make_float2(b[0], b[1]);
        mm2[r] = make_float2(d[0], d[1]);
    }
    const float2 dtdx2 = dup2(g.dtdx), dtdz2 = dup2(g.dtdz);
    // history rows as float pairs when every pair starts on 8 bytes
    const bool hist2 = ((g.pad | g.nx_dom) & 1) == 0;

    const bool plain = tile_plain4(g, c.i0, c.j0, T::TZH, T::M);
    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * STG;
        const float *own = S + T::S2;   // [sxx, szz, sxz][TZH][TX4] of the tile's own cells
        float *sxx = F + ((long long)s * F_N + F_EX) * g.fstride;
        float *szz = F + ((long long)s * F_N + F_EZ) * g.fstride;
        float *sxz = F + ((long long)s * F_N + F_ES) * g.fstride;
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, g.wait_polls))) {
            abort3(bar, it, nsh, out.status);
            return;
        }
        const float *sU = S, *sV = S + SN;
        float2 wU[T::W], wV[T::W];
        zwin2p<T::W, RPT>(wU, sU, ty, tx);
        zwin2p<T::W, RPT>(wV, sV, ty, tx);
        float *snap_s = out.snap ? out.snap + ((long long)s * out.slots + out.slot) * g.snf * g.nd : nullptr;
        if (plain && !in_tile4(sh.sz[s], sh.sx[s], c.i0, c.j0, T::TZH)) {
            // interior tile without this shot's source: no guards, paired arithmetic
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                const int qo = (ty * RPT + r) * TX4 + 2 * tx;
                const float2 e1 = *reinterpret_cast<const float2 *>(own + qo);
                const float2 e2 = *reinterpret_cast<const float2 *>(own + T::TZH * TX4 + qo);
                const float2 e3 = *reinterpret_cast<const float2 *>(own + 2 * T::TZH * TX4 + qo);
                float au[10], av[10];
                xrow(au, sU, q);
                xrow(av, sV, q);
                const float2 dxu = make_float2(a_dm<FD, false>(au, 0, 0, 0), a_dm<FD, false>(au, 1, 0, 0));
                const float2 dxv = make_float2(a_dp<FD, false>(av, 0, 0, 0), a_dp<FD, false>(av, 1, 0, 0));
                const float2 dex = mul2(dtdx2, dxu), dez = mul2(dtdz2, w_dm2<FD>(wV, r));
                const float2 des = mul2(dup2(0.5f), fma2(dtdx2, dxv, mul2(dtdz2, w_dp2<FD>(wU, r))));
                const float2 axx = fma2(ml[r], dez, fma2(ml2m[r], dex, e1));
                const float2 azz = fma2(ml2m[r], dez, fma2(ml[r], dex, e2));
                const float2 axz = fma2(mm2[r], des, e3);
                if (snap_s) {
                    float *sp = snap_s + (long long)(i - g.z0) * g.nx_dom + (jb - g.pad);
                    if (hist2) {
                        __stcs(reinterpret_cast<float2 *>(sp), axx);
                        __stcs(reinterpret_cast<float2 *>(sp + g.nd), azz);
                        __stcs(reinterpret_cast<float2 *>(sp + 2 * g.nd), axz);
                        if (g.snf == 5) {   // velocities of this step (density gradient)
                            __stcs(reinterpret_cast<float2 *>(sp + 3 * g.nd), make_float2(au[4], au[5]));
                            __stcs(reinterpret_cast<float2 *>(sp + 4 * g.nd), make_float2(av[4], av[5]));
                        }
                    } else {
                        __stcs(sp, axx.x); __stcs(sp + 1, axx.y);
                        __stcs(sp + g.nd, azz.x); __stcs(sp + g.nd + 1, azz.y);
                        __stcs(sp + 2 * g.nd, axz.x); __stcs(sp + 2 * g.nd + 1, axz.y);
                        if (g.snf == 5) {
                            __stcs(sp + 3 * g.nd, au[4]); __stcs(sp + 3 * g.nd + 1, au[5]);
                            __stcs(sp + 4 * g.nd, av[4]); __stcs(sp + 4 * g.nd + 1, av[5]);
                        }
                    }
                }
                if (ENERGY) {
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        float f;
                        if (out.energy_comp < 2) {
                            f = out.energy_comp == 0 ? au[4 + cc] : av[4 + cc];
                        } else {
                            float ex, ez, es;
                            strains_of(f2c(axx, cc), f2c(azz, cc), f2c(axz, cc), f2c(ml2m[r], cc), f2c(ml[r], cc),
                                       0.5f * f2c(mm2[r], cc), ex, ez, es);
                            f = out.energy_comp == 2 ? ex : ez;
                        }
                        eacc[r % RG][cc] += (double)f * (double)f;
                    }
                }
                const long long o = (long long)i * g.P + jb;
                *reinterpret_cast<float2 *>(sxx + o) = axx;
                *reinterpret_cast<float2 *>(szz + o) = azz;
                *reinterpret_cast<float2 *>(sxz + o) = axz;
            }
        } else {
            const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
            float *pDXU = px_ptr(g, PX, s, PX_DXU), *pDXV = px_ptr(g, PX, s, PX_DXV);
            float *pDZV = pz_ptr(g, PZ, s, PZ_DZV), *pDZU = pz_ptr(g, PZ, s, PZ_DZU);
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                if (i >= g.nz) continue;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                const int qo = (ty * RPT + r) * TX4 + 2 * tx;
                const float2 a2 = *reinterpret_cast<const float2 *>(own + qo);
                const float2 b2 = *reinterpret_cast<const float2 *>(own + T::TZH * TX4 + qo);
                const float2 d2 = *reinterpret_cast<const float2 *>(own + 2 * T::TZH * TX4 + qo);
                const float e1[2] = {a2.x, a2.y}, e2[2] = {b2.x, b2.y}, e3[2] = {d2.x, d2.y};
                float au[10], av[10];
                xrow(au, sU, q);
                xrow(av, sV, q);
                const int zs = zstrip_index(g, i);
                // this row's C-PML memories, requested before the stencils
                float pxo[2][2] = {{0.f, 0.f}, {0.f, 0.f}}, pzo[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
                float zb = 0.f, za = 0.f, zik = 1.f;
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc;
                    if (j >= g.nx) continue;
                    if (xs[cc] >= 0) {
                        const int px = i * g.xs_n + xs[cc];
                        if (j >= 1) pxo[cc][0] = pDXU[px];
                        if (i < g.nz - 1) pxo[cc][1] = pDXV[px];
                    }
                    if (zs >= 0) {
                        const int pz = zs * g.P + j;
                        if (j < g.nx - 1) pzo[cc][0] = pDZV[pz];
                        if (j >= 1) pzo[cc][1] = pDZU[pz];
                    }
                }
                if (zs >= 0) { zb = m.bz[i]; za = m.az[i]; zik = m.ikz[i]; }
                const float4 czm = zt[ty * RPT + r], czp = zt[T::TZH + ty * RPT + r];
                float nxx[2], nzz[2], nxz[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc;
                    nxx[cc] = e1[cc]; nzz[cc] = e2[cc]; nxz[cc] = e3[cc];
                    if (j >= g.nx) continue;
                    float dxu = a_dm_t<FD>(au, cc, xt[2 * tx + cc]);
                    float dxv = a_dp_t<FD>(av, cc, xt[TX4 + 2 * tx + cc]);
                    float dzv = w_dm_t<FD>(wV, r, cc, czm);
                    float dzu = w_dp_t<FD>(wU, r, cc, czp);
                    const int px = i * g.xs_n + xs[cc], pz = zs * g.P + j;
                    if (j >= 1 && xs[cc] >= 0)
                        dxu = pml_fwd_pre(dxu, bxv[cc], axv[cc], ikxv[cc], pxo[cc][0], pDXU + px);
                    if (j < g.nx - 1) {
                        if (g.fs && i == 0) dzv = Lr0[cc] * dxu * g.dzdx;
                        if (zs >= 0) dzv = pml_fwd_pre(dzv, zb, za, zik, pzo[cc][0], pDZV + pz);
                    } else {
                        dzv = 0.f;
                    }
                    if (j >= 1) {
                        if (zs >= 0) dzu = pml_fwd_pre(dzu, zb, za, zik, pzo[cc][1], pDZU + pz);
                    } else {
                        dzu = 0.f;
                    }
                    if (i < g.nz - 1) {
                        if (xs[cc] >= 0) dxv = pml_fwd_pre(dxv, bxv[cc], axv[cc], ikxv[cc], pxo[cc][1], pDXV + px);
                    } else {
                        dxv = 0.f;
                    }
                    const float dex = j >= 1 ? g.dtdx * dxu : 0.f;
                    const float dez = g.dtdz * dzv;
                    const float des = (i < g.nz - 1 && j < g.nx - 1) ? 0.5f * (g.dtdz * dzu + g.dtdx * dxv) : 0.f;
                    const float l2m = f2c(ml2m[r], cc), l = f2c(ml[r], cc);
                    float axx = e1[cc] + l2m * dex + l * dez;
                    float azz = e2[cc] + l * dex + l2m * dez;
                    const float axz = e3[cc] + f2c(mm2[r], cc) * des;
                    if (stype == 1 && i == ssz && j == ssx) {
                        const float stm = sh.wav[(long long)s * g.nt + n] * g.dt / sh.mcoef[s];
                        axx = axx + (l2m + l) * stm;
                        azz = azz + (l + l2m) * stm;
                    }
                    nxx[cc] = axx; nzz[cc] = azz; nxz[cc] = axz;
                    const int pi = i - g.z0, pj = j - g.pad;
                    const bool phys = pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom;
                    if (snap_s && phys) {
                        float *sp = snap_s + (long long)pi * g.nx_dom + pj;
                        __stcs(sp, axx);
                        __stcs(sp + g.nd, azz);
                        __stcs(sp + 2 * g.nd, axz);
                        if (g.snf == 5) {   // velocities of this step (density gradient)
                            __stcs(sp + 3 * g.nd, au[4 + cc]);
                            __stcs(sp + 4 * g.nd, av[4 + cc]);
                        }
                    }
                    if (out.row0 && g.fs && i == 0 && pj >= 0 && pj < g.nx_dom)
                        out.row0[((long long)s * out.slots + out.slot_row0) * g.nx_dom + pj] = dxu;
                    if (ENERGY) {
                        float f;
                        if (out.energy_comp < 2) {
                            f = out.energy_comp == 0 ? au[4 + cc] : av[4 + cc];
                        } else {
                            float ex, ez, es;
                            strains_of(axx, azz, axz, l2m, l, 0.5f * f2c(mm2[r], cc), ex, ez, es);
                            f = out.energy_comp == 2 ? ex : ez;
                        }
                        eacc[r % RG][cc] += (double)f * (double)f;
                    }
                }
                if (jb < g.nx) {
                    const long long o = (long long)i * g.P + jb;
                    if (jb + 1 < g.nx) {
                        *reinterpret_cast<float2 *>(sxx + o) = make_float2(nxx[0], nxx[1]);
                        *reinterpret_cast<float2 *>(szz + o) = make_float2(nzz[0], nzz[1]);
                        *reinterpret_cast<float2 *>(sxz + o) = make_float2(nxz[0], nxz[1]);
                    } else {
                        sxx[o] = nxx[0]; szz[o] = nzz[0]; sxz[o] = nxz[0];
                    }
                }
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4 + OWNB);
            tma_load_4d(S, &tmV, bar + (it & 1), c.j0 - XO4, c.i0 - K, F_U, s + 2);
            tma_load_4d(S + T::S2, &tmSo, bar + (it & 1), c.j0, c.i0, F_EX, s + 2);
        }
        const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
        const float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        const float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        for (int qq = r0 + tid; qq < r1; qq += NTHR) {
            const int rid = rv.tile_rec[qq];
            const long long o = (long long)rv.rz[rid] * g.P + rv.rx[rid];
            float ex, ez, es;
            strains_of(sxx[o], szz[o], sxz[o], m.L2M[o], m.L[o], m.M[o], ex, ez, es);
            const float v0 = U[o], v1 = V[o];
            float *dst = out.rec + (long long)s * 4 * g.nt * g.nrec + (long long)n * g.nrec + rid;
            dst[0] = v0;
            dst[(long long)g.nt * g.nrec] = v1;
            dst[2LL * g.nt * g.nrec] = ex;
            dst[3LL * g.nt * g.nrec] = ez;
            if (!(isfinite(v0) && isfinite(v1) && isfinite(ex) && isfinite(ez))) atomicOr(out.status, 1);
        }
    }
    if (ENERGY) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int i = c.i0 + ty * RPT + r, j = jb + cc;
                if (i < g.nz && j < g.nx) atomicAdd(out.energy + (long long)i * g.nx + j, eacc[r][cc]);
            }
    }
}

// ------------------------------------------------------------- adjoint: P = B U_a, Q = B V_a

template <int FD, int RPT>
__global__ void __launch_bounds__(NTHR, STFWI_MINBLOCKS)
    st_adj_a(Geo g, Mat m, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x, AdjIn in,
             int *status, const __grid_constant__ CUtensorMap tmE, const __grid_constant__ CUtensorMap tmPQo)
{
    using T = G4<FD, RPT>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH;
    constexpr int STG = L4<FD, RPT>::ADA_STAGE, OWNB = 2 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    constexpr int NCC = (SW4 + TX - 1) / TX;
    float *aDxV = sm + 2 * STG;
    float *tab = aDxV + T::S1;
    // coefficient tables: x sets (A, B of the transposed D- of exx_a, A, B of
    // the transposed D+ of exz_a), z sets (A, B of the transposed D+ of exz_a,
    // A, B of the transposed D- of ezz_a)
    float4 *xt = reinterpret_cast<float4 *>(sm + L4<FD, RPT>::ADA);
    float4 *zt = xt + 4 * TX4;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L5<FD, RPT>::ADA);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx5(g, spg, T::TZH, tiles_x, g.tordA, g.theavyA);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 3 * SN * 4 + OWNB);
            tma_load_4d(sm + b * STG, &tmE, bar + b, c.j0 - XO4, c.i0 - K, F_EX, c.s0 + b);
            tma_load_4d(sm + b * STG + T::S3, &tmPQo, bar + b, c.j0, c.i0, F_U, c.s0 + b);
        }
    }
    __syncthreads();
    const bool fix = box_special4(g, c.i0, c.j0, T::TZH, K);
    const bool lean = !fix && tile_plain4(g, c.i0, c.j0, T::TZH, T::M);
    if (fix) pml_table4<SH>(g, m, c.i0 - K, c.j0, tab, tid);   // ordered before use by the first wait's barrier
    for (int t = tid; t < 4 * TX4; t += NTHR) {
        const int j = c.j0 + t % TX4, set = t / TX4;
        xt[t] = set == 0 ? cv_tMA<FD>(j, g.nx, g.nx) : set == 1 ? cv_tMB<FD>(j, g.nx, g.nx)
              : set == 2 ? cv_tPA<FD>(j, g.nx) : cv_tPB<FD>(j, g.nx);
    }
    for (int t = tid; t < 4 * T::TZH; t += NTHR) {
        const int i = c.i0 + t % T::TZH, set = t / T::TZH;
        zt[t] = set == 0 ? cv_tPA<FD>(i, g.nz) : set == 1 ? cv_tPB<FD>(i, g.nz)
              : set == 2 ? cv_tMA<FD>(i, g.nz, g.nz) : cv_tMB<FD>(i, g.nz, g.nz);
    }
    const int rd = in.ping, wr = 1 - in.ping;
    const int jb = c.j0 + 2 * tx;
    const float hdtdz = 0.5f * g.dtdz, hdtdx = 0.5f * g.dtdx;
    float2 Bc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        float bc[2];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            bc[cc] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
        }
        Bc[r] = make_float2(bc[0], bc[1]);
    }
    double glr[2] = {0.0, 0.0};

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * STG;
        const float *own = S + T::S3;   // [P, Q][TZH][TX4] of the tile's own cells
        float *Pp = A + ((long long)s * F_N + F_U) * g.fstride;
        float *Qp = A + ((long long)s * F_N + F_V) * g.fstride;
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, g.wait_polls))) {
            abort3(bar, it, nsh, status);
            return;
        }
        if (fix) {
            const float *pDzU = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZU);
            const float *pDzV = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZV);
            const float *pDxU = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXU);
            const float *pDxV = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXV);
            float *wDzU = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZU);
            float *wDzV = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZV);
            float *wDxU = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXU);
            float *wDxV = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXV);
            // box columns [0, xl) and [xr, SW4) lie in the x-strips
            const int xl = g.pad - (c.j0 - XO4), xr = g.nx - g.pad - (c.j0 - XO4);
            const float *tbx = tab, *tax = tab + SW4, *tikx = tab + 2 * SW4, *tlr = tab + 3 * SW4;
            const int *txs = reinterpret_cast<const int *>(tab + 4 * SW4);
            const float *tbz = tab + 5 * SW4, *taz = tbz + SH, *tikz = taz + SH;
            const int *tzs = reinterpret_cast<const int *>(tikz + SH);
            for (int rr = ty; rr < SH; rr += NWARP) {
                const int i = c.i0 - K + rr;
                const int zs = tzs[rr];
                const bool rowsp = zs >= 0 || (g.fs && i == 0);
                const bool own_row = rr >= K && rr < K + T::TZH;
                // the C-PML memories of this row's cells, all requested before any is used
                float ps[NCC][4];
#pragma unroll
                for (int b = 0; b < NCC; ++b) {
                    const int cc = tx + b * TX, jj = c.j0 - XO4 + cc;
                    ps[b][0] = ps[b][1] = ps[b][2] = ps[b][3] = 0.f;
                    if (cc >= SW4) continue;
                    if (zs >= 0 && jj >= 0 && jj < g.nx) {
                        const long long pz = (long long)zs * g.P + jj;
                        ps[b][0] = pDzV[pz];
                        ps[b][1] = pDzU[pz];
                    }
                    const int xs = txs[cc];
                    if (xs >= 0 && i >= 0 && i < g.nz) {
                        const long long px = (long long)i * g.xs_n + xs;
                        ps[b][2] = pDxU[px];
                        ps[b][3] = pDxV[px];
                    }
                }
#pragma unroll
                for (int b = 0; b < NCC; ++b) {
                    const int cc = tx + b * TX;
                    if (cc >= SW4) continue;
                    const int jj = c.j0 - XO4 + cc, q = rr * SW4 + cc;
                    if (!rowsp && cc >= xl && cc < xr) {
                        // outside the strips and off the free-surface row the
                        // transform is the identity
                        aDxV[q] = S[2 * SN + q];
                        continue;
                    }
                    const float ea = S[q], za = S[SN + q], sa = S[2 * SN + q];
                    float vDxU = ea, vDzV = za, vDzU = sa, vDxV = sa;
                    if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                        const bool own = own_row && cc >= XO4 && cc < XO4 + TX4;
                        const int xs = txs[cc];
                        const long long pz = (long long)zs * g.P + jj, px = (long long)i * g.xs_n + xs;
                        if (zs >= 0) vDzV = pml_adj4(za, tbz[rr], taz[rr], tikz[rr], ps[b][0], wDzV + pz, own);
                        float din = (jj >= 1) ? ea : 0.f;
                        if (g.fs && i == 0 && jj < g.nx - 1) din = tlr[cc] * vDzV + din;
                        vDxU = din;
                        if (xs >= 0) vDxU = pml_adj4(din, tbx[cc], tax[cc], tikx[cc], ps[b][2], wDxU + px, own);
                        const float h = (i < g.nz - 1 && jj < g.nx - 1) ? sa : 0.f;
                        vDzU = h;
                        vDxV = h;
                        if (zs >= 0) vDzU = pml_adj4(h, tbz[rr], taz[rr], tikz[rr], ps[b][1], wDzU + pz, own);
                        if (xs >= 0) vDxV = pml_adj4(h, tbx[cc], tax[cc], tikx[cc], ps[b][3], wDxV + px, own);
                    }
                    S[q] = vDxU; S[SN + q] = vDzV; S[2 * SN + q] = vDzU; aDxV[q] = vDxV;
                }
            }
            __syncthreads();
        }
        const float *aDxU = S, *aDzV = S + SN, *aDzU = S + 2 * SN;
        const float *aXV = fix ? aDxV : aDzU;
        float2 wzu[T::W], wzv[T::W];
        zwin2p<T::W, RPT>(wzu, aDzU, ty, tx);
        zwin2p<T::W, RPT>(wzv, aDzV, ty, tx);
        if (lean) {
            // interior tile whose box needs no fix-up: no guards, paired arithmetic
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                float ad[10], av[10];
                xrow(ad, aDxU, q);
                xrow(av, aXV, q);
                const float2 p2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
                const float2 q2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
                const float2 tdm = make_float2(a_tdm<FD, false>(ad, 0, 0, 0, 0), a_tdm<FD, false>(ad, 1, 0, 0, 0));
                const float2 tdp = make_float2(a_tdp<FD, false>(av, 0, 0, 0), a_tdp<FD, false>(av, 1, 0, 0));
                const float2 gu = fma2(dup2(g.dtdx), tdm, mul2(dup2(hdtdz), w_tdp2<FD>(wzu, r)));
                const float2 gv = fma2(dup2(g.dtdz), w_tdm2<FD>(wzv, r), mul2(dup2(hdtdx), tdp));
                const long long o = (long long)i * g.P + jb;
                *reinterpret_cast<float2 *>(Pp + o) = fma2(Bc[r], gu, p2);
                *reinterpret_cast<float2 *>(Qp + o) = fma2(Bc[r], gv, q2);
            }
        } else {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = c.i0 + ty * RPT + r;
                if (i >= g.nz) continue;
                const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
                float ad[10], av[10];
                xrow(ad, aDxU, q);
                xrow(av, aXV, q);
                const float2 p2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
                const float2 q2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
                const float pr[2] = {p2.x, p2.y}, qr[2] = {q2.x, q2.y};
                const int zr = ty * RPT + r;
                const float4 zpa = zt[zr], zpb = zt[T::TZH + zr], zma = zt[2 * T::TZH + zr], zmb = zt[3 * T::TZH + zr];
                float np[2], nq[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc;
                    np[cc] = pr[cc]; nq[cc] = qr[cc];
                    if (j >= g.nx) continue;
                    const int col = 2 * tx + cc;
                    const float gu = (j >= 1 ? hdtdz * w_tdp_t<FD>(wzu, r, cc, zpa, zpb) : 0.f)
                                   + g.dtdx * a_tdm_t<FD>(ad, cc, xt[col], xt[TX4 + col]);
                    const float gv = (i < g.nz - 1 ? hdtdx * a_tdp_t<FD>(av, cc, xt[2 * TX4 + col], xt[3 * TX4 + col]) : 0.f)
                                   + (j < g.nx - 1 ? g.dtdz * w_tdm_t<FD>(wzv, r, cc, zma, zmb) : 0.f);
                    np[cc] = pr[cc] + f2c(Bc[r], cc) * gu;
                    nq[cc] = qr[cc] + f2c(Bc[r], cc) * gv;
                    if (in.want_exact && g.fs && i == 0) {
                        const int pj = j - g.pad;
                        if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) {
                            const float du = in.row0[((long long)s * in.slots + in.slot) * g.nx_dom + pj];
                            glr[cc] += (double)(g.dtdz * f2c(wzv[r + K], cc)) * (double)du * (double)g.dzdx;
                        }
                    }
                }
                if (jb < g.nx) {
                    const long long o = (long long)i * g.P + jb;
                    if (jb + 1 < g.nx) {
                        *reinterpret_cast<float2 *>(Pp + o) = make_float2(np[0], np[1]);
                        *reinterpret_cast<float2 *>(Qp + o) = make_float2(nq[0], nq[1]);
                    } else {
                        Pp[o] = np[0];
                        Qp[o] = nq[0];
                    }
                }
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4 + OWNB);
            tma_load_4d(S, &tmE, bar + (it & 1), c.j0 - XO4, c.i0 - K, F_EX, s + 2);
            tma_load_4d(S + T::S3, &tmPQo, bar + (it & 1), c.j0, c.i0, F_U, s + 2);
        }
        const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
        for (int qq = r0 + tid; qq < r1; qq += NTHR) {
            const int rid = rv.tile_rec[qq];
            const long long o = (long long)rv.rz[rid] * g.P + rv.rx[rid];
            const float *src = in.rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)n * g.nrec + rid;
            const float b = m.B[o];
            atomicAdd(Pp + o, b * src[0]);
            atomicAdd(Qp + o, b * src[(long long)g.nt * g.nrec]);
        }
    }
    if (in.want_exact && g.fs && c.i0 == 0 && ty == 0) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int j = jb + cc, pj = j - g.pad;
            if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) in.accLr[(long long)(c.s0 / spg) * g.nx_dom + pj] += glr[cc];
        }
    }
}

// ------------------------------------------------------------- adjoint: strains + gradient

template <int FD, int RPT, bool EXACT, bool IMG, bool RHO>
__global__ void __launch_bounds__(NTHR, STFWI_MINBLOCKS)
    st_adj_b(Geo g, Mat m, Shots sh, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x,
             AdjOut o, int *status, const __grid_constant__ CUtensorMap tmPQ,
             const __grid_constant__ CUtensorMap tmEo, const __grid_constant__ CUtensorMap tmH)
{
    using T = G4<FD, RPT>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH;
    constexpr int STG = L4<FD, RPT>::ADB_STAGE, OWNB = 3 * T::TZH * TX4 * 4, PL = T::TZH * TX4;
    extern __shared__ __align__(128) float sm[];
    constexpr int NCC = (SW4 + TX - 1) / TX;
    float *aZXZ = sm + 2 * STG, *aXXZ = aZXZ + T::S1;
    float *tab = aXXZ + T::S1;
    // coefficient tables: x sets (A, B of the transposed D+ of P, A, B of
    // the transposed D- of Q), z sets (A, B of the transposed D+ of Q, A, B
    // of the transposed D- of P)
    float4 *xt = reinterpret_cast<float4 *>(sm + L4<FD, RPT>::ADB);
    float4 *zt = xt + 4 * TX4;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L5<FD, RPT>::ADB);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx5(g, spg, T::TZH, tiles_x, g.tordB, g.theavyB);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    // the carry-in stresses of the exact gradient: one more box per shot from
    // the history [shot][slot * snf + field][nz_dom][nx_dom] at the tile's
    // physical coordinates (cells outside the physical domain arrive as 0)
    const bool htma = EXACT && o.hist_tma && o.slot_in >= 0;
    const int hbytes = htma ? OWNB : 0;
    const int hx = c.j0 - g.pad, hy = c.i0 - g.z0, hz = o.slot_in * g.snf;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 2 * SN * 4 + OWNB + hbytes);
            tma_load_4d(sm + b * STG, &tmPQ, bar + b, c.j0 - XO4, c.i0 - K, F_U, c.s0 + b);
            tma_load_4d(sm + b * STG + T::S2, &tmEo, bar + b, c.j0, c.i0, F_EX, c.s0 + b);
            if (htma)
                tma_load_4d_hint(sm + b * STG + T::S2 + L4<FD, RPT>::OWNB3, &tmH, bar + b, hx, hy, hz, c.s0 + b,
                                 l2_evict_first());
        }
    }
    __syncthreads();
    const bool fix = box_strips4(g, c.i0, c.j0, T::TZH, K);
    const bool lean = !fix && tile_plain4(g, c.i0, c.j0, T::TZH, T::M);
    if (fix) pml_table4<SH>(g, m, c.i0 - K, c.j0, tab, tid);   // ordered before use by the first wait's barrier
    for (int t = tid; t < 4 * TX4; t += NTHR) {
        const int j = c.j0 + t % TX4, set = t / TX4;
        xt[t] = set == 0 ? cv_tPA<FD>(j, g.nx) : set == 1 ? cv_tPB<FD>(j, g.nx)
              : set == 2 ? cv_tMA<FD>(j, g.nx, g.nx - 1) : cv_tMB<FD>(j, g.nx, g.nx - 1);
    }
    for (int t = tid; t < 4 * T::TZH; t += NTHR) {
        const int i = c.i0 + t % T::TZH, set = t / T::TZH;
        zt[t] = set == 0 ? cv_tPA<FD>(i, g.nz) : set == 1 ? cv_tPB<FD>(i, g.nz)
              : set == 2 ? cv_tMA<FD>(i, g.nz, g.nz - 1) : cv_tMB<FD>(i, g.nz, g.nz - 1);
    }
    const int rd = o.ping, wr = 1 - o.ping;
    const int jb = c.j0 + 2 * tx;
    const float2 dtdx2 = dup2(g.dtdx), dtdz2 = dup2(g.dtdz);
    constexpr int RE = EXACT ? RPT : 1, RI = IMG ? RPT : 1;
    float mL2M[RPT][2], mL[RPT][2], mM2[RPT][2], idet[RI][2], i2m[RI][2];
    // per-launch sums over the block's shots (at most a few terms) in FP32;
    // the sums over steps and shot groups are FP64 (the reductions below).
    // The exact gradient sums the carry-in stresses s against the stress
    // adjoints, sA = sum(s1 sxx_a + s2 szz_a), sB = sum(s2 sxx_a + s1 szz_a),
    // sC = sum(s3 sxz_a); the strain-recovery factors (constant per cell)
    // are applied once at the end: g_L2M = idet (L2M sA - L sB), g_L =
    // idet (L2M sB - L sA), g_M = sC / M.
    float sC[RE][2], sB[RE][2], sA[RE][2], glam[RI][2], gmu[RI][2];
    // density terms (history with velocities): dJ/dB of the exact gradient
    // and the rho term of the imaging formula
    constexpr int RB = (EXACT && RHO) ? RPT : 1, RR = (IMG && RHO) ? RPT : 1;
    float gB[RB][2], grl[RR][2];
#pragma unroll
    for (int r = 0; r < RB; ++r) gB[r][0] = gB[r][1] = 0.f;
#pragma unroll
    for (int r = 0; r < RR; ++r) grl[r][0] = grl[r][1] = 0.f;
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            const bool inb = i < g.nz && j < g.nx;
            const long long off = (long long)i * g.P + j;
            mL2M[r][cc] = inb ? m.L2M[off] : 0.f;
            mL[r][cc] = inb ? m.L[off] : 0.f;
            mM2[r][cc] = inb ? 2.f * m.M[off] : 0.f;
            if (IMG) {
                idet[r % RI][cc] = inb ? 1.0f / ((mL2M[r][cc] - mL[r][cc]) * (mL2M[r][cc] + mL[r][cc])) : 0.f;
                i2m[r % RI][cc] = inb ? 1.0f / mM2[r][cc] : 0.f;
            }
        }
#pragma unroll
    for (int r = 0; r < RE; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) sC[r][cc] = sB[r][cc] = sA[r][cc] = 0.f;
#pragma unroll
    for (int r = 0; r < RI; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) glam[r][cc] = gmu[r][cc] = 0.f;

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * STG;
        const float *own = S + T::S2;   // [ex_a, ez_a, es_a][TZH][TX4] of the tile's own cells
        const float *hown = own + L4<FD, RPT>::OWNB3;   // [sxx, szz, sxz][TZH][TX4] carry-in (htma)
        float *exa = A + ((long long)s * F_N + F_EX) * g.fstride;
        float *eza = A + ((long long)s * F_N + F_EZ) * g.fstride;
        float *esa = A + ((long long)s * F_N + F_ES) * g.fstride;
        const float *Pp = A + ((long long)s * F_N + F_U) * g.fstride;
        const float *Qp = A + ((long long)s * F_N + F_V) * g.fstride;
        const float *snap_in = ((EXACT || (IMG && RHO)) && o.slot_in >= 0)
                                   ? o.snap + ((long long)s * o.slots + o.slot_in) * g.snf * g.nd : nullptr;
        const float *snap_img = ((IMG || RHO) && o.slot_img >= 0)
                                    ? o.snap + ((long long)s * o.slots + o.slot_img) * g.snf * g.nd : nullptr;
        const float *snap_next = (IMG && RHO && o.slot_next >= 0)
                                     ? o.snap + ((long long)s * o.slots + o.slot_next) * g.snf * g.nd : nullptr;
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, g.wait_polls))) {
            abort3(bar, it, nsh, status);
            return;
        }
        if (fix) {
            const float *pXX = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XX);
            const float *pXXZ = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XXZ);
            const float *pZXZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZXZ);
            const float *pZZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZZ);
            float *wXX = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XX);
            float *wXXZ = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XXZ);
            float *wZXZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZXZ);
            float *wZZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZZ);
            const int xl = g.pad - (c.j0 - XO4), xr = g.nx - g.pad - (c.j0 - XO4);
            const float *tbx = tab, *tax = tab + SW4, *tikx = tab + 2 * SW4;
            const int *txs = reinterpret_cast<const int *>(tab + 4 * SW4);
            const float *tbz = tab + 5 * SW4, *taz = tbz + SH, *tikz = taz + SH;
            const int *tzs = reinterpret_cast<const int *>(tikz + SH);
            for (int rr = ty; rr < SH; rr += NWARP) {
                const int i = c.i0 - K + rr;
                const int zs = tzs[rr];
                const bool rowsp = zs >= 0;
                const bool own_row = rr >= K && rr < K + T::TZH;
                float ps[NCC][4];
#pragma unroll
                for (int b = 0; b < NCC; ++b) {
                    const int cc = tx + b * TX, jj = c.j0 - XO4 + cc;
                    ps[b][0] = ps[b][1] = ps[b][2] = ps[b][3] = 0.f;
                    if (cc >= SW4) continue;
                    const int xs = txs[cc];
                    if (xs >= 0 && i >= 0 && i < g.nz) {
                        const long long px = (long long)i * g.xs_n + xs;
                        ps[b][0] = pXX[px];
                        ps[b][1] = pXXZ[px];
                    }
                    if (zs >= 0 && jj >= 0 && jj < g.nx) {
                        const long long pz = (long long)zs * g.P + jj;
                        ps[b][2] = pZXZ[pz];
                        ps[b][3] = pZZ[pz];
                    }
                }
#pragma unroll
                for (int b = 0; b < NCC; ++b) {
                    const int cc = tx + b * TX;
                    if (cc >= SW4) continue;
                    const int jj = c.j0 - XO4 + cc, q = rr * SW4 + cc;
                    if (!rowsp && cc >= xl && cc < xr) {
                        // outside the strips: identity (cells off the grid are
                        // zero-filled by the tile copy already)
                        aZXZ[q] = S[q];
                        aXXZ[q] = S[SN + q];
                        continue;
                    }
                    float pv = 0.f, qq = 0.f;
                    if (i >= 0 && i < g.nz - 1 && jj >= 1 && jj < g.nx - 1) { pv = S[q]; qq = S[SN + q]; }
                    float vXX = pv, vZXZ = pv, vXXZ = qq, vZZ = qq;
                    if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                        const bool own = own_row && cc >= XO4 && cc < XO4 + TX4;
                        const int xs = txs[cc];
                        const long long px = (long long)i * g.xs_n + xs, pz = (long long)zs * g.P + jj;
                        if (xs >= 0) {
                            vXX = pml_adj4(pv, tbx[cc], tax[cc], tikx[cc], ps[b][0], wXX + px, own);
                            vXXZ = pml_adj4(qq, tbx[cc], tax[cc], tikx[cc], ps[b][1], wXXZ + px, own);
                        }
                        if (zs >= 0) {
                            vZXZ = pml_adj4(pv, tbz[rr], taz[rr], tikz[rr], ps[b][2], wZXZ + pz, own);
                            vZZ = pml_adj4(qq, tbz[rr], taz[rr], tikz[rr], ps[b][3], wZZ + pz, own);
                        }
                    }
                    S[q] = vXX; S[SN + q] = vZZ; aZXZ[q] = vZXZ; aXXZ[q] = vXXZ;
                }
            }
            __syncthreads();
        }
        const float *aXX = S, *aZZ = S + SN;
        const float *sZXZ = fix ? aZXZ : S, *sXXZ = fix ? aXXZ : S + SN;
        float2 wzz[T::W], wzxz[T::W];
        zwin2p<T::W, RPT>(wzz, aZZ, ty, tx);
        zwin2p<T::W, RPT>(wzxz, sZXZ, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
        // an interior tile whose box needs no fix-up, without this shot's
        // source: no per-cell guards, paired arithmetic
        auto lean_rows = [&]() {
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
            const int qo = (ty * RPT + r) * TX4 + 2 * tx;
            const float2 ea = *reinterpret_cast<const float2 *>(own + qo);
            const float2 za = *reinterpret_cast<const float2 *>(own + PL + qo);
            const float2 sa = *reinterpret_cast<const float2 *>(own + 2 * PL + qo);
            float axx[10], axz[10];
            xrow(axx, aXX, q);
            xrow(axz, sXXZ, q);
            const float2 sxx = mul2(dtdx2, make_float2(a_tdp<FD, false>(axx, 0, 0, 0), a_tdp<FD, false>(axx, 1, 0, 0)));
            const float2 szz = mul2(dtdz2, w_tdp2<FD>(wzz, r));
            const float2 sxz = fma2(dtdx2, make_float2(a_tdm<FD, false>(axz, 0, 0, 0, 0), a_tdm<FD, false>(axz, 1, 0, 0, 0)),
                                    mul2(dtdz2, w_tdm2<FD>(wzxz, r)));
            const float2 l2m = make_float2(mL2M[r][0], mL2M[r][1]), l = make_float2(mL[r][0], mL[r][1]);
            const float2 nex = fma2(l, szz, fma2(l2m, sxx, ea));
            const float2 nez = fma2(l2m, szz, fma2(l, sxx, za));
            const float2 nes = fma2(make_float2(mM2[r][0], mM2[r][1]), sxz, sa);
            const int pi = i - g.z0, pj0 = jb - g.pad;
            if (EXACT && (htma || snap_in)) {
                float2 h1, h2, h3;
                if (htma) {
                    h1 = *reinterpret_cast<const float2 *>(hown + qo);
                    h2 = *reinterpret_cast<const float2 *>(hown + PL + qo);
                    h3 = *reinterpret_cast<const float2 *>(hown + 2 * PL + qo);
                } else {
                    const long long pq = (long long)pi * g.nx_dom + pj0;
                    h1 = make_float2(__ldcs(snap_in + pq), __ldcs(snap_in + pq + 1));
                    h2 = make_float2(__ldcs(snap_in + g.nd + pq), __ldcs(snap_in + g.nd + pq + 1));
                    h3 = make_float2(__ldcs(snap_in + 2 * g.nd + pq), __ldcs(snap_in + 2 * g.nd + pq + 1));
                }
                float2 ta = make_float2(sA[r % RE][0], sA[r % RE][1]);
                float2 tb = make_float2(sB[r % RE][0], sB[r % RE][1]);
                float2 tc = make_float2(sC[r % RE][0], sC[r % RE][1]);
                ta = __fadd2_rn(ta, fma2(h1, sxx, mul2(h2, szz)));
                tb = __fadd2_rn(tb, fma2(h2, sxx, mul2(h1, szz)));
                tc = fma2(h3, sxz, tc);
                sA[r % RE][0] = ta.x; sA[r % RE][1] = ta.y;
                sB[r % RE][0] = tb.x; sB[r % RE][1] = tb.y;
                sC[r % RE][0] = tc.x; sC[r % RE][1] = tc.y;
            }
            if (RHO || IMG) {
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc, pj = pj0 + cc;
                    const long long off = (long long)i * g.P + j, pq = (long long)pi * g.nx_dom + pj;
                    if (RHO) {
                        const float pc = Pp[off], qc = Qp[off], bb = m.B[off];
                        if (EXACT && snap_in && snap_img) {
                            const float du = snap_img[3 * g.nd + pq] - snap_in[3 * g.nd + pq];
                            const float dv = snap_img[4 * g.nd + pq] - snap_in[4 * g.nd + pq];
                            gB[r % RB][cc] += (pc * du + qc * dv) / (bb * bb);
                        }
                        if (IMG) {
                            const float ua = pc / bb, va = qc / bb;
                            float t = 0.f;
                            if (n >= 2 && snap_in) t += ua * snap_in[3 * g.nd + pq] + va * snap_in[4 * g.nd + pq];
                            if (n <= g.nt - 3 && snap_next)
                                t -= ua * snap_next[3 * g.nd + pq] + va * snap_next[4 * g.nd + pq];
                            grl[r % RR][cc] -= 0.5f * t;
                        }
                    }
                    if (IMG && snap_img) {
                        const int ip = (i + 1) % g.nz, im = (i - 1 + g.nz) % g.nz;
                        const int jp = (j + 1) % g.nx, jm = (j - 1 + g.nx) % g.nx;
                        const long long oxp = (long long)i * g.P + jp, oxm = (long long)i * g.P + jm;
                        const long long ozp = (long long)ip * g.P + j, ozm = (long long)im * g.P + j;
                        const float dxBU = (Pp[oxp] - Pp[oxm]) * g.inv2dx;
                        const float dzBV = (Qp[ozp] - Qp[ozm]) * g.inv2dz;
                        const float dzBU = (Pp[ozp] - Pp[ozm]) * g.inv2dz;
                        const float dxBV = (Qp[oxp] - Qp[oxm]) * g.inv2dx;
                        const float t1 = snap_img[pq], t2 = snap_img[g.nd + pq], t3 = snap_img[2 * g.nd + pq];
                        const float e1 = (mL2M[r][cc] * t1 - mL[r][cc] * t2) * idet[r % RI][cc];
                        const float e2 = (mL2M[r][cc] * t2 - mL[r][cc] * t1) * idet[r % RI][cc];
                        const float e3 = t3 * i2m[r % RI][cc];
                        glam[r % RI][cc] -= g.dt * ((e1 + e2) * (dxBU + dzBV));
                        gmu[r % RI][cc] -= g.dt * (2.f * e1 * dxBU + 2.f * e2 * dzBV + e3 * (dzBU + dxBV));
                    }
                }
            }
            const long long off = (long long)i * g.P + jb;
            *reinterpret_cast<float2 *>(exa + off) = nex;
            *reinterpret_cast<float2 *>(eza + off) = nez;
            *reinterpret_cast<float2 *>(esa + off) = nes;
        }
        };
        // tiles with an edge, a C-PML strip, the free surface or the source:
        // table-driven stencils, per-cell guards
        auto rows = [&]() {
        constexpr bool LEAN = false;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (!LEAN && i >= g.nz) continue;
            const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
            const int qo = (ty * RPT + r) * TX4 + 2 * tx;
            const float2 a2 = *reinterpret_cast<const float2 *>(own + qo);
            const float2 b2 = *reinterpret_cast<const float2 *>(own + PL + qo);
            const float2 d2 = *reinterpret_cast<const float2 *>(own + 2 * PL + qo);
            const float ea[2] = {a2.x, a2.y}, za[2] = {b2.x, b2.y}, sa[2] = {d2.x, d2.y};
            float axx[10], axz[10];
            xrow(axx, aXX, q);
            xrow(axz, sXXZ, q);
            const int zr = ty * RPT + r;
            const float4 zpa = zt[zr], zpb = zt[T::TZH + zr], zma = zt[2 * T::TZH + zr], zmb = zt[3 * T::TZH + zr];
            float h1[2] = {0.f, 0.f}, h2[2] = {0.f, 0.f}, h3[2] = {0.f, 0.f};
            if (EXACT && htma) {
                const float2 x1 = *reinterpret_cast<const float2 *>(hown + qo);
                const float2 x2 = *reinterpret_cast<const float2 *>(hown + PL + qo);
                const float2 x3 = *reinterpret_cast<const float2 *>(hown + 2 * PL + qo);
                h1[0] = x1.x; h1[1] = x1.y; h2[0] = x2.x; h2[1] = x2.y; h3[0] = x3.x; h3[1] = x3.y;
            } else if (EXACT && snap_in) {
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int pi = i - g.z0, pj = jb + cc - g.pad;
                    if (LEAN || (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom)) {
                        const long long pq = (long long)pi * g.nx_dom + pj;
                        h1[cc] = __ldcs(snap_in + pq);
                        h2[cc] = __ldcs(snap_in + g.nd + pq);
                        h3[cc] = __ldcs(snap_in + 2 * g.nd + pq);
                    }
                }
            }
            float nex[2], nez[2], nes[2];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j = jb + cc;
                nex[cc] = ea[cc]; nez[cc] = za[cc]; nes[cc] = sa[cc];
                if (!LEAN && j >= g.nx) continue;
                float sxx = 0.f, szz = 0.f, sxz = 0.f;
                const int col = 2 * tx + cc;
                if (i < g.nz - 1) {
                    sxx = g.dtdx * a_tdp_t<FD>(axx, cc, xt[col], xt[TX4 + col]);
                    sxz = g.dtdx * a_tdm_t<FD>(axz, cc, xt[2 * TX4 + col], xt[3 * TX4 + col]);
                }
                if (j >= 1 && j < g.nx - 1) {
                    szz = g.dtdz * w_tdp_t<FD>(wzz, r, cc, zpa, zpb);
                    sxz += g.dtdz * w_tdm_t<FD>(wzxz, r, cc, zma, zmb);
                    if (g.fs && i == 0) sxz += 2.f * cf<FD>(1) * g.dtdz * f2c(wzxz[r + K], cc);
                }
                const long long off = (long long)i * g.P + j;
                if (!LEAN && i == ssz && j == ssx) {
                    const float w = sh.wav[(long long)s * g.nt + n];
                    if (stype == 0) {
                        if (o.src_a) o.src_a[(long long)s * g.nt + n] = g.dtdxdz * Qp[off];
                    } else {
                        if (o.src_a) o.src_a[(long long)s * g.nt + n] = (g.dt / sh.mcoef[s]) * (ea[cc] + za[cc]);
                        if (EXACT) {
                            // the moment factor's (L + M) term, straight into
                            // this group's FP64 sums of the source cell
                            const double lm = sh.lm[s];
                            const double glm = -((double)w * g.dt / ((double)sh.mcoef[s] / lm)) / (lm * lm)
                                               * (double)(ea[cc] + za[cc]);
                            const int pi = i - g.z0, pj = j - g.pad;
                            if (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                                double *acc = o.acc + (long long)(c.s0 / spg) * o.accp * g.nd +
                                              (long long)pi * g.nx_dom + pj;
                                atomicAdd(acc, glm);
                                atomicAdd(acc + g.nd, glm);
                            }
                        }
                    }
                }
                nex[cc] = ea[cc] + mL2M[r][cc] * sxx + mL[r][cc] * szz;
                nez[cc] = za[cc] + mL[r][cc] * sxx + mL2M[r][cc] * szz;
                nes[cc] = sa[cc] + mM2[r][cc] * sxz;
                if (EXACT) {
                    sA[r % RE][cc] += h1[cc] * sxx + h2[cc] * szz;
                    sB[r % RE][cc] += h2[cc] * sxx + h1[cc] * szz;
                    sC[r % RE][cc] += h3[cc] * sxz;
                }
                const int pi = i - g.z0, pj = j - g.pad;
                if (RHO && (LEAN || (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom))) {
                    const long long pq = (long long)pi * g.nx_dom + pj;
                    const float pc = Pp[off], qc = Qp[off], bb = m.B[off];
                    if (EXACT && snap_in && snap_img) {
                        // dJ/dB: U_a dU/B + V_a dV/B with U_a = P/B and the
                        // step's velocity increments from the history
                        const float du = snap_img[3 * g.nd + pq] - snap_in[3 * g.nd + pq];
                        const float dv = snap_img[4 * g.nd + pq] - snap_in[4 * g.nd + pq];
                        gB[r % RB][cc] += (pc * du + qc * dv) / (bb * bb);
                    }
                    if (IMG) {
                        // -1/2 U_a(n) (vx(n-1) - vx(n+1)), the rho term of the
                        // imaging formula regrouped by adjoint step
                        const float ua = pc / bb, va = qc / bb;
                        float t = 0.f;
                        if (n >= 2 && snap_in) t += ua * snap_in[3 * g.nd + pq] + va * snap_in[4 * g.nd + pq];
                        if (n <= g.nt - 3 && snap_next)
                            t -= ua * snap_next[3 * g.nd + pq] + va * snap_next[4 * g.nd + pq];
                        grl[r % RR][cc] -= 0.5f * t;
                    }
                }
                if (IMG && snap_img && (LEAN || (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom))) {
                    const long long pq = (long long)pi * g.nx_dom + pj;
                    const int ip = (i + 1) % g.nz, im = (i - 1 + g.nz) % g.nz;
                    const int jp = (j + 1) % g.nx, jm = (j - 1 + g.nx) % g.nx;
                    const long long oxp = (long long)i * g.P + jp, oxm = (long long)i * g.P + jm;
                    const long long ozp = (long long)ip * g.P + j, ozm = (long long)im * g.P + j;
                    const float dxBU = (Pp[oxp] - Pp[oxm]) * g.inv2dx;
                    const float dzBV = (Qp[ozp] - Qp[ozm]) * g.inv2dz;
                    const float dzBU = (Pp[ozp] - Pp[ozm]) * g.inv2dz;
                    const float dxBV = (Qp[oxp] - Qp[oxm]) * g.inv2dx;
                    const float t1 = snap_img[pq], t2 = snap_img[g.nd + pq], t3 = snap_img[2 * g.nd + pq];
                    const float e1 = (mL2M[r][cc] * t1 - mL[r][cc] * t2) * idet[r % RI][cc];
                    const float e2 = (mL2M[r][cc] * t2 - mL[r][cc] * t1) * idet[r % RI][cc];
                    const float e3 = t3 * i2m[r % RI][cc];
                    glam[r % RI][cc] -= g.dt * ((e1 + e2) * (dxBU + dzBV));
                    gmu[r % RI][cc] -= g.dt * (2.f * e1 * dxBU + 2.f * e2 * dzBV + e3 * (dzBU + dxBV));
                }
            }
            if (LEAN || jb < g.nx) {
                const long long off = (long long)i * g.P + jb;
                if (LEAN || jb + 1 < g.nx) {
                    *reinterpret_cast<float2 *>(exa + off) = make_float2(nex[0], nex[1]);
                    *reinterpret_cast<float2 *>(eza + off) = make_float2(nez[0], nez[1]);
                    *reinterpret_cast<float2 *>(esa + off) = make_float2(nes[0], nes[1]);
                } else {
                    exa[off] = nex[0]; eza[off] = nez[0]; esa[off] = nes[0];
                }
            }
        }
        };
        if (lean && !in_tile4(ssz, ssx, c.i0, c.j0, T::TZH)) lean_rows();
        else rows();
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4 + OWNB + hbytes);
            tma_load_4d(S, &tmPQ, bar + (it & 1), c.j0 - XO4, c.i0 - K, F_U, s + 2);
            tma_load_4d(S + T::S2, &tmEo, bar + (it & 1), c.j0, c.i0, F_EX, s + 2);
            if (htma)
                tma_load_4d_hint(S + T::S2 + L4<FD, RPT>::OWNB3, &tmH, bar + (it & 1), hx, hy, hz, s + 2,
                                 l2_evict_first());
        }
        if (n > 0) {
            const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
            for (int qq = r0 + tid; qq < r1; qq += NTHR) {
                const int rid = rv.tile_rec[qq];
                const long long off = (long long)rv.rz[rid] * g.P + rv.rx[rid];
                const float *src = o.rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)(n - 1) * g.nrec + rid;
                atomicAdd(exa + off, src[2LL * g.nt * g.nrec]);
                atomicAdd(eza + off, src[3LL * g.nt * g.nrec]);
            }
        }
    }
    if (EXACT || IMG) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int i = c.i0 + ty * RPT + r, j = jb + cc;
                const int pi = i - g.z0, pj = j - g.pad;
                if (i < g.nz && j < g.nx && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                    // one block per (tile, shot group) adds to these cells in a
                    // launch: the atomic adds only avoid waiting for the loads
                    double *acc = o.acc + (long long)(c.s0 / spg) * o.accp * g.nd + (long long)pi * g.nx_dom + pj;
                    if (EXACT) {
                        const double l2m = mL2M[r][cc], l = mL[r][cc];
                        const double id = 1.0 / ((l2m - l) * (l2m + l));
                        const double a = sA[r % RE][cc], b = sB[r % RE][cc];
                        atomicAdd(acc, 2.0 * (double)sC[r % RE][cc] / (double)mM2[r][cc]);
                        atomicAdd(acc + g.nd, id * (l2m * b - l * a));
                        atomicAdd(acc + 2 * g.nd, id * (l2m * a - l * b));
                    }
                    if (IMG) {
                        atomicAdd(acc + 3 * g.nd, (double)glam[r % RI][cc]);
                        atomicAdd(acc + 4 * g.nd, (double)gmu[r % RI][cc]);
                    }
                    if (EXACT && RHO) atomicAdd(acc + 5 * g.nd, (double)gB[r % RB][cc]);
                    if (IMG && RHO) atomicAdd(acc + 6 * g.nd, (double)grl[r % RR][cc]);
                }
            }
    }
}

}  // namespace stfwi
