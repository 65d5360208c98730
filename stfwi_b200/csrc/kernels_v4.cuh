// Two-column register-blocked stencil kernels (sm_100a), the default path.
//
// The same four phases, state variables and arithmetic as kernels_v3.cuh
// (stress-state forward, buoyancy-scaled adjoint; kernels.cuh documents the
// correspondence with the reference), with each thread owning TWO adjacent
// columns of RPT rows: a tile is 64 columns wide, the x-neighbourhood of a
// thread's two columns on one row is five aligned float2 shared loads
// (columns j-4 .. j+5), and the z-stencils come from a float2 register
// window of RPT + 2K rows.  Halo tiles arrive by TMA (one 4-D bulk tensor
// copy per shot, double-buffered over the shots a block owns).
#pragma once
#include <type_traits>

#include "common.cuh"

namespace stfwi {

#ifndef STFWI_V4_MINBLOCKS
#define STFWI_V4_MINBLOCKS 2
#endif

constexpr int TX4 = 64;               // tile width: 32 lanes x 2 columns
constexpr int XO4 = 4;                // x halo of the staged tile
constexpr int SW4 = TX4 + 2 * XO4;    // 72 floats = 288 B rows

template <int FD, int RPT> struct G4 {
    static constexpr int K = FD / 2;
    static constexpr int TZH = RPT * NWARP;
    static constexpr int SH = TZH + 2 * K;
    static constexpr int SN = SH * SW4;
    static constexpr int W = RPT + 2 * K;
    static constexpr int M = 2 * K + 1;
    static constexpr int S1 = al32_3(SN), S2 = al32_3(2 * SN), S3 = al32_3(3 * SN);
};

#ifndef STFWI_V4_RPT
#define STFWI_V4_RPT 2
#endif
#ifndef STFWI_V4_RPTB
#define STFWI_V4_RPTB 2
#endif
constexpr int RPT4 = STFWI_V4_RPT;    // rows per thread: fwd_vel, fwd_str, adj_a
constexpr int RPT4B = STFWI_V4_RPTB;  // rows per thread: adj_b (FP64 sums per cell in registers)

template <int FD> struct L4 {
    using A = G4<FD, RPT4>;
    using B = G4<FD, RPT4B>;
    // own-cell boxes (no halo) staged beside the halo boxes: U, V for the
    // velocity phase, sxx, szz, sxz for the stress phase
    static constexpr int OWN2 = al32_3(2 * A::TZH * TX4), OWN3 = al32_3(3 * A::TZH * TX4);
    static constexpr int VEL_STAGE = A::S3 + OWN2, STR_STAGE = A::S2 + OWN3;
    static constexpr int VEL = 2 * VEL_STAGE;
    static constexpr int STR = 2 * STR_STAGE;
    // C-PML coefficient tables of a staged box: bx, ax, ikx, Lr per column, bz, az, ikz per row
    static constexpr int TABA = al32_3(5 * SW4 + 4 * A::SH);
    static constexpr int TABB = al32_3(5 * SW4 + 4 * B::SH);
    static constexpr int ADA_STAGE = A::S3 + OWN2;   // + P, Q of the own cells
    static constexpr int ADA = 2 * ADA_STAGE + A::S1 + TABA;
    static constexpr int OWNB3 = al32_3(3 * B::TZH * TX4);   // strain adjoints of the own cells
    // + the carry-in stresses of the own cells from the history (exact gradient)
    static constexpr int ADB_STAGE = B::S2 + 2 * OWNB3;
    static constexpr int ADB = 2 * ADB_STAGE + 2 * B::S1 + TABB;
    static constexpr size_t bytes(int floats, int nbar) { return (size_t)floats * 4 + 8 * nbar; }
};

// a[i] = f[j - 4 + i], i in [0, 10): the x-neighbourhood of columns j, j+1
__device__ __forceinline__ void xrow(float (&a)[10], const float *s, int q)
{
    const float2 *p = reinterpret_cast<const float2 *>(s + q - 4);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const float2 t = p[m];
        a[2 * m] = t.x;
        a[2 * m + 1] = t.y;
    }
}

// stencils on a (output column c of the pair, global column jc)
template <int FD, bool MASK>
__device__ __forceinline__ float a_dp(const float (&a)[10], int c, int jc, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mP(jc, k, n)) d += cf<FD>(k) * (a[4 + c + k] - a[5 + c - k]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float a_dm(const float (&a)[10], int c, int jc, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mM(jc, k, n)) d += cf<FD>(k) * (a[3 + c + k] - a[4 + c - k]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float a_tdp(const float (&a)[10], int c, int jc, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        if (!MASK || mP(jc - k, k, n)) d += cf<FD>(k) * a[4 + c - k];
        if (!MASK || mP(jc + k - 1, k, n)) d -= cf<FD>(k) * a[3 + c + k];
    }
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float a_tdm(const float (&a)[10], int c, int jc, int n, int lim)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const int t1 = jc - k + 1, t2 = jc + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += cf<FD>(k) * a[5 + c - k];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= cf<FD>(k) * a[4 + c + k];
    }
    return d;
}

// z window of the pair: w[m][c] = f(row ty*RPT + m - K relative to the tile, column c)
template <int W, int RPT>
__device__ __forceinline__ void zwin2(float (&w)[W][2], const float *s, int ty, int tx)
{
#pragma unroll
    for (int m = 0; m < W; ++m) {
        const float2 t = *reinterpret_cast<const float2 *>(s + (ty * RPT + m) * SW4 + XO4 + 2 * tx);
        w[m][0] = t.x;
        w[m][1] = t.y;
    }
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float w_dp(const float (&w)[W][2], int r, int c, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k)
        if (!MASK || mP(i, k, n)) d += cf<FD>(k) * (w[r + K + k][c] - w[r + K - k + 1][c]);
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float w_dm(const float (&w)[W][2], int r, int c, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k)
        if (!MASK || mM(i, k, n)) d += cf<FD>(k) * (w[r + K + k - 1][c] - w[r + K - k][c]);
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float w_tdp(const float (&w)[W][2], int r, int c, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        if (!MASK || mP(i - k, k, n)) d += cf<FD>(k) * w[r + K - k][c];
        if (!MASK || mP(i + k - 1, k, n)) d -= cf<FD>(k) * w[r + K + k - 1][c];
    }
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float w_tdm(const float (&w)[W][2], int r, int c, int i, int n, int lim)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        const int t1 = i - k + 1, t2 = i + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += cf<FD>(k) * w[r + K - k + 1][c];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= cf<FD>(k) * w[r + K + k][c];
    }
    return d;
}

__device__ __forceinline__ Ctx3 ctx4(const Geo &g, int spg, int tzh, int tiles_x)
{
    Ctx3 c;
    c.tile = blockIdx.x;
    c.j0 = (c.tile % tiles_x) * TX4;
    c.i0 = (c.tile / tiles_x) * tzh;
    c.s0 = blockIdx.y * spg;
    c.s1 = min(c.s0 + spg, g.nshot);
    return c;
}

__device__ __forceinline__ bool box_special4(const Geo &g, int i0, int j0, int tzh, int K)
{
    const int r0 = i0 - K, r1 = i0 + tzh + K - 1, c0 = j0 - XO4, c1 = j0 + TX4 + XO4 - 1;
    if (c0 < g.pad || c1 >= g.nx - g.pad) return true;
    if (r1 >= g.nz - g.pad) return true;
    if (r0 <= 0) return true;
    if (!g.fs && r0 < g.pad) return true;
    return false;
}

// do the tile's own cells lie where no slice mask, edge rule, C-PML strip or
// free-surface row applies (margin M from every edge, outside the strips)?
// Such tiles take a code path without per-cell guards.
__device__ __forceinline__ bool tile_plain4(const Geo &g, int i0, int j0, int tzh, int M)
{
    const int i1 = i0 + tzh - 1, j1 = j0 + TX4 - 1;
    if (i0 < M || i1 > g.nz - 1 - M || j0 < M || j1 > g.nx - 1 - M) return false;
    if (j0 < g.pad || j1 >= g.nx - g.pad) return false;
    if (i1 >= g.nz - g.pad) return false;
    if (!g.fs && i0 < g.pad) return false;
    return true;
}

__device__ __forceinline__ bool in_tile4(int i, int j, int i0, int j0, int tzh)
{
    return i >= i0 && i < i0 + tzh && j >= j0 && j < j0 + TX4;
}

// the strain-phase fix-up only applies C-PML transposes and edge limits, which
// all lie in the strips: the free-surface row needs none there
__device__ __forceinline__ bool box_strips4(const Geo &g, int i0, int j0, int tzh, int K)
{
    const int r0 = i0 - K, r1 = i0 + tzh + K - 1, c0 = j0 - XO4, c1 = j0 + TX4 + XO4 - 1;
    if (c0 < g.pad || c1 >= g.nx - g.pad) return true;
    if (r1 >= g.nz - g.pad) return true;
    if (!g.fs && r0 < g.pad) return true;
    return false;
}

// pml_fwd with the old memory already loaded (the load is issued early)
__device__ __forceinline__ float pml_fwd_pre(float D, float b, float a, float ik, float old, float *psi)
{
    const float pn = b * old + a * D;
    *psi = pn;
    return D * ik + pn;
}

// C-PML coefficients of the box's columns and rows in shared memory (read by
// the fix-up passes instead of per-cell global loads): per column bx, ax,
// ikx, Lr (free-surface term) and the x-strip index (-1 outside the strips),
// per row bz, az, ikz and the z-strip index
template <int SH>
__device__ __forceinline__ void pml_table4(const Geo &g, const Mat &m, int i0, int j0, float *tab, int tid)
{
    int *itab = reinterpret_cast<int *>(tab);
    for (int t = tid; t < SW4; t += NTHR) {
        const int jj = j0 - XO4 + t;
        const bool in = jj >= 0 && jj < g.nx;
        const int xs = in ? xstrip_index(g, jj) : -1;
        tab[t] = xs >= 0 ? m.bx[jj] : 0.f;
        tab[SW4 + t] = xs >= 0 ? m.ax[jj] : 0.f;
        tab[2 * SW4 + t] = xs >= 0 ? m.ikx[jj] : 1.f;
        tab[3 * SW4 + t] = (in && g.fs) ? m.Lr[jj] : 0.f;
        itab[4 * SW4 + t] = xs;
    }
    for (int t = tid; t < SH; t += NTHR) {
        const int i = i0 + t;
        const int zs = (i >= 0 && i < g.nz) ? zstrip_index(g, i) : -1;
        tab[5 * SW4 + t] = zs >= 0 ? m.bz[i] : 0.f;
        tab[5 * SW4 + SH + t] = zs >= 0 ? m.az[i] : 0.f;
        tab[5 * SW4 + 2 * SH + t] = zs >= 0 ? m.ikz[i] : 1.f;
        itab[5 * SW4 + 3 * SH + t] = zs;
    }
}

// transposed C-PML on a staged value x with the memory kept in the scaled
// form phi = psi / (dt / d) of the adjoint step (so the step's factor drops
// out): returns (1/k + a) x + a phi and stores the new memory b (x + phi)
__device__ __forceinline__ float pml_adj4(float x, float b, float a, float ik, float phi, float *dst, bool own)
{
    if (own) *dst = b * (x + phi);
    return (ik + a) * x + a * phi;
}

// ------------------------------------------------------------- forward: velocities

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_V4_MINBLOCKS)
    k4_fwd_vel(Geo g, Mat m, Shots sh, float *F, float *PX, float *PZ, int n, int spg, int tiles_x, int *status,
               const __grid_constant__ CUtensorMap tmS, const __grid_constant__ CUtensorMap tmUo)
{
    using T = G4<FD, RPT4>;
    constexpr int K = T::K, SN = T::SN, RPT = RPT4;
    constexpr int STG = L4<FD>::VEL_STAGE, OWNB = 2 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L4<FD>::VEL);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx4(g, spg, T::TZH, tiles_x);
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
    __syncthreads();
    const int jb = c.j0 + 2 * tx;
    int xs[2];
    float bxv[2], axv[2], ikxv[2];
    bool colin[2];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int j = jb + cc;
        xs[cc] = (j < g.nx) ? xstrip_index(g, j) : -1;
        bxv[cc] = xs[cc] >= 0 ? m.bx[j] : 0.f;
        axv[cc] = xs[cc] >= 0 ? m.ax[j] : 0.f;
        ikxv[cc] = xs[cc] >= 0 ? m.ikx[j] : 1.f;
        colin[cc] = j >= T::M && j <= g.nx - 1 - T::M;
    }
    float Bc[RPT][2];
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            Bc[r][cc] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
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
        float *pSXX = px_ptr(g, PX, s, PX_SXX), *pSXZx = px_ptr(g, PX, s, PX_SXZ);
        float *pSXZz = pz_ptr(g, PZ, s, PZ_SXZ), *pSZZ = pz_ptr(g, PZ, s, PZ_SZZ);
        float wxz[T::W][2], wzz[T::W][2];
        zwin2<T::W, RPT>(wxz, sxz, ty, tx);
        zwin2<T::W, RPT>(wzz, szz, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
        // LEAN: an interior tile without this shot's source (no per-cell guards)
        auto rows = [&](auto lean_c) {
        constexpr bool LEAN = decltype(lean_c)::value;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
            float ax[10], az[10];
            xrow(ax, sxx, q);
            xrow(az, sxz, q);
            const bool rowin = i >= T::M && i <= g.nz - 1 - T::M;
            const int zs = zstrip_index(g, i);
            // this row's C-PML memories, requested before the stencils
            float pxo[2][2] = {{0.f, 0.f}, {0.f, 0.f}}, pzo[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
            float zb = 0.f, za = 0.f, zik = 1.f;
            if (!LEAN && i < g.nz - 1) {
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int j = jb + cc;
                    if (j < 1 || j >= g.nx - 1) continue;
                    if (xs[cc] >= 0) {
                        const long long px = (long long)i * g.xs_n + xs[cc];
                        pxo[cc][0] = pSXX[px];
                        pxo[cc][1] = pSXZx[px];
                    }
                    if (zs >= 0) {
                        const long long pz = (long long)zs * g.P + j;
                        pzo[cc][0] = pSXZz[pz];
                        pzo[cc][1] = pSZZ[pz];
                    }
                }
                if (zs >= 0) { zb = m.bz[i]; za = m.az[i]; zik = m.ikz[i]; }
            }
            const float2 u2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
            const float2 v2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
            const float u[2] = {u2.x, u2.y}, v[2] = {v2.x, v2.y};
            float un[2], vn[2];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j = jb + cc;
                un[cc] = u[cc];
                vn[cc] = v[cc];
                if (!LEAN && (i >= g.nz - 1 || j < 1 || j >= g.nx - 1)) continue;
                float dxx, dzxz, dxxz, dzz;
                if (LEAN || (colin[cc] && rowin)) {
                    dxx = a_dp<FD, false>(ax, cc, j, g.nx);
                    dxxz = a_dm<FD, false>(az, cc, j, g.nx);
                    dzxz = w_dm<FD, false>(wxz, r, cc, i, g.nz);
                    dzz = w_dp<FD, false>(wzz, r, cc, i, g.nz);
                } else {
                    dxx = a_dp<FD, true>(ax, cc, j, g.nx);
                    dxxz = a_dm<FD, true>(az, cc, j, g.nx);
                    dzxz = w_dm<FD, true>(wxz, r, cc, i, g.nz);
                    dzz = w_dp<FD, true>(wzz, r, cc, i, g.nz);
                    if (g.fs && i == 0) dzxz = 2.f * cf<FD>(1) * wxz[r + K][cc];
                }
                if (!LEAN && xs[cc] >= 0) {
                    const long long px = (long long)i * g.xs_n + xs[cc];
                    dxx = pml_fwd_pre(dxx, bxv[cc], axv[cc], ikxv[cc], pxo[cc][0], pSXX + px);
                    dxxz = pml_fwd_pre(dxxz, bxv[cc], axv[cc], ikxv[cc], pxo[cc][1], pSXZx + px);
                }
                if (!LEAN && zs >= 0) {
                    const long long pz = (long long)zs * g.P + j;
                    dzxz = pml_fwd_pre(dzxz, zb, za, zik, pzo[cc][0], pSXZz + pz);
                    dzz = pml_fwd_pre(dzz, zb, za, zik, pzo[cc][1], pSZZ + pz);
                }
                un[cc] = u[cc] + g.dtdx * Bc[r][cc] * dxx + g.dtdz * Bc[r][cc] * dzxz;
                float vv = v[cc] + g.dtdx * Bc[r][cc] * dxxz + g.dtdz * Bc[r][cc] * dzz;
                if (!LEAN && stype == 0 && i == ssz && j == ssx) vv = vv + sh.fcoef[s] * sh.wav[(long long)s * g.nt + n];
                vn[cc] = vv;
            }
            // cells outside the update region keep their value (column 0, nx-1, row nz-1)
            if (LEAN || (i < g.nz - 1 && jb < g.nx)) {
                const long long o = (long long)i * g.P + jb;
                if (LEAN || jb + 1 < g.nx) {
                    *reinterpret_cast<float2 *>(U + o) = make_float2(un[0], un[1]);
                    *reinterpret_cast<float2 *>(V + o) = make_float2(vn[0], vn[1]);
                } else {
                    U[o] = un[0];
                    V[o] = vn[0];
                }
            }
        }
        };
        if (plain && !in_tile4(ssz, ssx, c.i0, c.j0, T::TZH)) rows(std::true_type{});
        else rows(std::false_type{});
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

template <int FD, bool ENERGY>
__global__ void __launch_bounds__(NTHR, STFWI_V4_MINBLOCKS)
    k4_fwd_str(Geo g, Mat m, Shots sh, Recv rv, float *F, float *PX, float *PZ, int n, int spg, int tiles_x,
               FwdOut out, const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmSo)
{
    using T = G4<FD, RPT4>;
    constexpr int K = T::K, SN = T::SN, RPT = RPT4;
    constexpr int STG = L4<FD>::STR_STAGE, OWNB = 3 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L4<FD>::STR);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx4(g, spg, T::TZH, tiles_x);
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
    __syncthreads();
    const int jb = c.j0 + 2 * tx;
    int xs[2];
    float bxv[2], axv[2], ikxv[2], Lr0[2];
    bool colin[2];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int j = jb + cc;
        xs[cc] = (j < g.nx) ? xstrip_index(g, j) : -1;
        bxv[cc] = xs[cc] >= 0 ? m.bx[j] : 0.f;
        axv[cc] = xs[cc] >= 0 ? m.ax[j] : 0.f;
        ikxv[cc] = xs[cc] >= 0 ? m.ikx[j] : 1.f;
        Lr0[cc] = (g.fs && j < g.nx) ? m.Lr[j] : 0.f;
        colin[cc] = j >= T::M && j <= g.nx - 1 - T::M;
    }
    float ml2m[RPT][2], ml[RPT][2], mm2[RPT][2];
    constexpr int RG = ENERGY ? RPT : 1;
    double eacc[RG][2];
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            ml2m[r][cc] = ok ? m.L2M[o] : 0.f;
            ml[r][cc] = ok ? m.L[o] : 0.f;
            mm2[r][cc] = ok ? 2.f * m.M[o] : 0.f;
            if (r < RG) eacc[r][cc] = 0.0;
        }

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
        float *pDXU = px_ptr(g, PX, s, PX_DXU), *pDXV = px_ptr(g, PX, s, PX_DXV);
        float *pDZV = pz_ptr(g, PZ, s, PZ_DZV), *pDZU = pz_ptr(g, PZ, s, PZ_DZU);
        float wU[T::W][2], wV[T::W][2];
        zwin2<T::W, RPT>(wU, sU, ty, tx);
        zwin2<T::W, RPT>(wV, sV, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
        // LEAN: an interior tile without this shot's source (no per-cell guards)
        auto rows = [&](auto lean_c) {
        constexpr bool LEAN = decltype(lean_c)::value;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (!LEAN && i >= g.nz) continue;
            const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
            const int qo = (ty * RPT + r) * TX4 + 2 * tx;
            const float2 a2 = *reinterpret_cast<const float2 *>(own + qo);
            const float2 b2 = *reinterpret_cast<const float2 *>(own + T::TZH * TX4 + qo);
            const float2 d2 = *reinterpret_cast<const float2 *>(own + 2 * T::TZH * TX4 + qo);
            const float e1[2] = {a2.x, a2.y}, e2[2] = {b2.x, b2.y}, e3[2] = {d2.x, d2.y};
            float au[10], av[10];
            xrow(au, sU, q);
            xrow(av, sV, q);
            const bool rowin = i >= T::M && i <= g.nz - 1 - T::M;
            const int zs = zstrip_index(g, i);
            // this row's C-PML memories, requested before the stencils
            float pxo[2][2] = {{0.f, 0.f}, {0.f, 0.f}}, pzo[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
            float zb = 0.f, za = 0.f, zik = 1.f;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j = jb + cc;
                if (LEAN || j >= g.nx) continue;
                if (xs[cc] >= 0) {
                    const long long px = (long long)i * g.xs_n + xs[cc];
                    if (j >= 1) pxo[cc][0] = pDXU[px];
                    if (i < g.nz - 1) pxo[cc][1] = pDXV[px];
                }
                if (zs >= 0) {
                    const long long pz = (long long)zs * g.P + j;
                    if (j < g.nx - 1) pzo[cc][0] = pDZV[pz];
                    if (j >= 1) pzo[cc][1] = pDZU[pz];
                }
            }
            if (!LEAN && zs >= 0) { zb = m.bz[i]; za = m.az[i]; zik = m.ikz[i]; }
            float nxx[2], nzz[2], nxz[2];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j = jb + cc;
                nxx[cc] = e1[cc]; nzz[cc] = e2[cc]; nxz[cc] = e3[cc];
                if (!LEAN && j >= g.nx) continue;
                float dxu, dzv, dzu, dxv;
                if (LEAN || (colin[cc] && rowin)) {
                    dxu = a_dm<FD, false>(au, cc, j, g.nx);
                    dxv = a_dp<FD, false>(av, cc, j, g.nx);
                    dzv = w_dm<FD, false>(wV, r, cc, i, g.nz);
                    dzu = w_dp<FD, false>(wU, r, cc, i, g.nz);
                } else {
                    dxu = a_dm<FD, true>(au, cc, j, g.nx);
                    dxv = a_dp<FD, true>(av, cc, j, g.nx);
                    dzv = w_dm<FD, true>(wV, r, cc, i, g.nz);
                    dzu = w_dp<FD, true>(wU, r, cc, i, g.nz);
                }
                const long long px = (long long)i * g.xs_n + xs[cc], pz = (long long)zs * g.P + j;
                if (!LEAN) {
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
                }
                const float dex = (LEAN || j >= 1) ? g.dtdx * dxu : 0.f;
                const float dez = g.dtdz * dzv;
                const float des = (LEAN || (i < g.nz - 1 && j < g.nx - 1)) ? 0.5f * (g.dtdz * dzu + g.dtdx * dxv) : 0.f;
                const float l2m = ml2m[r][cc], l = ml[r][cc];
                float axx = e1[cc] + l2m * dex + l * dez;
                float azz = e2[cc] + l * dex + l2m * dez;
                const float axz = e3[cc] + mm2[r][cc] * des;
                if (!LEAN && stype == 1 && i == ssz && j == ssx) {
                    const float stm = sh.wav[(long long)s * g.nt + n] * g.dt / sh.mcoef[s];
                    axx = axx + (l2m + l) * stm;
                    azz = azz + (l + l2m) * stm;
                }
                nxx[cc] = axx; nzz[cc] = azz; nxz[cc] = axz;
                const int pi = i - g.z0, pj = j - g.pad;
                const bool phys = LEAN || (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom);
                if (out.snap && phys) {
                    float *sp = out.snap + ((long long)s * out.slots + out.slot) * g.snf * g.nd + (long long)pi * g.nx_dom + pj;
                    __stcs(sp, axx);
                    __stcs(sp + g.nd, azz);
                    __stcs(sp + 2 * g.nd, axz);
                    if (g.snf == 5) {   // velocities of this step (density gradient)
                        __stcs(sp + 3 * g.nd, au[4 + cc]);
                        __stcs(sp + 4 * g.nd, av[4 + cc]);
                    }
                }
                if (!LEAN && out.row0 && g.fs && i == 0 && pj >= 0 && pj < g.nx_dom)
                    out.row0[((long long)s * out.slots + out.slot_row0) * g.nx_dom + pj] = dxu;
                if (ENERGY) {
                    float f;
                    if (out.energy_comp < 2) {
                        f = out.energy_comp == 0 ? au[4 + cc] : av[4 + cc];
                    } else {
                        float ex, ez, es;
                        strains_of(axx, azz, axz, l2m, l, 0.5f * mm2[r][cc], ex, ez, es);
                        f = out.energy_comp == 2 ? ex : ez;
                    }
                    eacc[r % RG][cc] += (double)f * (double)f;
                }
            }
            if (LEAN || jb < g.nx) {
                const long long o = (long long)i * g.P + jb;
                if (LEAN || jb + 1 < g.nx) {
                    *reinterpret_cast<float2 *>(sxx + o) = make_float2(nxx[0], nxx[1]);
                    *reinterpret_cast<float2 *>(szz + o) = make_float2(nzz[0], nzz[1]);
                    *reinterpret_cast<float2 *>(sxz + o) = make_float2(nxz[0], nxz[1]);
                } else {
                    sxx[o] = nxx[0]; szz[o] = nzz[0]; sxz[o] = nxz[0];
                }
            }
        }
        };
        if (plain && !in_tile4(ssz, ssx, c.i0, c.j0, T::TZH)) rows(std::true_type{});
        else rows(std::false_type{});
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

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_V4_MINBLOCKS)
    k4_adj_a(Geo g, Mat m, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x, AdjIn in,
             int *status, const __grid_constant__ CUtensorMap tmE, const __grid_constant__ CUtensorMap tmPQo)
{
    using T = G4<FD, RPT4>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH, RPT = RPT4;
    constexpr int STG = L4<FD>::ADA_STAGE, OWNB = 2 * T::TZH * TX4 * 4;
    extern __shared__ __align__(128) float sm[];
    constexpr int NCC = (SW4 + TX - 1) / TX;
    float *aDxV = sm + 2 * STG;
    float *tab = aDxV + T::S1;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L4<FD>::ADA);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx4(g, spg, T::TZH, tiles_x);
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
    const int rd = in.ping, wr = 1 - in.ping;
    const int jb = c.j0 + 2 * tx;
    bool colin[2];
    colin[0] = jb >= T::M && jb <= g.nx - 1 - T::M;
    colin[1] = jb + 1 >= T::M && jb + 1 <= g.nx - 1 - T::M;
    const float hdtdz = 0.5f * g.dtdz, hdtdx = 0.5f * g.dtdx;
    float Bc[RPT][2];
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int i = c.i0 + ty * RPT + r, j = jb + cc;
            Bc[r][cc] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
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
        float wzu[T::W][2], wzv[T::W][2];
        zwin2<T::W, RPT>(wzu, aDzU, ty, tx);
        zwin2<T::W, RPT>(wzv, aDzV, ty, tx);
        // LEAN: an interior tile whose box needs no fix-up (no per-cell guards)
        auto rows = [&](auto lean_c) {
        constexpr bool LEAN = decltype(lean_c)::value;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (!LEAN && i >= g.nz) continue;
            const int q = (ty * RPT + r + K) * SW4 + XO4 + 2 * tx;
            float ad[10], av[10];
            xrow(ad, aDxU, q);
            xrow(av, aXV, q);
            const float2 p2 = *reinterpret_cast<const float2 *>(own + (ty * RPT + r) * TX4 + 2 * tx);
            const float2 q2 = *reinterpret_cast<const float2 *>(own + (T::TZH + ty * RPT + r) * TX4 + 2 * tx);
            const float pr[2] = {p2.x, p2.y}, qr[2] = {q2.x, q2.y};
            const bool rowin = i >= T::M && i <= g.nz - 1 - T::M;
            float np[2], nq[2];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j = jb + cc;
                np[cc] = pr[cc]; nq[cc] = qr[cc];
                if (!LEAN && j >= g.nx) continue;
                float gu, gv;
                if (LEAN || (colin[cc] && rowin)) {
                    gu = hdtdz * w_tdp<FD, false>(wzu, r, cc, i, g.nz) + g.dtdx * a_tdm<FD, false>(ad, cc, j, g.nx, g.nx);
                    gv = hdtdx * a_tdp<FD, false>(av, cc, j, g.nx) + g.dtdz * w_tdm<FD, false>(wzv, r, cc, i, g.nz, g.nz);
                } else {
                    gu = (j >= 1 ? hdtdz * w_tdp<FD, true>(wzu, r, cc, i, g.nz) : 0.f)
                       + g.dtdx * a_tdm<FD, true>(ad, cc, j, g.nx, g.nx);
                    gv = (i < g.nz - 1 ? hdtdx * a_tdp<FD, true>(av, cc, j, g.nx) : 0.f)
                       + (j < g.nx - 1 ? g.dtdz * w_tdm<FD, true>(wzv, r, cc, i, g.nz, g.nz) : 0.f);
                }
                np[cc] = pr[cc] + Bc[r][cc] * gu;
                nq[cc] = qr[cc] + Bc[r][cc] * gv;
                if (!LEAN && in.want_exact && g.fs && i == 0) {
                    const int pj = j - g.pad;
                    if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) {
                        const float du = in.row0[((long long)s * in.slots + in.slot) * g.nx_dom + pj];
                        glr[cc] += (double)(g.dtdz * wzv[r + K][cc]) * (double)du * (double)g.dzdx;
                    }
                }
            }
            if (LEAN || jb < g.nx) {
                const long long o = (long long)i * g.P + jb;
                if (LEAN || jb + 1 < g.nx) {
                    *reinterpret_cast<float2 *>(Pp + o) = make_float2(np[0], np[1]);
                    *reinterpret_cast<float2 *>(Qp + o) = make_float2(nq[0], nq[1]);
                } else {
                    Pp[o] = np[0];
                    Qp[o] = nq[0];
                }
            }
        }
        };
        if (lean) rows(std::true_type{});
        else rows(std::false_type{});
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
            if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) in.accLr[(long long)blockIdx.y * g.nx_dom + pj] += glr[cc];
        }
    }
}

// ------------------------------------------------------------- adjoint: strains + gradient

template <int FD, bool EXACT, bool IMG, bool RHO>
__global__ void __launch_bounds__(NTHR, STFWI_V4_MINBLOCKS)
    k4_adj_b(Geo g, Mat m, Shots sh, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x,
             AdjOut o, int *status, const __grid_constant__ CUtensorMap tmPQ,
             const __grid_constant__ CUtensorMap tmEo, const __grid_constant__ CUtensorMap tmH)
{
    using T = G4<FD, RPT4B>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH, RPT = RPT4B;
    constexpr int STG = L4<FD>::ADB_STAGE, OWNB = 3 * T::TZH * TX4 * 4, PL = T::TZH * TX4;
    extern __shared__ __align__(128) float sm[];
    constexpr int NCC = (SW4 + TX - 1) / TX;
    float *aZXZ = sm + 2 * STG, *aXXZ = aZXZ + T::S1;
    float *tab = aXXZ + T::S1;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L4<FD>::ADB);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx4(g, spg, T::TZH, tiles_x);
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
            if (htma) tma_load_4d(sm + b * STG + T::S2 + L4<FD>::OWNB3, &tmH, bar + b, hx, hy, hz, c.s0 + b);
        }
    }
    __syncthreads();
    const bool fix = box_strips4(g, c.i0, c.j0, T::TZH, K);
    const bool lean = !fix && tile_plain4(g, c.i0, c.j0, T::TZH, T::M);
    if (fix) pml_table4<SH>(g, m, c.i0 - K, c.j0, tab, tid);   // ordered before use by the first wait's barrier
    const int rd = o.ping, wr = 1 - o.ping;
    const int jb = c.j0 + 2 * tx;
    bool colin[2];
    colin[0] = jb >= T::M && jb <= g.nx - 1 - T::M;
    colin[1] = jb + 1 >= T::M && jb + 1 <= g.nx - 1 - T::M;
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
        const float *hown = own + L4<FD>::OWNB3;   // [sxx, szz, sxz][TZH][TX4] carry-in (htma)
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
        float wzz[T::W][2], wzxz[T::W][2];
        zwin2<T::W, RPT>(wzz, aZZ, ty, tx);
        zwin2<T::W, RPT>(wzxz, sZXZ, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
        // LEAN: an interior tile whose box needs no fix-up, without this
        // shot's source (no per-cell guards)
        auto rows = [&](auto lean_c) {
        constexpr bool LEAN = decltype(lean_c)::value;
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
            const bool rowin = i >= T::M && i <= g.nz - 1 - T::M;
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
                if (LEAN || (colin[cc] && rowin)) {
                    sxx = g.dtdx * a_tdp<FD, false>(axx, cc, j, g.nx);
                    szz = g.dtdz * w_tdp<FD, false>(wzz, r, cc, i, g.nz);
                    sxz = g.dtdz * w_tdm<FD, false>(wzxz, r, cc, i, g.nz, g.nz - 1)
                        + g.dtdx * a_tdm<FD, false>(axz, cc, j, g.nx, g.nx - 1);
                } else {
                    if (i < g.nz - 1) {
                        sxx = g.dtdx * a_tdp<FD, true>(axx, cc, j, g.nx);
                        sxz = g.dtdx * a_tdm<FD, true>(axz, cc, j, g.nx, g.nx - 1);
                    }
                    if (j >= 1 && j < g.nx - 1) {
                        szz = g.dtdz * w_tdp<FD, true>(wzz, r, cc, i, g.nz);
                        sxz += g.dtdz * w_tdm<FD, true>(wzxz, r, cc, i, g.nz, g.nz - 1);
                        if (g.fs && i == 0) sxz += 2.f * cf<FD>(1) * g.dtdz * wzxz[r + K][cc];
                    }
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
                                double *acc = o.acc + (long long)blockIdx.y * o.accp * g.nd +
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
        if (lean && !in_tile4(ssz, ssx, c.i0, c.j0, T::TZH)) rows(std::true_type{});
        else rows(std::false_type{});
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4 + OWNB + hbytes);
            tma_load_4d(S, &tmPQ, bar + (it & 1), c.j0 - XO4, c.i0 - K, F_U, s + 2);
            tma_load_4d(S + T::S2, &tmEo, bar + (it & 1), c.j0, c.i0, F_EX, s + 2);
            if (htma) tma_load_4d(S + T::S2 + L4<FD>::OWNB3, &tmH, bar + (it & 1), hx, hy, hz, s + 2);
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
                    double *acc = o.acc + (long long)blockIdx.y * o.accp * g.nd + (long long)pi * g.nx_dom + pj;
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
