// Register-blocked, TMA-fed stencil kernels (sm_100a), the default path.
//
// Same operator as kernels.cuh (which documents the correspondence with the
// reference, fwi/forward.py:250-469 and fwi/adjoint_jax_kernel.py:189-476),
// with two changes of variables that are exact in real arithmetic:
//  * forward state in stresses: sxx = L2M ex + L ez, szz = L ex + L2M ez,
//    sxz = 2 M es are carried instead of the strains.  The velocity phase
//    then differentiates the state directly; the strain phase updates the
//    stresses pointwise from the strain increments.  Strains are recovered
//    pointwise where they are needed (receivers, history, illumination);
//  * adjoint velocities scaled by the buoyancy: P = B U_a, Q = B V_a.  The
//    adjoint phases then read their staged inputs without a transform,
//    except in tiles that touch a C-PML strip or the free surface, where a
//    fix-up pass applies the C-PML transpose and the boundary terms in place.
// Each thread owns one column of RPT consecutive rows: z-stencils come from a
// register window of RPT + 2K values, x-stencils from the staged tile.
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace stfwi {

#ifndef STFWI_V3_MINBLOCKS
#define STFWI_V3_MINBLOCKS 4
#endif
#ifndef STFWI_V3_MINBLOCKS_HEAVY
#define STFWI_V3_MINBLOCKS_HEAVY 3   // fwd_str and adj_b hold more per-thread state
#endif
#ifndef STFWI_V3_RPT
#define STFWI_V3_RPT 4
#endif
constexpr int RPT3 = STFWI_V3_RPT;   // rows per thread of fwd_vel, fwd_str, adj_a

constexpr int XO3 = 4;               // x halo of the staged tile (box width 40 floats = 160 B)
constexpr int SW3 = TX + 2 * XO3;
constexpr uint32_t WAIT3 = 1u << 22; // mbarrier polls before a wait gives up
constexpr int ST_TIMEOUT3 = 2;

__host__ __device__ constexpr int al32_3(int x) { return (x + 31) / 32 * 32; }

template <int FD, int RPT> struct G3 {
    static constexpr int K = FD / 2;
    static constexpr int TZH = RPT * NWARP;  // tile height
    static constexpr int SH = TZH + 2 * K;
    static constexpr int SN = SH * SW3;
    static constexpr int W = RPT + 2 * K;   // z window
    static constexpr int M = 2 * K + 1;     // interior margin: no slice mask applies
    static constexpr int S1 = al32_3(SN), S2 = al32_3(2 * SN), S3 = al32_3(3 * SN);
};

template <int FD> struct L3 {               // shared-memory plans (floats)
    using A = G3<FD, RPT3>;                 // RPT3*8-row tiles: fwd_vel, fwd_str, adj_a
    using B = G3<FD, 4>;                    // 32-row tiles: adj_b (FP64 sums in registers)
    static constexpr int VEL = 2 * A::S3;
    static constexpr int STR = 2 * A::S2;
    static constexpr int ADA = 2 * A::S3 + A::S1;
    static constexpr int ADB = 2 * B::S2 + 2 * B::S1;
    static constexpr size_t bytes(int floats, int nbar) { return (size_t)floats * 4 + 8 * nbar; }
};

// ------------------------------------------------------------- stencil pieces

template <int FD, bool MASK>
__device__ __forceinline__ float x_dp(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mP(j, k, n)) d += cf<FD>(k) * (s[q + k] - s[q - k + 1]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float x_dm(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mM(j, k, n)) d += cf<FD>(k) * (s[q + k - 1] - s[q - k]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float x_tdp(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        if (!MASK || mP(j - k, k, n)) d += cf<FD>(k) * s[q - k];
        if (!MASK || mP(j + k - 1, k, n)) d -= cf<FD>(k) * s[q + k - 1];
    }
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float x_tdm(const float *s, int q, int j, int n, int lim)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const int t1 = j - k + 1, t2 = j + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += cf<FD>(k) * s[q - k + 1];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= cf<FD>(k) * s[q + k];
    }
    return d;
}
// z stencils on a register window w (row r of the thread at w[r + K])
template <int FD, bool MASK, int W>
__device__ __forceinline__ float z_dp(const float (&w)[W], int r, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k)
        if (!MASK || mP(i, k, n)) d += cf<FD>(k) * (w[r + K + k] - w[r + K - k + 1]);
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float z_dm(const float (&w)[W], int r, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k)
        if (!MASK || mM(i, k, n)) d += cf<FD>(k) * (w[r + K + k - 1] - w[r + K - k]);
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float z_tdp(const float (&w)[W], int r, int i, int n)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        if (!MASK || mP(i - k, k, n)) d += cf<FD>(k) * w[r + K - k];
        if (!MASK || mP(i + k - 1, k, n)) d -= cf<FD>(k) * w[r + K + k - 1];
    }
    return d;
}
template <int FD, bool MASK, int W>
__device__ __forceinline__ float z_tdm(const float (&w)[W], int r, int i, int n, int lim)
{
    constexpr int K = FD / 2;
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        const int t1 = i - k + 1, t2 = i + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += cf<FD>(k) * w[r + K - k + 1];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= cf<FD>(k) * w[r + K + k];
    }
    return d;
}

template <int W, int RPT>
__device__ __forceinline__ void load_window(float (&w)[W], const float *s, int ty, int tx)
{
#pragma unroll
    for (int m = 0; m < W; ++m) w[m] = s[(ty * RPT + m) * SW3 + tx + XO3];
}

struct Ctx3 {
    int tile, j0, i0, s0, s1;
};

__device__ __forceinline__ Ctx3 ctx3(const Geo &g, int spg, int tzh, int tiles_x)
{
    Ctx3 c;
    c.tile = blockIdx.x;
    c.j0 = (c.tile % tiles_x) * TX;
    c.i0 = (c.tile / tiles_x) * tzh;
    c.s0 = blockIdx.y * spg;
    c.s1 = min(c.s0 + spg, g.nshot);
    return c;
}

__device__ __forceinline__ void abort3(uint64_t *bar, int nbar, int *status)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicOr(status, ST_TIMEOUT3);
        for (int b = 0; b < nbar; ++b) {
            mbar_wait_bounded(bar + b, 0, WAIT3);
            mbar_wait_bounded(bar + b, 1, WAIT3);
        }
    }
}

// does the staged box [i0-K, i0+tzh+K) x [j0-XO3, j0+TX+XO3) contain a cell of
// a C-PML strip or the free-surface row (the cells needing the fix-up pass)?
__device__ __forceinline__ bool box_special(const Geo &g, int i0, int j0, int tzh, int K)
{
    const int r0 = i0 - K, r1 = i0 + tzh + K - 1, c0 = j0 - XO3, c1 = j0 + TX + XO3 - 1;
    if (c0 < g.pad || c1 >= g.nx - g.pad) return true;
    if (r1 >= g.nz - g.pad) return true;
    if (r0 <= 0) return true;                 // free-surface row 0, or the top strip
    if (!g.fs && r0 < g.pad) return true;
    return false;
}

// strains from stresses at one cell (inverse of the 2x2 normal-stress law and sxz = 2 M es)
__device__ __forceinline__ void strains_of(float sxx, float szz, float sxz, float l2m, float l, float mm,
                                           float &ex, float &ez, float &es)
{
    const float idet = 1.0f / ((l2m - l) * (l2m + l));
    ex = (l2m * sxx - l * szz) * idet;
    ez = (l2m * szz - l * sxx) * idet;
    es = sxz / (2.f * mm);
}

// ------------------------------------------------------------- forward: velocities

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_V3_MINBLOCKS)
    k3_fwd_vel(Geo g, Mat m, Shots sh, float *F, float *PX, float *PZ, int n, int spg, int tiles_x, int *status,
               const __grid_constant__ CUtensorMap tmS)
{
    using T = G3<FD, RPT3>;
    constexpr int K = T::K, SN = T::SN, RPT = RPT3;
    extern __shared__ __align__(128) float sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L3<FD>::VEL);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx3(g, spg, T::TZH, tiles_x);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 3 * SN * 4);
            tma_load_4d(sm + b * T::S3, &tmS, bar + b, c.j0 - XO3, c.i0 - K, F_EX, c.s0 + b);
        }
    }
    __syncthreads();
    const int j = c.j0 + tx;
    const int xs = (j < g.nx) ? xstrip_index(g, j) : -1;
    float bxv = 0.f, axv = 0.f, ikxv = 1.f;
    if (xs >= 0) { bxv = m.bx[j]; axv = m.ax[j]; ikxv = m.ikx[j]; }
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    float Bc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = c.i0 + ty * RPT + r;
        Bc[r] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
    }

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * T::S3;
        float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        float u[RPT], v[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz - 1 && j >= 1 && j < g.nx - 1;
            u[r] = ok ? U[o] : 0.f;
            v[r] = ok ? V[o] : 0.f;
        }
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT3))) {
            abort3(bar, 2, status);
            return;
        }
        const float *sxx = S, *szz = S + SN, *sxz = S + 2 * SN;
        float wxz[T::W], wzz[T::W];
        load_window<T::W, RPT>(wxz, sxz, ty, tx);
        load_window<T::W, RPT>(wzz, szz, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz - 1 || j < 1 || j >= g.nx - 1) continue;
            const int q = (ty * RPT + r + K) * SW3 + tx + XO3;
            float dxx, dzxz, dxxz, dzz;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                dxx = x_dp<FD, false>(sxx, q, j, g.nx);
                dxxz = x_dm<FD, false>(sxz, q, j, g.nx);
                dzxz = z_dm<FD, false>(wxz, r, i, g.nz);
                dzz = z_dp<FD, false>(wzz, r, i, g.nz);
            } else {
                dxx = x_dp<FD, true>(sxx, q, j, g.nx);
                dxxz = x_dm<FD, true>(sxz, q, j, g.nx);
                dzxz = z_dm<FD, true>(wxz, r, i, g.nz);
                dzz = z_dp<FD, true>(wzz, r, i, g.nz);
                if (g.fs && i == 0) dzxz = 2.f * cf<FD>(1) * wxz[r + K];
            }
            if (xs >= 0) {
                dxx = pml_fwd(dxx, bxv, axv, ikxv, px_ptr(g, PX, s, PX_SXX) + (long long)i * g.xs_n + xs);
                dxxz = pml_fwd(dxxz, bxv, axv, ikxv, px_ptr(g, PX, s, PX_SXZ) + (long long)i * g.xs_n + xs);
            }
            const int zs = zstrip_index(g, i);
            if (zs >= 0) {
                const float b = m.bz[i], a = m.az[i], ik = m.ikz[i];
                dzxz = pml_fwd(dzxz, b, a, ik, pz_ptr(g, PZ, s, PZ_SXZ) + (long long)zs * g.P + j);
                dzz = pml_fwd(dzz, b, a, ik, pz_ptr(g, PZ, s, PZ_SZZ) + (long long)zs * g.P + j);
            }
            const long long o = (long long)i * g.P + j;
            U[o] = u[r] + g.dtdx * Bc[r] * dxx + g.dtdz * Bc[r] * dzxz;
            float vv = v[r] + g.dtdx * Bc[r] * dxxz + g.dtdz * Bc[r] * dzz;
            if (stype == 0 && i == ssz && j == ssx) vv = vv + sh.fcoef[s] * sh.wav[(long long)s * g.nt + n];
            V[o] = vv;
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4);
            tma_load_4d(S, &tmS, bar + (it & 1), c.j0 - XO3, c.i0 - K, F_EX, s + 2);
        }
    }
}

// ------------------------------------------------------------- forward: stresses

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_V3_MINBLOCKS_HEAVY)
    k3_fwd_str(Geo g, Mat m, Shots sh, Recv rv, float *F, float *PX, float *PZ, int n, int spg, int tiles_x,
               FwdOut out, const __grid_constant__ CUtensorMap tmV)
{
    using T = G3<FD, RPT3>;
    constexpr int K = T::K, SN = T::SN, RPT = RPT3;
    extern __shared__ __align__(128) float sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L3<FD>::STR);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx3(g, spg, T::TZH, tiles_x);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 2 * SN * 4);
            tma_load_4d(sm + b * T::S2, &tmV, bar + b, c.j0 - XO3, c.i0 - K, F_U, c.s0 + b);
        }
    }
    __syncthreads();
    const int j = c.j0 + tx;
    const int xs = (j < g.nx) ? xstrip_index(g, j) : -1;
    float bxv = 0.f, axv = 0.f, ikxv = 1.f;
    if (xs >= 0) { bxv = m.bx[j]; axv = m.ax[j]; ikxv = m.ikx[j]; }
    const float Lr0 = (g.fs && j < g.nx) ? m.Lr[j] : 0.f;
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    double eacc[RPT];
    float ml2m[RPT], ml[RPT], mm2[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        eacc[r] = 0.0;
        const int i = c.i0 + ty * RPT + r;
        const long long o = (long long)i * g.P + j;
        const bool ok = i < g.nz && j < g.nx;
        ml2m[r] = ok ? m.L2M[o] : 0.f;
        ml[r] = ok ? m.L[o] : 0.f;
        mm2[r] = ok ? 2.f * m.M[o] : 0.f;
    }

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * T::S2;
        float *sxx = F + ((long long)s * F_N + F_EX) * g.fstride;
        float *szz = F + ((long long)s * F_N + F_EZ) * g.fstride;
        float *sxz = F + ((long long)s * F_N + F_ES) * g.fstride;
        float e1[RPT], e2[RPT], e3[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            e1[r] = ok ? sxx[o] : 0.f;
            e2[r] = ok ? szz[o] : 0.f;
            e3[r] = ok ? sxz[o] : 0.f;
        }
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT3))) {
            abort3(bar, 2, out.status);
            return;
        }
        const float *sU = S, *sV = S + SN;
        float wU[T::W], wV[T::W];
        load_window<T::W, RPT>(wU, sU, ty, tx);
        load_window<T::W, RPT>(wV, sV, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SW3 + tx + XO3;
            const int zs = zstrip_index(g, i);
            float dxu, dzv, dzu, dxv;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                dxu = x_dm<FD, false>(sU, q, j, g.nx);
                dxv = x_dp<FD, false>(sV, q, j, g.nx);
                dzv = z_dm<FD, false>(wV, r, i, g.nz);
                dzu = z_dp<FD, false>(wU, r, i, g.nz);
            } else {
                dxu = x_dm<FD, true>(sU, q, j, g.nx);
                dxv = x_dp<FD, true>(sV, q, j, g.nx);
                dzv = z_dm<FD, true>(wV, r, i, g.nz);
                dzu = z_dp<FD, true>(wU, r, i, g.nz);
            }
            if (j >= 1 && xs >= 0)
                dxu = pml_fwd(dxu, bxv, axv, ikxv, px_ptr(g, PX, s, PX_DXU) + (long long)i * g.xs_n + xs);
            if (j < g.nx - 1) {
                if (g.fs && i == 0) dzv = Lr0 * dxu * g.dzdx;
                if (zs >= 0)
                    dzv = pml_fwd(dzv, m.bz[i], m.az[i], m.ikz[i], pz_ptr(g, PZ, s, PZ_DZV) + (long long)zs * g.P + j);
            } else {
                dzv = 0.f;
            }
            if (j >= 1) {
                if (zs >= 0)
                    dzu = pml_fwd(dzu, m.bz[i], m.az[i], m.ikz[i], pz_ptr(g, PZ, s, PZ_DZU) + (long long)zs * g.P + j);
            } else {
                dzu = 0.f;
            }
            if (i < g.nz - 1) {
                if (xs >= 0)
                    dxv = pml_fwd(dxv, bxv, axv, ikxv, px_ptr(g, PX, s, PX_DXV) + (long long)i * g.xs_n + xs);
            } else {
                dxv = 0.f;
            }
            // strain increments of the reference's updates, applied to the stresses
            const float dex = (j >= 1) ? g.dtdx * dxu : 0.f;
            const float dez = g.dtdz * dzv;
            const float des = (i < g.nz - 1 && j < g.nx - 1) ? 0.5f * (g.dtdz * dzu + g.dtdx * dxv) : 0.f;
            const long long o = (long long)i * g.P + j;
            const float l2m = ml2m[r], l = ml[r];
            float axx = e1[r] + l2m * dex + l * dez;
            float azz = e2[r] + l * dex + l2m * dez;
            const float axz = e3[r] + mm2[r] * des;
            if (stype == 1 && i == ssz && j == ssx) {
                const float stm = sh.wav[(long long)s * g.nt + n] * g.dt / sh.mcoef[s];
                axx = axx + (l2m + l) * stm;
                azz = azz + (l + l2m) * stm;
            }
            sxx[o] = axx; szz[o] = azz; sxz[o] = axz;
            const int pi = i - g.z0, pj = j - g.pad;
            const bool phys = pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom;
            if (out.snap && phys) {
                float *sp = out.snap + ((long long)s * out.slots + out.slot) * g.snf * g.nd + (long long)pi * g.nx_dom + pj;
                __stcs(sp, axx);
                __stcs(sp + g.nd, azz);
                __stcs(sp + 2 * g.nd, axz);
            }
            if (out.row0 && g.fs && i == 0 && pj >= 0 && pj < g.nx_dom)
                out.row0[((long long)s * out.slots + out.slot_row0) * g.nx_dom + pj] = dxu;
            if (out.energy) {
                float f;
                if (out.energy_comp < 2) {
                    f = out.energy_comp == 0 ? sU[q] : sV[q];
                } else {
                    float ex, ez, es;
                    strains_of(axx, azz, axz, l2m, l, 0.5f * mm2[r], ex, ez, es);
                    f = out.energy_comp == 2 ? ex : ez;
                }
                eacc[r] += (double)f * (double)f;
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4);
            tma_load_4d(S, &tmV, bar + (it & 1), c.j0 - XO3, c.i0 - K, F_U, s + 2);
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
    if (out.energy) {
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i < g.nz && j < g.nx) atomicAdd(out.energy + (long long)i * g.nx + j, eacc[r]);
        }
    }
}

// ------------------------------------------------------------- adjoint: P = B U_a, Q = B V_a

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_V3_MINBLOCKS)
    k3_adj_a(Geo g, Mat m, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x, AdjIn in,
             int *status, const __grid_constant__ CUtensorMap tmE)
{
    using T = G3<FD, RPT3>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH, RPT = RPT3;
    extern __shared__ __align__(128) float sm[];
    float *aDxV = sm + 2 * T::S3;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L3<FD>::ADA);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx3(g, spg, T::TZH, tiles_x);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 3 * SN * 4);
            tma_load_4d(sm + b * T::S3, &tmE, bar + b, c.j0 - XO3, c.i0 - K, F_EX, c.s0 + b);
        }
    }
    __syncthreads();
    const bool fix = box_special(g, c.i0, c.j0, T::TZH, K);
    const int rd = in.ping, wr = 1 - in.ping;
    const int j = c.j0 + tx;
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    const float hdtdz = 0.5f * g.dtdz, hdtdx = 0.5f * g.dtdx;
    float Bc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = c.i0 + ty * RPT + r;
        Bc[r] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
    }
    double glr = 0.0;

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * T::S3;   // exa, eza, esa -> Dx_U_a/dtdx, Dz_V_a/dtdz, Dz_U_a/(dtdz/2)
        float *Pp = A + ((long long)s * F_N + F_U) * g.fstride;
        float *Qp = A + ((long long)s * F_N + F_V) * g.fstride;
        float p[RPT], qv[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            p[r] = ok ? Pp[o] : 0.f;
            qv[r] = ok ? Qp[o] : 0.f;
        }
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT3))) {
            abort3(bar, 2, status);
            return;
        }
        if (fix) {
            // the C-PML transpose (fwi/adjoint_jax_kernel.py:51-54), the
            // free-surface term and the slice limits of the strain updates,
            // in the scaled units the gathers use
            const float *pDzU = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZU);
            const float *pDzV = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZV);
            const float *pDxU = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXU);
            const float *pDxV = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXV);
            float *wDzU = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZU);
            float *wDzV = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZV);
            float *wDxU = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXU);
            float *wDxV = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXV);
            for (int rr = ty; rr < SH; rr += NWARP) {
                const int i = c.i0 - K + rr;
                for (int cc = tx; cc < SW3; cc += TX) {
                    const int jj = c.j0 - XO3 + cc, q = rr * SW3 + cc;
                    const float ea = S[q], za = S[SN + q], sa = S[2 * SN + q];
                    float vDxU = ea, vDzV = za, vDzU = sa, vDxV = sa;
                    if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                        const bool own = rr >= K && rr < K + T::TZH && cc >= XO3 && cc < XO3 + TX;
                        const int xs = xstrip_index(g, jj), zs = zstrip_index(g, i);
                        if (zs >= 0) {
                            const long long pz = (long long)zs * g.P + jj;
                            const float b = m.bz[i], a = m.az[i], ik = m.ikz[i], ps = pDzV[pz];
                            vDzV = (ik + a) * za + a * ps / g.dtdz;
                            if (own) wDzV[pz] = b * (g.dtdz * za + ps);
                        }
                        float din = (jj >= 1) ? ea : 0.f;
                        if (g.fs && i == 0 && jj < g.nx - 1) din = m.Lr[jj] * vDzV + din;
                        vDxU = din;
                        if (xs >= 0) {
                            const long long px = (long long)i * g.xs_n + xs;
                            const float b = m.bx[jj], a = m.ax[jj], ik = m.ikx[jj], ps = pDxU[px];
                            vDxU = (ik + a) * din + a * ps / g.dtdx;
                            if (own) wDxU[px] = b * (g.dtdx * din + ps);
                        }
                        const float h = (i < g.nz - 1 && jj < g.nx - 1) ? sa : 0.f;
                        vDzU = h;
                        vDxV = h;
                        if (zs >= 0) {
                            const long long pz = (long long)zs * g.P + jj;
                            const float b = m.bz[i], a = m.az[i], ik = m.ikz[i], ps = pDzU[pz];
                            vDzU = (ik + a) * h + a * ps / hdtdz;
                            if (own) wDzU[pz] = b * (hdtdz * h + ps);
                        }
                        if (xs >= 0) {
                            const long long px = (long long)i * g.xs_n + xs;
                            const float b = m.bx[jj], a = m.ax[jj], ik = m.ikx[jj], ps = pDxV[px];
                            vDxV = (ik + a) * h + a * ps / hdtdx;
                            if (own) wDxV[px] = b * (hdtdx * h + ps);
                        }
                    }
                    S[q] = vDxU; S[SN + q] = vDzV; S[2 * SN + q] = vDzU; aDxV[q] = vDxV;
                }
            }
            __syncthreads();
        }
        const float *aDxU = S, *aDzV = S + SN, *aDzU = S + 2 * SN;
        const float *aXV = fix ? aDxV : aDzU;
        float wzu[T::W], wzv[T::W];
        load_window<T::W, RPT>(wzu, aDzU, ty, tx);
        load_window<T::W, RPT>(wzv, aDzV, ty, tx);
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SW3 + tx + XO3;
            float gu, gv;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                gu = hdtdz * z_tdp<FD, false>(wzu, r, i, g.nz) + g.dtdx * x_tdm<FD, false>(aDxU, q, j, g.nx, g.nx);
                gv = hdtdx * x_tdp<FD, false>(aXV, q, j, g.nx) + g.dtdz * z_tdm<FD, false>(wzv, r, i, g.nz, g.nz);
            } else {
                gu = (j >= 1 ? hdtdz * z_tdp<FD, true>(wzu, r, i, g.nz) : 0.f)
                   + g.dtdx * x_tdm<FD, true>(aDxU, q, j, g.nx, g.nx);
                gv = (i < g.nz - 1 ? hdtdx * x_tdp<FD, true>(aXV, q, j, g.nx) : 0.f)
                   + (j < g.nx - 1 ? g.dtdz * z_tdm<FD, true>(wzv, r, i, g.nz, g.nz) : 0.f);
            }
            const long long o = (long long)i * g.P + j;
            Pp[o] = p[r] + Bc[r] * gu;
            Qp[o] = qv[r] + Bc[r] * gv;
            if (in.want_exact && g.fs && i == 0) {
                const int pj = j - g.pad;
                if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) {
                    const float du = in.row0[((long long)s * in.slots + in.slot) * g.nx_dom + pj];
                    glr += (double)(g.dtdz * wzv[r + K]) * (double)du * (double)g.dzdx;
                }
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4);
            tma_load_4d(S, &tmE, bar + (it & 1), c.j0 - XO3, c.i0 - K, F_EX, s + 2);
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
        const int pj = j - g.pad;
        if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) in.accLr[(long long)blockIdx.y * g.nx_dom + pj] += glr;
    }
}

// ------------------------------------------------------------- adjoint: strains + gradient

template <int FD, bool EXACT, bool IMG>
__global__ void __launch_bounds__(NTHR, STFWI_V3_MINBLOCKS_HEAVY)
    k3_adj_b(Geo g, Mat m, Shots sh, Recv rv, float *A, float *PX, float *PZ, int n, int spg, int tiles_x,
             AdjOut o, int *status, const __grid_constant__ CUtensorMap tmPQ)
{
    using T = G3<FD, 4>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH, RPT = 4;
    extern __shared__ __align__(128) float sm[];
    float *aZXZ = sm + 2 * T::S2, *aXXZ = aZXZ + T::S1;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L3<FD>::ADB);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const Ctx3 c = ctx3(g, spg, T::TZH, tiles_x);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        for (int b = 0; b < 2 && b < nsh; ++b) {
            mbar_arrive_expect_tx(bar + b, 2 * SN * 4);
            tma_load_4d(sm + b * T::S2, &tmPQ, bar + b, c.j0 - XO3, c.i0 - K, F_U, c.s0 + b);
        }
    }
    __syncthreads();
    const bool fix = box_special(g, c.i0, c.j0, T::TZH, K);
    const int rd = o.ping, wr = 1 - o.ping;
    const int j = c.j0 + tx;
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    float mL2M[RPT], mL[RPT], mM2[RPT], idet[RPT], i2m[RPT];
    constexpr int RE = EXACT ? RPT : 1, RI = IMG ? RPT : 1;
    double gM[RE], gL[RE], gL2M[RE], glam[RI], gmu[RI];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = c.i0 + ty * RPT + r;
        const bool inb = i < g.nz && j < g.nx;
        const long long off = (long long)i * g.P + j;
        mL2M[r] = inb ? m.L2M[off] : 0.f;
        mL[r] = inb ? m.L[off] : 0.f;
        mM2[r] = inb ? 2.f * m.M[off] : 0.f;
        // strain recovery factors (physical cells have M > 0 and L2M > |L|)
        idet[r] = inb ? 1.0f / ((mL2M[r] - mL[r]) * (mL2M[r] + mL[r])) : 0.f;
        i2m[r] = inb ? 1.0f / mM2[r] : 0.f;
    }
#pragma unroll
    for (int r = 0; r < RE; ++r) gM[r] = gL[r] = gL2M[r] = 0.0;
#pragma unroll
    for (int r = 0; r < RI; ++r) glam[r] = gmu[r] = 0.0;

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S = sm + (it & 1) * T::S2;   // P, Q -> A_XX/dtdx, A_ZZ/dtdz
        float *exa = A + ((long long)s * F_N + F_EX) * g.fstride;
        float *eza = A + ((long long)s * F_N + F_EZ) * g.fstride;
        float *esa = A + ((long long)s * F_N + F_ES) * g.fstride;
        const float *Pp = A + ((long long)s * F_N + F_U) * g.fstride;
        const float *Qp = A + ((long long)s * F_N + F_V) * g.fstride;
        const float *snap_in = (EXACT && o.slot_in >= 0)
                                   ? o.snap + ((long long)s * o.slots + o.slot_in) * g.snf * g.nd : nullptr;
        const float *snap_img = (IMG && o.slot_img >= 0)
                                    ? o.snap + ((long long)s * o.slots + o.slot_img) * g.snf * g.nd : nullptr;
        float ea[RPT], za[RPT], sa[RPT], h1[RPT], h2[RPT], h3[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long off = (long long)i * g.P + j;
            const bool inb = i < g.nz && j < g.nx;
            ea[r] = inb ? exa[off] : 0.f;
            za[r] = inb ? eza[off] : 0.f;
            sa[r] = inb ? esa[off] : 0.f;
            h1[r] = h2[r] = h3[r] = 0.f;
            const int pi = i - g.z0, pj = j - g.pad;
            if (EXACT && snap_in && inb && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                const long long pq = (long long)pi * g.nx_dom + pj;
                h1[r] = __ldcs(snap_in + pq);
                h2[r] = __ldcs(snap_in + g.nd + pq);
                h3[r] = __ldcs(snap_in + 2 * g.nd + pq);
            }
        }
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT3))) {
            abort3(bar, 2, status);
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
            for (int rr = ty; rr < SH; rr += NWARP) {
                const int i = c.i0 - K + rr;
                for (int cc = tx; cc < SW3; cc += TX) {
                    const int jj = c.j0 - XO3 + cc, q = rr * SW3 + cc;
                    float pv = 0.f, qq = 0.f;
                    if (i >= 0 && i < g.nz - 1 && jj >= 1 && jj < g.nx - 1) { pv = S[q]; qq = S[SN + q]; }
                    float vXX = pv, vZXZ = pv, vXXZ = qq, vZZ = qq;
                    if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                        const bool own = rr >= K && rr < K + T::TZH && cc >= XO3 && cc < XO3 + TX;
                        const int xs = xstrip_index(g, jj), zs = zstrip_index(g, i);
                        if (xs >= 0) {
                            const long long px = (long long)i * g.xs_n + xs;
                            const float b = m.bx[jj], a = m.ax[jj], ik = m.ikx[jj];
                            const float p0 = pXX[px], p1 = pXXZ[px];
                            vXX = (ik + a) * pv + a * p0 / g.dtdx;
                            vXXZ = (ik + a) * qq + a * p1 / g.dtdx;
                            if (own) {
                                wXX[px] = b * (g.dtdx * pv + p0);
                                wXXZ[px] = b * (g.dtdx * qq + p1);
                            }
                        }
                        if (zs >= 0) {
                            const long long pz = (long long)zs * g.P + jj;
                            const float b = m.bz[i], a = m.az[i], ik = m.ikz[i];
                            const float p0 = pZXZ[pz], p1 = pZZ[pz];
                            vZXZ = (ik + a) * pv + a * p0 / g.dtdz;
                            vZZ = (ik + a) * qq + a * p1 / g.dtdz;
                            if (own) {
                                wZXZ[pz] = b * (g.dtdz * pv + p0);
                                wZZ[pz] = b * (g.dtdz * qq + p1);
                            }
                        }
                    }
                    S[q] = vXX; S[SN + q] = vZZ; aZXZ[q] = vZXZ; aXXZ[q] = vXXZ;
                }
            }
            __syncthreads();
        }
        const float *aXX = S, *aZZ = S + SN;
        const float *sZXZ = fix ? aZXZ : S, *sXXZ = fix ? aXXZ : S + SN;
        float wzz[T::W], wzxz[T::W];
        load_window<T::W, RPT>(wzz, aZZ, ty, tx);
        load_window<T::W, RPT>(wzxz, sZXZ, ty, tx);
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SW3 + tx + XO3;
            float sxx = 0.f, szz = 0.f, sxz = 0.f;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                sxx = g.dtdx * x_tdp<FD, false>(aXX, q, j, g.nx);
                szz = g.dtdz * z_tdp<FD, false>(wzz, r, i, g.nz);
                sxz = g.dtdz * z_tdm<FD, false>(wzxz, r, i, g.nz, g.nz - 1)
                    + g.dtdx * x_tdm<FD, false>(sXXZ, q, j, g.nx, g.nx - 1);
            } else {
                if (i < g.nz - 1) {
                    sxx = g.dtdx * x_tdp<FD, true>(aXX, q, j, g.nx);
                    sxz = g.dtdx * x_tdm<FD, true>(sXXZ, q, j, g.nx, g.nx - 1);
                }
                if (j >= 1 && j < g.nx - 1) {
                    szz = g.dtdz * z_tdp<FD, true>(wzz, r, i, g.nz);
                    sxz += g.dtdz * z_tdm<FD, true>(wzxz, r, i, g.nz, g.nz - 1);
                    if (g.fs && i == 0) sxz += 2.f * cf<FD>(1) * g.dtdz * wzxz[r + K];
                }
            }
            const long long off = (long long)i * g.P + j;
            if (i == ssz && j == ssx) {
                const float w = sh.wav[(long long)s * g.nt + n];
                if (stype == 0) {
                    // dt/(dx dz) B V_a = dt/(dx dz) Q
                    if (o.src_a) o.src_a[(long long)s * g.nt + n] = g.dtdxdz * Qp[off];
                } else {
                    if (o.src_a) o.src_a[(long long)s * g.nt + n] = (g.dt / sh.mcoef[s]) * (ea[r] + za[r]);
                    if (EXACT) {
                        const double lm = sh.lm[s];
                        const double glm = -((double)w * g.dt / ((double)sh.mcoef[s] / lm)) / (lm * lm)
                                           * (double)(ea[r] + za[r]);
                        gM[r % RE] += glm;
                        gL[r % RE] += glm;
                    }
                }
            }
            exa[off] = ea[r] + mL2M[r] * sxx + mL[r] * szz;
            eza[off] = za[r] + mL[r] * sxx + mL2M[r] * szz;
            esa[off] = sa[r] + mM2[r] * sxz;
            if (EXACT) {
                // forward strains of the carry-in, from the stored stresses
                const float e1 = (mL2M[r] * h1[r] - mL[r] * h2[r]) * idet[r];
                const float e2 = (mL2M[r] * h2[r] - mL[r] * h1[r]) * idet[r];
                const float e3 = h3[r] * i2m[r];
                gL2M[r % RE] += (double)e1 * sxx + (double)e2 * szz;
                gL[r % RE] += (double)e2 * sxx + (double)e1 * szz;
                gM[r % RE] += 2.0 * (double)e3 * sxz;
            }
            const int pi = i - g.z0, pj = j - g.pad;
            if (IMG && snap_img && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                const long long pq = (long long)pi * g.nx_dom + pj;
                const int ip = (i + 1) % g.nz, im = (i - 1 + g.nz) % g.nz;
                const int jp = (j + 1) % g.nx, jm = (j - 1 + g.nx) % g.nx;
                const long long oxp = (long long)i * g.P + jp, oxm = (long long)i * g.P + jm;
                const long long ozp = (long long)ip * g.P + j, ozm = (long long)im * g.P + j;
                // fwi/imaging.py:125-141 on B U_a = P and B V_a = Q
                const float dxBU = (Pp[oxp] - Pp[oxm]) * g.inv2dx;
                const float dzBV = (Qp[ozp] - Qp[ozm]) * g.inv2dz;
                const float dzBU = (Pp[ozp] - Pp[ozm]) * g.inv2dz;
                const float dxBV = (Qp[oxp] - Qp[oxm]) * g.inv2dx;
                const float t1 = snap_img[pq], t2 = snap_img[g.nd + pq], t3 = snap_img[2 * g.nd + pq];
                const float e1 = (mL2M[r] * t1 - mL[r] * t2) * idet[r];
                const float e2 = (mL2M[r] * t2 - mL[r] * t1) * idet[r];
                const float e3 = t3 * i2m[r];
                glam[r % RI] -= (double)g.dt * (double)((e1 + e2) * (dxBU + dzBV));
                gmu[r % RI] -= (double)g.dt * (double)(2.f * e1 * dxBU + 2.f * e2 * dzBV + e3 * (dzBU + dxBV));
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4);
            tma_load_4d(S, &tmPQ, bar + (it & 1), c.j0 - XO3, c.i0 - K, F_U, s + 2);
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
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const int pi = i - g.z0, pj = j - g.pad;
            if (i < g.nz && j < g.nx && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                double *acc = o.acc + (long long)blockIdx.y * o.accp * g.nd + (long long)pi * g.nx_dom + pj;
                if (EXACT) {
                    acc[0] += gM[r % RE];
                    acc[g.nd] += gL[r % RE];
                    acc[2 * g.nd] += gL2M[r % RE];
                }
                if (IMG) {
                    acc[3 * g.nd] += glam[r % RI];
                    acc[4 * g.nd] += gmu[r % RI];
                }
            }
        }
    }
}

}  // namespace stfwi
