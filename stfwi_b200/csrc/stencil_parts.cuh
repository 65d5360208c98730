// Tiling, staging plans and stencil pieces of the stencil kernels (sm_100a).
//
// Every thread owns TWO adjacent columns of RPT rows: a tile is 64 columns
// wide, the x-neighbourhood of a thread's two columns on one row is five
// aligned float2 shared loads (columns j-4 .. j+5), and the z-stencils come
// from a register window of RPT + 2K rows.  Halo tiles arrive by TMA (one 4-D
// bulk tensor copy per shot, double-buffered over the shots a block owns).
// The forward carries stresses (sxx = L2M ex + L ez, szz = L ex + L2M ez,
// sxz = 2 M es) instead of strains and the adjoint the buoyancy-scaled
// velocities P = B U_a, Q = B V_a: exact changes of variables that remove
// the halo transforms from the interior tiles.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace stfwi {

#ifndef STFWI_MINBLOCKS
#define STFWI_MINBLOCKS 2
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

// rows per thread: every kernel is built for 1 and 2 (8- and 16-row tiles);
// a handle runs fwd_vel, fwd_str and adj_a on one tile height and adj_b on
// another, chosen by the autotuner (2 and 2 until it has run)
constexpr int RPT_MIN = 1, RPT_DEFAULT = 2;

// shared-memory plan of R rows per thread; the velocity, stress and adj_a
// kernels use the A-layout members, adj_b the B-layout ones
template <int FD, int R> struct L4 {
    using A = G4<FD, R>;
    using B = G4<FD, R>;
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

}  // namespace stfwi
