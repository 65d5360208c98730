// TMA-pipelined stencil kernels (sm_100a).
//
// Same four phases and the same arithmetic as kernels.cuh (which documents
// the reference correspondence), restructured for throughput:
//  * a block owns one 32x32 tile and loops over a group of shots;
//  * one thread issues, per shot, a single 4-D bulk tensor copy of the tile
//    plus its halo for every field the phase reads (strains, velocities or
//    their adjoints: adjacent field slots of the [shot][field][z][x] layout);
//    cells outside the grid arrive as zeros;
//  * the copies are double-buffered: shot s+2 streams in while shot s+1
//    waits and shot s computes;
//  * the padded material tile is copied once per block;
//  * cells at least 2K+1 cells from every grid edge skip the per-term slice
//    masks (all of them hold there); the others evaluate them exactly;
//  * every mbarrier wait is bounded: on expiry the block sets status bit 2
//    and returns.
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace stfwi {

#ifndef STFWI_TMA_MINBLOCKS
#define STFWI_TMA_MINBLOCKS 4
#endif
constexpr int XO = 4;                 // x halo staged by the copies (box width 40 floats = 160 B)
constexpr int SWT = TX + 2 * XO;      // smem row stride
constexpr uint32_t WAIT_LIMIT = 1u << 22;
constexpr int ST_TIMEOUT = 2;

__host__ __device__ constexpr int al32(int x) { return (x + 31) / 32 * 32; }

template <int FD> struct TileT {
    static constexpr int K = FD / 2;
    static constexpr int SH = TZ + 2 * K;
    static constexpr int SN = SH * SWT;   // one staged field
    static constexpr int M = 2 * K + 1;   // interior margin (mask-free cells)
    // shared-memory layouts (floats); copy destinations start on 128-byte boundaries
    static constexpr int S3 = al32(3 * SN), S2 = al32(2 * SN), S1 = al32(SN), S4 = al32(4 * SN);
    static constexpr int VEL = 2 * S3 + S4;       // fwd_vel: 2 stages x (ex,ez,es) + (B,L2M,L,M)
    static constexpr int STR = 2 * S2;            // fwd_str: 2 stages x (U,V)
    static constexpr int ADA = 2 * S3 + S1;       // adj_a: 2 stages x (exa,eza,esa) + Dx_V_a
    static constexpr int ADB = 2 * S2 + 3 * S1;   // adj_b: 2 stages x (Ua,Va) + ZXZ, XXZ, B
    static constexpr size_t bytes(int floats, int nbar) { return (size_t)floats * 4 + 8 * nbar; }
};

// ------------------------------------------------------------- masked / unmasked stencils
// q indexes the staged tile; SW is its row stride.

template <int FD, bool MASK>
__device__ __forceinline__ float st_dxp(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mP(j, k, n)) d += cf<FD>(k) * (s[q + k] - s[q - k + 1]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_dxm(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mM(j, k, n)) d += cf<FD>(k) * (s[q + k - 1] - s[q - k]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_dzp(const float *s, int q, int i, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mP(i, k, n)) d += cf<FD>(k) * (s[q + k * SWT] - s[q - (k - 1) * SWT]);
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_dzm(const float *s, int q, int i, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k)
        if (!MASK || mM(i, k, n)) d += cf<FD>(k) * (s[q + (k - 1) * SWT] - s[q - k * SWT]);
    return d;
}
// transposes: (D+x)^T, (D-x)^T, (D+z)^T, (D-z)^T; `lim` excludes source
// indices >= lim (the reference's narrower slice of some derivatives)
template <int FD, bool MASK>
__device__ __forceinline__ float st_tdxp(const float *s, int q, int j, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const float c = cf<FD>(k);
        if (!MASK || mP(j - k, k, n)) d += c * s[q - k];
        if (!MASK || mP(j + k - 1, k, n)) d -= c * s[q + k - 1];
    }
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_tdxm(const float *s, int q, int j, int n, int lim)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const float c = cf<FD>(k);
        const int t1 = j - k + 1, t2 = j + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += c * s[q - k + 1];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= c * s[q + k];
    }
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_tdzp(const float *s, int q, int i, int n)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const float c = cf<FD>(k);
        if (!MASK || mP(i - k, k, n)) d += c * s[q - k * SWT];
        if (!MASK || mP(i + k - 1, k, n)) d -= c * s[q + (k - 1) * SWT];
    }
    return d;
}
template <int FD, bool MASK>
__device__ __forceinline__ float st_tdzm(const float *s, int q, int i, int n, int lim)
{
    float d = 0.f;
#pragma unroll
    for (int k = 1; k <= FD / 2; ++k) {
        const float c = cf<FD>(k);
        const int t1 = i - k + 1, t2 = i + k;
        if (!MASK || (mM(t1, k, n) && t1 < lim)) d += c * s[q - (k - 1) * SWT];
        if (!MASK || (mM(t2, k, n) && t2 < lim)) d -= c * s[q + k * SWT];
    }
    return d;
}

// ------------------------------------------------------------- pipeline scaffolding

struct TmaCtx {
    int tile, j0, i0, s0, s1;
};

__device__ __forceinline__ TmaCtx tma_ctx(const Geo &g, int spg)
{
    TmaCtx c;
    c.tile = blockIdx.x;
    const int tx_ = c.tile % g.tiles_x, tz_ = c.tile / g.tiles_x;
    c.j0 = tx_ * TX;
    c.i0 = tz_ * TZ;
    c.s0 = blockIdx.y * spg;
    c.s1 = min(c.s0 + spg, g.nshot);
    return c;
}

// after a failed wait: flag it, then give the copies still in flight a bounded
// chance to land before the block's shared memory is released
__device__ __forceinline__ void tma_abort(uint64_t *bar, int nbar, int *status)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicOr(status, ST_TIMEOUT);
        for (int b = 0; b < nbar; ++b) {
            mbar_wait_bounded(bar + b, 0, WAIT_LIMIT);
            mbar_wait_bounded(bar + b, 1, WAIT_LIMIT);
        }
    }
}

// ------------------------------------------------------------- forward: velocities

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_TMA_MINBLOCKS)
    k_fwd_vel_t(Geo g, Mat m, Shots sh, float *F, float *PX, float *PZ, int n, int spg, int *status,
                const __grid_constant__ CUtensorMap tmF, const __grid_constant__ CUtensorMap tmM)
{
    using T = TileT<FD>;
    constexpr int K = T::K, SN = T::SN;
    extern __shared__ __align__(128) float sm[];
    float *stage0 = sm, *stage1 = sm + T::S3, *mat = sm + 2 * T::S3;  // mat: B, L2M, L, M
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + T::VEL);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const TmaCtx c = tma_ctx(g, spg);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1); mbar_init(bar + 2, 1);
        fence_async_shared();
        mbar_arrive_expect_tx(bar + 2, 4 * SN * 4);
        tma_load_3d(mat, &tmM, bar + 2, c.j0 - XO, c.i0 - K, 0);
        mbar_arrive_expect_tx(bar + 0, 3 * SN * 4);
        tma_load_4d(stage0, &tmF, bar + 0, c.j0 - XO, c.i0 - K, F_EX, c.s0);
        if (nsh > 1) {
            mbar_arrive_expect_tx(bar + 1, 3 * SN * 4);
            tma_load_4d(stage1, &tmF, bar + 1, c.j0 - XO, c.i0 - K, F_EX, c.s0 + 1);
        }
    }
    __syncthreads();
    const int j = c.j0 + tx;
    const int xs = (j < g.nx) ? xstrip_index(g, j) : -1;
    float bxv = 0.f, axv = 0.f, ikxv = 1.f;
    if (xs >= 0) { bxv = m.bx[j]; axv = m.ax[j]; ikxv = m.ikx[j]; }
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    if (!__syncthreads_and(mbar_wait_bounded(bar + 2, 0, WAIT_LIMIT))) { tma_abort(bar, 2, status); return; }

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S3 = (it & 1) ? stage1 : stage0;
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
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT_LIMIT))) {
            tma_abort(bar, 2, status);
            return;
        }
        // stresses in place: ex -> sxx, ez -> szz, es -> sxz
        for (int q = tid; q < SN; q += NTHR) {
            const float e1 = S3[q], e2 = S3[SN + q], e3 = S3[2 * SN + q];
            const float l2m = mat[SN + q], l = mat[2 * SN + q], mm = mat[3 * SN + q];
            S3[q] = l2m * e1 + l * e2;
            S3[SN + q] = l * e1 + l2m * e2;
            S3[2 * SN + q] = 2.f * mm * e3;
        }
        __syncthreads();
        const float *sxx = S3, *szz = S3 + SN, *sxz = S3 + 2 * SN;
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz - 1 || j < 1 || j >= g.nx - 1) continue;
            const int q = (ty * RPT + r + K) * SWT + tx + XO;
            float dxx, dzxz, dxxz, dzz;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                dxx = st_dxp<FD, false>(sxx, q, j, g.nx);
                dzxz = st_dzm<FD, false>(sxz, q, i, g.nz);
                dxxz = st_dxm<FD, false>(sxz, q, j, g.nx);
                dzz = st_dzp<FD, false>(szz, q, i, g.nz);
            } else {
                dxx = st_dxp<FD, true>(sxx, q, j, g.nx);
                dzxz = st_dzm<FD, true>(sxz, q, i, g.nz);
                dxxz = st_dxm<FD, true>(sxz, q, j, g.nx);
                dzz = st_dzp<FD, true>(szz, q, i, g.nz);
                if (g.fs && i == 0) dzxz = 2.f * cf<FD>(1) * sxz[q];
            }
            if (xs >= 0) {
                float *p0 = px_ptr(g, PX, s, PX_SXX) + (long long)i * g.xs_n + xs;
                float *p1 = px_ptr(g, PX, s, PX_SXZ) + (long long)i * g.xs_n + xs;
                dxx = pml_fwd(dxx, bxv, axv, ikxv, p0);
                dxxz = pml_fwd(dxxz, bxv, axv, ikxv, p1);
            }
            const int zs = zstrip_index(g, i);
            if (zs >= 0) {
                const float b = m.bz[i], a = m.az[i], ik = m.ikz[i];
                dzxz = pml_fwd(dzxz, b, a, ik, pz_ptr(g, PZ, s, PZ_SXZ) + (long long)zs * g.P + j);
                dzz = pml_fwd(dzz, b, a, ik, pz_ptr(g, PZ, s, PZ_SZZ) + (long long)zs * g.P + j);
            }
            const long long o = (long long)i * g.P + j;
            const float Bv = mat[q];
            U[o] = u[r] + g.dtdx * Bv * dxx + g.dtdz * Bv * dzxz;
            float vv = v[r] + g.dtdx * Bv * dxxz + g.dtdz * Bv * dzz;
            if (stype == 0 && i == ssz && j == ssx) vv = vv + sh.fcoef[s] * sh.wav[(long long)s * g.nt + n];
            V[o] = vv;
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4);
            tma_load_4d(S3, &tmF, bar + (it & 1), c.j0 - XO, c.i0 - K, F_EX, s + 2);
        }
    }
}

// ------------------------------------------------------------- forward: strains

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_TMA_MINBLOCKS)
    k_fwd_str_t(Geo g, Mat m, Shots sh, Recv rv, float *F, float *PX, float *PZ, int n, int spg, FwdOut out,
                const __grid_constant__ CUtensorMap tmF)
{
    using T = TileT<FD>;
    constexpr int K = T::K, SN = T::SN;
    extern __shared__ __align__(128) float sm[];
    float *stage0 = sm, *stage1 = sm + T::S2;  // U, V
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + T::STR);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const TmaCtx c = tma_ctx(g, spg);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        mbar_arrive_expect_tx(bar + 0, 2 * SN * 4);
        tma_load_4d(stage0, &tmF, bar + 0, c.j0 - XO, c.i0 - K, F_U, c.s0);
        if (nsh > 1) {
            mbar_arrive_expect_tx(bar + 1, 2 * SN * 4);
            tma_load_4d(stage1, &tmF, bar + 1, c.j0 - XO, c.i0 - K, F_U, c.s0 + 1);
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
#pragma unroll
    for (int r = 0; r < RPT; ++r) eacc[r] = 0.0;

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *SU = (it & 1) ? stage1 : stage0;
        const float *sU = SU, *sV = SU + SN;
        float *ex = F + ((long long)s * F_N + F_EX) * g.fstride;
        float *ez = F + ((long long)s * F_N + F_EZ) * g.fstride;
        float *es = F + ((long long)s * F_N + F_ES) * g.fstride;
        float e1[RPT], e2[RPT], e3[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            e1[r] = ok ? ex[o] : 0.f;
            e2[r] = ok ? ez[o] : 0.f;
            e3[r] = ok ? es[o] : 0.f;
        }
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT_LIMIT))) {
            tma_abort(bar, 2, out.status);
            return;
        }
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SWT + tx + XO;
            const int zs = zstrip_index(g, i);
            float dxu, dzv, dzu, dxv;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                dxu = st_dxm<FD, false>(sU, q, j, g.nx);
                dzv = st_dzm<FD, false>(sV, q, i, g.nz);
                dzu = st_dzp<FD, false>(sU, q, i, g.nz);
                dxv = st_dxp<FD, false>(sV, q, j, g.nx);
            } else {
                dxu = st_dxm<FD, true>(sU, q, j, g.nx);
                dzv = st_dzm<FD, true>(sV, q, i, g.nz);
                dzu = st_dzp<FD, true>(sU, q, i, g.nz);
                dxv = st_dxp<FD, true>(sV, q, j, g.nx);
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
            const long long o = (long long)i * g.P + j;
            float exn = e1[r], ezn = e2[r], esn = e3[r];
            if (j >= 1) exn = exn + g.dtdx * dxu;
            ezn = ezn + g.dtdz * dzv;
            if (stype == 1 && i == ssz && j == ssx) {
                const float stm = sh.wav[(long long)s * g.nt + n] * g.dt / sh.mcoef[s];
                exn = exn + stm;
                ezn = ezn + stm;
            }
            if (i < g.nz - 1 && j < g.nx - 1) esn = esn + 0.5f * (g.dtdz * dzu + g.dtdx * dxv);
            ex[o] = exn; ez[o] = ezn; es[o] = esn;
            const int pi = i - g.z0, pj = j - g.pad;
            const bool phys = pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom;
            if (out.snap && phys) {
                float *sp = out.snap + ((long long)s * out.slots + out.slot) * 3 * g.nd + (long long)pi * g.nx_dom + pj;
                __stcs(sp, exn);
                __stcs(sp + g.nd, ezn);
                __stcs(sp + 2 * g.nd, esn);
            }
            if (out.row0 && g.fs && i == 0 && pj >= 0 && pj < g.nx_dom)
                out.row0[((long long)s * out.slots + out.slot) * g.nx_dom + pj] = dxu;
            if (out.energy) {
                const float f = out.energy_comp == 2 ? exn : out.energy_comp == 3 ? ezn
                              : out.energy_comp == 0 ? sU[q] : sV[q];
                eacc[r] += (double)f * (double)f;
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4);
            tma_load_4d(SU, &tmF, bar + (it & 1), c.j0 - XO, c.i0 - K, F_U, s + 2);
        }
        // receivers of this tile: the tile's cells are final (read from global)
        const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
        const float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        const float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        for (int q = r0 + tid; q < r1; q += NTHR) {
            const int rid = rv.tile_rec[q];
            const long long o = (long long)rv.rz[rid] * g.P + rv.rx[rid];
            const float v0 = U[o], v1 = V[o], v2 = ex[o], v3 = ez[o];
            float *dst = out.rec + (long long)s * 4 * g.nt * g.nrec + (long long)n * g.nrec + rid;
            dst[0] = v0;
            dst[(long long)g.nt * g.nrec] = v1;
            dst[2LL * g.nt * g.nrec] = v2;
            dst[3LL * g.nt * g.nrec] = v3;
            if (!(isfinite(v0) && isfinite(v1) && isfinite(v2) && isfinite(v3))) atomicOr(out.status, 1);
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

// ------------------------------------------------------------- adjoint: velocities

template <int FD>
__global__ void __launch_bounds__(NTHR, STFWI_TMA_MINBLOCKS)
    k_adj_a_t(Geo g, Mat m, Recv rv, float *A, float *PX, float *PZ, int n, int spg, AdjIn in, int *status,
              const __grid_constant__ CUtensorMap tmA)
{
    using T = TileT<FD>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH;
    extern __shared__ __align__(128) float sm[];
    float *stage0 = sm, *stage1 = sm + T::S3, *aDxV = sm + 2 * T::S3;  // stage: exa, eza, esa
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + T::ADA);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const TmaCtx c = tma_ctx(g, spg);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1);
        fence_async_shared();
        mbar_arrive_expect_tx(bar + 0, 3 * SN * 4);
        tma_load_4d(stage0, &tmA, bar + 0, c.j0 - XO, c.i0 - K, F_EX, c.s0);
        if (nsh > 1) {
            mbar_arrive_expect_tx(bar + 1, 3 * SN * 4);
            tma_load_4d(stage1, &tmA, bar + 1, c.j0 - XO, c.i0 - K, F_EX, c.s0 + 1);
        }
    }
    __syncthreads();
    const int rd = in.ping, wr = 1 - in.ping;
    const int j = c.j0 + tx;
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    double glr = 0.0;

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S3 = (it & 1) ? stage1 : stage0;
        float *Ua = A + ((long long)s * F_N + F_U) * g.fstride;
        float *Va = A + ((long long)s * F_N + F_V) * g.fstride;
        float u[RPT], v[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            const long long o = (long long)i * g.P + j;
            const bool ok = i < g.nz && j < g.nx;
            u[r] = ok ? Ua[o] : 0.f;
            v[r] = ok ? Va[o] : 0.f;
        }
        const float *pDzU = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZU);
        const float *pDzV = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZV);
        const float *pDxU = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXU);
        const float *pDxV = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXV);
        float *wDzU = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZU);
        float *wDzV = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZV);
        float *wDxU = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXU);
        float *wDxV = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXV);
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT_LIMIT))) {
            tma_abort(bar, 2, status);
            return;
        }
        // derivative adjoints after the C-PML transpose, in place:
        // exa -> Dx_U_a, eza -> Dz_V_a, esa -> Dz_U_a, and Dx_V_a separately
        for (int rr = ty; rr < SH; rr += NWARP) {
            const int i = c.i0 - K + rr;
            for (int cc = tx; cc < SWT; cc += TX) {
                const int jj = c.j0 - XO + cc, q = rr * SWT + cc;
                float vDzU = 0.f, vDxU = 0.f, vDxV = 0.f, vDzV = 0.f;
                if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                    const bool own = rr >= K && rr < K + TZ && cc >= XO && cc < XO + TX;
                    const int xs = xstrip_index(g, jj), zs = zstrip_index(g, i);
                    const float ea = S3[q], za = S3[SN + q], sa = S3[2 * SN + q];
                    vDzV = g.dtdz * za;
                    if (zs >= 0) {
                        const long long pz = (long long)zs * g.P + jj;
                        vDzV = pml_adj(vDzV, m.bz[i], m.az[i], m.ikz[i], pDzV[pz], own ? wDzV + pz : nullptr);
                    }
                    float din = 0.f;
                    if (g.fs && i == 0 && jj < g.nx - 1) din = m.Lr[jj] * g.dzdx * vDzV;
                    if (jj >= 1) din = din + g.dtdx * ea;
                    vDxU = din;
                    if (xs >= 0) {
                        const long long px = (long long)i * g.xs_n + xs;
                        vDxU = pml_adj(din, m.bx[jj], m.ax[jj], m.ikx[jj], pDxU[px], own ? wDxU + px : nullptr);
                    }
                    const float h = (i < g.nz - 1 && jj < g.nx - 1) ? sa : 0.f;
                    vDzU = 0.5f * g.dtdz * h;
                    vDxV = 0.5f * g.dtdx * h;
                    if (zs >= 0) {
                        const long long pz = (long long)zs * g.P + jj;
                        vDzU = pml_adj(vDzU, m.bz[i], m.az[i], m.ikz[i], pDzU[pz], own ? wDzU + pz : nullptr);
                    }
                    if (xs >= 0) {
                        const long long px = (long long)i * g.xs_n + xs;
                        vDxV = pml_adj(vDxV, m.bx[jj], m.ax[jj], m.ikx[jj], pDxV[px], own ? wDxV + px : nullptr);
                    }
                }
                S3[q] = vDxU; S3[SN + q] = vDzV; S3[2 * SN + q] = vDzU; aDxV[q] = vDxV;
            }
        }
        __syncthreads();
        const float *aDxU = S3, *aDzV = S3 + SN, *aDzU = S3 + 2 * SN;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SWT + tx + XO;
            float gu, gv;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                gu = st_tdzp<FD, false>(aDzU, q, i, g.nz) + st_tdxm<FD, false>(aDxU, q, j, g.nx, g.nx);
                gv = st_tdxp<FD, false>(aDxV, q, j, g.nx) + st_tdzm<FD, false>(aDzV, q, i, g.nz, g.nz);
            } else {
                gu = (j >= 1 ? st_tdzp<FD, true>(aDzU, q, i, g.nz) : 0.f) + st_tdxm<FD, true>(aDxU, q, j, g.nx, g.nx);
                gv = (i < g.nz - 1 ? st_tdxp<FD, true>(aDxV, q, j, g.nx) : 0.f)
                   + (j < g.nx - 1 ? st_tdzm<FD, true>(aDzV, q, i, g.nz, g.nz) : 0.f);
            }
            const long long o = (long long)i * g.P + j;
            Ua[o] = u[r] + gu;
            Va[o] = v[r] + gv;
            if (in.want_exact && g.fs && i == 0) {
                const int pj = j - g.pad;
                if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) {
                    const float du = in.row0[((long long)s * in.slots + in.slot) * g.nx_dom + pj];
                    glr += (double)aDzV[q] * (double)du * (double)g.dzdx;
                }
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 3 * SN * 4);
            tma_load_4d(S3, &tmA, bar + (it & 1), c.j0 - XO, c.i0 - K, F_EX, s + 2);
        }
        const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
        for (int q = r0 + tid; q < r1; q += NTHR) {
            const int rid = rv.tile_rec[q];
            const long long o = (long long)rv.rz[rid] * g.P + rv.rx[rid];
            const float *src = in.rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)n * g.nrec + rid;
            atomicAdd(Ua + o, src[0]);
            atomicAdd(Va + o, src[(long long)g.nt * g.nrec]);
        }
    }
    if (in.want_exact && g.fs && c.i0 == 0 && ty == 0) {
        const int pj = j - g.pad;
        if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) in.accLr[(long long)blockIdx.y * g.nx_dom + pj] += glr;
    }
}

// ------------------------------------------------------------- adjoint: strains + gradient

template <int FD, bool EXACT, bool IMG>
__global__ void __launch_bounds__(NTHR, STFWI_TMA_MINBLOCKS)
    k_adj_b_t(Geo g, Mat m, Shots sh, Recv rv, float *A, float *PX, float *PZ, int n, int spg, AdjOut o,
              int *status, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB)
{
    using T = TileT<FD>;
    constexpr int K = T::K, SN = T::SN, SH = T::SH;
    extern __shared__ __align__(128) float sm[];
    float *stage0 = sm, *stage1 = sm + T::S2;            // U_a, V_a -> A_XX, A_ZZ
    float *aZXZ = sm + 2 * T::S2, *aXXZ = aZXZ + T::S1, *sB = aXXZ + T::S1;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + T::ADB);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const TmaCtx c = tma_ctx(g, spg);
    const int nsh = c.s1 - c.s0;
    if (nsh <= 0) return;
    if (tid == 0) {
        mbar_init(bar + 0, 1); mbar_init(bar + 1, 1); mbar_init(bar + 2, 1);
        fence_async_shared();
        mbar_arrive_expect_tx(bar + 2, SN * 4);
        tma_load_3d(sB, &tmB, bar + 2, c.j0 - XO, c.i0 - K, 0);
        mbar_arrive_expect_tx(bar + 0, 2 * SN * 4);
        tma_load_4d(stage0, &tmA, bar + 0, c.j0 - XO, c.i0 - K, F_U, c.s0);
        if (nsh > 1) {
            mbar_arrive_expect_tx(bar + 1, 2 * SN * 4);
            tma_load_4d(stage1, &tmA, bar + 1, c.j0 - XO, c.i0 - K, F_U, c.s0 + 1);
        }
    }
    __syncthreads();
    const int rd = o.ping, wr = 1 - o.ping;
    const int j = c.j0 + tx;
    const bool colin = j >= T::M && j <= g.nx - 1 - T::M;
    float mL2M[RPT], mL[RPT], mM2[RPT];
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
    }
#pragma unroll
    for (int r = 0; r < RE; ++r) gM[r] = gL[r] = gL2M[r] = 0.0;
#pragma unroll
    for (int r = 0; r < RI; ++r) glam[r] = gmu[r] = 0.0;
    if (!__syncthreads_and(mbar_wait_bounded(bar + 2, 0, WAIT_LIMIT))) { tma_abort(bar, 2, status); return; }

    for (int it = 0; it < nsh; ++it) {
        const int s = c.s0 + it;
        float *S2 = (it & 1) ? stage1 : stage0;
        float *exa = A + ((long long)s * F_N + F_EX) * g.fstride;
        float *eza = A + ((long long)s * F_N + F_EZ) * g.fstride;
        float *esa = A + ((long long)s * F_N + F_ES) * g.fstride;
        const float *Ua = A + ((long long)s * F_N + F_U) * g.fstride;
        const float *Va = A + ((long long)s * F_N + F_V) * g.fstride;
        const float *snap_in = (EXACT && o.slot_in >= 0)
                                   ? o.snap + ((long long)s * o.slots + o.slot_in) * 3 * g.nd : nullptr;
        const float *snap_img = (IMG && o.slot_img >= 0)
                                    ? o.snap + ((long long)s * o.slots + o.slot_img) * 3 * g.nd : nullptr;
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
        const float *pXX = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XX);
        const float *pXXZ = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XXZ);
        const float *pZXZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZXZ);
        const float *pZZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZZ);
        float *wXX = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XX);
        float *wXXZ = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XXZ);
        float *wZXZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZXZ);
        float *wZZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZZ);
        if (!__syncthreads_and(mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1, WAIT_LIMIT))) {
            tma_abort(bar, 2, status);
            return;
        }
        // 1-T / 2-T inputs after the C-PML transpose, in place: U_a -> A_XX, V_a -> A_ZZ
        for (int rr = ty; rr < SH; rr += NWARP) {
            const int i = c.i0 - K + rr;
            for (int cc = tx; cc < SWT; cc += TX) {
                const int jj = c.j0 - XO + cc, q = rr * SWT + cc;
                float vXX = 0.f, vZXZ = 0.f, vXXZ = 0.f, vZZ = 0.f;
                if (i >= 0 && i < g.nz - 1 && jj >= 1 && jj < g.nx - 1) {
                    const float ua = S2[q], va = S2[SN + q], Bv = sB[q];
                    vXX = g.dtdx * Bv * ua;
                    vZXZ = g.dtdz * Bv * ua;
                    vXXZ = g.dtdx * Bv * va;
                    vZZ = g.dtdz * Bv * va;
                }
                if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                    const bool own = rr >= K && rr < K + TZ && cc >= XO && cc < XO + TX;
                    const int xs = xstrip_index(g, jj), zs = zstrip_index(g, i);
                    if (xs >= 0) {
                        const long long px = (long long)i * g.xs_n + xs;
                        const float b = m.bx[jj], a = m.ax[jj], ik = m.ikx[jj];
                        vXX = pml_adj(vXX, b, a, ik, pXX[px], own ? wXX + px : nullptr);
                        vXXZ = pml_adj(vXXZ, b, a, ik, pXXZ[px], own ? wXXZ + px : nullptr);
                    }
                    if (zs >= 0) {
                        const long long pz = (long long)zs * g.P + jj;
                        const float b = m.bz[i], a = m.az[i], ik = m.ikz[i];
                        vZXZ = pml_adj(vZXZ, b, a, ik, pZXZ[pz], own ? wZXZ + pz : nullptr);
                        vZZ = pml_adj(vZZ, b, a, ik, pZZ[pz], own ? wZZ + pz : nullptr);
                    }
                }
                S2[q] = vXX; S2[SN + q] = vZZ; aZXZ[q] = vZXZ; aXXZ[q] = vXXZ;
            }
        }
        __syncthreads();
        const float *aXX = S2, *aZZ = S2 + SN;
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = c.i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + K) * SWT + tx + XO;
            float sxx = 0.f, szz = 0.f, sxz = 0.f;
            if (colin && i >= T::M && i <= g.nz - 1 - T::M) {
                sxx = st_tdxp<FD, false>(aXX, q, j, g.nx);
                szz = st_tdzp<FD, false>(aZZ, q, i, g.nz);
                sxz = st_tdzm<FD, false>(aZXZ, q, i, g.nz, g.nz - 1) + st_tdxm<FD, false>(aXXZ, q, j, g.nx, g.nx - 1);
            } else {
                if (i < g.nz - 1) {
                    sxx = st_tdxp<FD, true>(aXX, q, j, g.nx);
                    sxz = st_tdxm<FD, true>(aXXZ, q, j, g.nx, g.nx - 1);
                }
                if (j >= 1 && j < g.nx - 1) {
                    szz = st_tdzp<FD, true>(aZZ, q, i, g.nz);
                    sxz += st_tdzm<FD, true>(aZXZ, q, i, g.nz, g.nz - 1);
                    if (g.fs && i == 0) sxz += 2.f * cf<FD>(1) * aZXZ[q];
                }
            }
            const long long off = (long long)i * g.P + j;
            if (i == ssz && j == ssx) {
                const float w = sh.wav[(long long)s * g.nt + n];
                if (stype == 0) {
                    if (o.src_a) o.src_a[(long long)s * g.nt + n] = sh.fcoef[s] * Va[off];
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
                const double e1 = h1[r], e2 = h2[r], e3 = h3[r];
                gL2M[r % RE] += e1 * sxx + e2 * szz;
                gL[r % RE] += e2 * sxx + e1 * szz;
                gM[r % RE] += 2.0 * e3 * sxz;
            }
            const int pi = i - g.z0, pj = j - g.pad;
            if (IMG && snap_img && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                const long long pq = (long long)pi * g.nx_dom + pj;
                const int ip = (i + 1) % g.nz, im = (i - 1 + g.nz) % g.nz;
                const int jp = (j + 1) % g.nx, jm = (j - 1 + g.nx) % g.nx;
                const long long oxp = (long long)i * g.P + jp, oxm = (long long)i * g.P + jm;
                const long long ozp = (long long)ip * g.P + j, ozm = (long long)im * g.P + j;
                const float bxp = m.B[oxp], bxm = m.B[oxm], bzp = m.B[ozp], bzm = m.B[ozm];
                const float dxBU = (bxp * Ua[oxp] - bxm * Ua[oxm]) * g.inv2dx;
                const float dzBV = (bzp * Va[ozp] - bzm * Va[ozm]) * g.inv2dz;
                const float dzBU = (bzp * Ua[ozp] - bzm * Ua[ozm]) * g.inv2dz;
                const float dxBV = (bxp * Va[oxp] - bxm * Va[oxm]) * g.inv2dx;
                const float e1 = snap_img[pq], e2 = snap_img[g.nd + pq], e3 = snap_img[2 * g.nd + pq];
                glam[r % RI] -= (double)g.dt * (double)((e1 + e2) * (dxBU + dzBV));
                gmu[r % RI] -= (double)g.dt * (double)(2.f * e1 * dxBU + 2.f * e2 * dzBV + e3 * (dzBU + dxBV));
            }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0 && it + 2 < nsh) {
            mbar_arrive_expect_tx(bar + (it & 1), 2 * SN * 4);
            tma_load_4d(S2, &tmA, bar + (it & 1), c.j0 - XO, c.i0 - K, F_U, s + 2);
        }
        if (n > 0) {
            const int r0 = rv.tile_start[c.tile], r1 = rv.tile_start[c.tile + 1];
            for (int q = r0 + tid; q < r1; q += NTHR) {
                const int rid = rv.tile_rec[q];
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
                double *acc = o.acc + (long long)blockIdx.y * 5 * g.nd + (long long)pi * g.nx_dom + pj;
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
