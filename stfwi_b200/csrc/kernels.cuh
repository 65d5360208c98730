// Device kernels of the B200 elastic velocity-strain solver (sm_100a).
//
// Time step of the reference (fwi/forward.py:250-469) split in two gather
// phases, each one launch over every tile of every shot of the batch:
//   fwd_vel : U, V from the strain-derived stresses (forward.py:253-367)
//   fwd_str : exx, ezz, exz from the new U, V (forward.py:369-444)
// and the discrete adjoint (fwi/adjoint_jax_kernel.py:189-476) in the
// mirror order, written as gathers (the transpose of a stencil is a stencil):
//   adj_a   : U_a, V_a from the strain adjoints (its 0-T .. 2-T part)
//   adj_b   : exx_a, ezz_a, exz_a from U_a, V_a (its 2-T, 1-T, constitutive-T)
//             + the model-gradient accumulation.
//
// Every finite-difference term c_k is applied exactly where the reference
// applies it: a D+ term k at index t needs f[t+k] and f[t-k+1] in range, a D-
// term needs f[t+k-1] and f[t-k] in range, and each derivative is only
// formed inside the rectangle the reference slices it on.  This reproduces
// the reference's per-term slice ranges (its high-order terms are dropped
// near the edges, not zero-padded).
//
// Stresses are merged: sxx = L2M ex + L ez and szz = L ex + L2M ez carry one
// C-PML memory variable each, where the reference carries two whose sum is
// all it ever uses (and whose adjoints are identical).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace stfwi {

constexpr int TX = 32;            // tile width  = one warp of columns
constexpr int TZ = 32;            // tile height
constexpr int NWARP = 8;          // warps per block
constexpr int NTHR = TX * NWARP;  // threads per block
constexpr int RPT = TZ / NWARP;   // rows per thread

// psi (C-PML memory) arrays per shot: x-strips and z-strips
enum { PX_SXX = 0, PX_SXZ, PX_DXU, PX_DXV, PX_NFWD };
enum { PZ_SXZ = 0, PZ_SZZ, PZ_DZV, PZ_DZU, PZ_NFWD };
// adjoint psi: 4 x + 4 z, double-buffered (slot 0/1)
enum { PXA_DXU = 0, PXA_DXV, PXA_XX, PXA_XXZ, PXA_N };
enum { PZA_DZU = 0, PZA_DZV, PZA_ZXZ, PZA_ZZ, PZA_N };
constexpr int NPX = PX_NFWD + 2 * PXA_N;  // 12
constexpr int NPZ = PZ_NFWD + 2 * PZA_N;  // 12

// field slots per shot
enum { F_U = 0, F_V, F_EX, F_EZ, F_ES, F_N };

struct Geo {
    int nz, nx, P;             // padded grid and row pitch (floats)
    int nz_dom, nx_dom, z0, pad;
    int fs;                    // free surface
    int xs_n, zs_n;            // strip widths: 2*pad columns, pad or 2*pad rows
    int nt, nrec, nshot;
    int tiles_x, tiles_z;
    float dtdx, dtdz, dzdx, dt;
    float inv2dx, inv2dz;      // 1/(2 dx), 1/(2 dz) (imaging condition)
    float dtdxdz;              // dt / (dx dz) (force source)
    long long fstride;         // nz*P
    long long xstride;         // nz*xs_n  (one x-psi array)
    long long zstride;         // zs_n*P   (one z-psi array)
    long long nd;              // nz_dom*nx_dom
    int snf;                   // history fields per slot: 3 (stresses) or 5 (+ U, V)
};

struct Mat {
    const float *B, *L2M, *L, *M;   // padded grid [nz][P]
    const float *Lr;                // row 0 of -L/L2M [P] (free surface)
    const float *bx, *ax, *ikx;     // per column [nx]
    const float *bz, *az, *ikz;     // per row [nz]
};

struct Shots {
    const int *sx, *sz, *type;      // padded-grid source position, type
    const float *wav;               // [nshot][nt]
    const float *fcoef;             // dt/(dx dz) * B[src]          (force)
    const float *mcoef;             // 2 (L+M)[src] dx dz           (moment denominator)
    const float *lm;                // (L+M)[src]
};

struct Recv {
    const int *tile_start;          // [tiles+1]
    const int *tile_rec;            // receiver ids grouped by tile
    const int *rx, *rz;             // padded-grid receiver position
};

// ---------------------------------------------------------------- stencils

template <int FD> struct Sten { static constexpr int K = FD / 2; };

template <int FD>
__device__ __forceinline__ float cf(int k)
{
    if (FD == 8) {
        return k == 1 ? (float)(1225.0 / 1024.0)
             : k == 2 ? (float)(-245.0 / 3072.0)
             : k == 3 ? (float)(49.0 / 5120.0)
                      : (float)(-5.0 / 7168.0);
    }
    if (FD == 4) return k == 1 ? (float)(9.0 / 8.0) : (float)(-1.0 / 24.0);
    return 1.0f;
}

// term k of D+ at index t exists (f[t+k], f[t-k+1] in [0,n))
__device__ __forceinline__ bool mP(int t, int k, int n) { return t >= k - 1 && t <= n - 1 - k; }
// term k of D- at index t exists (f[t+k-1], f[t-k] in [0,n))
__device__ __forceinline__ bool mM(int t, int k, int n) { return t >= k && t <= n - k; }

__device__ __forceinline__ int xstrip_index(const Geo &g, int j)
{
    if (j < g.pad) return j;
    if (j >= g.nx - g.pad) return j - (g.nx - 2 * g.pad);
    return -1;
}
__device__ __forceinline__ int zstrip_index(const Geo &g, int i)
{
    if (i >= g.nz - g.pad) return i - (g.nz - g.pad);
    if (!g.fs && i < g.pad) return g.pad + i;
    return -1;
}

__device__ __forceinline__ float *px_ptr(const Geo &g, float *PX, int s, int a)
{
    return PX + ((long long)s * NPX + a) * g.xstride;
}
__device__ __forceinline__ float *pz_ptr(const Geo &g, float *PZ, int s, int a)
{
    return PZ + ((long long)s * NPZ + a) * g.zstride;
}

// forward C-PML (fwi/forward.py:107-112): psi' = b psi + a D ; D' = D/k + psi'
__device__ __forceinline__ float pml_fwd(float D, float b, float a, float ik, float *psi)
{
    float pn = b * (*psi) + a * D;
    *psi = pn;
    return D * ik + pn;
}

// ---------------------------------------------------------------- forward: velocities

template <int FD>
__global__ void __launch_bounds__(NTHR) k_fwd_vel(Geo g, Mat m, Shots sh, float *F, float *PX,
                                                  float *PZ, int n, int spg)
{
    constexpr int K = Sten<FD>::K, H = K;
    constexpr int SW = TX + 2 * H, SH = TZ + 2 * H, SN = SW * SH;
    __shared__ float sL2M[SN], sL[SN], sM[SN], sxx[SN], szz[SN], sxz[SN];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int tile_x = blockIdx.x % g.tiles_x, tile_z = blockIdx.x / g.tiles_x;
    const int j0 = tile_x * TX, i0 = tile_z * TZ;
    const int s0 = blockIdx.y * spg, s1 = min(s0 + spg, g.nshot);

    for (int q = tid; q < SN; q += NTHR) {
        const int i = i0 - H + q / SW, j = j0 - H + q % SW;
        const bool in = i >= 0 && i < g.nz && j >= 0 && j < g.nx;
        const long long o = (long long)i * g.P + j;
        sL2M[q] = in ? m.L2M[o] : 0.f;
        sL[q] = in ? m.L[o] : 0.f;
        sM[q] = in ? m.M[o] : 0.f;
    }
    const int j = j0 + tx;
    const int xs = (j < g.nx) ? xstrip_index(g, j) : -1;
    float bxv = 0.f, axv = 0.f, ikxv = 1.f;
    if (xs >= 0) { bxv = m.bx[j]; axv = m.ax[j]; ikxv = m.ikx[j]; }
    float Bc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = i0 + ty * RPT + r;
        Bc[r] = (i < g.nz && j < g.nx) ? m.B[(long long)i * g.P + j] : 0.f;
    }

    for (int s = s0; s < s1; ++s) {
        const float *ex = F + ((long long)s * F_N + F_EX) * g.fstride;
        const float *ez = F + ((long long)s * F_N + F_EZ) * g.fstride;
        const float *es = F + ((long long)s * F_N + F_ES) * g.fstride;
        __syncthreads();
        for (int q = tid; q < SN; q += NTHR) {
            const int i = i0 - H + q / SW, jj = j0 - H + q % SW;
            float a = 0.f, b = 0.f, c = 0.f;
            if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                const long long o = (long long)i * g.P + jj;
                const float e1 = ex[o], e2 = ez[o], e3 = es[o];
                a = sL2M[q] * e1 + sL[q] * e2;
                b = sL[q] * e1 + sL2M[q] * e2;
                c = 2.f * sM[q] * e3;
            }
            sxx[q] = a; szz[q] = b; sxz[q] = c;
        }
        __syncthreads();
        float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = i0 + ty * RPT + r;
            if (i >= g.nz - 1 || j < 1 || j >= g.nx - 1) continue;
            const int q = (ty * RPT + r + H) * SW + tx + H;
            float dxx = 0.f, dzxz = 0.f, dxxz = 0.f, dzz = 0.f;
#pragma unroll
            for (int k = 1; k <= K; ++k) {
                const float c = cf<FD>(k);
                if (mP(j, k, g.nx)) dxx += c * (sxx[q + k] - sxx[q - k + 1]);
                if (mM(i, k, g.nz)) dzxz += c * (sxz[q + (k - 1) * SW] - sxz[q - k * SW]);
                if (mM(j, k, g.nx)) dxxz += c * (sxz[q + k - 1] - sxz[q - k]);
                if (mP(i, k, g.nz)) dzz += c * (szz[q + k * SW] - szz[q - (k - 1) * SW]);
            }
            if (g.fs && i == 0) dzxz = 2.f * cf<FD>(1) * sxz[q];
            if (xs >= 0) {
                float *p0 = px_ptr(g, PX, s, PX_SXX) + (long long)i * g.xs_n + xs;
                float *p1 = px_ptr(g, PX, s, PX_SXZ) + (long long)i * g.xs_n + xs;
                dxx = pml_fwd(dxx, bxv, axv, ikxv, p0);
                dxxz = pml_fwd(dxxz, bxv, axv, ikxv, p1);
            }
            const int zs = zstrip_index(g, i);
            if (zs >= 0) {
                const float b = m.bz[i], a = m.az[i], ik = m.ikz[i];
                float *p0 = pz_ptr(g, PZ, s, PZ_SXZ) + (long long)zs * g.P + j;
                float *p1 = pz_ptr(g, PZ, s, PZ_SZZ) + (long long)zs * g.P + j;
                dzxz = pml_fwd(dzxz, b, a, ik, p0);
                dzz = pml_fwd(dzz, b, a, ik, p1);
            }
            const long long o = (long long)i * g.P + j;
            const float Bv = Bc[r];
            U[o] = U[o] + g.dtdx * Bv * dxx + g.dtdz * Bv * dzxz;
            float v = V[o] + g.dtdx * Bv * dxxz + g.dtdz * Bv * dzz;
            if (stype == 0 && i == ssz && j == ssx) v = v + sh.fcoef[s] * sh.wav[(long long)s * g.nt + n];
            V[o] = v;
        }
    }
}

// ---------------------------------------------------------------- forward: strains

struct FwdOut {
    float *rec;          // [nshot][4][nt][nrec]
    float *snap;         // history: + (s*slots + slot)*snf*nd, or null
    float *row0;         // post-PML d(vx)/dx at row 0 (free surface): + (s*slots+slot_row0)*nx_dom, or null
    int slots, slot;     // history slot written by this step (its carry-out)
    int slot_row0;       // row-0 slot of this step
    double *energy;      // illumination accumulator [nz][nx] (padded grid, pitch nx), or null
    int energy_comp;     // 0 vx, 1 vz, 2 exx, 3 ezz
    int *status;         // bit 0: non-finite receiver sample
};

template <int FD>
__global__ void __launch_bounds__(NTHR) k_fwd_str(Geo g, Mat m, Shots sh, Recv rv, float *F,
                                                  float *PX, float *PZ, int n, int spg, FwdOut out)
{
    constexpr int K = Sten<FD>::K, H = K;
    constexpr int SW = TX + 2 * H, SH = TZ + 2 * H, SN = SW * SH;
    __shared__ float sU[SN], sV[SN];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int tile = blockIdx.x;
    const int tile_x = tile % g.tiles_x, tile_z = tile / g.tiles_x;
    const int j0 = tile_x * TX, i0 = tile_z * TZ;
    const int s0 = blockIdx.y * spg, s1 = min(s0 + spg, g.nshot);
    const int j = j0 + tx;
    const int xs = (j < g.nx) ? xstrip_index(g, j) : -1;
    float bxv = 0.f, axv = 0.f, ikxv = 1.f;
    if (xs >= 0) { bxv = m.bx[j]; axv = m.ax[j]; ikxv = m.ikx[j]; }
    const float Lr0 = (g.fs && j < g.nx) ? m.Lr[j] : 0.f;
    double eacc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) eacc[r] = 0.0;

    for (int s = s0; s < s1; ++s) {
        const float *U = F + ((long long)s * F_N + F_U) * g.fstride;
        const float *V = F + ((long long)s * F_N + F_V) * g.fstride;
        float *ex = F + ((long long)s * F_N + F_EX) * g.fstride;
        float *ez = F + ((long long)s * F_N + F_EZ) * g.fstride;
        float *es = F + ((long long)s * F_N + F_ES) * g.fstride;
        __syncthreads();
        for (int q = tid; q < SN; q += NTHR) {
            const int i = i0 - H + q / SW, jj = j0 - H + q % SW;
            const bool in = i >= 0 && i < g.nz && jj >= 0 && jj < g.nx;
            const long long o = (long long)i * g.P + jj;
            sU[q] = in ? U[o] : 0.f;
            sV[q] = in ? V[o] : 0.f;
        }
        __syncthreads();
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + H) * SW + tx + H;
            const int zs = zstrip_index(g, i);
            float dxu = 0.f, dzv = 0.f, dzu = 0.f, dxv = 0.f;
#pragma unroll
            for (int k = 1; k <= K; ++k) {
                const float c = cf<FD>(k);
                if (mM(j, k, g.nx)) dxu += c * (sU[q + k - 1] - sU[q - k]);
                if (mM(i, k, g.nz)) dzv += c * (sV[q + (k - 1) * SW] - sV[q - k * SW]);
                if (mP(i, k, g.nz)) dzu += c * (sU[q + k * SW] - sU[q - (k - 1) * SW]);
                if (mP(j, k, g.nx)) dxv += c * (sV[q + k] - sV[q - k + 1]);
            }
            // exx (forward.py:370-383): D-x U on all rows, columns [1, nx)
            if (j >= 1 && xs >= 0)
                dxu = pml_fwd(dxu, bxv, axv, ikxv, px_ptr(g, PX, s, PX_DXU) + (long long)i * g.xs_n + xs);
            // ezz (forward.py:386-404): D-z V on columns [0, nx-1); free-surface row 0
            if (j < g.nx - 1) {
                if (g.fs && i == 0) dzv = Lr0 * dxu * g.dzdx;
                if (zs >= 0)
                    dzv = pml_fwd(dzv, m.bz[i], m.az[i], m.ikz[i],
                                  pz_ptr(g, PZ, s, PZ_DZV) + (long long)zs * g.P + j);
            } else {
                dzv = 0.f;
            }
            // exz (forward.py:414-444): D+z U on columns [1, nx), D+x V on rows [0, nz-1)
            if (j >= 1) {
                if (zs >= 0)
                    dzu = pml_fwd(dzu, m.bz[i], m.az[i], m.ikz[i],
                                  pz_ptr(g, PZ, s, PZ_DZU) + (long long)zs * g.P + j);
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
            float exn = ex[o], ezn = ez[o], esn = es[o];
            if (j >= 1) exn = exn + g.dtdx * dxu;
            ezn = ezn + g.dtdz * dzv;
            if (stype == 1 && i == ssz && j == ssx) {
                const float st = sh.wav[(long long)s * g.nt + n] * g.dt / sh.mcoef[s];
                exn = exn + st;
                ezn = ezn + st;
            }
            if (i < g.nz - 1 && j < g.nx - 1) esn = esn + 0.5f * (g.dtdz * dzu + g.dtdx * dxv);
            ex[o] = exn; ez[o] = ezn; es[o] = esn;
            const int pi = i - g.z0, pj = j - g.pad;
            const bool phys = pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom;
            if (out.snap && phys) {
                float *sp = out.snap + ((long long)s * out.slots + out.slot) * g.snf * g.nd + (long long)pi * g.nx_dom + pj;
                __stcs(sp, exn);
                __stcs(sp + g.nd, ezn);
                __stcs(sp + 2 * g.nd, esn);
            }
            if (out.row0 && g.fs && i == 0 && pj >= 0 && pj < g.nx_dom)
                out.row0[((long long)s * out.slots + out.slot_row0) * g.nx_dom + pj] = dxu;
            if (out.energy) {
                float f = out.energy_comp == 2 ? exn : out.energy_comp == 3 ? ezn
                        : out.energy_comp == 0 ? U[o] : V[o];
                eacc[r] += (double)f * (double)f;
            }
        }
        // receivers of this tile (the tile's own cells are final now)
        __syncthreads();
        const int r0 = rv.tile_start[tile], r1 = rv.tile_start[tile + 1];
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
            const int i = i0 + ty * RPT + r;
            if (i < g.nz && j < g.nx) atomicAdd(out.energy + (long long)i * g.nx + j, eacc[r]);
        }
    }
}

// ---------------------------------------------------------------- adjoint: velocities

// adjoint C-PML (fwi/adjoint_jax_kernel.py:51-54) with the old memory value
__device__ __forceinline__ float pml_adj(float Din, float b, float a, float ik, float psi_old,
                                         float *psi_new)
{
    if (psi_new) *psi_new = b * (Din + psi_old);
    return (ik + a) * Din + a * psi_old;
}

struct AdjIn {
    const float *rec_adj;  // [nshot][4][nt][nrec]
    const float *row0;     // forward post-PML d(vx)/dx at row 0: + (s*slots + slot)*nx_dom
    int slots, slot;
    double *accLr;         // [groups][nx_dom] FP64: dJ/dLr on row 0
    int want_exact;
    int ping;              // psi slot read (ping) / written (1-ping)
};

template <int FD>
__global__ void __launch_bounds__(NTHR) k_adj_a(Geo g, Mat m, Recv rv, float *A, float *PX,
                                                float *PZ, int n, int spg, AdjIn in)
{
    constexpr int K = Sten<FD>::K, H = K;
    constexpr int SW = TX + 2 * H, SH = TZ + 2 * H, SN = SW * SH;
    __shared__ float aDzU[SN], aDxU[SN], aDxV[SN], aDzV[SN];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int tile = blockIdx.x;
    const int tile_x = tile % g.tiles_x, tile_z = tile / g.tiles_x;
    const int j0 = tile_x * TX, i0 = tile_z * TZ;
    const int grp = blockIdx.y;
    const int s0 = grp * spg, s1 = min(s0 + spg, g.nshot);
    const int rd = in.ping, wr = 1 - in.ping;
    const int j = j0 + tx;
    double glr = 0.0;

    for (int s = s0; s < s1; ++s) {
        const float *exa = A + ((long long)s * F_N + F_EX) * g.fstride;
        const float *eza = A + ((long long)s * F_N + F_EZ) * g.fstride;
        const float *esa = A + ((long long)s * F_N + F_ES) * g.fstride;
        const float *pDzU = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZU);
        const float *pDzV = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_DZV);
        const float *pDxU = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXU);
        const float *pDxV = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_DXV);
        float *wDzU = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZU);
        float *wDzV = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_DZV);
        float *wDxU = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXU);
        float *wDxV = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_DXV);
        __syncthreads();
        // derivative adjoints after the C-PML transpose, on tile + halo
        for (int q = tid; q < SN; q += NTHR) {
            const int ti = q / SW, tj = q % SW;
            const int i = i0 - H + ti, jj = j0 - H + tj;
            float vDzU = 0.f, vDxU = 0.f, vDxV = 0.f, vDzV = 0.f;
            if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                const long long o = (long long)i * g.P + jj;
                const bool own = ti >= H && ti < H + TZ && tj >= H && tj < H + TX;
                const int xs = xstrip_index(g, jj), zs = zstrip_index(g, i);
                const float ea = exa[o], za = eza[o], sa = esa[o];
                // 4-T: Dz_V_used_a = dt/dz ezz_a on the whole grid
                vDzV = g.dtdz * za;
                if (zs >= 0) {
                    const long long pz = (long long)zs * g.P + jj;
                    vDzV = pml_adj(vDzV, m.bz[i], m.az[i], m.ikz[i], pDzV[pz], own ? wDzV + pz : nullptr);
                }
                // 4-T free surface + 3-T: Dx_U_a
                float din = 0.f;
                if (g.fs && i == 0 && jj < g.nx - 1) din = m.Lr[jj] * g.dzdx * vDzV;
                if (jj >= 1) din = din + g.dtdx * ea;
                vDxU = din;
                if (xs >= 0) {
                    const long long px = (long long)i * g.xs_n + xs;
                    vDxU = pml_adj(din, m.bx[jj], m.ax[jj], m.ikx[jj], pDxU[px], own ? wDxU + px : nullptr);
                }
                // 5-T: 0.5 dt/dz exz_a and 0.5 dt/dx exz_a on [0,nz-1) x [0,nx-1)
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
            aDzU[q] = vDzU; aDxU[q] = vDxU; aDxV[q] = vDxV; aDzV[q] = vDzV;
        }
        __syncthreads();
        float *Ua = A + ((long long)s * F_N + F_U) * g.fstride;
        float *Va = A + ((long long)s * F_N + F_V) * g.fstride;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + H) * SW + tx + H;
            float gu = 0.f, gv = 0.f;
#pragma unroll
            for (int k = 1; k <= K; ++k) {
                const float c = cf<FD>(k);
                // U_a += (D+z)^T Dz_U_a   (forward D+z U on columns [1, nx))
                if (j >= 1) {
                    if (mP(i - k, k, g.nz)) gu += c * aDzU[q - k * SW];
                    if (mP(i + k - 1, k, g.nz)) gu -= c * aDzU[q + (k - 1) * SW];
                }
                // U_a += (D-x)^T Dx_U_a   (forward D-x U on all rows)
                if (mM(j - k + 1, k, g.nx)) gu += c * aDxU[q - k + 1];
                if (mM(j + k, k, g.nx)) gu -= c * aDxU[q + k];
                // V_a += (D+x)^T Dx_V_a   (forward D+x V on rows [0, nz-1))
                if (i < g.nz - 1) {
                    if (mP(j - k, k, g.nx)) gv += c * aDxV[q - k];
                    if (mP(j + k - 1, k, g.nx)) gv -= c * aDxV[q + k - 1];
                }
                // V_a += (D-z)^T Dz_V_a   (forward D-z V on columns [0, nx-1))
                if (j < g.nx - 1) {
                    if (mM(i - k + 1, k, g.nz)) gv += c * aDzV[q - (k - 1) * SW];
                    if (mM(i + k, k, g.nz)) gv -= c * aDzV[q + k * SW];
                }
            }
            const long long o = (long long)i * g.P + j;
            Ua[o] = Ua[o] + gu;
            Va[o] = Va[o] + gv;
            // exact gradient: Dz_V[0,j] = Lr * Dx_U' * dz/dx  ->  dJ/dLr (row 0 is ty=0, r=0)
            if (in.want_exact && g.fs && i == 0) {
                const int pj = j - g.pad;
                if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) {
                    const float du = in.row0[((long long)s * in.slots + in.slot) * g.nx_dom + pj];
                    glr += (double)aDzV[q] * (double)du * (double)g.dzdx;
                }
            }
        }
        // receiver injection of this step into U_a, V_a (0-T)
        __syncthreads();
        const int r0 = rv.tile_start[tile], r1 = rv.tile_start[tile + 1];
        for (int q = r0 + tid; q < r1; q += NTHR) {
            const int rid = rv.tile_rec[q];
            const long long o = (long long)rv.rz[rid] * g.P + rv.rx[rid];
            const float *src = in.rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)n * g.nrec + rid;
            atomicAdd(Ua + o, src[0]);
            atomicAdd(Va + o, src[(long long)g.nt * g.nrec]);
        }
    }
    if (in.want_exact && g.fs && i0 == 0 && ty == 0) {
        const int pj = j - g.pad;
        if (pj >= 0 && pj < g.nx_dom && j < g.nx - 1) in.accLr[(long long)grp * g.nx_dom + pj] += glr;
    }
}

// ---------------------------------------------------------------- adjoint: strains + gradient

struct AdjOut {
    const float *snap;     // history base (s*slots + slot)*snf*nd
    int slots;
    int slot_in;           // slot of the forward carry-in of this step (-1: zero state)
    int slot_img;          // slot of the forward carry-out of this step (imaging), -1 if none
    int slot_next;         // slot of the carry-out of the next step (density imaging term), -1 if none
    int accp;              // accumulator planes per group (5, or 7 with the density terms)
    double *acc;           // [groups][accp][nd]: gM, gL, gL2M (exact), glam, gmu (imaging), gB (exact), g_rho_lame (imaging)
    int want_exact, want_img;
    float *src_a;          // [nshot][nt] or null
    const float *rec_adj;  // [nshot][4][nt][nrec]
    int ping;
    int hist_tma;          // two-column kernels: the carry-in stresses arrive by TMA (history map valid)
};

template <int FD, bool EXACT, bool IMG>
__global__ void __launch_bounds__(NTHR) k_adj_b(Geo g, Mat m, Shots sh, Recv rv, float *A,
                                                float *PX, float *PZ, int n, int spg, AdjOut o)
{
    constexpr int K = Sten<FD>::K, H = K;
    constexpr int SW = TX + 2 * H, SH = TZ + 2 * H, SN = SW * SH;
    __shared__ float aXX[SN], aZXZ[SN], aXXZ[SN], aZZ[SN], sB[SN];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int tile = blockIdx.x;
    const int tile_x = tile % g.tiles_x, tile_z = tile / g.tiles_x;
    const int j0 = tile_x * TX, i0 = tile_z * TZ;
    const int grp = blockIdx.y;
    const int s0 = grp * spg, s1 = min(s0 + spg, g.nshot);
    const int rd = o.ping, wr = 1 - o.ping;
    const int j = j0 + tx;

    for (int q = tid; q < SN; q += NTHR) {
        const int i = i0 - H + q / SW, jj = j0 - H + q % SW;
        const bool in = i >= 0 && i < g.nz && jj >= 0 && jj < g.nx;
        sB[q] = in ? m.B[(long long)i * g.P + jj] : 0.f;
    }
    float mL2M[RPT], mL[RPT], mM2[RPT];
    constexpr int RE = EXACT ? RPT : 1, RI = IMG ? RPT : 1;
    double gM[RE], gL[RE], gL2M[RE], glam[RI], gmu[RI];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = i0 + ty * RPT + r;
        const bool in = i < g.nz && j < g.nx;
        const long long off = (long long)i * g.P + j;
        mL2M[r] = in ? m.L2M[off] : 0.f;
        mL[r] = in ? m.L[off] : 0.f;
        mM2[r] = in ? 2.f * m.M[off] : 0.f;
    }
#pragma unroll
    for (int r = 0; r < RE; ++r) gM[r] = gL[r] = gL2M[r] = 0.0;
#pragma unroll
    for (int r = 0; r < RI; ++r) glam[r] = gmu[r] = 0.0;

    for (int s = s0; s < s1; ++s) {
        const float *Ua = A + ((long long)s * F_N + F_U) * g.fstride;
        const float *Va = A + ((long long)s * F_N + F_V) * g.fstride;
        const float *pXX = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XX);
        const float *pXXZ = px_ptr(g, PX, s, PX_NFWD + rd * PXA_N + PXA_XXZ);
        const float *pZXZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZXZ);
        const float *pZZ = pz_ptr(g, PZ, s, PZ_NFWD + rd * PZA_N + PZA_ZZ);
        float *wXX = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XX);
        float *wXXZ = px_ptr(g, PX, s, PX_NFWD + wr * PXA_N + PXA_XXZ);
        float *wZXZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZXZ);
        float *wZZ = pz_ptr(g, PZ, s, PZ_NFWD + wr * PZA_N + PZA_ZZ);
        __syncthreads();
        for (int q = tid; q < SN; q += NTHR) {
            const int ti = q / SW, tj = q % SW;
            const int i = i0 - H + ti, jj = j0 - H + tj;
            float vXX = 0.f, vZXZ = 0.f, vXXZ = 0.f, vZZ = 0.f;
            if (i >= 0 && i < g.nz && jj >= 0 && jj < g.nx) {
                const long long off = (long long)i * g.P + jj;
                const bool own = ti >= H && ti < H + TZ && tj >= H && tj < H + TX;
                float ua = 0.f, va = 0.f;
                if (i < g.nz - 1 && jj >= 1 && jj < g.nx - 1) { ua = Ua[off]; va = Va[off]; }
                const float Bv = sB[q];
                // 1-T / 2-T inputs: dt/dx B U_a, dt/dz B U_a, dt/dx B V_a, dt/dz B V_a
                vXX = g.dtdx * Bv * ua;
                vZXZ = g.dtdz * Bv * ua;
                vXXZ = g.dtdx * Bv * va;
                vZZ = g.dtdz * Bv * va;
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
            aXX[q] = vXX; aZXZ[q] = vZXZ; aXXZ[q] = vXXZ; aZZ[q] = vZZ;
        }
        __syncthreads();
        float *exa = A + ((long long)s * F_N + F_EX) * g.fstride;
        float *eza = A + ((long long)s * F_N + F_EZ) * g.fstride;
        float *esa = A + ((long long)s * F_N + F_ES) * g.fstride;
        const int ssx = sh.sx[s], ssz = sh.sz[s], stype = sh.type[s];
        const float *snap_in = (EXACT && o.slot_in >= 0)
                                   ? o.snap + ((long long)s * o.slots + o.slot_in) * g.snf * g.nd : nullptr;
        const float *snap_img = (IMG && o.slot_img >= 0)
                                    ? o.snap + ((long long)s * o.slots + o.slot_img) * g.snf * g.nd : nullptr;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = i0 + ty * RPT + r;
            if (i >= g.nz || j >= g.nx) continue;
            const int q = (ty * RPT + r + H) * SW + tx + H;
            float sxx = 0.f, szz = 0.f, sxz = 0.f;
#pragma unroll
            for (int k = 1; k <= K; ++k) {
                const float c = cf<FD>(k);
                // Dx_L2M_ex / Dx_L_ez: D+x on rows [0, nz-1)
                if (i < g.nz - 1) {
                    if (mP(j - k, k, g.nx)) sxx += c * aXX[q - k];
                    if (mP(j + k - 1, k, g.nx)) sxx -= c * aXX[q + k - 1];
                }
                if (j >= 1 && j < g.nx - 1) {
                    // Dz_L2M_ez / Dz_L_ex: D+z on columns [1, nx-1)
                    if (mP(i - k, k, g.nz)) szz += c * aZZ[q - k * SW];
                    if (mP(i + k - 1, k, g.nz)) szz -= c * aZZ[q + (k - 1) * SW];
                    // Dz_M_es: D-z on rows [1, nz-1), columns [1, nx-1)
                    const int t1 = i - k + 1, t2 = i + k;
                    if (mM(t1, k, g.nz) && t1 < g.nz - 1) sxz += c * aZXZ[q - (k - 1) * SW];
                    if (mM(t2, k, g.nz) && t2 < g.nz - 1) sxz -= c * aZXZ[q + k * SW];
                }
                // Dx_M_es: D-x on rows [0, nz-1), columns [1, nx-1)
                if (i < g.nz - 1) {
                    const int t1 = j - k + 1, t2 = j + k;
                    if (mM(t1, k, g.nx) && t1 < g.nx - 1) sxz += c * aXXZ[q - k + 1];
                    if (mM(t2, k, g.nx) && t2 < g.nx - 1) sxz -= c * aXXZ[q + k];
                }
            }
            if (g.fs && i == 0 && j >= 1 && j < g.nx - 1) sxz += 2.f * cf<FD>(1) * aZXZ[q];
            const long long off = (long long)i * g.P + j;
            const float ea = exa[off], za = eza[off];
            // source-wavelet adjoint and the source terms of the model gradient
            if (i == ssz && j == ssx) {
                const float w = sh.wav[(long long)s * g.nt + n];
                if (stype == 0) {
                    if (o.src_a) o.src_a[(long long)s * g.nt + n] = sh.fcoef[s] * Va[off];
                } else {
                    if (o.src_a) o.src_a[(long long)s * g.nt + n] = (g.dt / sh.mcoef[s]) * (ea + za);
                    if (EXACT) {
                        const double lm = sh.lm[s];
                        const double glm = -((double)w * g.dt / ((double)sh.mcoef[s] / lm)) / (lm * lm)
                                           * (double)(ea + za);
                        gM[r % RE] += glm;
                        gL[r % RE] += glm;
                    }
                }
            }
            exa[off] = ea + mL2M[r] * sxx + mL[r] * szz;
            eza[off] = za + mL[r] * sxx + mL2M[r] * szz;
            esa[off] = esa[off] + mM2[r] * sxz;
            const int pi = i - g.z0, pj = j - g.pad;
            if (pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                const long long pq = (long long)pi * g.nx_dom + pj;
                if (EXACT && snap_in) {
                    const double e1 = snap_in[pq], e2 = snap_in[g.nd + pq], e3 = snap_in[2 * g.nd + pq];
                    gL2M[r % RE] += e1 * sxx + e2 * szz;
                    gL[r % RE] += e2 * sxx + e1 * szz;
                    gM[r % RE] += 2.0 * e3 * sxz;
                }
                if (IMG && snap_img) {
                    // fwi/imaging.py:125-141: periodic centred differences of B U_a, B V_a
                    const int ip = (i + 1) % g.nz, im = (i - 1 + g.nz) % g.nz;
                    const int jp = (j + 1) % g.nx, jm = (j - 1 + g.nx) % g.nx;
                    const long long oxp = (long long)i * g.P + jp, oxm = (long long)i * g.P + jm;
                    const long long ozp = (long long)ip * g.P + j, ozm = (long long)im * g.P + j;
                    const float bxp = m.B[oxp], bxm = m.B[oxm], bzp = m.B[ozp], bzm = m.B[ozm];
                    const float inv2dx = g.inv2dx, inv2dz = g.inv2dz;
                    const float dxBU = (bxp * Ua[oxp] - bxm * Ua[oxm]) * inv2dx;
                    const float dzBV = (bzp * Va[ozp] - bzm * Va[ozm]) * inv2dz;
                    const float dzBU = (bzp * Ua[ozp] - bzm * Ua[ozm]) * inv2dz;
                    const float dxBV = (bxp * Va[oxp] - bxm * Va[oxm]) * inv2dx;
                    const float e1 = snap_img[pq], e2 = snap_img[g.nd + pq], e3 = snap_img[2 * g.nd + pq];
                    glam[r % RI] -= (double)g.dt * (double)((e1 + e2) * (dxBU + dzBV));
                    gmu[r % RI] -= (double)g.dt * (double)(2.f * e1 * dxBU + 2.f * e2 * dzBV + e3 * (dzBU + dxBV));
                }
            }
        }
        // receiver injection of step n-1 into exx_a, ezz_a (0-T of the next adjoint step)
        __syncthreads();
        if (n > 0) {
            const int r0 = rv.tile_start[tile], r1 = rv.tile_start[tile + 1];
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
            const int i = i0 + ty * RPT + r;
            const int pi = i - g.z0, pj = j - g.pad;
            if (i < g.nz && j < g.nx && pi >= 0 && pi < g.nz_dom && pj >= 0 && pj < g.nx_dom) {
                double *acc = o.acc + (long long)grp * o.accp * g.nd + (long long)pi * g.nx_dom + pj;
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
