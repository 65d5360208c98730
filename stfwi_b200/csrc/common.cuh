// Shared definitions of the stencil kernels (sm_100a): the state layout of a
// handle (field slots, C-PML memory arrays of the strips), the geometry and
// material views the kernels receive, the staggered finite-difference
// coefficients and the per-term slice masks of the reference's operator.
//
// The operator is the reference's time step (fwi/forward.py:250-469) and its
// discrete adjoint (fwi/adjoint_jax_kernel.py:189-476).  Every
// finite-difference term c_k is applied exactly where the reference applies
// it: a D+ term k at index t needs f[t+k] and f[t-k+1] in range, a D- term
// needs f[t+k-1] and f[t-k] in range, and each derivative is only formed
// inside the rectangle the reference slices it on, so the reference's
// high-order terms are dropped near the edges, not zero-padded.
//
// Stresses are merged: sxx = L2M ex + L ez and szz = L ex + L2M ez carry one
// C-PML memory variable each, where the reference carries two whose sum is
// all it ever uses (and whose adjoints are identical).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tma.cuh"

namespace stfwi {

constexpr int TX = 32;            // lanes of a warp across the tile
constexpr int NWARP = 8;          // warps per block
constexpr int NTHR = TX * NWARP;  // threads per block

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
    float dtdx, dtdz, dzdx, dt;
    float inv2dx, inv2dz;      // 1/(2 dx), 1/(2 dz) (imaging condition)
    float dtdxdz;              // dt / (dx dz) (force source)
    long long fstride;         // nz*P
    long long xstride;         // nz*xs_n  (one x-psi array)
    long long zstride;         // zs_n*P   (one z-psi array)
    long long nd;              // nz_dom*nx_dom
    int snf;                   // history fields per slot: 3 (stresses) or 5 (+ U, V)
    uint32_t wait_polls;       // mbarrier polls before a tile wait gives up (WAIT3 by default)
    // dispatch order of the tiles of the staged tilings (A: fwd_vel, fwd_str,
    // adj_a; B: adj_b): the `heavy` tiles that touch an edge, a C-PML strip
    // or the free surface first, or null for the plain order
    const int *tordA, *tordB;
    int theavyA, theavyB;
    int goff;                  // first shot group of the launch (a pass split into two chains)
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

// forward outputs of the strain phase
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

// inputs of the adjoint velocity phase
struct AdjIn {
    const float *rec_adj;  // [nshot][4][nt][nrec]
    const float *row0;     // forward post-PML d(vx)/dx at row 0: + (s*slots + slot)*nx_dom
    int slots, slot;
    double *accLr;         // [groups][nx_dom] FP64: dJ/dLr on row 0
    int want_exact;
    int ping;              // psi slot read (ping) / written (1-ping)
};

// inputs and outputs of the adjoint strain phase
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

constexpr uint32_t WAIT3 = 1u << 22; // mbarrier polls before a wait gives up
constexpr int ST_TIMEOUT3 = 2;

__host__ __device__ constexpr int al32_3(int x) { return (x + 31) / 32 * 32; }

struct Ctx3 {
    int tile, j0, i0, s0, s1;
};

// on a wait that ran out (the copy of shot `it` of the block): record the
// timeout and, before the block returns, drain the copies still in flight,
// which are those of shots it and it + 1 (each shot's copy is issued two
// shots ahead, on barrier it & 1); these waits are bounded too
__device__ __forceinline__ void abort3(uint64_t *bar, int it, int nsh, int *status)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicOr(status, ST_TIMEOUT3);
        for (int k = it; k < it + 2 && k < nsh; ++k) mbar_wait_bounded(bar + (k & 1), (k >> 1) & 1, WAIT3);
    }
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

}  // namespace stfwi
