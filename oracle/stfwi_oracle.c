/*
 * stfwi_oracle.c -- CPU restatement of the reference's elastic velocity-strain
 * solver, for TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).
 * Nothing in the product path links or calls this file.
 *
 * It restates, slice for slice, the reference's
 *   fwi/forward.py            _pml_coefficients (:35-104), _pml_apply (:107-112),
 *                             forward_jax setup (:167-247) and time_step (:250-469)
 *   fwi/adjoint_jax_kernel.py pml_apply_T (:51-54), adjoint_step (:189-476)
 *   fwi/imaging.py            imaging_condition time sums (:108-141), with the
 *                             periodic jnp.roll centred differences (:47-53)
 * and adds the exact discrete model gradient (what JAX reverse-mode AD of
 * forward_jax returns, fwi/gradient.py:106-132), derived by hand from
 * time_step: at every adjoint step the adjoint of each material-weighted
 * product is multiplied by the forward value it scaled.
 *
 * Every derivative is written as the same sequence of "set"/"add" slabs as
 * the reference (one helper call per `.at[...].set/add` line), and every
 * adjoint transpose as the same sequence of scatters, so the boundary index
 * ranges are the reference's by construction.
 *
 * Compiled twice: ORACLE_F32 undefined -> oracle64_* (FP64, the parity
 * oracle); ORACLE_F32 defined -> oracle32_* (FP32, the timed CPU baseline in
 * the reference's default dtype, every multiply and add rounded as written).
 * OpenMP parallelism is over shots.  A third, tuned build (ORACLE_FAST ->
 * oraclefast_*, liboracle_fast.so, made on the machine that times it) keeps
 * the FP32 arithmetic but lets the compiler contract and vectorise for the
 * host's own ISA.  (Splitting each slab's rows over threads was measured
 * ten times slower: a slab is too small for a parallel region of its own.)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_FAST
/* the tuned timing build: FP32, native ISA, contraction allowed */
typedef float real;
#define ORACLE(n) oraclefast_##n
#elif defined(ORACLE_F32)
typedef float real;
#define ORACLE(n) oracle32_##n
#else
typedef double real;
#define ORACLE(n) oracle64_##n
#endif

typedef struct {
    int32_t nz_dom, nx_dom, pad, fd_order, free_surface, nt, nrec;
    /* 1: build d0 of the PML profile with float32 arithmetic, which is what
     * JAX does when Vp arrives as float32 with x64 enabled
     * (fwi/forward.py:48: f32 Vp_max times weak-typed Python scalars). */
    int32_t d0_f32;
    double dx, dz, dt, fc;
} oracle_desc;

enum { SRC_FORCE = 0, SRC_MOMENT = 1 };

/* carry layout, fwi/forward.py:251 */
enum {
    C_U, C_V, C_EX, C_EZ, C_ES,
    P_DX_L2M_EX, P_DX_L_EZ, P_DZ_M_ES, P_DZ_L2M_EZ, P_DZ_L_EX, P_DX_M_ES,
    P_DX_U, P_DZ_V, P_DZ_U, P_DX_V, NCARRY
};

/* forward intermediates kept for the model gradient (post-PML derivatives) */
enum {
    I_DX_L2M_EX, I_DX_L_EZ, I_DZ_M_ES, I_DX_M_ES, I_DZ_L2M_EZ, I_DZ_L_EX,
    I_DX_U, NINTER
};

typedef struct {
    int nz, nx, nz_dom, nx_dom, pad, z_start, fd, fs, src_type;
    real c1, c2, c3, c4, dx, dz, dt;
    real *M, *L2M, *L, *B, *Lr;
    real *kx, *kz, *bx, *bz, *ax, *az;
    int sx, sz;
    int nrec;
    int *rx, *rz;
    real *work; /* scratch: products and derivative arrays */
} grid_t;

#define IDX(i, j) ((size_t)(i) * (size_t)nx + (size_t)(j))

static real *zalloc(size_t n) { return (real *)calloc(n ? n : 1, sizeof(real)); }

/* D[i,j] (=|+=) c * (f[i+ar, j+ac] - f[i+br, j+bc]) for i in [r0,r1), j in [c0,c1) */
static void slab(real *D, const real *f, int nx, int r0, int r1, int c0, int c1,
                 real c, int ar, int ac, int br, int bc, int add)
{
    for (int i = r0; i < r1; ++i)
        for (int j = c0; j < c1; ++j) {
            real v = c * (f[IDX(i + ar, j + ac)] - f[IDX(i + br, j + bc)]);
            D[IDX(i, j)] = add ? D[IDX(i, j)] + v : v;
        }
}

/* T[i,j] += coef * S[i+dr, j+dc] for i in [r0,r1), j in [c0,c1) */
static void scat(real *T, const real *S, int nx, int r0, int r1, int c0, int c1,
                 real coef, int dr, int dc)
{
    for (int i = r0; i < r1; ++i)
        for (int j = c0; j < c1; ++j)
            T[IDX(i, j)] += coef * S[IDX(i + dr, j + dc)];
}

/* fwi/forward.py:107-112 */
static void pml_apply(real *D, const real *k, real *psi, const real *b, const real *a, size_t n)
{
    for (size_t q = 0; q < n; ++q) {
        real pn = b[q] * psi[q] + a[q] * D[q];
        D[q] = D[q] / k[q] + pn;
        psi[q] = pn;
    }
}

/* fwi/adjoint_jax_kernel.py:51-54 (in place: D holds D_new_a on entry, D_a on exit) */
static void pml_apply_T(real *D, real *psi, const real *k, const real *b, const real *a, size_t n)
{
    for (size_t q = 0; q < n; ++q) {
        real Dn = D[q], pn = psi[q];
        D[q] = ((real)1.0 / k[q] + a[q]) * Dn + a[q] * pn;
        psi[q] = b[q] * (Dn + pn);
    }
}

/* ---------------------------------------------------------------- setup */

static void grid_free(grid_t *g)
{
    free(g->M); free(g->L2M); free(g->L); free(g->B); free(g->Lr);
    free(g->kx); free(g->kz); free(g->bx); free(g->bz); free(g->ax); free(g->az);
    free(g->rx); free(g->rz); free(g->work);
    memset(g, 0, sizeof(*g));
}

/* fwi/forward.py:177-242 and :35-104 */
static int grid_init(grid_t *g, const oracle_desc *d, const double *vs, const double *vp,
                     const double *rho, int src_x, int src_z, int src_type,
                     const int32_t *rec_x, const int32_t *rec_z)
{
    memset(g, 0, sizeof(*g));
    if (d->fd_order != 2 && d->fd_order != 4 && d->fd_order != 8) return -1;
    const int pad = d->pad, nzd = d->nz_dom, nxd = d->nx_dom, fs = d->free_surface ? 1 : 0;
    g->fd = d->fd_order; g->fs = fs; g->pad = pad; g->nz_dom = nzd; g->nx_dom = nxd;
    g->src_type = src_type;
    if (g->fd == 8) {
        g->c1 = (real)(1225.0 / 1024.0); g->c2 = (real)(-245.0 / 3072.0);
        g->c3 = (real)(49.0 / 5120.0);   g->c4 = (real)(-5.0 / 7168.0);
    } else if (g->fd >= 4) {
        g->c1 = (real)(9.0 / 8.0); g->c2 = (real)(-1.0 / 24.0); g->c3 = 0; g->c4 = 0;
    } else {
        g->c1 = 1; g->c2 = 0; g->c3 = 0; g->c4 = 0;
    }
    const int nx = nxd + 2 * pad;
    const int nz = fs ? nzd + pad : nzd + 2 * pad;
    const int z0 = fs ? 0 : pad;
    g->nz = nz; g->nx = nx; g->z_start = z0;
    g->dx = (real)d->dx; g->dz = (real)d->dz; g->dt = (real)d->dt;
    const size_t N = (size_t)nz * nx;

    /* model embedding + nearest-neighbour extension (fwi/forward.py:195-212) */
    real *vsf = zalloc(N), *vpf = zalloc(N), *rof = zalloc(N);
    for (int i = 0; i < nz; ++i) {
        int si = i - z0;
        if (si < 0) si = 0;
        if (si > nzd - 1) si = nzd - 1;
        for (int j = 0; j < nx; ++j) {
            int sj = j - pad;
            if (sj < 0) sj = 0;
            if (sj > nxd - 1) sj = nxd - 1;
            size_t s = (size_t)si * nxd + sj;
            vsf[IDX(i, j)] = (real)vs[s];
            vpf[IDX(i, j)] = (real)vp[s];
            rof[IDX(i, j)] = (real)rho[s];
        }
    }
    /* materials (fwi/forward.py:222-231) */
    g->M = zalloc(N); g->L2M = zalloc(N); g->L = zalloc(N); g->B = zalloc(N); g->Lr = zalloc(N);
    for (size_t q = 0; q < N; ++q) {
        g->M[q] = rof[q] * (vsf[q] * vsf[q]);
        g->L2M[q] = rof[q] * (vpf[q] * vpf[q]);
        g->L[q] = g->L2M[q] - 2 * g->M[q];
        g->B[q] = (real)1.0 / rof[q];
        g->Lr[q] = -g->L[q] / g->L2M[q];
    }
    free(vsf); free(vpf); free(rof);

    /* C-PML coefficients (fwi/forward.py:35-104) */
    double vpmax = vp[0];
    for (size_t q = 1; q < (size_t)nzd * nxd; ++q) if (vp[q] > vpmax) vpmax = vp[q];
    const double Lpml = pad * d->dx;
    double d0;
    if (d->d0_f32) {
        float t = (float)(-3.0f * (float)vpmax);
        t = t * (float)log(1e-3);
        t = t / (float)(2.0 * Lpml);
        d0 = (double)t;
    } else {
        d0 = -(2 + 1) * vpmax * log(1e-3) / (2 * Lpml);
    }
    g->kx = zalloc(N); g->kz = zalloc(N); g->bx = zalloc(N); g->bz = zalloc(N);
    g->ax = zalloc(N); g->az = zalloc(N);
    double *dxa = (double *)calloc(N, sizeof(double)), *dza = (double *)calloc(N, sizeof(double));
    double *kxa = (double *)malloc(N * sizeof(double)), *kza = (double *)malloc(N * sizeof(double));
    double *alx = (double *)calloc(N, sizeof(double)), *alz = (double *)calloc(N, sizeof(double));
    for (size_t q = 0; q < N; ++q) { kxa[q] = 1.0; kza[q] = 1.0; }
    for (int i = 0; i < pad; ++i) {
        double dist = (i + 1) * d->dx / Lpml;
        double dp = d0 * (dist * dist), kp = 1.0 + (2.0 - 1.0) * (dist * dist);
        double ap = M_PI * d->fc * (1.0 - dist);
        int cl = pad - 1 - i, cr = nx - pad + i;
        for (int r = 0; r < nz; ++r) {
            dxa[IDX(r, cl)] = dp; kxa[IDX(r, cl)] = kp; alx[IDX(r, cl)] = ap;
            dxa[IDX(r, cr)] = dp; kxa[IDX(r, cr)] = kp; alx[IDX(r, cr)] = ap;
        }
        int rb = (fs ? nzd : pad + nzd) + i;
        for (int c = 0; c < nx; ++c) { dza[IDX(rb, c)] = dp; kza[IDX(rb, c)] = kp; alz[IDX(rb, c)] = ap; }
        if (!fs) {
            int rt = pad - 1 - i;
            for (int c = 0; c < nx; ++c) { dza[IDX(rt, c)] = dp; kza[IDX(rt, c)] = kp; alz[IDX(rt, c)] = ap; }
        }
    }
    for (size_t q = 0; q < N; ++q) {
        double bx = exp(-(dxa[q] / kxa[q] + alx[q]) * d->dt);
        double bz = exp(-(dza[q] / kza[q] + alz[q]) * d->dt);
        double dnx = kxa[q] * (dxa[q] + kxa[q] * alx[q]);
        double dnz = kza[q] * (dza[q] + kza[q] * alz[q]);
        g->bx[q] = (real)bx; g->bz[q] = (real)bz;
        g->kx[q] = (real)kxa[q]; g->kz[q] = (real)kza[q];
        g->ax[q] = (real)(dnx > 1e-10 ? dxa[q] * (bx - 1.0) / dnx : 0.0);
        g->az[q] = (real)(dnz > 1e-10 ? dza[q] * (bz - 1.0) / dnz : 0.0);
    }
    free(dxa); free(dza); free(kxa); free(kza); free(alx); free(alz);

    /* source / receivers in padded coordinates (fwi/forward.py:241-242) */
    g->sx = src_x + pad; g->sz = src_z + z0;
    if (g->sx < 0 || g->sx >= nx || g->sz < 0 || g->sz >= nz) { grid_free(g); return -2; }
    g->nrec = rec_x ? d->nrec : 0;
    g->rx = (int *)malloc(sizeof(int) * (g->nrec ? g->nrec : 1));
    g->rz = (int *)malloc(sizeof(int) * (g->nrec ? g->nrec : 1));
    for (int r = 0; r < g->nrec; ++r) {
        g->rx[r] = rec_x[r] + pad; g->rz[r] = rec_z[r] + z0;
        if (g->rx[r] < 0 || g->rx[r] >= nx || g->rz[r] < 0 || g->rz[r] >= nz) { grid_free(g); return -3; }
    }
    g->work = zalloc(N * 24);
    return 0;
}

/* ---------------------------------------------------------------- forward step */

/* fwi/forward.py:250-469.  C: carry (15 arrays), w: src_wavelet[it].
 * inter (NINTER arrays, optional): post-PML derivatives used by the step. */
static void fwd_step(grid_t *g, real **C, real w, real **inter)
{
    const int nz = g->nz, nx = g->nx, fd = g->fd;
    const size_t N = (size_t)nz * nx;
    const real c1 = g->c1, c2 = g->c2, c3 = g->c3, c4 = g->c4;
    const real dx = g->dx, dz = g->dz, dt = g->dt;
    real *U = C[C_U], *V = C[C_V], *ex = C[C_EX], *ez = C[C_EZ], *es = C[C_ES];
    real *W = g->work;
    real *L2M_ex = W, *L_ez = W + N, *M_es = W + 2 * N, *L2M_ez = W + 3 * N, *L_ex = W + 4 * N;
    real *Dx_L2M_ex = W + 5 * N, *Dx_L_ez = W + 6 * N, *Dz_M_es = W + 7 * N, *Dx_M_es = W + 8 * N;
    real *Dz_L2M_ez = W + 9 * N, *Dz_L_ex = W + 10 * N, *Dx_U = W + 11 * N, *Dz_V = W + 12 * N;
    real *Dz_U = W + 13 * N, *Dx_V = W + 14 * N;
    const real *M = g->M, *L2M = g->L2M, *L = g->L, *B = g->B;

    /* 1) U update (:253-308) */
    for (size_t q = 0; q < N; ++q) { L2M_ex[q] = L2M[q] * ex[q]; L_ez[q] = L[q] * ez[q]; M_es[q] = 2 * M[q] * es[q]; }

    memset(Dx_L2M_ex, 0, N * sizeof(real));
    slab(Dx_L2M_ex, L2M_ex, nx, 0, nz - 1, 0, nx - 1, c1, 0, 1, 0, 0, 0);
    if (fd >= 4) slab(Dx_L2M_ex, L2M_ex, nx, 0, nz - 1, 1, nx - 2, c2, 0, 2, 0, -1, 1);
    if (fd >= 8) {
        slab(Dx_L2M_ex, L2M_ex, nx, 0, nz - 1, 2, nx - 3, c3, 0, 3, 0, -2, 1);
        slab(Dx_L2M_ex, L2M_ex, nx, 0, nz - 1, 3, nx - 4, c4, 0, 4, 0, -3, 1);
    }
    pml_apply(Dx_L2M_ex, g->kx, C[P_DX_L2M_EX], g->bx, g->ax, N);

    memset(Dx_L_ez, 0, N * sizeof(real));
    slab(Dx_L_ez, L_ez, nx, 0, nz - 1, 0, nx - 1, c1, 0, 1, 0, 0, 0);
    if (fd >= 4) slab(Dx_L_ez, L_ez, nx, 0, nz - 1, 1, nx - 2, c2, 0, 2, 0, -1, 1);
    if (fd >= 8) {
        slab(Dx_L_ez, L_ez, nx, 0, nz - 1, 2, nx - 3, c3, 0, 3, 0, -2, 1);
        slab(Dx_L_ez, L_ez, nx, 0, nz - 1, 3, nx - 4, c4, 0, 4, 0, -3, 1);
    }
    pml_apply(Dx_L_ez, g->kx, C[P_DX_L_EZ], g->bx, g->ax, N);

    memset(Dz_M_es, 0, N * sizeof(real));
    slab(Dz_M_es, M_es, nx, 1, nz - 1, 1, nx - 1, c1, 0, 0, -1, 0, 0);
    if (fd >= 4) slab(Dz_M_es, M_es, nx, 2, nz - 1, 1, nx - 1, c2, 1, 0, -2, 0, 1);
    if (fd >= 8) {
        slab(Dz_M_es, M_es, nx, 3, nz - 2, 1, nx - 1, c3, 2, 0, -3, 0, 1);
        slab(Dz_M_es, M_es, nx, 4, nz - 3, 1, nx - 1, c4, 3, 0, -4, 0, 1);
    }
    if (g->fs)
        for (int j = 1; j < nx - 1; ++j) Dz_M_es[IDX(0, j)] = 2 * c1 * M_es[IDX(0, j)];
    pml_apply(Dz_M_es, g->kz, C[P_DZ_M_ES], g->bz, g->az, N);

    for (int i = 0; i < nz - 1; ++i)
        for (int j = 1; j < nx - 1; ++j) {
            size_t q = IDX(i, j);
            U[q] = U[q] + dt / dx * B[q] * Dx_L2M_ex[q] + dt / dx * B[q] * Dx_L_ez[q]
                 + dt / dz * B[q] * Dz_M_es[q];
        }

    /* 2) V update (:310-367) */
    for (size_t q = 0; q < N; ++q) { L2M_ez[q] = L2M[q] * ez[q]; L_ex[q] = L[q] * ex[q]; }

    memset(Dx_M_es, 0, N * sizeof(real));
    slab(Dx_M_es, M_es, nx, 0, nz - 1, 1, nx - 1, c1, 0, 0, 0, -1, 0);
    if (fd >= 4) slab(Dx_M_es, M_es, nx, 0, nz - 1, 2, nx - 1, c2, 0, 1, 0, -2, 1);
    if (fd >= 8) {
        slab(Dx_M_es, M_es, nx, 0, nz - 1, 3, nx - 2, c3, 0, 2, 0, -3, 1);
        slab(Dx_M_es, M_es, nx, 0, nz - 1, 4, nx - 3, c4, 0, 3, 0, -4, 1);
    }
    pml_apply(Dx_M_es, g->kx, C[P_DX_M_ES], g->bx, g->ax, N);

    memset(Dz_L2M_ez, 0, N * sizeof(real));
    slab(Dz_L2M_ez, L2M_ez, nx, 0, nz - 1, 1, nx - 1, c1, 1, 0, 0, 0, 0);
    if (fd >= 4) slab(Dz_L2M_ez, L2M_ez, nx, 1, nz - 2, 1, nx - 1, c2, 2, 0, -1, 0, 1);
    if (fd >= 8) {
        slab(Dz_L2M_ez, L2M_ez, nx, 2, nz - 3, 1, nx - 1, c3, 3, 0, -2, 0, 1);
        slab(Dz_L2M_ez, L2M_ez, nx, 3, nz - 4, 1, nx - 1, c4, 4, 0, -3, 0, 1);
    }
    pml_apply(Dz_L2M_ez, g->kz, C[P_DZ_L2M_EZ], g->bz, g->az, N);

    memset(Dz_L_ex, 0, N * sizeof(real));
    slab(Dz_L_ex, L_ex, nx, 0, nz - 1, 1, nx - 1, c1, 1, 0, 0, 0, 0);
    if (fd >= 4) slab(Dz_L_ex, L_ex, nx, 1, nz - 2, 1, nx - 1, c2, 2, 0, -1, 0, 1);
    if (fd >= 8) {
        slab(Dz_L_ex, L_ex, nx, 2, nz - 3, 1, nx - 1, c3, 3, 0, -2, 0, 1);
        slab(Dz_L_ex, L_ex, nx, 3, nz - 4, 1, nx - 1, c4, 4, 0, -3, 0, 1);
    }
    pml_apply(Dz_L_ex, g->kz, C[P_DZ_L_EX], g->bz, g->az, N);

    for (int i = 0; i < nz - 1; ++i)
        for (int j = 1; j < nx - 1; ++j) {
            size_t q = IDX(i, j);
            V[q] = V[q] + dt / dx * B[q] * Dx_M_es[q] + dt / dz * B[q] * Dz_L2M_ez[q]
                 + dt / dz * B[q] * Dz_L_ex[q];
        }
    if (g->src_type == SRC_FORCE) {
        size_t q = IDX(g->sz, g->sx);
        V[q] = V[q] + dt / (dx * dz) * B[q] * w;
    }

    /* 3) exx update (:369-383) */
    memset(Dx_U, 0, N * sizeof(real));
    slab(Dx_U, U, nx, 0, nz, 1, nx, c1, 0, 0, 0, -1, 0);
    if (fd >= 4) slab(Dx_U, U, nx, 0, nz, 2, nx - 1, c2, 0, 1, 0, -2, 1);
    if (fd >= 8) {
        slab(Dx_U, U, nx, 0, nz, 3, nx - 2, c3, 0, 2, 0, -3, 1);
        slab(Dx_U, U, nx, 0, nz, 4, nx - 3, c4, 0, 3, 0, -4, 1);
    }
    pml_apply(Dx_U, g->kx, C[P_DX_U], g->bx, g->ax, N);
    for (int i = 0; i < nz; ++i)
        for (int j = 1; j < nx; ++j) ex[IDX(i, j)] = ex[IDX(i, j)] + dt / dx * Dx_U[IDX(i, j)];

    /* 4) ezz update + free surface (:385-404) */
    memset(Dz_V, 0, N * sizeof(real));
    if (g->fs)
        for (int j = 0; j < nx - 1; ++j)
            Dz_V[IDX(0, j)] = g->Lr[IDX(0, j)] * Dx_U[IDX(0, j)] * dz / dx;
    slab(Dz_V, V, nx, 1, nz, 0, nx - 1, c1, 0, 0, -1, 0, 0);
    if (fd >= 4) slab(Dz_V, V, nx, 2, nz - 1, 0, nx - 1, c2, 1, 0, -2, 0, 1);
    if (fd >= 8) {
        slab(Dz_V, V, nx, 3, nz - 2, 0, nx - 1, c3, 2, 0, -3, 0, 1);
        slab(Dz_V, V, nx, 4, nz - 3, 0, nx - 1, c4, 3, 0, -4, 0, 1);
    }
    pml_apply(Dz_V, g->kz, C[P_DZ_V], g->bz, g->az, N);
    for (size_t q = 0; q < N; ++q) ez[q] = ez[q] + dt / dz * Dz_V[q];

    /* 5) moment source (:406-411) */
    if (g->src_type == SRC_MOMENT) {
        size_t q = IDX(g->sz, g->sx);
        real lam_mu_s = L[q] + M[q];
        real src_term = w * dt / (2 * lam_mu_s * dx * dz);
        ex[q] = ex[q] + src_term;
        ez[q] = ez[q] + src_term;
    }

    /* 6) exz update (:413-444) */
    memset(Dz_U, 0, N * sizeof(real));
    slab(Dz_U, U, nx, 0, nz - 1, 1, nx, c1, 1, 0, 0, 0, 0);
    if (fd >= 4) slab(Dz_U, U, nx, 1, nz - 2, 1, nx, c2, 2, 0, -1, 0, 1);
    if (fd >= 8) {
        slab(Dz_U, U, nx, 2, nz - 3, 1, nx, c3, 3, 0, -2, 0, 1);
        slab(Dz_U, U, nx, 3, nz - 4, 1, nx, c4, 4, 0, -3, 0, 1);
    }
    pml_apply(Dz_U, g->kz, C[P_DZ_U], g->bz, g->az, N);

    memset(Dx_V, 0, N * sizeof(real));
    slab(Dx_V, V, nx, 0, nz - 1, 0, nx - 1, c1, 0, 1, 0, 0, 0);
    if (fd >= 4) slab(Dx_V, V, nx, 0, nz - 1, 1, nx - 2, c2, 0, 2, 0, -1, 1);
    if (fd >= 8) {
        slab(Dx_V, V, nx, 0, nz - 1, 2, nx - 3, c3, 0, 3, 0, -2, 1);
        slab(Dx_V, V, nx, 0, nz - 1, 3, nx - 4, c4, 0, 4, 0, -3, 1);
    }
    pml_apply(Dx_V, g->kx, C[P_DX_V], g->bx, g->ax, N);

    for (int i = 0; i < nz - 1; ++i)
        for (int j = 0; j < nx - 1; ++j) {
            size_t q = IDX(i, j);
            es[q] = es[q] + (real)0.5 * (dt / dz * Dz_U[q] + dt / dx * Dx_V[q]);
        }

    if (inter) {
        memcpy(inter[I_DX_L2M_EX], Dx_L2M_ex, N * sizeof(real));
        memcpy(inter[I_DX_L_EZ], Dx_L_ez, N * sizeof(real));
        memcpy(inter[I_DZ_M_ES], Dz_M_es, N * sizeof(real));
        memcpy(inter[I_DX_M_ES], Dx_M_es, N * sizeof(real));
        memcpy(inter[I_DZ_L2M_EZ], Dz_L2M_ez, N * sizeof(real));
        memcpy(inter[I_DZ_L_EX], Dz_L_ex, N * sizeof(real));
        memcpy(inter[I_DX_U], Dx_U, N * sizeof(real));
    }
}

/* ---------------------------------------------------------------- adjoint step */

/* fwi/adjoint_jax_kernel.py:189-476.  A: adjoint carry (15 arrays, modified in
 * place from carry-out adjoint to carry-in adjoint).  recy: receiver adjoints
 * at this step, [4][nrec] with stride `rstride` between components (or NULL).
 * Returns src_wavelet_a[it].
 *
 * Model gradient (optional, gm != NULL): gm[0..3] accumulate dJ/dM, dJ/dL,
 * dJ/dL2M, dJ/dB on the full grid, treating M, L, L2M, B as independent; the
 * free-surface ratio and the moment-source factor are chained into L, L2M, M
 * here.  fin: forward carry-in of this step; inter: forward intermediates of
 * this step; w: src_wavelet[it]. */
static real adj_step(grid_t *g, real **A, const real *recy, size_t rstride,
                     real **gm, real **fin, real **inter, real w)
{
    const int nz = g->nz, nx = g->nx, fd = g->fd;
    const size_t N = (size_t)nz * nx;
    const real c1 = g->c1, c2 = g->c2, c3 = g->c3, c4 = g->c4;
    const real dx = g->dx, dz = g->dz, dt = g->dt;
    const real *M = g->M, *L2M = g->L2M, *L = g->L, *B = g->B;
    real *U_a = A[C_U], *V_a = A[C_V], *ex_a = A[C_EX], *ez_a = A[C_EZ], *es_a = A[C_ES];
    real *W = g->work;
    real *Dz_U_a = W, *Dx_V_a = W + N, *Dz_V_a = W + 2 * N, *Dx_U_a = W + 3 * N;
    real *Dx_M_es_a = W + 4 * N, *Dz_L2M_ez_a = W + 5 * N, *Dz_L_ex_a = W + 6 * N;
    real *M_es_a = W + 7 * N, *L2M_ez_a = W + 8 * N, *L_ex_a = W + 9 * N;
    real *Dx_L2M_ex_a = W + 10 * N, *Dx_L_ez_a = W + 11 * N, *Dz_M_es_a = W + 12 * N;
    real *L2M_ex_a = W + 13 * N, *L_ez_a = W + 14 * N;
    real src_wav_a_t = 0;
    const size_t qs = IDX(g->sz, g->sx);

    /* 0-T) receiver injection (:203-206) */
    if (recy)
        for (int r = 0; r < g->nrec; ++r) {
            size_t q = IDX(g->rz[r], g->rx[r]);
            U_a[q] += recy[r];
            V_a[q] += recy[rstride + r];
            ex_a[q] += recy[2 * rstride + r];
            ez_a[q] += recy[3 * rstride + r];
        }

    /* 5-T) exz update (:212-250) */
    memset(Dz_U_a, 0, N * sizeof(real));
    memset(Dx_V_a, 0, N * sizeof(real));
    for (int i = 0; i < nz - 1; ++i)
        for (int j = 0; j < nx - 1; ++j) {
            Dz_U_a[IDX(i, j)] = (real)0.5 * dt / dz * es_a[IDX(i, j)];
            Dx_V_a[IDX(i, j)] = (real)0.5 * dt / dx * es_a[IDX(i, j)];
        }
    pml_apply_T(Dz_U_a, A[P_DZ_U], g->kz, g->bz, g->az, N);
    pml_apply_T(Dx_V_a, A[P_DX_V], g->kx, g->bx, g->ax, N);

    scat(U_a, Dz_U_a, nx, 1, nz, 1, nx, c1, -1, 0);
    scat(U_a, Dz_U_a, nx, 0, nz - 1, 1, nx, -c1, 0, 0);
    if (fd >= 4) {
        scat(U_a, Dz_U_a, nx, 3, nz, 1, nx, c2, -2, 0);
        scat(U_a, Dz_U_a, nx, 0, nz - 3, 1, nx, -c2, 1, 0);
    }
    if (fd >= 8) {
        scat(U_a, Dz_U_a, nx, 5, nz, 1, nx, c3, -3, 0);
        scat(U_a, Dz_U_a, nx, 0, nz - 5, 1, nx, -c3, 2, 0);
        scat(U_a, Dz_U_a, nx, 7, nz, 1, nx, c4, -4, 0);
        scat(U_a, Dz_U_a, nx, 0, nz - 7, 1, nx, -c4, 3, 0);
    }
    scat(V_a, Dx_V_a, nx, 0, nz - 1, 1, nx, c1, 0, -1);
    scat(V_a, Dx_V_a, nx, 0, nz - 1, 0, nx - 1, -c1, 0, 0);
    if (fd >= 4) {
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 3, nx, c2, 0, -2);
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 0, nx - 3, -c2, 0, 1);
    }
    if (fd >= 8) {
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 5, nx, c3, 0, -3);
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 0, nx - 5, -c3, 0, 2);
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 7, nx, c4, 0, -4);
        scat(V_a, Dx_V_a, nx, 0, nz - 1, 0, nx - 7, -c4, 0, 3);
    }

    /* 4.5-T) moment source (:259-262); its model term: d(src)/d(L+M) */
    if (g->src_type == SRC_MOMENT) {
        real lam_mu_s = L[qs] + M[qs];
        src_wav_a_t = (dt / (2 * lam_mu_s * dx * dz)) * (ex_a[qs] + ez_a[qs]);
        if (gm) {
            real glm = -(w * dt / (2 * dx * dz)) / (lam_mu_s * lam_mu_s) * (ex_a[qs] + ez_a[qs]);
            gm[0][qs] += glm; /* M */
            gm[1][qs] += glm; /* L */
        }
    }

    /* 4-T) ezz update (:266-294) */
    for (size_t q = 0; q < N; ++q) Dz_V_a[q] = dt / dz * ez_a[q];
    pml_apply_T(Dz_V_a, A[P_DZ_V], g->kz, g->bz, g->az, N);
    memset(Dx_U_a, 0, N * sizeof(real));
    if (g->fs) {
        for (int j = 0; j < nx - 1; ++j)
            Dx_U_a[IDX(0, j)] += g->Lr[IDX(0, j)] * (dz / dx) * Dz_V_a[IDX(0, j)];
        if (gm) {
            /* Dz_V[0,j] = Lr*Dx_U'*dz/dx with Lr = -L/L2M */
            for (int j = 0; j < nx - 1; ++j) {
                size_t q = IDX(0, j);
                real glr = Dz_V_a[q] * inter[I_DX_U][q] * dz / dx;
                gm[1][q] += -glr / L2M[q];
                gm[2][q] += glr * L[q] / (L2M[q] * L2M[q]);
            }
        }
    }
    scat(V_a, Dz_V_a, nx, 1, nz, 0, nx - 1, c1, 0, 0);
    scat(V_a, Dz_V_a, nx, 0, nz - 1, 0, nx - 1, -c1, 1, 0);
    if (fd >= 4) {
        scat(V_a, Dz_V_a, nx, 3, nz, 0, nx - 1, c2, -1, 0);
        scat(V_a, Dz_V_a, nx, 0, nz - 3, 0, nx - 1, -c2, 2, 0);
    }
    if (fd >= 8) {
        scat(V_a, Dz_V_a, nx, 5, nz, 0, nx - 1, c3, -2, 0);
        scat(V_a, Dz_V_a, nx, 0, nz - 5, 0, nx - 1, -c3, 3, 0);
        scat(V_a, Dz_V_a, nx, 7, nz, 0, nx - 1, c4, -3, 0);
        scat(V_a, Dz_V_a, nx, 0, nz - 7, 0, nx - 1, -c4, 4, 0);
    }

    /* 3-T) exx update (:299-317) */
    for (int i = 0; i < nz; ++i)
        for (int j = 1; j < nx; ++j) Dx_U_a[IDX(i, j)] += dt / dx * ex_a[IDX(i, j)];
    pml_apply_T(Dx_U_a, A[P_DX_U], g->kx, g->bx, g->ax, N);
    scat(U_a, Dx_U_a, nx, 0, nz, 1, nx, c1, 0, 0);
    scat(U_a, Dx_U_a, nx, 0, nz, 0, nx - 1, -c1, 0, 1);
    if (fd >= 4) {
        scat(U_a, Dx_U_a, nx, 0, nz, 3, nx, c2, 0, -1);
        scat(U_a, Dx_U_a, nx, 0, nz, 0, nx - 3, -c2, 0, 2);
    }
    if (fd >= 8) {
        scat(U_a, Dx_U_a, nx, 0, nz, 5, nx, c3, 0, -2);
        scat(U_a, Dx_U_a, nx, 0, nz, 0, nx - 5, -c3, 0, 3);
        scat(U_a, Dx_U_a, nx, 0, nz, 7, nx, c4, 0, -3);
        scat(U_a, Dx_U_a, nx, 0, nz, 0, nx - 7, -c4, 0, 4);
    }

    /* 2-T) force source (:322-323); its model term: d(src)/dB */
    if (g->src_type == SRC_FORCE) {
        src_wav_a_t = (dt / (dx * dz)) * B[qs] * V_a[qs];
        if (gm) gm[3][qs] += (dt / (dx * dz)) * w * V_a[qs];
    }

    /* 2-T) V update (:328-385) */
    memset(Dx_M_es_a, 0, N * sizeof(real));
    memset(Dz_L2M_ez_a, 0, N * sizeof(real));
    memset(Dz_L_ex_a, 0, N * sizeof(real));
    for (int i = 0; i < nz - 1; ++i)
        for (int j = 1; j < nx - 1; ++j) {
            size_t q = IDX(i, j);
            Dx_M_es_a[q] = (dt / dx) * B[q] * V_a[q];
            Dz_L2M_ez_a[q] = (dt / dz) * B[q] * V_a[q];
            Dz_L_ex_a[q] = (dt / dz) * B[q] * V_a[q];
            if (gm)
                gm[3][q] += V_a[q] * ((dt / dx) * inter[I_DX_M_ES][q] + (dt / dz) * inter[I_DZ_L2M_EZ][q]
                                      + (dt / dz) * inter[I_DZ_L_EX][q]);
        }
    pml_apply_T(Dx_M_es_a, A[P_DX_M_ES], g->kx, g->bx, g->ax, N);
    pml_apply_T(Dz_L2M_ez_a, A[P_DZ_L2M_EZ], g->kz, g->bz, g->az, N);
    pml_apply_T(Dz_L_ex_a, A[P_DZ_L_EX], g->kz, g->bz, g->az, N);

    memset(M_es_a, 0, N * sizeof(real));
    scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 1, nx - 1, c1, 0, 0);
    scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 0, nx - 2, -c1, 0, 1);
    if (fd >= 4) {
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 3, nx, c2, 0, -1);
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 0, nx - 3, -c2, 0, 2);
    }
    if (fd >= 8) {
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 5, nx, c3, 0, -2);
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 0, nx - 5, -c3, 0, 3);
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 7, nx, c4, 0, -3);
        scat(M_es_a, Dx_M_es_a, nx, 0, nz - 1, 0, nx - 7, -c4, 0, 4);
    }
    memset(L2M_ez_a, 0, N * sizeof(real));
    scat(L2M_ez_a, Dz_L2M_ez_a, nx, 1, nz, 1, nx - 1, c1, -1, 0);
    scat(L2M_ez_a, Dz_L2M_ez_a, nx, 0, nz - 1, 1, nx - 1, -c1, 0, 0);
    if (fd >= 4) {
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 3, nz, 1, nx - 1, c2, -2, 0);
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 0, nz - 3, 1, nx - 1, -c2, 1, 0);
    }
    if (fd >= 8) {
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 5, nz, 1, nx - 1, c3, -3, 0);
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 0, nz - 5, 1, nx - 1, -c3, 2, 0);
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 7, nz, 1, nx - 1, c4, -4, 0);
        scat(L2M_ez_a, Dz_L2M_ez_a, nx, 0, nz - 7, 1, nx - 1, -c4, 3, 0);
    }
    memset(L_ex_a, 0, N * sizeof(real));
    scat(L_ex_a, Dz_L_ex_a, nx, 1, nz, 1, nx - 1, c1, -1, 0);
    scat(L_ex_a, Dz_L_ex_a, nx, 0, nz - 1, 1, nx - 1, -c1, 0, 0);
    if (fd >= 4) {
        scat(L_ex_a, Dz_L_ex_a, nx, 3, nz, 1, nx - 1, c2, -2, 0);
        scat(L_ex_a, Dz_L_ex_a, nx, 0, nz - 3, 1, nx - 1, -c2, 1, 0);
    }
    if (fd >= 8) {
        scat(L_ex_a, Dz_L_ex_a, nx, 5, nz, 1, nx - 1, c3, -3, 0);
        scat(L_ex_a, Dz_L_ex_a, nx, 0, nz - 5, 1, nx - 1, -c3, 2, 0);
        scat(L_ex_a, Dz_L_ex_a, nx, 7, nz, 1, nx - 1, c4, -4, 0);
        scat(L_ex_a, Dz_L_ex_a, nx, 0, nz - 7, 1, nx - 1, -c4, 3, 0);
    }

    /* 1-T) U update (:390-455) */
    memset(Dx_L2M_ex_a, 0, N * sizeof(real));
    memset(Dx_L_ez_a, 0, N * sizeof(real));
    memset(Dz_M_es_a, 0, N * sizeof(real));
    for (int i = 0; i < nz - 1; ++i)
        for (int j = 1; j < nx - 1; ++j) {
            size_t q = IDX(i, j);
            Dx_L2M_ex_a[q] = (dt / dx) * B[q] * U_a[q];
            Dx_L_ez_a[q] = (dt / dx) * B[q] * U_a[q];
            Dz_M_es_a[q] = (dt / dz) * B[q] * U_a[q];
            if (gm)
                gm[3][q] += U_a[q] * ((dt / dx) * inter[I_DX_L2M_EX][q] + (dt / dx) * inter[I_DX_L_EZ][q]
                                      + (dt / dz) * inter[I_DZ_M_ES][q]);
        }
    pml_apply_T(Dx_L2M_ex_a, A[P_DX_L2M_EX], g->kx, g->bx, g->ax, N);
    pml_apply_T(Dx_L_ez_a, A[P_DX_L_EZ], g->kx, g->bx, g->ax, N);
    pml_apply_T(Dz_M_es_a, A[P_DZ_M_ES], g->kz, g->bz, g->az, N);

    memset(L2M_ex_a, 0, N * sizeof(real));
    scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 1, nx, c1, 0, -1);
    scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 0, nx - 1, -c1, 0, 0);
    if (fd >= 4) {
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 3, nx, c2, 0, -2);
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 0, nx - 3, -c2, 0, 1);
    }
    if (fd >= 8) {
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 5, nx, c3, 0, -3);
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 0, nx - 5, -c3, 0, 2);
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 7, nx, c4, 0, -4);
        scat(L2M_ex_a, Dx_L2M_ex_a, nx, 0, nz - 1, 0, nx - 7, -c4, 0, 3);
    }
    memset(L_ez_a, 0, N * sizeof(real));
    scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 1, nx, c1, 0, -1);
    scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 0, nx - 1, -c1, 0, 0);
    if (fd >= 4) {
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 3, nx, c2, 0, -2);
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 0, nx - 3, -c2, 0, 1);
    }
    if (fd >= 8) {
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 5, nx, c3, 0, -3);
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 0, nx - 5, -c3, 0, 2);
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 7, nx, c4, 0, -4);
        scat(L_ez_a, Dx_L_ez_a, nx, 0, nz - 1, 0, nx - 7, -c4, 0, 3);
    }
    scat(M_es_a, Dz_M_es_a, nx, 1, nz - 1, 1, nx - 1, c1, 0, 0);
    scat(M_es_a, Dz_M_es_a, nx, 0, nz - 2, 1, nx - 1, -c1, 1, 0);
    if (fd >= 4) {
        scat(M_es_a, Dz_M_es_a, nx, 3, nz, 1, nx - 1, c2, -1, 0);
        scat(M_es_a, Dz_M_es_a, nx, 0, nz - 3, 1, nx - 1, -c2, 2, 0);
    }
    if (fd >= 8) {
        scat(M_es_a, Dz_M_es_a, nx, 5, nz, 1, nx - 1, c3, -2, 0);
        scat(M_es_a, Dz_M_es_a, nx, 0, nz - 5, 1, nx - 1, -c3, 3, 0);
        scat(M_es_a, Dz_M_es_a, nx, 7, nz, 1, nx - 1, c4, -3, 0);
        scat(M_es_a, Dz_M_es_a, nx, 0, nz - 7, 1, nx - 1, -c4, 4, 0);
    }
    if (g->fs)
        for (int j = 1; j < nx - 1; ++j) M_es_a[IDX(0, j)] += (real)2.0 * c1 * Dz_M_es_a[IDX(0, j)];

    /* model gradient from the constitutive products (forward :254, :311) */
    if (gm) {
        const real *exi = fin[C_EX], *ezi = fin[C_EZ], *esi = fin[C_ES];
        for (size_t q = 0; q < N; ++q) {
            gm[0][q] += M_es_a[q] * 2 * esi[q];
            gm[1][q] += L_ez_a[q] * ezi[q] + L_ex_a[q] * exi[q];
            gm[2][q] += L2M_ex_a[q] * exi[q] + L2M_ez_a[q] * ezi[q];
        }
    }

    /* constitutive transpose (:462-464) */
    for (size_t q = 0; q < N; ++q) {
        ex_a[q] = ex_a[q] + L2M[q] * L2M_ex_a[q] + L[q] * L_ex_a[q];
        ez_a[q] = ez_a[q] + L[q] * L_ez_a[q] + L2M[q] * L2M_ez_a[q];
        es_a[q] = es_a[q] + (real)2.0 * M[q] * M_es_a[q];
    }
    return src_wav_a_t;
}

/* fwi/imaging.py:125-141 for one time frame: U_a/V_a (adjoint velocities of
 * frame it) and the forward strains of frame it; periodic centred differences
 * as jnp.roll gives them. g_lam/g_mu accumulate on the full padded grid. */
static void imaging_frame(grid_t *g, const real *U_a, const real *V_a, const real *ex,
                          const real *ez, const real *es, double *g_lam, double *g_mu)
{
    const int nz = g->nz, nx = g->nx;
    const real dx = g->dx, dz = g->dz, dt = g->dt;
    const real *B = g->B;
    for (int i = 0; i < nz; ++i) {
        int ip = (i + 1) % nz, im = (i - 1 + nz) % nz;
        for (int j = 0; j < nx; ++j) {
            int jp = (j + 1) % nx, jm = (j - 1 + nx) % nx;
            real dx_BU = (B[IDX(i, jp)] * U_a[IDX(i, jp)] - B[IDX(i, jm)] * U_a[IDX(i, jm)]) / (2 * dx);
            real dz_BV = (B[IDX(ip, j)] * V_a[IDX(ip, j)] - B[IDX(im, j)] * V_a[IDX(im, j)]) / (2 * dz);
            real dz_BU = (B[IDX(ip, j)] * U_a[IDX(ip, j)] - B[IDX(im, j)] * U_a[IDX(im, j)]) / (2 * dz);
            real dx_BV = (B[IDX(i, jp)] * V_a[IDX(i, jp)] - B[IDX(i, jm)] * V_a[IDX(i, jm)]) / (2 * dx);
            size_t q = IDX(i, j);
            g_lam[q] -= (double)dt * (double)((ex[q] + ez[q]) * (dx_BU + dz_BV));
            g_mu[q] -= (double)dt * (double)(2 * ex[q] * dx_BU + 2 * ez[q] * dz_BV + es[q] * (dz_BU + dx_BV));
        }
    }
}

/* ---------------------------------------------------------------- public API */

static real **carry_alloc(size_t N)
{
    real **C = (real **)malloc(sizeof(real *) * NCARRY);
    for (int k = 0; k < NCARRY; ++k) C[k] = zalloc(N);
    return C;
}
static void carry_free(real **C)
{
    if (!C) return;
    for (int k = 0; k < NCARRY; ++k) free(C[k]);
    free(C);
}

int ORACLE(grid_shape)(const oracle_desc *d, int32_t *nz, int32_t *nx)
{
    *nx = d->nx_dom + 2 * d->pad;
    *nz = d->free_surface ? d->nz_dom + d->pad : d->nz_dom + 2 * d->pad;
    return 0;
}

/* PML profile arrays as _pml_coefficients returns them (full grid), for tests:
 * out = [6][nz][nx] in the order kx, kz, bx, bz, ax, az. */
int ORACLE(pml_profiles)(const oracle_desc *d, const double *vp_dom, double *out)
{
    grid_t g;
    const size_t nd = (size_t)d->nz_dom * d->nx_dom;
    double *ones = (double *)malloc(nd * sizeof(double));
    for (size_t q = 0; q < nd; ++q) ones[q] = 1.0;
    int rc = grid_init(&g, d, ones, vp_dom, ones, 0, 0, SRC_FORCE, NULL, NULL);
    free(ones);
    if (rc) return rc;
    const size_t N = (size_t)g.nz * g.nx;
    const real *arrs[6] = {g.kx, g.kz, g.bx, g.bz, g.ax, g.az};
    for (int k = 0; k < 6; ++k)
        for (size_t q = 0; q < N; ++q) out[k * N + q] = (double)arrs[k][q];
    grid_free(&g);
    return 0;
}

/* Forward modelling of one shot (fwi/forward.py:119-501).
 * rec_out  [4][nt][nrec] (vx, vz, ex, ez), optional.
 * full_mask bits 0..4 (vx, vz, ex, ez, es): frames written to full_out in bit
 *           order, [nfull][nt][nz][nx], optional.
 * energy_mask bits 0..4: Sum_t field^2 into energy_out [ne][nz][nx] (FP64,
 *           accumulated with +=), optional (fwi/illumination.py:38-41). */
int ORACLE(forward)(const oracle_desc *d, const double *vs, const double *vp, const double *rho,
                    int32_t src_x, int32_t src_z, int32_t src_type, const double *wavelet,
                    const int32_t *rec_x, const int32_t *rec_z, double *rec_out,
                    int32_t full_mask, double *full_out, int32_t energy_mask, double *energy_out)
{
    grid_t g;
    int rc = grid_init(&g, d, vs, vp, rho, src_x, src_z, src_type, rec_x, rec_z);
    if (rc) return rc;
    const int nz = g.nz, nx = g.nx, nt = d->nt, nrec = d->nrec;
    const size_t N = (size_t)nz * nx;
    real **C = carry_alloc(N);
    const int fmap[5] = {C_U, C_V, C_EX, C_EZ, C_ES};
    for (int it = 0; it < nt; ++it) {
        fwd_step(&g, C, (real)wavelet[it], NULL);
        if (rec_out)
            for (int r = 0; r < nrec; ++r) {
                size_t q = (size_t)g.rz[r] * nx + g.rx[r];
                for (int c = 0; c < 4; ++c)
                    rec_out[((size_t)c * nt + it) * nrec + r] = (double)C[fmap[c]][q];
            }
        int kf = 0, ke = 0;
        for (int b = 0; b < 5; ++b) {
            if (full_out && (full_mask >> b & 1)) {
                double *dst = full_out + ((size_t)kf * nt + it) * N;
                for (size_t q = 0; q < N; ++q) dst[q] = (double)C[fmap[b]][q];
                ++kf;
            }
            if (energy_out && (energy_mask >> b & 1)) {
                double *dst = energy_out + (size_t)ke * N;
                for (size_t q = 0; q < N; ++q) { double v = (double)C[fmap[b]][q]; dst[q] += v * v; }
                ++ke;
            }
        }
    }
    carry_free(C);
    grid_free(&g);
    return 0;
}

/* Adjoint sweep of one shot (fwi/adjoint_jax_kernel.py:61-483), optionally
 * with the exact model gradient and the reference imaging formula.
 * rec_adj   [4][nt][nrec] receiver-data adjoints (vx, vz, ex, ez).
 * src_wav_a [nt] source-wavelet adjoint, optional.
 * gmat      [4][nz][nx] += dJ/d(M, L, L2M, B) on the full grid, optional.
 * img       [3][nz][nx] += (g_lam, g_mu, g_rho_lame) of fwi/imaging.py on the
 *           full grid (before cropping), optional; g_rho_lame is the density
 *           term of fwi/imaging.py:145-154, -dt sum_{n=1}^{nt-2} (vx[n] (U_a[n+1]
 *           - U_a[n-1]) + vz[n] (V_a[n+1] - V_a[n-1])) / (2 dt), with vx[n] the
 *           forward velocity after step n and U_a[n] the adjoint carry of step n.
 * hist_mask bits 0..4 (U_a, V_a, ex_a, ez_a, es_a): frames written to
 *           hist_out [nh][nt][nz][nx]; frame it is the carry of adjoint step
 *           it, as adjoint_jax(return_wavefields=...) returns them.
 * wavelet   needed when gmat or img is requested (forward recompute).
 * ckpt      forward checkpoint interval for the recompute (>=1). */
int ORACLE(adjoint)(const oracle_desc *d, const double *vs, const double *vp, const double *rho,
                    int32_t src_x, int32_t src_z, int32_t src_type, const double *wavelet,
                    const int32_t *rec_x, const int32_t *rec_z, const double *rec_adj,
                    double *src_wav_a, double *gmat, double *img,
                    int32_t hist_mask, double *hist_out, int32_t ckpt)
{
    grid_t g;
    int rc = grid_init(&g, d, vs, vp, rho, src_x, src_z, src_type, rec_x, rec_z);
    if (rc) return rc;
    const int nz = g.nz, nx = g.nx, nt = d->nt, nrec = d->nrec;
    const size_t N = (size_t)nz * nx;
    const int need_fwd = (gmat != NULL) || (img != NULL);
    if (ckpt < 1) ckpt = 1;
    real **A = carry_alloc(N);
    real *recy = (real *)malloc(sizeof(real) * 4 * (size_t)(nrec ? nrec : 1));
    real **gm = NULL;
    double *glam = NULL, *gmu = NULL, *grl = NULL;
    real *vnx = NULL, *vnz = NULL;   /* velocities after the first step of the segment processed before */
    if (gmat) { gm = (real **)malloc(4 * sizeof(real *)); for (int k = 0; k < 4; ++k) gm[k] = zalloc(N); }
    if (img) {
        glam = (double *)calloc(N, sizeof(double)); gmu = (double *)calloc(N, sizeof(double));
        grl = (double *)calloc(N, sizeof(double));
        vnx = zalloc(N); vnz = zalloc(N);
    }

    /* forward checkpoints (carry-in of steps 0, ckpt, 2*ckpt, ...) */
    const int nseg = (nt + ckpt - 1) / ckpt;
    real ***ck = NULL, ***seg = NULL, **inter = NULL, **tmp = NULL;
    /* ckpt >= nt keeps every step of the first forward pass (one segment, no
     * recompute of it); otherwise checkpoints and a recompute per segment */
    const int store_all = need_fwd && nseg == 1;
    if (need_fwd) {
        ck = (real ***)malloc(sizeof(real **) * nseg);
        seg = (real ***)malloc(sizeof(real **) * (ckpt + 1));
        for (int k = 0; k <= ckpt; ++k) seg[k] = carry_alloc(N);
        if (store_all) {
            ck[0] = NULL;
            for (int it = 0; it < nt; ++it) {
                for (int k = 0; k < NCARRY; ++k) memcpy(seg[it + 1][k], seg[it][k], N * sizeof(real));
                fwd_step(&g, seg[it + 1], (real)wavelet[it], NULL);
            }
        } else {
            real **C = carry_alloc(N);
            for (int it = 0; it < nt; ++it) {
                if (it % ckpt == 0) {
                    ck[it / ckpt] = carry_alloc(N);
                    for (int k = 0; k < NCARRY; ++k) memcpy(ck[it / ckpt][k], C[k], N * sizeof(real));
                }
                fwd_step(&g, C, (real)wavelet[it], NULL);
            }
            carry_free(C);
        }
        inter = (real **)malloc(sizeof(real *) * NINTER);
        for (int k = 0; k < NINTER; ++k) inter[k] = zalloc(N);
        tmp = carry_alloc(N);
    }

    const int hmap[5] = {C_U, C_V, C_EX, C_EZ, C_ES};
    for (int s = nseg - 1; s >= 0; --s) {
        const int t0 = s * ckpt, t1 = (t0 + ckpt < nt) ? t0 + ckpt : nt;
        if (need_fwd && !store_all) {
            /* seg[k] = carry-in of step t0+k, for k = 0 .. t1-t0 (last = carry-out of t1-1) */
            for (int k = 0; k < NCARRY; ++k) memcpy(seg[0][k], ck[s][k], N * sizeof(real));
            for (int it = t0; it < t1; ++it) {
                for (int k = 0; k < NCARRY; ++k) memcpy(seg[it - t0 + 1][k], seg[it - t0][k], N * sizeof(real));
                fwd_step(&g, seg[it - t0 + 1], (real)wavelet[it], NULL);
            }
        }
        for (int it = t1 - 1; it >= t0; --it) {
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < nrec; ++r)
                    recy[(size_t)c * nrec + r] = (real)rec_adj[((size_t)c * nt + it) * nrec + r];
            if (need_fwd) {
                /* regenerate this step's forward intermediates */
                for (int k = 0; k < NCARRY; ++k) memcpy(tmp[k], seg[it - t0][k], N * sizeof(real));
                fwd_step(&g, tmp, (real)wavelet[it], inter);
            }
            real sa = adj_step(&g, A, recy, (size_t)nrec, gm, need_fwd ? seg[it - t0] : NULL, inter,
                               need_fwd ? (real)wavelet[it] : 0);
            if (src_wav_a) src_wav_a[it] = (double)sa;
            if (img) {
                real **fo = seg[it - t0 + 1]; /* forward carry-out of step it = frame it */
                imaging_frame(&g, A[C_U], A[C_V], fo[C_EX], fo[C_EZ], fo[C_ES], glam, gmu);
                /* density term regrouped by adjoint step it: the reference's sum
                 * over n of vx[n] U_a[n+1] meets this step at n = it-1 (it >= 2),
                 * its sum of vx[n] U_a[n-1] at n = it+1 (it <= nt-3) */
                const real *um = seg[it - t0][C_U], *wm = seg[it - t0][C_V];   /* vx, vz after step it-1 */
                const real *up = (it + 1 < t1) ? seg[it - t0 + 2][C_U] : vnx;    /* after step it+1 */
                const real *wp = (it + 1 < t1) ? seg[it - t0 + 2][C_V] : vnz;
                for (size_t q = 0; q < N; ++q) {
                    double t = 0.0;
                    if (it >= 2 && it <= nt - 1) t += (double)um[q] * A[C_U][q] + (double)wm[q] * A[C_V][q];
                    if (it <= nt - 3) t -= (double)up[q] * A[C_U][q] + (double)wp[q] * A[C_V][q];
                    grl[q] -= 0.5 * t;
                }
            }
            if (hist_out) {
                int kh = 0;
                for (int b = 0; b < 5; ++b)
                    if (hist_mask >> b & 1) {
                        double *dst = hist_out + ((size_t)kh * nt + it) * N;
                        for (size_t q = 0; q < N; ++q) dst[q] = (double)A[hmap[b]][q];
                        ++kh;
                    }
            }
        }
        if (img && need_fwd) {   /* velocities after step t0, for step t0 - 1 of the next (earlier) segment */
            memcpy(vnx, seg[1][C_U], N * sizeof(real));
            memcpy(vnz, seg[1][C_V], N * sizeof(real));
        }
    }

    if (gmat)
        for (int k = 0; k < 4; ++k)
            for (size_t q = 0; q < N; ++q) gmat[k * N + q] += (double)gm[k][q];
    if (img)
        for (size_t q = 0; q < N; ++q) { img[q] += glam[q]; img[N + q] += gmu[q]; img[2 * N + q] += grl[q]; }

    if (need_fwd) {
        for (int k = 0; k < nseg; ++k)
            if (ck[k]) carry_free(ck[k]);
        free(ck);
        for (int k = 0; k <= ckpt; ++k) carry_free(seg[k]);
        free(seg);
        for (int k = 0; k < NINTER; ++k) free(inter[k]);
        free(inter);
        carry_free(tmp);
    }
    if (gm) { for (int k = 0; k < 4; ++k) free(gm[k]); free(gm); }
    free(glam); free(gmu); free(grl); free(vnx); free(vnz);
    free(recy);
    carry_free(A);
    grid_free(&g);
    return 0;
}

/* Many shots at once, OpenMP over shots (the timed CPU baseline).  Runs the
 * forward with receiver output for every shot: src [nshot][3] = (x, z, type),
 * wavelet [nt] shared, rec_out [nshot][4][nt][nrec]. */
int ORACLE(forward_batch)(const oracle_desc *d, const double *vs, const double *vp, const double *rho,
                          int32_t nshot, const int32_t *src, const double *wavelet,
                          const int32_t *rec_x, const int32_t *rec_z, double *rec_out)
{
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int s = 0; s < nshot; ++s) {
        int rc = ORACLE(forward)(d, vs, vp, rho, src[3 * s], src[3 * s + 1], src[3 * s + 2], wavelet,
                                 rec_x, rec_z,
                                 rec_out ? rec_out + (size_t)s * 4 * d->nt * d->nrec : NULL,
                                 0, NULL, 0, NULL);
        if (rc) bad |= 1;
    }
    return bad ? -1 : 0;
}

/* Forward + adjoint + exact gradient for many shots (OpenMP over shots).
 * rec_adj [nshot][4][nt][nrec]; gmat_out [nshot][4][nz][nx] (per shot). */
int ORACLE(gradient_batch)(const oracle_desc *d, const double *vs, const double *vp, const double *rho,
                           int32_t nshot, const int32_t *src, const double *wavelet,
                           const int32_t *rec_x, const int32_t *rec_z, const double *rec_adj,
                           double *gmat_out, double *img_out, int32_t ckpt)
{
    int32_t nz, nx;
    ORACLE(grid_shape)(d, &nz, &nx);
    const size_t N = (size_t)nz * nx;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int s = 0; s < nshot; ++s) {
        int rc = ORACLE(adjoint)(d, vs, vp, rho, src[3 * s], src[3 * s + 1], src[3 * s + 2], wavelet,
                                 rec_x, rec_z, rec_adj + (size_t)s * 4 * d->nt * d->nrec, NULL,
                                 gmat_out ? gmat_out + (size_t)s * 4 * N : NULL,
                                 img_out ? img_out + (size_t)s * 3 * N : NULL, 0, NULL, ckpt);
        if (rc) bad |= 1;
    }
    return bad ? -1 : 0;
}
