// C ABI of the B200 elastic velocity-strain solver: handle, workspace plan,
// model/geometry set-up kernels, launch sequences (captured into CUDA graphs)
// and the residual/misfit kernel.  Declarations: include/stfwi.h.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/stfwi.h"
#include "stencils.cuh"
#include "post.cuh"

using namespace stfwi;

namespace {

constexpr int MAX_SOS = 16;
constexpr int MAX_CHAINS = 4;   // chains a pass may be split into (streams per handle)

struct GraphKey {
    int kind;    // 0 forward, 1 adjoint, 2 illumination
    uint32_t flags;
    int nshot;
    bool operator<(const GraphKey &o) const
    {
        if (kind != o.kind) return kind < o.kind;
        if (flags != o.flags) return flags < o.flags;
        return nshot < o.nshot;
    }
};

}  // namespace

struct stfwi_handle {
    stfwi_desc d{};
    Geo g{};
    int device = 0;
    std::string err;

    // model
    float *vs = nullptr, *vp = nullptr, *rho = nullptr;     // physical [nd]
    float *B = nullptr, *L2M = nullptr, *L = nullptr, *M = nullptr, *Lr = nullptr;
    float *bx = nullptr, *ax = nullptr, *ikx = nullptr, *bz = nullptr, *az = nullptr, *ikz = nullptr;
    float *vpmax = nullptr;
    float *MATS = nullptr;  // [4][nz][P]: B, L2M, L, M
    bool model_set = false;
    // tensor maps of the staged tiles and per-kernel shot groups
    int sms = 148;
    int accp = 5;   // accumulator planes per shot group (7 with the density terms)
    CUtensorMap tmS{}, tmV{}, tmE{}, tmPQ{};
    CUtensorMap tmUo{}, tmSo{}, tmPQo{}, tmEo{};   // own-cell boxes of the two-column kernels
    CUtensorMap tmH{};        // history [shot][slot*snf + field][nz_dom][nx_dom] (own-cell carry-in boxes)
    bool hist_tma = false;    // tmH valid: pad and nx_dom multiples of 4 (16-byte box rows)
    // staged tilings: tiles tw columns wide; fwd_vel/fwd_str/adj_a tiles tha
    // = ra * NWARP rows high, adj_b tiles thb = rb * NWARP rows high (ra, rb:
    // rows per thread, 1 or 2, set by set_tiling)
    int tw = TX4, ra = RPT_DEFAULT, rb = RPT_DEFAULT, tha = RPT_DEFAULT * NWARP, thb = RPT_DEFAULT * NWARP;
    int ntx = 1, ntza = 1, ntzb = 1;                       // tile counts
    int ntz_max = 1;                                       // tile rows of the lowest tiles (array sizes)
    int *tile_startA = nullptr, *tile_recA = nullptr;      // receivers grouped by the tw x tha tiles
    int *tile_startB = nullptr, *tile_recB = nullptr;      // receivers grouped by the tw x thb tiles
    int *tordA = nullptr, *tordB = nullptr;                // tile dispatch orders, boundary tiles first
    int grp[4] = {1, 1, 1, 1}, spgk[4] = {1, 1, 1, 1};
    int acc_groups = 1, acc_used = 1;
    int lr_used = 1;  // rows of accLr written by the U_a/V_a phase (one per block row of shots)
    int tuned[4] = {0, 0, 0, 0};  // shots per block chosen by stfwi_autotune (0: default)

    // shots / receivers
    int nshot = 0;
    int *sx = nullptr, *sz = nullptr, *stype = nullptr;
    float *wav = nullptr, *fcoef = nullptr, *mcoef = nullptr, *lm = nullptr;
    int *rx = nullptr, *rz = nullptr;
    bool shots_set = false, recv_set = false;
    std::vector<int> rec_x_h, rec_z_h;   // physical-domain receiver indices (preconditioner geometry)

    // gradient post-processing (fwi/gradient.py:266-277) and preconditioners
    double post_sigma = 0.0;
    int post_radius = 0;
    bool post_taper = false, post_illum = false;
    double *pw = nullptr;      // Gaussian weights [2 * POST_MAX_RADIUS + 1]
    double *ptaper = nullptr, *pillum = nullptr, *ptmp = nullptr;   // [nd] each
    double *pscr = nullptr;    // [nz][nx] scratch (eprecond3)
    double *pmax = nullptr;    // reductions

    // state
    float *F = nullptr, *A = nullptr, *PX = nullptr, *PZ = nullptr;
    float *rec = nullptr, *rec_adj = nullptr;
    float *snap = nullptr, *row0 = nullptr;
    int slots = 0;
    // checkpointing: history of ck steps (slots = ck + 1, slot 0 = carry-in of
    // the segment); ncp > 0 state checkpoints every ck steps (ncp = 0: the
    // history covers all nt steps)
    int ck = 0, ncp = 0;
    float *CKF = nullptr, *CKPX = nullptr, *CKPZ = nullptr;
    double *acc = nullptr, *accLr = nullptr, *gtmp = nullptr;
    double *energy = nullptr;
    double *mis_trace = nullptr, *mis_shot = nullptr;
    float *src_a = nullptr;
    float *obs = nullptr;
    int *status = nullptr;
    bool stored = false;  // last forward kept its strain history

    cudaStream_t hs = nullptr;
    // a pass split into chains over the shot groups: the chains it may use
    // (1-4, stfwi_set_chains), the chains of the pass being recorded, and
    // the streams of chains 1.. (chain 0 runs on the pass's own stream)
    int chains = 2, nchain_cur = 1;
    cudaStream_t hsx[MAX_CHAINS - 1] = {};
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr;
    cudaEvent_t ev_join[MAX_CHAINS - 1] = {};
    // sampled kernel timing: pev[k] holds (start, stop) pairs per sampled step
    int prof_every = 0;
    std::vector<cudaEvent_t> pev[4];
    double prof_ms[4] = {0, 0, 0, 0};
    long long prof_cnt[4] = {0, 0, 0, 0};
    std::map<GraphKey, cudaGraphExec_t> graphs;
    size_t bytes = 0;
};

namespace {

stfwi_status fail(stfwi_handle *h, stfwi_status st, const char *fmt, ...)
{
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return st;
}

#define CK(h, call)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), STFWI_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                \
    } while (0)

struct Plan {
    long long nz, nx, P, nd, zs_n, xs_n;
    size_t fields, psi, snap, row0, acc, rec, misc, ckpt;
    size_t total() const { return fields + psi + snap + row0 + acc + rec + misc + ckpt; }
};

// FP64 gradient accumulator groups: one per group of shots of the strain
// phase, at least two shots per group unless the descriptor asks otherwise
int acc_groups_of(const stfwi_desc *d)
{
    const int spg0 = d->shot_group > 0 ? d->shot_group : 2;
    return std::max(1, (d->max_shots + spg0 - 1) / spg0);
}

// k: history segment length (k = nt: every step kept, no checkpoints)
Plan make_plan(const stfwi_desc *d, int k)
{
    Plan p{};
    p.nx = d->nx_dom + 2LL * d->pad;
    p.nz = d->free_surface ? d->nz_dom + (long long)d->pad : d->nz_dom + 2LL * d->pad;
    p.P = (p.nx + 31) / 32 * 32;
    p.nd = (long long)d->nz_dom * d->nx_dom;
    p.xs_n = 2LL * d->pad;
    p.zs_n = d->free_surface ? d->pad : 2LL * d->pad;
    const long long S = d->max_shots;
    const int G = acc_groups_of(d);
    p.fields = (size_t)2 * S * F_N * p.nz * p.P * sizeof(float);
    p.psi = (size_t)S * (NPX * p.nz * p.xs_n + NPZ * p.zs_n * p.P) * sizeof(float);
    // history fields per slot: the stresses, plus U and V for the density
    // gradient (want_gradient == 2); with checkpoints and velocities one more
    // slot holds the first output of the following segment
    const int snf = d->want_gradient == 2 ? 5 : 3;
    const int slots = k + 1 + ((snf == 5 && k < d->nt) ? 1 : 0);
    p.snap = d->want_gradient ? (size_t)S * slots * snf * p.nd * sizeof(float) : 0;
    p.row0 = (d->want_gradient && d->free_surface) ? (size_t)S * slots * d->nx_dom * sizeof(float) : 0;
    const long long ncp = (d->want_gradient && k < d->nt) ? (d->nt + k - 1) / k : 0;
    p.ckpt = (size_t)ncp * S * (F_N * p.nz * p.P + PX_NFWD * p.nz * p.xs_n + PZ_NFWD * p.zs_n * p.P) * sizeof(float);
    p.acc = (size_t)G * ((snf == 5 ? 7 : 5) * p.nd + d->nx_dom) * sizeof(double) + 3 * p.nd * 2 * sizeof(double);
    p.rec = (size_t)2 * S * 4 * d->nt * std::max(d->nrec, 1) * sizeof(float)
          + (size_t)S * d->nt * std::max(d->nrec, 1) * sizeof(float);
    p.misc = (size_t)(8 * p.nz * p.P + 4 * p.nd) * sizeof(float) + (size_t)2 * p.nz * p.nx * sizeof(double)
           + (size_t)3 * p.nd * sizeof(double)
           + (size_t)S * (d->nt + 16) * sizeof(float) + (size_t)S * (std::max(d->nrec, 1) + 1) * sizeof(double)
           + (1 << 20);
    return p;
}

// ---------------------------------------------------------------- set-up kernels

__global__ void k_materials(int nz, int nx, int P, int nz_dom, int nx_dom, int z0, int pad,
                            const float *vs, const float *vp, const float *rho, float *B, float *L2M,
                            float *L, float *M, float *Lr)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nx || i >= nz) return;
    // nearest-neighbour extension into the PML (fwi/forward.py:195-212)
    const int si = min(max(i - z0, 0), nz_dom - 1), sj = min(max(j - pad, 0), nx_dom - 1);
    const long long s = (long long)si * nx_dom + sj;
    const float r = rho[s], a = vs[s], b = vp[s];
    // fwi/forward.py:222-231
    const float m = r * (a * a), l2m = r * (b * b), l = l2m - 2.f * m;
    const long long o = (long long)i * P + j;
    B[o] = 1.0f / r;
    L2M[o] = l2m;
    L[o] = l;
    M[o] = m;
    if (i == 0) Lr[j] = -l / l2m;
}

__global__ void k_vpmax(const float *vp, long long n, float *out)
{
    __shared__ float red[1024];
    float m = -INFINITY;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) m = fmaxf(m, vp[q]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// C-PML profiles (fwi/forward.py:35-104), as 1-D arrays: the reference's
// 2-D coefficient arrays are constant along rows (x) / columns (z).
__global__ void k_pml(int nz, int nx, int nz_dom, int pad, int fs, double dx, double dt, double fc,
                      const float *vpmax, float *bx, float *ax, float *ikx, float *bz, float *az,
                      float *ikz)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double Lp = pad * dx;
    // d0 with the float32 arithmetic of the reference's promotion rules
    float d0f = -3.0f * vpmax[0];
    d0f = d0f * (float)log(1e-3);
    d0f = d0f / (float)(2.0 * Lp);
    const double d0 = d0f;
    auto coef = [&](int i, float *b, float *a, float *ik) {
        if (i < 0) { *b = 1.f; *a = 0.f; *ik = 1.f; return; }
        const double dist = (i + 1) * dx / Lp;
        const double dd = d0 * (dist * dist), kk = 1.0 + (2.0 - 1.0) * (dist * dist);
        const double al = M_PI * fc * (1.0 - dist);
        const double bb = exp(-(dd / kk + al) * dt);
        const double den = kk * (dd + kk * al);
        *b = (float)bb;
        *a = (float)(den > 1e-10 ? dd * (bb - 1.0) / den : 0.0);
        *ik = (float)(1.0 / kk);
    };
    if (t < nx) {
        int i = -1;
        if (t < pad) i = pad - 1 - t;
        else if (t >= nx - pad) i = t - (nx - pad);
        coef(i, bx + t, ax + t, ikx + t);
    }
    if (t < nz) {
        int i = -1;
        const int bottom = fs ? nz_dom : pad + nz_dom;
        if (t >= bottom) i = t - bottom;
        else if (!fs && t < pad) i = pad - 1 - t;
        coef(i, bz + t, az + t, ikz + t);
    }
}

__global__ void k_src_coefs(int nshot, const int *sx, const int *sz, int P, const float *B,
                            const float *L, const float *M, float dtdxdz, float dx, float dz,
                            float *fcoef, float *mcoef, float *lm)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshot) return;
    const long long o = (long long)sz[s] * P + sx[s];
    fcoef[s] = dtdxdz * B[o];
    const float lms = L[o] + M[o];
    lm[s] = lms;
    mcoef[s] = 2.f * lms * dx * dz;
}

// adjoint prologue: receiver injection of the last step into exx_a, ezz_a
__global__ void k_inject_last(Geo g, const int *rx, const int *rz, const float *rec_adj, float *A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nshot * g.nrec) return;
    const int s = t / g.nrec, r = t % g.nrec;
    const long long o = (long long)rz[r] * g.P + rx[r];
    const float *src = rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)(g.nt - 1) * g.nrec + r;
    atomicAdd(A + ((long long)s * F_N + F_EX) * g.fstride + o, src[2LL * g.nt * g.nrec]);
    atomicAdd(A + ((long long)s * F_N + F_EZ) * g.fstride + o, src[3LL * g.nt * g.nrec]);
}

// Residual preparation (fwi/gradient.py:139-156, fwi/filters.py), one thread
// per trace: r = F T (pred - obs); misfit = scale/nshot * mean(r^2);
// cotangent = 2 scale/(nshot N) T^T F^T r, F^T being the time-reversed cascade.
struct SosParams {
    int nsos;
    double c[MAX_SOS][5];  // b0 b1 b2 a1 a2, normalised by a0
};

__global__ void k_misfit(Geo g, int comp, int n_taper, SosParams sp, double scale, int nshot_norm,
                         const float *rec, const float *obs, float *rec_adj, double *mis_trace)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nshot * g.nrec) return;
    const int s = t / g.nrec, r = t % g.nrec;
    const long long NR = g.nrec, NT = g.nt;
    const float *pred = rec + (long long)s * 4 * NT * NR + comp * NT * NR + r;
    const float *ob = obs + (long long)s * NT * NR + r;
    float *out = rec_adj + (long long)s * 4 * NT * NR;
    for (int c = 0; c < 4; ++c)
        if (c != comp)
            for (long long n = 0; n < NT; ++n) out[c * NT * NR + n * NR + r] = 0.f;
    float *cot = out + comp * NT * NR + r;
    const int tstart = g.nt - min(n_taper, g.nt);
    const double npi = M_PI;
    auto taper = [&](int n) -> double {
        if (n_taper <= 0 || n < tstart) return 1.0;
        const int m = n - tstart + 1;
        return (cos((double)m / n_taper * npi) + 1.0) / 2.0;
    };
    double st[MAX_SOS][4];
    for (int k = 0; k < sp.nsos; ++k) st[k][0] = st[k][1] = st[k][2] = st[k][3] = 0.0;
    double sum = 0.0;
    for (int n = 0; n < g.nt; ++n) {
        const double tp = taper(n);
        double x = tp * (double)pred[n * NR] - tp * (double)ob[n * NR];
        for (int k = 0; k < sp.nsos; ++k) {
            const double y = sp.c[k][0] * x + sp.c[k][1] * st[k][0] + sp.c[k][2] * st[k][1]
                           - sp.c[k][3] * st[k][2] - sp.c[k][4] * st[k][3];
            st[k][1] = st[k][0]; st[k][0] = x; st[k][3] = st[k][2]; st[k][2] = y;
            x = y;
        }
        sum += x * x;
        cot[n * NR] = (float)x;
    }
    const double coef = 2.0 * scale / ((double)nshot_norm * (double)NT * (double)NR);
    for (int k = 0; k < sp.nsos; ++k) st[k][0] = st[k][1] = st[k][2] = st[k][3] = 0.0;
    for (int n = g.nt - 1; n >= 0; --n) {
        double x = coef * (double)cot[n * NR];
        for (int k = sp.nsos - 1; k >= 0; --k) {
            const double y = sp.c[k][0] * x + sp.c[k][1] * st[k][0] + sp.c[k][2] * st[k][1]
                           - sp.c[k][3] * st[k][2] - sp.c[k][4] * st[k][3];
            st[k][1] = st[k][0]; st[k][0] = x; st[k][3] = st[k][2]; st[k][2] = y;
            x = y;
        }
        cot[n * NR] = (float)(taper(n) * x);
    }
    mis_trace[t] = scale / nshot_norm * sum / ((double)NT * (double)NR);
}

__global__ void k_misfit_reduce(int nshot, int nrec, const double *mis_trace, double *mis_shot)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshot) return;
    double a = 0.0;
    for (int r = 0; r < nrec; ++r) a += mis_trace[(long long)s * nrec + r];
    mis_shot[s] = a;
}

// (M, L, L2M) or (lambda, mu) partial sums -> (Vs, Vp, rho) gradients on the
// physical grid.  EXACT: M = rho Vs^2, L2M = rho Vp^2, L = L2M - 2M; the
// free-surface ratio Lr = -L/L2M contributes on row 0.  IMAGING:
// fwi/imaging.py:165-167.
__global__ void k_finalize(Geo g, int groups, int accp, int lr_rows, const double *acc, const double *accLr,
                           const float *L2M, const float *L, const float *vs, const float *vp,
                           const float *rho, int want_exact, int want_img, double *out_exact,
                           double *out_img)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= g.nd) return;
    const int pi = (int)(q / g.nx_dom), pj = (int)(q % g.nx_dom);
    double gM = 0, gL = 0, gL2M = 0, gla = 0, gmu = 0, gB = 0, grl = 0;
    for (int k = 0; k < groups; ++k) {
        const double *a = acc + (long long)k * accp * g.nd + q;
        gM += a[0]; gL += a[g.nd]; gL2M += a[2 * g.nd]; gla += a[3 * g.nd]; gmu += a[4 * g.nd];
        if (accp == 7) { gB += a[5 * g.nd]; grl += a[6 * g.nd]; }
    }
    const double r = rho[q], a = vs[q], b = vp[q];
    if (want_exact) {
        if (g.fs && pi == 0) {
            double glr = 0;
            for (int k = 0; k < lr_rows; ++k) glr += accLr[(long long)k * g.nx_dom + pj];
            const long long o = (long long)(pi + g.z0) * g.P + pj + g.pad;
            const double l2m = L2M[o], l = L[o];
            gL += -glr / l2m;
            gL2M += glr * l / (l2m * l2m);
        }
        out_exact[q] = 2.0 * r * a * (gM - 2.0 * gL);
        out_exact[g.nd + q] = 2.0 * r * b * (gL2M + gL);
        // M = rho Vs^2, L2M = rho Vp^2, L = rho (Vp^2 - 2 Vs^2), B = 1/rho
        out_exact[2 * g.nd + q] = accp == 7 ? a * a * gM + b * b * gL2M + (b * b - 2.0 * a * a) * gL - gB / (r * r) : 0.0;
    }
    if (want_img) {
        out_img[q] = 2.0 * r * a * (gmu - 2.0 * gla);
        out_img[g.nd + q] = 2.0 * r * b * gla;
        out_img[2 * g.nd + q] = (b * b - 2.0 * a * a) * gla + a * a * gmu + grl;
    }
}

// ---------------------------------------------------------------- launch helpers

Mat mat_of(stfwi_handle *h)
{
    return Mat{h->B, h->L2M, h->L, h->M, h->Lr, h->bx, h->ax, h->ikx, h->bz, h->az, h->ikz};
}
Shots shots_of(stfwi_handle *h)
{
    return Shots{h->sx, h->sz, h->stype, h->wav, h->fcoef, h->mcoef, h->lm};
}

// event pair of sampled step n around kernel k (0 fwd_vel, 1 fwd_str, 2 adj_a, 3 adj_b)
inline void prof_mark(stfwi_handle *h, int k, int n, int which, cudaStream_t st)
{
    if (h->prof_every <= 0 || n % h->prof_every) return;
    const size_t idx = 2 * (size_t)(n / h->prof_every) + which;
    // inside stream capture only an external record becomes an event node of
    // the graph; outside (the autotuner's passes) a plain record
    if (idx >= h->pev[k].size()) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(h->pev[k][idx], st, cudaEventRecordExternal);
    else cudaEventRecord(h->pev[k][idx], st);
}

// the shot groups of kernel k that a launch covers: all of them (part < 0)
// or chain `part`'s share of the h->nchain_cur chains of a split pass
// (consecutive groups); the Geo of the launch carries the first group
Geo part_geo(const stfwi_handle *h, int k, int part, int *ngroups)
{
    Geo g = h->g;
    const int G = h->grp[k], C = h->nchain_cur;
    if (part < 0) {
        *ngroups = G;
        return g;
    }
    const int a = G * part / C, b = G * (part + 1) / C;
    g.goff = a;
    *ngroups = b - a;
    return g;
}

// chains a pass may run as: independent chains over the shot groups (the
// shots never interact, the shared sums are atomic) when every stencil
// kernel groups the shots the same way -- a chain's kernels then touch
// exactly its own shots -- and no sampled timing is on; at most one chain
// per group
int pass_chains(const stfwi_handle *h)
{
    for (int k = 1; k < 4; ++k)
        if (h->spgk[k] != h->spgk[0] || h->grp[k] != h->grp[0]) return 1;
    if (h->prof_every != 0) return 1;
    return std::max(1, std::min(h->chains, h->grp[0]));
}

template <int FD, int R>
void launch_fwd_step_r(stfwi_handle *h, int n, const FwdOut &o, cudaStream_t st, int part)
{
    using Lk = L5<FD, R>;
    const int tiles = h->ntx * h->ntza;
    dim3 block(TX, NWARP);
    Recv rva{h->tile_startA, h->tile_recA, h->rx, h->rz};
    int ng = 0;
    const Geo g0 = part_geo(h, 0, part, &ng);
    prof_mark(h, 0, n, 0, st);
    st_fwd_vel<FD, R><<<dim3(tiles, ng), block, Lk::bytes(Lk::VEL, 2), st>>>(
        g0, mat_of(h), shots_of(h), h->F, h->PX, h->PZ, n, h->spgk[0], h->ntx, h->status, h->tmS, h->tmUo);
    prof_mark(h, 0, n, 1, st);
    prof_mark(h, 1, n, 0, st);
    const Geo g1 = part_geo(h, 1, part, &ng);
    auto str = o.energy ? st_fwd_str<FD, R, true> : st_fwd_str<FD, R, false>;
    str<<<dim3(tiles, ng), block, Lk::bytes(Lk::STR, 2), st>>>(
        g1, mat_of(h), shots_of(h), rva, h->F, h->PX, h->PZ, n, h->spgk[1], h->ntx, o, h->tmV, h->tmSo);
    prof_mark(h, 1, n, 1, st);
}

template <int FD>
void launch_fwd_step(stfwi_handle *h, int n, const FwdOut &o, cudaStream_t st, int part)
{
    if (h->ra == 1) launch_fwd_step_r<FD, 1>(h, n, o, st, part);
    else launch_fwd_step_r<FD, 2>(h, n, o, st, part);
}

template <int FD, int R>
void launch_adj_a_r(stfwi_handle *h, int n, const AdjIn &ai, cudaStream_t st, int part)
{
    using Lk = L5<FD, R>;
    Recv rva{h->tile_startA, h->tile_recA, h->rx, h->rz};
    int ng = 0;
    const Geo ga = part_geo(h, 2, part, &ng);
    st_adj_a<FD, R><<<dim3(h->ntx * h->ntza, ng), dim3(TX, NWARP), Lk::bytes(Lk::ADA, 2), st>>>(
        ga, mat_of(h), rva, h->A, h->PX, h->PZ, n, h->spgk[2], h->ntx, ai, h->status, h->tmE, h->tmPQo);
}

template <int FD, int R>
void launch_adj_b_r(stfwi_handle *h, int n, const AdjOut &ao, cudaStream_t st, int part)
{
    using Lk = L5<FD, R>;
    Recv rvb{h->tile_startB, h->tile_recB, h->rx, h->rz};
    int ng = 0;
    const Geo gb = part_geo(h, 3, part, &ng);
    auto launch = [&](auto kern) {
        kern<<<dim3(h->ntx * h->ntzb, ng), dim3(TX, NWARP), Lk::bytes(Lk::ADB, 2), st>>>(
            gb, mat_of(h), shots_of(h), rvb, h->A, h->PX, h->PZ, n, h->spgk[3], h->ntx, ao, h->status,
            h->tmPQ, h->tmEo, h->tmH);
    };
    const bool rho = h->g.snf == 5;
    if (ao.want_exact && ao.want_img) rho ? launch(st_adj_b<FD, R, true, true, true>) : launch(st_adj_b<FD, R, true, true, false>);
    else if (ao.want_exact) rho ? launch(st_adj_b<FD, R, true, false, true>) : launch(st_adj_b<FD, R, true, false, false>);
    else if (ao.want_img) rho ? launch(st_adj_b<FD, R, false, true, true>) : launch(st_adj_b<FD, R, false, true, false>);
    else launch(st_adj_b<FD, R, false, false, false>);
}

template <int FD>
void launch_adj_step(stfwi_handle *h, int n, const AdjIn &ai, const AdjOut &ao, cudaStream_t st, int part = -1)
{
    prof_mark(h, 2, n, 0, st);
    if (h->ra == 1) launch_adj_a_r<FD, 1>(h, n, ai, st, part);
    else launch_adj_a_r<FD, 2>(h, n, ai, st, part);
    prof_mark(h, 2, n, 1, st);
    prof_mark(h, 3, n, 0, st);
    if (h->rb == 1) launch_adj_b_r<FD, 1>(h, n, ao, st, part);
    else launch_adj_b_r<FD, 2>(h, n, ao, st, part);
    prof_mark(h, 3, n, 1, st);
}


stfwi_status zero_forward_state(stfwi_handle *h, cudaStream_t st)
{
    const Geo &g = h->g;
    CK(h, cudaMemsetAsync(h->F, 0, (size_t)h->nshot * F_N * g.fstride * sizeof(float), st));
    for (int s = 0; s < h->nshot; ++s) {
        CK(h, cudaMemsetAsync(h->PX + (long long)s * NPX * g.xstride, 0,
                              (size_t)PX_NFWD * g.xstride * sizeof(float), st));
        CK(h, cudaMemsetAsync(h->PZ + (long long)s * NPZ * g.zstride, 0,
                              (size_t)PZ_NFWD * g.zstride * sizeof(float), st));
    }
    CK(h, cudaMemsetAsync(h->status, 0, sizeof(int), st));
    return STFWI_OK;
}

stfwi_status zero_adjoint_state(stfwi_handle *h, cudaStream_t st)
{
    const Geo &g = h->g;
    CK(h, cudaMemsetAsync(h->A, 0, (size_t)h->nshot * F_N * g.fstride * sizeof(float), st));
    for (int s = 0; s < h->nshot; ++s) {
        CK(h, cudaMemsetAsync(h->PX + ((long long)s * NPX + PX_NFWD) * g.xstride, 0,
                              (size_t)2 * PXA_N * g.xstride * sizeof(float), st));
        CK(h, cudaMemsetAsync(h->PZ + ((long long)s * NPZ + PZ_NFWD) * g.zstride, 0,
                              (size_t)2 * PZA_N * g.zstride * sizeof(float), st));
    }
    CK(h, cudaMemsetAsync(h->acc, 0, (size_t)h->acc_used * h->accp * g.nd * sizeof(double), st));
    CK(h, cudaMemsetAsync(h->accLr, 0, (size_t)h->lr_used * g.nx_dom * sizeof(double), st));
    return STFWI_OK;
}

// history slot 0 of every shot = the physical cells of the current state
// (the carry-in of the first step of a history segment)
__global__ void k_snap_state(Geo g, int slots, const float *F, float *snap)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (q >= g.nd) return;
    const int pi = (int)(q / g.nx_dom), pj = (int)(q % g.nx_dom);
    const long long o = (long long)(pi + g.z0) * g.P + pj + g.pad;
    float *dst = snap + (long long)s * slots * g.snf * g.nd + q;
#pragma unroll
    for (int f = 0; f < 3; ++f) dst[f * g.nd] = F[((long long)s * F_N + F_EX + f) * g.fstride + o];
    if (g.snf == 5) {
        dst[3 * g.nd] = F[((long long)s * F_N + F_U) * g.fstride + o];
        dst[4 * g.nd] = F[((long long)s * F_N + F_V) * g.fstride + o];
    }
}

void snap_state(stfwi_handle *h, cudaStream_t st)
{
    const Geo &g = h->g;
    k_snap_state<<<dim3((unsigned)((g.nd + 255) / 256), h->nshot), 256, 0, st>>>(g, h->slots, h->F, h->snap);
}

// state of the forward (fields + forward C-PML memories) <-> checkpoint c
stfwi_status copy_ckpt(stfwi_handle *h, int c, bool save, cudaStream_t st)
{
    const Geo &g = h->g;
    const size_t S = (size_t)h->d.max_shots, ns = (size_t)h->nshot;
    float *cf = h->CKF + (size_t)c * S * F_N * g.fstride;
    float *cx = h->CKPX + (size_t)c * S * PX_NFWD * g.xstride;
    float *cz = h->CKPZ + (size_t)c * S * PZ_NFWD * g.zstride;
    const size_t fb = ns * F_N * g.fstride * 4;
    const size_t xw = PX_NFWD * g.xstride * 4, xp = NPX * g.xstride * 4;
    const size_t zw = PZ_NFWD * g.zstride * 4, zp = NPZ * g.zstride * 4;
    if (save) {
        CK(h, cudaMemcpyAsync(cf, h->F, fb, cudaMemcpyDeviceToDevice, st));
        CK(h, cudaMemcpy2DAsync(cx, xw, h->PX, xp, xw, ns, cudaMemcpyDeviceToDevice, st));
        CK(h, cudaMemcpy2DAsync(cz, zw, h->PZ, zp, zw, ns, cudaMemcpyDeviceToDevice, st));
    } else {
        CK(h, cudaMemcpyAsync(h->F, cf, fb, cudaMemcpyDeviceToDevice, st));
        CK(h, cudaMemcpy2DAsync(h->PX, xp, cx, xw, xw, ns, cudaMemcpyDeviceToDevice, st));
        CK(h, cudaMemcpy2DAsync(h->PZ, zp, cz, zw, zw, ns, cudaMemcpyDeviceToDevice, st));
    }
    return STFWI_OK;
}

void fwd_step(stfwi_handle *h, int n, const FwdOut &o, cudaStream_t st, int part = -1)
{
    switch (h->d.fd_order) {
    case 2: launch_fwd_step<2>(h, n, o, st, part); break;
    case 4: launch_fwd_step<4>(h, n, o, st, part); break;
    default: launch_fwd_step<8>(h, n, o, st, part); break;
    }
}

// fork the streams of chains 1 .. C-1 off `st` / join them back (event
// edges of the captured graph); C = h->nchain_cur
stfwi_status fork_chains(stfwi_handle *h, cudaStream_t st)
{
    CK(h, cudaEventRecord(h->ev_fork, st));
    for (int c = 1; c < h->nchain_cur; ++c) CK(h, cudaStreamWaitEvent(h->hsx[c - 1], h->ev_fork, 0));
    return STFWI_OK;
}
stfwi_status join_chains(stfwi_handle *h, cudaStream_t st)
{
    for (int c = 1; c < h->nchain_cur; ++c) {
        CK(h, cudaEventRecord(h->ev_join[c - 1], h->hsx[c - 1]));
        CK(h, cudaStreamWaitEvent(st, h->ev_join[c - 1], 0));
    }
    return STFWI_OK;
}
cudaStream_t chain_stream(const stfwi_handle *h, cudaStream_t st, int c) { return c == 0 ? st : h->hsx[c - 1]; }

// record the whole forward pass (kind 0) or illumination pass (kind 2)
stfwi_status enqueue_forward(stfwi_handle *h, uint32_t flags, int comp, cudaStream_t st)
{
    stfwi_status rc = zero_forward_state(h, st);
    if (rc) return rc;
    FwdOut o{};
    o.rec = h->rec;
    o.status = h->status;
    o.slots = h->slots;
    const bool store = (flags & STFWI_FWD_STORE) != 0;
    if (comp >= 0) {
        CK(h, cudaMemsetAsync(h->energy, 0, (size_t)h->g.nz * h->g.nx * sizeof(double), st));
        o.energy = h->energy;
        o.energy_comp = comp;
    }
    // with checkpoints the history is written later, segment by segment
    const bool hist = store && h->ncp == 0;
    if (hist) snap_state(h, st);
    h->nchain_cur = pass_chains(h);
    const bool split = h->nchain_cur > 1;
    const bool ckpt = store && h->ncp > 0;
    if (split && !ckpt && (rc = fork_chains(h, st))) return rc;
    for (int n = 0; n < h->g.nt; ++n) {
        if (ckpt && n % h->ck == 0) {
            // the checkpoint copy takes every shot: the chains join before
            // it and fork again after it
            if (split && n > 0 && (rc = join_chains(h, st))) return rc;
            stfwi_status r = copy_ckpt(h, n / h->ck, true, st);
            if (r) return r;
            if (split && (rc = fork_chains(h, st))) return rc;
        }
        o.snap = hist ? h->snap : nullptr;
        o.row0 = (hist && h->g.fs) ? h->row0 : nullptr;
        o.slot = n + 1;
        o.slot_row0 = n;
        if (split) {
            for (int c = 0; c < h->nchain_cur; ++c) fwd_step(h, n, o, chain_stream(h, st, c), c);
        } else {
            fwd_step(h, n, o, st);
        }
    }
    if (split && (rc = join_chains(h, st))) return rc;
    CK(h, cudaGetLastError());
    return STFWI_OK;
}

// run `fn` on the handle's stream, ordered after `user` work, replaying a
// captured graph when one exists for `key`
template <class Fn>
stfwi_status run_graph(stfwi_handle *h, GraphKey key, cudaStream_t user, Fn fn)
{
    CK(h, cudaEventRecord(h->ev_in, user));
    CK(h, cudaStreamWaitEvent(h->hs, h->ev_in, 0));
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
        cudaGraph_t graph = nullptr;
        CK(h, cudaStreamBeginCapture(h->hs, cudaStreamCaptureModeThreadLocal));
        stfwi_status rc = fn(h->hs);
        cudaError_t e = cudaStreamEndCapture(h->hs, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fail(h, STFWI_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(h, STFWI_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        it = h->graphs.emplace(key, exec).first;
    }
    CK(h, cudaGraphLaunch(it->second, h->hs));
    CK(h, cudaEventRecord(h->ev_out, h->hs));
    CK(h, cudaStreamWaitEvent(user, h->ev_out, 0));
    return STFWI_OK;
}

void drop_graphs(stfwi_handle *h)
{
    for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
    h->graphs.clear();
}

// add the elapsed times of kernel kind k's sampled pairs (after its pass completed)
void prof_accumulate(stfwi_handle *h, int k)
{
    for (size_t i = 0; i + 1 < h->pev[k].size(); i += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->pev[k][i], h->pev[k][i + 1]) == cudaSuccess) {
            h->prof_ms[k] += ms;
            h->prof_cnt[k] += 1;
        }
    }
    cudaGetLastError();
}

// ---------------------------------------------------------------- TMA set-up

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// row-major float32 array of `rank` dims (x fastest), box of `box` elements
stfwi_status encode(stfwi_handle *h, CUtensorMap *m, void *base, int rank, const cuuint64_t *dims,
                    const cuuint64_t *strides_bytes, const cuuint32_t *box)
{
    auto fn = encode_fn();
    if (!fn) return fail(h, STFWI_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, base, dims, strides_bytes, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(h, STFWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return STFWI_OK;
}

template <typename Lk>
stfwi_status set_smem(stfwi_handle *h, const void *const (&kern)[7])
{
    const size_t bytes[] = {Lk::bytes(Lk::VEL, 2), Lk::bytes(Lk::STR, 2), Lk::bytes(Lk::ADA, 2), Lk::bytes(Lk::ADB, 2),
                            Lk::bytes(Lk::ADB, 2), Lk::bytes(Lk::ADB, 2), Lk::bytes(Lk::ADB, 2)};
    for (int k = 0; k < 7; ++k)
        CK(h, cudaFuncSetAttribute(kern[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes[k]));
    return STFWI_OK;
}

template <int FD, int R>
stfwi_status setup_tma_kernels_r(stfwi_handle *h)
{
    using Lk = L5<FD, R>;
    const void *const kern[7] = {
        (const void *)st_fwd_vel<FD, R>, (const void *)st_fwd_str<FD, R, false>, (const void *)st_adj_a<FD, R>,
        (const void *)st_adj_b<FD, R, true, false, false>, (const void *)st_adj_b<FD, R, true, true, false>,
        (const void *)st_adj_b<FD, R, false, true, false>, (const void *)st_adj_b<FD, R, false, false, false>};
    stfwi_status r = set_smem<Lk>(h, kern);
    if (r) return r;
    CK(h, cudaFuncSetAttribute((const void *)st_fwd_str<FD, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Lk::bytes(Lk::STR, 2)));
    const void *const rho_kern[3] = {(const void *)st_adj_b<FD, R, true, false, true>,
                                     (const void *)st_adj_b<FD, R, true, true, true>,
                                     (const void *)st_adj_b<FD, R, false, true, true>};
    for (const void *k : rho_kern)
        CK(h, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lk::bytes(Lk::ADB, 2)));
    return STFWI_OK;
}

// both tile heights of every kernel of the fd order
template <int FD>
stfwi_status setup_tma_kernels(stfwi_handle *h)
{
    stfwi_status r = setup_tma_kernels_r<FD, 1>(h);
    return r ? r : setup_tma_kernels_r<FD, 2>(h);
}

stfwi_status setup_tensor_maps(stfwi_handle *h)
{
    const Geo &g = h->g;
    const int H = h->d.fd_order / 2;
    const cuuint64_t S = (cuuint64_t)h->d.max_shots;
    const cuuint64_t fdims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.nz, (cuuint64_t)F_N, S};
    const cuuint64_t fstr[3] = {(cuuint64_t)g.P * 4, (cuuint64_t)g.nz * g.P * 4, (cuuint64_t)F_N * g.nz * g.P * 4};
    // staged boxes: the tile plus a 4-column and an H-row halo on each side
    const cuuint32_t bw = (cuuint32_t)(h->tw + 8);
    const cuuint32_t box3[4] = {bw, (cuuint32_t)(h->tha + 2 * H), 3, 1};
    const cuuint32_t box2[4] = {bw, (cuuint32_t)(h->tha + 2 * H), 2, 1};
    const cuuint32_t box2s[4] = {bw, (cuuint32_t)(h->thb + 2 * H), 2, 1};
    stfwi_status r;
    if ((r = encode(h, &h->tmS, h->F, 4, fdims, fstr, box3))) return r;
    if ((r = encode(h, &h->tmV, h->F, 4, fdims, fstr, box2))) return r;
    if ((r = encode(h, &h->tmE, h->A, 4, fdims, fstr, box3))) return r;
    if ((r = encode(h, &h->tmPQ, h->A, 4, fdims, fstr, box2s))) return r;
    {
        const cuuint32_t own2[4] = {(cuuint32_t)h->tw, (cuuint32_t)h->tha, 2, 1};
        const cuuint32_t own3[4] = {(cuuint32_t)h->tw, (cuuint32_t)h->tha, 3, 1};
        if ((r = encode(h, &h->tmUo, h->F, 4, fdims, fstr, own2))) return r;
        if ((r = encode(h, &h->tmSo, h->F, 4, fdims, fstr, own3))) return r;
        if ((r = encode(h, &h->tmPQo, h->A, 4, fdims, fstr, own2))) return r;
        const cuuint32_t own3b[4] = {(cuuint32_t)h->tw, (cuuint32_t)h->thb, 3, 1};
        if ((r = encode(h, &h->tmEo, h->A, 4, fdims, fstr, own3b))) return r;
        // the history box starts at column j0 - pad and its rows are nx_dom
        // floats: both must be multiples of 16 bytes for a tensor copy
        if (h->snap && h->d.pad % 4 == 0 && g.nx_dom % 4 == 0) {
            const cuuint64_t hdims[4] = {(cuuint64_t)g.nx_dom, (cuuint64_t)g.nz_dom,
                                         (cuuint64_t)g.snf * h->slots, S};
            const cuuint64_t hstr[3] = {(cuuint64_t)g.nx_dom * 4, (cuuint64_t)g.nd * 4,
                                        (cuuint64_t)h->slots * g.snf * g.nd * 4};
            if ((r = encode(h, &h->tmH, h->snap, 4, hdims, hstr, own3b))) return r;
            h->hist_tma = true;
        }
    }
    return STFWI_OK;
}

// shots per block of each staged kernel (balanced groups; the strain phase
// keeps at most acc_groups accumulator groups)
void set_groups(stfwi_handle *h, const int spg_in[4])
{
    const int nshot = h->nshot;
    for (int k = 0; k < 4; ++k) {
        const int spg = std::max(1, spg_in[k]);
        int G = (nshot + spg - 1) / spg;
        if (k == 3) G = std::min(G, h->acc_groups);
        h->spgk[k] = (nshot + G - 1) / G;
        h->grp[k] = (nshot + h->spgk[k] - 1) / h->spgk[k];
    }
    h->acc_used = h->grp[3];
    h->lr_used = h->grp[2];
}

}  // namespace

// tiles of a tw x th tiling in dispatch order, the `heavy` tiles first: those
// whose own cells touch an edge margin, a C-PML strip or the free-surface
// row, or whose staged box (one halo of K rows and 4 columns) reaches a strip
// or the free-surface row, i.e. the tiles that take the guarded path
std::vector<int> tile_order(const Geo &g, int K, int tw, int th, int ntx, int ntz, int *heavy)
{
    const int M = 2 * K + 1;
    std::vector<int> hv, lt;
    for (int t = 0; t < ntx * ntz; ++t) {
        const int i0 = (t / ntx) * th, j0 = (t % ntx) * tw, i1 = i0 + th - 1, j1 = j0 + tw - 1;
        bool plain = i0 >= M && i1 <= g.nz - 1 - M && j0 >= M && j1 <= g.nx - 1 - M && j0 >= g.pad &&
                     j1 < g.nx - g.pad && i1 < g.nz - g.pad && (g.fs || i0 >= g.pad);
        const int r0 = i0 - K, r1 = i1 + K, c0 = j0 - 4, c1 = j1 + 4;
        const bool box = c0 < g.pad || c1 >= g.nx - g.pad || r1 >= g.nz - g.pad || r0 <= 0 || (!g.fs && r0 < g.pad);
        (plain && !box ? lt : hv).push_back(t);
    }
    *heavy = (int)hv.size();
    hv.insert(hv.end(), lt.begin(), lt.end());
    return hv;
}

// receivers grouped by the tiles of the two staged tilings (CSR: start per
// tile, receiver indices)
static stfwi_status group_receivers(stfwi_handle *h)
{
    const Geo &g = h->g;
    const int nrec = (int)h->rec_x_h.size();
    auto tile_of = [&](int r, int th) { return ((h->rec_z_h[r] + g.z0) / th) * h->ntx + (h->rec_x_h[r] + g.pad) / h->tw; };
    auto group = [&](int th, int ntz, int *d_start, int *d_list) -> stfwi_status {
        const int ntl = h->ntx * ntz;
        std::vector<int> c(ntl + 1, 0), st(ntl + 1, 0), l(std::max(nrec, 1));
        for (int r = 0; r < nrec; ++r) c[tile_of(r, th)]++;
        for (int t = 0; t < ntl; ++t) st[t + 1] = st[t] + c[t];
        std::vector<int> f(st.begin(), st.end() - 1);
        for (int r = 0; r < nrec; ++r) l[f[tile_of(r, th)]++] = r;
        CK(h, cudaMemcpy(d_start, st.data(), st.size() * 4, cudaMemcpyHostToDevice));
        CK(h, cudaMemcpy(d_list, l.data(), l.size() * 4, cudaMemcpyHostToDevice));
        return STFWI_OK;
    };
    stfwi_status r = group(h->tha, h->ntza, h->tile_startA, h->tile_recA);
    return r ? r : group(h->thb, h->ntzb, h->tile_startB, h->tile_recB);
}

// tile heights of the staged tilings: ra rows per thread (ra * NWARP rows a
// tile) for fwd_vel, fwd_str and adj_a, rb for adj_b, each 1 or 2; sets the
// tile counts, the dispatch orders, the receivers' tile lists and the tensor
// maps whose boxes follow the heights, and drops the captured graphs
static stfwi_status set_tiling(stfwi_handle *h, int ra, int rb)
{
    if ((ra != 1 && ra != 2) || (rb != 1 && rb != 2))
        return fail(h, STFWI_ERR_INVALID, "rows per thread (%d, %d): use 1 or 2", ra, rb);
    if (h->hs) CK(h, cudaStreamSynchronize(h->hs));   // no launch of the handle reads the old tables
    Geo &g = h->g;
    h->ra = ra; h->rb = rb;
    h->tha = ra * NWARP; h->thb = rb * NWARP;
    h->ntza = (g.nz + h->tha - 1) / h->tha;
    h->ntzb = (g.nz + h->thb - 1) / h->thb;
    const int K = h->d.fd_order / 2;
    int ha = 0, hb = 0;
    const std::vector<int> oa = tile_order(g, K, h->tw, h->tha, h->ntx, h->ntza, &ha);
    const std::vector<int> ob = tile_order(g, K, h->tw, h->thb, h->ntx, h->ntzb, &hb);
    CK(h, cudaMemcpy(h->tordA, oa.data(), oa.size() * 4, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->tordB, ob.data(), ob.size() * 4, cudaMemcpyHostToDevice));
    g.tordA = h->tordA; g.tordB = h->tordB; g.theavyA = ha; g.theavyB = hb;
    stfwi_status r = setup_tensor_maps(h);
    if (r) return r;
    if (h->recv_set && (r = group_receivers(h))) return r;
    drop_graphs(h);
    return STFWI_OK;
}

// ================================================================ C ABI


// ---------------------------------------------------------------- full wavefield frames

namespace {

// frame of the forward state of every shot after a step: U, V and the
// strains recovered from the carried stresses, on the padded grid (no pitch)
__global__ void k_frames_fwd(Geo g, Mat m, const float *F, uint32_t fields, int nf, float *out)
{
    const long long N = (long long)g.nz * g.nx;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (q >= N) return;
    const int i = (int)(q / g.nx), j = (int)(q % g.nx);
    const long long o = (long long)i * g.P + j;
    const float *f = F + (long long)s * F_N * g.fstride;
    float v[5];
    v[0] = f[F_U * g.fstride + o];
    v[1] = f[F_V * g.fstride + o];
    strains_of(f[F_EX * g.fstride + o], f[F_EZ * g.fstride + o], f[F_ES * g.fstride + o], m.L2M[o], m.L[o],
               m.M[o], v[2], v[3], v[4]);
    int k = 0;
#pragma unroll
    for (int b = 0; b < 5; ++b)
        if (fields >> b & 1u) out[((long long)s * nf + k++) * N + q] = v[b];
}

// frame of the adjoint state after adjoint step n: U_a = P / B, V_a = Q / B
// and the three strain adjoints
__global__ void k_frames_adj(Geo g, Mat m, const float *A, uint32_t fields, int nf, float *out)
{
    const long long N = (long long)g.nz * g.nx;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (q >= N) return;
    const int i = (int)(q / g.nx), j = (int)(q % g.nx);
    const long long o = (long long)i * g.P + j;
    const float *a = A + (long long)s * F_N * g.fstride;
    const float b = m.B[o];
    const float v[5] = {a[F_U * g.fstride + o] / b, a[F_V * g.fstride + o] / b, a[F_EX * g.fstride + o],
                        a[F_EZ * g.fstride + o], a[F_ES * g.fstride + o]};
    int k = 0;
#pragma unroll
    for (int b2 = 0; b2 < 5; ++b2)
        if (fields >> b2 & 1u) out[((long long)s * nf + k++) * N + q] = v[b2];
}

// the strain-phase kernel of adjoint step n already added the exx / ezz
// receiver sources of step n - 1 (the start of the next adjoint step): take
// them out of the frame of step n
__global__ void k_frames_unpick(Geo g, const int *rx, const int *rz, const float *rec_adj, int n, int kex,
                                int kez, int nf, float *out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nshot * g.nrec || n < 1) return;
    const int s = t / g.nrec, r = t % g.nrec;
    const long long N = (long long)g.nz * g.nx, q = (long long)rz[r] * g.nx + rx[r];
    const float *src = rec_adj + (long long)s * 4 * g.nt * g.nrec + (long long)(n - 1) * g.nrec + r;
    if (kex >= 0) atomicAdd(out + ((long long)s * nf + kex) * N + q, -src[2LL * g.nt * g.nrec]);
    if (kez >= 0) atomicAdd(out + ((long long)s * nf + kez) * N + q, -src[3LL * g.nt * g.nrec]);
}

// fwi/imaging.py:83-169 on histories held by the caller: one thread per
// physical cell sums, over the frames [t0, t1) of a chunk, the Lame terms
// with the periodic centred differences of B U_a and B V_a (jnp.roll wraps
// across the padded grid) and, with the forward velocities, the density
// term with the centred time derivative of the adjoint velocities.  The
// chunk arrays hold frames [c0, c0 + ...) (ua, va from c0 - 1 when t0 > 0).
struct ImgArgs {
    int nz, nx, nz_dom, nx_dom, z0, pad, nt;
    double dt, inv2dx, inv2dz;
    const float *rho;                       // physical [nz_dom][nx_dom]
    const float *ex, *ez, *es, *vx, *vz;    // frames t0.. of the chunk
    const float *ua, *va;                   // frames ua0.. (one before t0 when t0 > 0)
    int t0, t1, ua0;
    double *acc;                            // [3][nd]: g_lam, g_mu, g_rho_lame
};

__device__ __forceinline__ double b_ext(const ImgArgs &a, int i, int j)
{
    // buoyancy of the nearest-neighbour extension of rho (fwi/imaging.py:56-80)
    const int pi = min(max(i - a.z0, 0), a.nz_dom - 1), pj = min(max(j - a.pad, 0), a.nx_dom - 1);
    return 1.0 / (double)a.rho[(long long)pi * a.nx_dom + pj];
}

__global__ void k_imaging_hist(ImgArgs a)
{
    const long long nd = (long long)a.nz_dom * a.nx_dom;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nd) return;
    const int i = (int)(q / a.nx_dom) + a.z0, j = (int)(q % a.nx_dom) + a.pad;
    const long long N = (long long)a.nz * a.nx;
    const int ip = (i + 1) % a.nz, im = (i - 1 + a.nz) % a.nz, jp = (j + 1) % a.nx, jm = (j - 1 + a.nx) % a.nx;
    const long long o = (long long)i * a.nx + j;
    const long long oxp = (long long)i * a.nx + jp, oxm = (long long)i * a.nx + jm;
    const long long ozp = (long long)ip * a.nx + j, ozm = (long long)im * a.nx + j;
    const double bxp = b_ext(a, i, jp), bxm = b_ext(a, i, jm), bzp = b_ext(a, ip, j), bzm = b_ext(a, im, j);
    double glam = 0.0, gmu = 0.0, grl = 0.0;
    for (int t = a.t0; t < a.t1; ++t) {
        const float *u = a.ua + (long long)(t - a.ua0) * N, *v = a.va + (long long)(t - a.ua0) * N;
        const long long f = (long long)(t - a.t0) * N;
        const double dxBU = (bxp * u[oxp] - bxm * u[oxm]) * a.inv2dx;
        const double dzBU = (bzp * u[ozp] - bzm * u[ozm]) * a.inv2dz;
        const double dxBV = (bxp * v[oxp] - bxm * v[oxm]) * a.inv2dx;
        const double dzBV = (bzp * v[ozp] - bzm * v[ozm]) * a.inv2dz;
        const double e1 = a.ex[f + o], e2 = a.ez[f + o], e3 = a.es[f + o];
        glam -= a.dt * ((e1 + e2) * (dxBU + dzBV));
        gmu -= a.dt * (2.0 * e1 * dxBU + 2.0 * e2 * dzBV + e3 * (dzBU + dxBV));
        if (a.vx && t >= 1 && t <= a.nt - 2) {
            const double dua = ((double)u[N + o] - (double)u[o - N]) / (2.0 * a.dt);
            const double dva = ((double)v[N + o] - (double)v[o - N]) / (2.0 * a.dt);
            grl -= a.dt * ((double)a.vx[f + o] * dua + (double)a.vz[f + o] * dva);
        }
    }
    a.acc[q] += glam;
    a.acc[nd + q] += gmu;
    a.acc[2 * nd + q] += grl;
}

// chain rule to (Vs, Vp, rho) after the crop (fwi/imaging.py:165-167)
__global__ void k_imaging_chain(long long nd, const float *vs, const float *vp, const float *rho, const double *acc,
                                double *g)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nd) return;
    const double Vs = vs[q], Vp = vp[q], r = rho[q], gl = acc[q], gm = acc[nd + q], grl = acc[2 * nd + q];
    g[q] = 2.0 * r * Vs * (gm - 2.0 * gl);
    g[nd + q] = 2.0 * r * Vp * gl;
    g[2 * nd + q] = (Vp * Vp - 2.0 * Vs * Vs) * gl + Vs * Vs * gm + grl;
    g[3 * nd + q] = gl;
    g[4 * nd + q] = gm;
    g[5 * nd + q] = grl;
}

bool device_resident(const void *p)
{
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int popc5(uint32_t f)
{
    int n = 0;
    for (int b = 0; b < 5; ++b) n += (f >> b) & 1u;
    return n;
}

}  // namespace

extern "C" {

void stfwi_grid_shape(const stfwi_desc *d, int32_t *nz_t, int32_t *nx_t)
{
    *nx_t = d->nx_dom + 2 * d->pad;
    *nz_t = d->free_surface ? d->nz_dom + d->pad : d->nz_dom + 2 * d->pad;
}

size_t stfwi_workspace_bytes(const stfwi_desc *d)
{
    if (!d || d->nt < 1) return 0;
    const int k = d->ckpt_interval > 0 ? std::min(d->ckpt_interval, d->nt) : d->nt;
    return make_plan(d, k).total();
}

const char *stfwi_last_error(const stfwi_handle *h) { return h ? h->err.c_str() : "null handle"; }

stfwi_status stfwi_create(const stfwi_desc *d, stfwi_handle **out)
{
    if (!d || !out) return STFWI_ERR_INVALID;
    *out = nullptr;
    if (d->fd_order != 2 && d->fd_order != 4 && d->fd_order != 8) return STFWI_ERR_UNSUPPORTED;
    // one kernel family: the field is kept for the ABI, other values are refused
    if (d->kernel_variant != 0) return STFWI_ERR_UNSUPPORTED;
    if (d->want_gradient < 0 || d->want_gradient > 2) return STFWI_ERR_INVALID;
    const int H = d->fd_order / 2;
    if (d->nz_dom < 1 || d->nx_dom < 1 || d->pad < H || d->nt < 1 || d->nrec < 0 || d->max_shots < 1 ||
        !(d->dx > 0) || !(d->dz > 0) || !(d->dt > 0))
        return STFWI_ERR_INVALID;
    stfwi_handle *h = new stfwi_handle();
    h->d = *d;
    cudaGetDevice(&h->device);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        delete h;
        return STFWI_ERR_CUDA;
    }
    const double budget = d->mem_budget_gb > 0 ? d->mem_budget_gb * 1e9 : 0.85 * (double)fr;
    // history plan: every step if it fits, else the longest checkpoint
    // segment that fits (the recompute costs one forward whatever k is)
    int k = d->nt;
    if (d->want_gradient) {
        if (d->ckpt_interval > 0) {
            k = std::min(d->ckpt_interval, d->nt);
        } else if ((double)make_plan(d, d->nt).total() > budget) {
            k = 0;
            for (int kk = d->nt - 1; kk >= 1; --kk)
                if ((double)make_plan(d, kk).total() <= budget) { k = kk; break; }
            if (k == 0) k = 1;
        }
    }
    Plan p = make_plan(d, k);
    h->ck = k;
    h->ncp = (d->want_gradient && k < d->nt) ? (d->nt + k - 1) / k : 0;
    if ((double)p.total() > budget) {
        h->err = "workspace of " + std::to_string(p.total() / 1e9) + " GB exceeds the budget of " +
                 std::to_string(budget / 1e9) + " GB";
        fprintf(stderr, "stfwi_create: %s\n", h->err.c_str());
        delete h;
        return STFWI_ERR_OOM;
    }
    Geo &g = h->g;
    g.nz = (int)p.nz; g.nx = (int)p.nx; g.P = (int)p.P;
    g.nz_dom = d->nz_dom; g.nx_dom = d->nx_dom; g.z0 = d->free_surface ? 0 : d->pad; g.pad = d->pad;
    g.fs = d->free_surface ? 1 : 0;
    g.xs_n = (int)p.xs_n; g.zs_n = (int)p.zs_n;
    g.nt = d->nt; g.nrec = d->nrec; g.nshot = 0;
    g.dtdx = (float)(d->dt / d->dx); g.dtdz = (float)(d->dt / d->dz); g.dzdx = (float)(d->dz / d->dx);
    g.dt = (float)d->dt;
    g.inv2dx = (float)(1.0 / (2.0 * d->dx)); g.inv2dz = (float)(1.0 / (2.0 * d->dz));
    g.dtdxdz = (float)(d->dt / (d->dx * d->dz));
    g.fstride = p.nz * p.P; g.xstride = p.nz * p.xs_n; g.zstride = p.zs_n * p.P; g.nd = p.nd;
    g.snf = d->want_gradient == 2 ? 5 : 3;
    g.wait_polls = WAIT3;
    h->accp = g.snf == 5 ? 7 : 5;
    h->tw = TX4;
    h->ntx = (int)((p.nx + h->tw - 1) / h->tw);
    h->ntz_max = (int)((p.nz + RPT_MIN * NWARP - 1) / (RPT_MIN * NWARP));
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
    {
        stfwi_status r = STFWI_OK;
        switch (d->fd_order) {
        case 2: r = setup_tma_kernels<2>(h); break;
        case 4: r = setup_tma_kernels<4>(h); break;
        default: r = setup_tma_kernels<8>(h); break;
        }
        if (r) { delete h; return r; }
        h->acc_groups = acc_groups_of(d);
    }
    h->acc_used = h->acc_groups;
    h->slots = k + 1 + ((g.snf == 5 && h->ncp > 0) ? 1 : 0);

    auto alloc = [&](void **ptr, size_t bytes) -> bool {
        if (bytes == 0) { *ptr = nullptr; return true; }
        if (cudaMalloc(ptr, bytes) != cudaSuccess) return false;
        h->bytes += bytes;
        return true;
    };
    const long long S = d->max_shots, NP = p.nz * p.P, nd = p.nd;
    const long long nrec = std::max(d->nrec, 1);
    bool ok = true;
    ok &= alloc((void **)&h->vs, nd * 4) && alloc((void **)&h->vp, nd * 4) && alloc((void **)&h->rho, nd * 4);
    ok &= alloc((void **)&h->MATS, 4 * NP * 4) && alloc((void **)&h->Lr, p.P * 4);
    if (ok) { h->B = h->MATS; h->L2M = h->MATS + NP; h->L = h->MATS + 2 * NP; h->M = h->MATS + 3 * NP; }
    ok &= alloc((void **)&h->bx, p.P * 4) && alloc((void **)&h->ax, p.P * 4) && alloc((void **)&h->ikx, p.P * 4);
    ok &= alloc((void **)&h->bz, p.nz * 4) && alloc((void **)&h->az, p.nz * 4) && alloc((void **)&h->ikz, p.nz * 4);
    ok &= alloc((void **)&h->vpmax, 16) && alloc((void **)&h->status, 16);
    ok &= alloc((void **)&h->sx, S * 4) && alloc((void **)&h->sz, S * 4) && alloc((void **)&h->stype, S * 4);
    ok &= alloc((void **)&h->wav, S * d->nt * 4) && alloc((void **)&h->fcoef, S * 4) &&
          alloc((void **)&h->mcoef, S * 4) && alloc((void **)&h->lm, S * 4);
    // tile arrays sized for the lowest tiles (set_tiling picks the heights)
    const size_t ntl_max = (size_t)h->ntx * h->ntz_max;
    ok &= alloc((void **)&h->tile_startA, (ntl_max + 1) * 4) && alloc((void **)&h->tile_recA, nrec * 4) &&
          alloc((void **)&h->tile_startB, (ntl_max + 1) * 4) && alloc((void **)&h->tile_recB, nrec * 4);
    ok &= alloc((void **)&h->rx, nrec * 4) && alloc((void **)&h->rz, nrec * 4);
    ok &= alloc((void **)&h->tordA, ntl_max * 4) && alloc((void **)&h->tordB, ntl_max * 4);
    ok &= alloc((void **)&h->F, (size_t)S * F_N * NP * 4) && alloc((void **)&h->A, (size_t)S * F_N * NP * 4);
    ok &= alloc((void **)&h->PX, (size_t)S * NPX * p.nz * p.xs_n * 4) &&
          alloc((void **)&h->PZ, (size_t)S * NPZ * p.zs_n * p.P * 4);
    ok &= alloc((void **)&h->rec, (size_t)S * 4 * d->nt * nrec * 4) &&
          alloc((void **)&h->rec_adj, (size_t)S * 4 * d->nt * nrec * 4) &&
          alloc((void **)&h->obs, (size_t)S * d->nt * nrec * 4);
    ok &= alloc((void **)&h->snap, p.snap) && alloc((void **)&h->row0, p.row0);
    if (h->ncp > 0) {
        ok &= alloc((void **)&h->CKF, (size_t)h->ncp * S * F_N * NP * 4) &&
              alloc((void **)&h->CKPX, (size_t)h->ncp * S * PX_NFWD * p.nz * p.xs_n * 4) &&
              alloc((void **)&h->CKPZ, (size_t)h->ncp * S * PZ_NFWD * p.zs_n * p.P * 4);
    }
    ok &= alloc((void **)&h->acc, (size_t)h->acc_groups * h->accp * nd * 8) &&
          alloc((void **)&h->accLr, (size_t)std::max(h->acc_groups, d->max_shots) * std::max(d->nx_dom, 1) * 8) &&
          alloc((void **)&h->gtmp, (size_t)6 * nd * 8);
    ok &= alloc((void **)&h->energy, (size_t)p.nz * p.nx * 8);
    ok &= alloc((void **)&h->pw, (2 * POST_MAX_RADIUS + 1) * 8) && alloc((void **)&h->ptaper, (size_t)nd * 8) &&
          alloc((void **)&h->pillum, (size_t)nd * 8) && alloc((void **)&h->ptmp, (size_t)nd * 8) &&
          alloc((void **)&h->pscr, (size_t)p.nz * p.nx * 8) && alloc((void **)&h->pmax, 64);
    ok &= alloc((void **)&h->mis_trace, (size_t)S * nrec * 8) && alloc((void **)&h->mis_shot, (size_t)S * 8);
    ok &= alloc((void **)&h->src_a, (size_t)S * d->nt * 4);
    if (!ok) {
        cudaGetLastError();
        stfwi_destroy(h);
        return STFWI_ERR_OOM;
    }
    bool sok = cudaStreamCreateWithFlags(&h->hs, cudaStreamNonBlocking) == cudaSuccess &&
               cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int c = 0; c < MAX_CHAINS - 1 && sok; ++c)
        sok = cudaStreamCreateWithFlags(&h->hsx[c], cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&h->ev_join[c], cudaEventDisableTiming) == cudaSuccess;
    if (!sok) {
        stfwi_destroy(h);
        return STFWI_ERR_CUDA;
    }
    cudaMemset(h->status, 0, 16);
    // pitch padding and never-written cells read as zero by the tile copies
    cudaMemset(h->MATS, 0, (size_t)4 * NP * 4);
    cudaMemset(h->F, 0, (size_t)S * F_N * NP * 4);
    cudaMemset(h->A, 0, (size_t)S * F_N * NP * 4);
    {
        stfwi_status r = set_tiling(h, RPT_DEFAULT, RPT_DEFAULT);
        if (r) {
            fprintf(stderr, "stfwi_create: %s\n", h->err.c_str());
            stfwi_destroy(h);
            return r;
        }
    }
    *out = h;
    return STFWI_OK;
}

void stfwi_destroy(stfwi_handle *h)
{
    if (!h) return;
    if (h->hs) cudaStreamSynchronize(h->hs);
    drop_graphs(h);
    void *bufs[] = {h->vs, h->vp, h->rho, h->MATS, h->Lr, h->bx, h->ax, h->ikx, h->bz,
                    h->az, h->ikz, h->vpmax, h->status, h->sx, h->sz, h->stype, h->wav, h->fcoef, h->mcoef,
                    h->lm, h->rx, h->rz, h->F, h->A, h->PX, h->PZ, h->rec,
                    h->rec_adj, h->obs, h->snap, h->row0, h->acc, h->accLr, h->gtmp, h->energy,
                    h->mis_trace, h->mis_shot, h->src_a, h->pw, h->ptaper, h->pillum, h->ptmp, h->pscr, h->pmax,
                    h->tile_startA, h->tile_recA, h->tile_startB, h->tile_recB, h->tordA, h->tordB, h->CKF, h->CKPX,
                    h->CKPZ};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (int k = 0; k < 4; ++k)
        for (cudaEvent_t e : h->pev[k]) cudaEventDestroy(e);
    if (h->ev_in) cudaEventDestroy(h->ev_in);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    for (int c = 0; c < MAX_CHAINS - 1; ++c) {
        if (h->ev_join[c]) cudaEventDestroy(h->ev_join[c]);
        if (h->hsx[c]) cudaStreamDestroy(h->hsx[c]);
    }
    if (h->hs) cudaStreamDestroy(h->hs);
    delete h;
}

stfwi_status stfwi_set_model(stfwi_handle *h, const float *vs, const float *vp, const float *rho,
                             void *stream)
{
    if (!h || !vs || !vp || !rho) return fail(h, STFWI_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    const size_t nb = (size_t)g.nd * sizeof(float);
    CK(h, cudaMemcpyAsync(h->vs, vs, nb, cudaMemcpyDefault, st));
    CK(h, cudaMemcpyAsync(h->vp, vp, nb, cudaMemcpyDefault, st));
    CK(h, cudaMemcpyAsync(h->rho, rho, nb, cudaMemcpyDefault, st));
    dim3 blk(128), grd((g.nx + 127) / 128, g.nz);
    k_materials<<<grd, blk, 0, st>>>(g.nz, g.nx, g.P, g.nz_dom, g.nx_dom, g.z0, g.pad, h->vs, h->vp, h->rho,
                                     h->B, h->L2M, h->L, h->M, h->Lr);
    k_vpmax<<<1, 1024, 0, st>>>(h->vp, g.nd, h->vpmax);
    const int nmax = std::max(g.nx, g.nz);
    k_pml<<<(nmax + 127) / 128, 128, 0, st>>>(g.nz, g.nx, g.nz_dom, g.pad, g.fs, h->d.dx, h->d.dt, h->d.fc,
                                              h->vpmax, h->bx, h->ax, h->ikx, h->bz, h->az, h->ikz);
    CK(h, cudaGetLastError());
    h->model_set = true;
    if (h->shots_set) {
        k_src_coefs<<<(h->nshot + 127) / 128, 128, 0, st>>>(h->nshot, h->sx, h->sz, g.P, h->B, h->L, h->M,
                                                           (float)(h->d.dt / (h->d.dx * h->d.dz)),
                                                           (float)h->d.dx, (float)h->d.dz, h->fcoef,
                                                           h->mcoef, h->lm);
        CK(h, cudaGetLastError());
    }
    return STFWI_OK;
}

stfwi_status stfwi_set_receivers(stfwi_handle *h, int32_t nrec, const int32_t *rec_x, const int32_t *rec_z)
{
    if (!h) return STFWI_ERR_INVALID;
    const Geo &g = h->g;
    if (nrec != g.nrec) return fail(h, STFWI_ERR_INVALID, "nrec %d != descriptor nrec %d", nrec, g.nrec);
    if (nrec > 0 && (!rec_x || !rec_z)) return fail(h, STFWI_ERR_INVALID, "null receiver array");
    std::vector<int> rx(std::max(nrec, 1)), rz(std::max(nrec, 1));
    for (int r = 0; r < nrec; ++r) {
        rx[r] = rec_x[r] + g.pad;
        rz[r] = rec_z[r] + g.z0;
        if (rx[r] < 0 || rx[r] >= g.nx || rz[r] < 0 || rz[r] >= g.nz)
            return fail(h, STFWI_ERR_INVALID, "receiver %d at (%d,%d) is outside the grid", r, rec_z[r], rec_x[r]);
    }
    CK(h, cudaMemcpy(h->rx, rx.data(), rx.size() * 4, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->rz, rz.data(), rz.size() * 4, cudaMemcpyHostToDevice));
    h->rec_x_h.assign(rec_x, rec_x + nrec);
    h->rec_z_h.assign(rec_z, rec_z + nrec);
    h->recv_set = false;
    stfwi_status gr = group_receivers(h);
    if (gr) return gr;
    h->recv_set = true;
    return STFWI_OK;
}

stfwi_status stfwi_set_shots(stfwi_handle *h, int32_t nshot, const int32_t *src, const float *wavelets,
                             void *stream)
{
    if (!h || !src || !wavelets) return fail(h, STFWI_ERR_INVALID, "null argument");
    if (nshot < 1 || nshot > h->d.max_shots)
        return fail(h, STFWI_ERR_INVALID, "nshot %d outside [1, %d]", nshot, h->d.max_shots);
    cudaStream_t st = (cudaStream_t)stream;
    Geo &g = h->g;
    std::vector<int> sx(nshot), sz(nshot), ty(nshot);
    for (int s = 0; s < nshot; ++s) {
        sx[s] = src[3 * s] + g.pad;
        sz[s] = src[3 * s + 1] + g.z0;
        ty[s] = src[3 * s + 2];
        if (ty[s] != STFWI_SRC_FORCE && ty[s] != STFWI_SRC_MOMENT)
            return fail(h, STFWI_ERR_UNSUPPORTED, "src_type %d not supported (use force=0 or moment=1)", ty[s]);
        if (sx[s] < 0 || sx[s] >= g.nx || sz[s] < 0 || sz[s] >= g.nz)
            return fail(h, STFWI_ERR_INVALID, "source %d at (%d,%d) is outside the grid", s, src[3 * s + 1], src[3 * s]);
    }
    CK(h, cudaStreamSynchronize(st));
    CK(h, cudaMemcpy(h->sx, sx.data(), nshot * 4, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->sz, sz.data(), nshot * 4, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->stype, ty.data(), nshot * 4, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpyAsync(h->wav, wavelets, (size_t)nshot * g.nt * 4, cudaMemcpyDefault, st));
    if (nshot != h->nshot) drop_graphs(h);
    h->nshot = nshot;
    g.nshot = nshot;
    {
        // shots per block by default (measured on B200, 50 shots of 172 x 540):
        // enough blocks to keep every SM busy, copies of the next shots in
        // flight while one computes; the strain phase keeps FP64 sums per cell
        // over its shots and gains from larger groups
        static const int dflt4[4] = {3, 3, 3, 4};
        int spg[4];
        for (int k = 0; k < 4; ++k)
            spg[k] = h->d.shot_group > 0 ? h->d.shot_group : h->tuned[k] > 0 ? h->tuned[k] : dflt4[k];
        set_groups(h, spg);
    }
    h->shots_set = true;
    h->stored = false;
    if (h->model_set) {
        k_src_coefs<<<(nshot + 127) / 128, 128, 0, st>>>(nshot, h->sx, h->sz, g.P, h->B, h->L, h->M,
                                                        (float)(h->d.dt / (h->d.dx * h->d.dz)),
                                                        (float)h->d.dx, (float)h->d.dz, h->fcoef, h->mcoef,
                                                        h->lm);
        CK(h, cudaGetLastError());
    }
    return STFWI_OK;
}

static stfwi_status ready(stfwi_handle *h)
{
    if (!h) return STFWI_ERR_INVALID;
    if (!h->model_set || !h->shots_set || !h->recv_set)
        return fail(h, STFWI_ERR_STATE, "set the model, receivers and shots first");
    return STFWI_OK;
}

stfwi_status stfwi_forward(stfwi_handle *h, uint32_t flags, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if ((flags & STFWI_FWD_STORE) && !h->snap)
        return fail(h, STFWI_ERR_STATE, "handle was created without want_gradient");
    GraphKey key{0, flags & STFWI_FWD_STORE, h->nshot};
    rc = run_graph(h, key, (cudaStream_t)stream,
                   [&](cudaStream_t st) { return enqueue_forward(h, flags, -1, st); });
    if (rc) return rc;
    h->stored = (flags & STFWI_FWD_STORE) != 0;
    if (h->prof_every > 0) {
        CK(h, cudaStreamSynchronize(h->hs));
        prof_accumulate(h, 0);
        prof_accumulate(h, 1);
    }
    return STFWI_OK;
}

stfwi_status stfwi_get_records(stfwi_handle *h, float *out, void *stream)
{
    if (!h || !out) return fail(h, STFWI_ERR_INVALID, "null argument");
    CK(h, cudaMemcpyAsync(out, h->rec, (size_t)h->nshot * 4 * h->g.nt * h->g.nrec * 4, cudaMemcpyDefault,
                          (cudaStream_t)stream));
    return STFWI_OK;
}

stfwi_status stfwi_misfit(stfwi_handle *h, const float *obs, const stfwi_misfit_desc *m,
                          double *misfit_out, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if (!obs || !m) return fail(h, STFWI_ERR_INVALID, "null argument");
    if (m->component < 0 || m->component > 3) return fail(h, STFWI_ERR_INVALID, "component %d", m->component);
    if (m->nsos < 0 || m->nsos > MAX_SOS || (m->nsos > 0 && !m->sos))
        return fail(h, STFWI_ERR_INVALID, "nsos %d outside [0, %d]", m->nsos, MAX_SOS);
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    SosParams sp{};
    sp.nsos = m->nsos;
    for (int k = 0; k < m->nsos; ++k) {
        const double *s = m->sos + 6 * k;
        if (s[3] == 0.0) return fail(h, STFWI_ERR_INVALID, "sos section %d has a0 = 0", k);
        sp.c[k][0] = s[0] / s[3]; sp.c[k][1] = s[1] / s[3]; sp.c[k][2] = s[2] / s[3];
        sp.c[k][3] = s[4] / s[3]; sp.c[k][4] = s[5] / s[3];
    }
    const int nnorm = m->nshot_norm > 0 ? m->nshot_norm : h->nshot;
    CK(h, cudaMemcpyAsync(h->obs, obs, (size_t)h->nshot * g.nt * g.nrec * 4, cudaMemcpyDefault, st));
    const int n = h->nshot * g.nrec, thr = 128;
    if (n > 0) {
        const int ntap = std::min(std::max(m->n_taper, 0), g.nt);  // fwi/filters.py:28
        k_misfit<<<(n + thr - 1) / thr, thr, 0, st>>>(g, m->component, ntap, sp, m->scale, nnorm, h->rec,
                                                     h->obs, h->rec_adj, h->mis_trace);
        k_misfit_reduce<<<(h->nshot + 127) / 128, 128, 0, st>>>(h->nshot, g.nrec, h->mis_trace, h->mis_shot);
    } else {
        CK(h, cudaMemsetAsync(h->mis_shot, 0, h->nshot * 8, st));
    }
    CK(h, cudaGetLastError());
    if (misfit_out) CK(h, cudaMemcpyAsync(misfit_out, h->mis_shot, h->nshot * 8, cudaMemcpyDefault, st));
    return STFWI_OK;
}

stfwi_status stfwi_set_adjoint_sources(stfwi_handle *h, const float *rec_adj, void *stream)
{
    if (!h || !rec_adj) return fail(h, STFWI_ERR_INVALID, "null argument");
    CK(h, cudaMemcpyAsync(h->rec_adj, rec_adj, (size_t)h->nshot * 4 * h->g.nt * h->g.nrec * 4,
                          cudaMemcpyDefault, (cudaStream_t)stream));
    return STFWI_OK;
}

stfwi_status stfwi_gradient(stfwi_handle *h, uint32_t mode, double *g_out, float *src_wav_a, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    const bool ex = mode & STFWI_GRAD_EXACT, im = mode & STFWI_GRAD_IMAGING, sr = mode & STFWI_GRAD_SRC;
    if (!ex && !im && !sr) return fail(h, STFWI_ERR_INVALID, "empty gradient mode");
    if ((ex || im) && !g_out) return fail(h, STFWI_ERR_INVALID, "g_out is null");
    if (sr && !src_wav_a) return fail(h, STFWI_ERR_INVALID, "src_wav_a is null");
    if ((ex || im) && !h->stored)
        return fail(h, STFWI_ERR_STATE, "model gradients need a preceding stfwi_forward(STFWI_FWD_STORE)");
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    float *src_dev = sr ? h->src_a : nullptr;
    GraphKey key{1, mode, h->nshot};
    rc = run_graph(h, key, st, [&](cudaStream_t s) {
        stfwi_status r = zero_adjoint_state(h, s);
        if (r) return r;
        const int thr = 256;
        if (g.nrec > 0)
            k_inject_last<<<(g.nshot * g.nrec + thr - 1) / thr, thr, 0, s>>>(g, h->rx, h->rz, h->rec_adj, h->A);
        auto adj = [&](int n, int seg0, int seg1, cudaStream_t as, int part) {
            const int ping = (g.nt - 1 - n) & 1;
            AdjIn ai{};
            ai.rec_adj = h->rec_adj; ai.row0 = h->row0; ai.slots = h->slots; ai.slot = n - seg0;
            ai.accLr = h->accLr; ai.want_exact = ex; ai.ping = ping;
            AdjOut ao{};
            ao.snap = h->snap; ao.slots = h->slots; ao.slot_in = n - seg0; ao.slot_img = n - seg0 + 1;
            ao.accp = h->accp;
            // outputs of step n + 1: the next slot inside a segment, else the
            // extra slot filled from the following segment (checkpoints)
            ao.slot_next = (n + 1 < seg1) ? n - seg0 + 2 : (h->ncp > 0 && n + 1 < g.nt ? h->ck + 1 : -1);
            ao.acc = h->acc; ao.want_exact = ex; ao.want_img = im; ao.hist_tma = h->hist_tma ? 1 : 0;
            ao.src_a = sr ? src_dev : nullptr; ao.rec_adj = h->rec_adj; ao.ping = ping;
            switch (h->d.fd_order) {
            case 2: launch_adj_step<2>(h, n, ai, ao, as, part); break;
            case 4: launch_adj_step<4>(h, n, ai, ao, as, part); break;
            default: launch_adj_step<8>(h, n, ai, ao, as, part); break;
            }
        };
        if ((ex || im) && h->ncp > 0) {
            // segments from the last: restore the checkpoint, recompute the
            // segment's history, run its adjoint steps
            for (int c = h->ncp - 1; c >= 0; --c) {
                const int seg0 = c * h->ck, seg1 = std::min(seg0 + h->ck, g.nt);
                if (g.snf == 5 && c + 1 < h->ncp) {
                    // keep the velocities of step seg1 (slot 1 of the segment
                    // just processed) for the density term of step seg1 - 1
                    const size_t ps = (size_t)h->slots * g.snf * g.nd * sizeof(float);
                    CK(h, cudaMemcpy2DAsync(h->snap + ((size_t)h->ck + 1) * g.snf * g.nd + 3 * g.nd, ps,
                                            h->snap + (size_t)g.snf * g.nd + 3 * g.nd, ps,
                                            (size_t)2 * g.nd * sizeof(float), h->nshot, cudaMemcpyDeviceToDevice, s));
                }
                r = copy_ckpt(h, c, false, s);
                if (r) return r;
                snap_state(h, s);
                FwdOut o{};
                o.rec = h->rec; o.status = h->status; o.slots = h->slots;
                o.snap = h->snap; o.row0 = g.fs ? h->row0 : nullptr;
                // the segment's recompute and adjoint steps in chains over
                // the shot groups; the copies above take every shot
                const int C = h->nchain_cur = pass_chains(h);
                if (C > 1 && (r = fork_chains(h, s))) return r;
                for (int n = seg0; n < seg1; ++n) {
                    o.slot = n - seg0 + 1;
                    o.slot_row0 = n - seg0;
                    if (C > 1)
                        for (int q = 0; q < C; ++q) fwd_step(h, n, o, chain_stream(h, s, q), q);
                    else
                        fwd_step(h, n, o, s);
                }
                for (int n = seg1 - 1; n >= seg0; --n) {
                    if (C > 1)
                        for (int q = 0; q < C; ++q) adj(n, seg0, seg1, chain_stream(h, s, q), q);
                    else
                        adj(n, seg0, seg1, s, -1);
                }
                if (C > 1 && (r = join_chains(h, s))) return r;
            }
        } else if ((h->nchain_cur = pass_chains(h)) > 1) {
            if ((r = fork_chains(h, s))) return r;
            for (int n = g.nt - 1; n >= 0; --n)
                for (int c = 0; c < h->nchain_cur; ++c) adj(n, 0, g.nt, chain_stream(h, s, c), c);
            if ((r = join_chains(h, s))) return r;
        } else {
            for (int n = g.nt - 1; n >= 0; --n) adj(n, 0, g.nt, s, -1);
        }
        if (ex || im)
            k_finalize<<<(unsigned)((g.nd + 255) / 256), 256, 0, s>>>(g, h->acc_used, h->accp, h->lr_used, h->acc, h->accLr, h->L2M,
                                                                      h->L, h->vs, h->vp, h->rho, ex, im,
                                                                      h->gtmp, h->gtmp + 3 * g.nd);
        CK(h, cudaGetLastError());
        return STFWI_OK;
    });
    if (rc) return rc;
    if (h->prof_every > 0) {
        CK(h, cudaStreamSynchronize(h->hs));
        prof_accumulate(h, 2);
        prof_accumulate(h, 3);
    }
    if ((ex || im) && (h->post_radius > 0 || h->post_taper || h->post_illum)) {
        // fwi/gradient.py:266-277 on the device: Gaussian smoothing, then the
        // source taper and the illumination multiplies, on every output plane
        double *base = ex ? h->gtmp : h->gtmp + 3 * g.nd;
        const int planes = 3 * (int(ex) + int(im));
        const unsigned nb = (unsigned)((g.nd + 255) / 256);
        if (h->post_radius > 0)
            for (int p = 0; p < planes; ++p) {
                double *pl = base + (size_t)p * g.nd;
                k_gauss_axis<<<nb, 256, 0, st>>>(g.nz_dom, g.nx_dom, 1, h->post_radius, h->pw, pl, h->ptmp);
                k_gauss_axis<<<nb, 256, 0, st>>>(g.nz_dom, g.nx_dom, 0, h->post_radius, h->pw, h->ptmp, pl);
            }
        if (h->post_taper || h->post_illum)
            k_mul_planes<<<nb, 256, 0, st>>>(g.nd, planes, base, h->post_taper ? h->ptaper : nullptr,
                                             h->post_illum ? h->pillum : nullptr);
        CK(h, cudaGetLastError());
    }
    if (sr) CK(h, cudaMemcpyAsync(src_wav_a, src_dev, (size_t)h->nshot * g.nt * 4, cudaMemcpyDefault, st));
    size_t off = 0;
    if (ex) {
        CK(h, cudaMemcpyAsync(g_out, h->gtmp, (size_t)3 * g.nd * 8, cudaMemcpyDefault, st));
        off += 3 * g.nd;
    }
    if (im) CK(h, cudaMemcpyAsync(g_out + off, h->gtmp + 3 * g.nd, (size_t)3 * g.nd * 8, cudaMemcpyDefault, st));
    return STFWI_OK;
}

stfwi_status stfwi_illumination(stfwi_handle *h, int32_t component, double *ws_out, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if (component < 0 || component > 3 || !ws_out) return fail(h, STFWI_ERR_INVALID, "bad illumination request");
    GraphKey key{2, (uint32_t)component, h->nshot};
    rc = run_graph(h, key, (cudaStream_t)stream,
                   [&](cudaStream_t st) { return enqueue_forward(h, 0, component, st); });
    if (rc) return rc;
    h->stored = false;
    CK(h, cudaMemcpyAsync(ws_out, h->energy, (size_t)h->g.nz * h->g.nx * 8, cudaMemcpyDefault,
                          (cudaStream_t)stream));
    return STFWI_OK;
}

stfwi_status stfwi_set_postprocess(stfwi_handle *h, double grad_smooth_sigma, const double *source_taper,
                                   const double *illumination, void *stream)
{
    if (!h) return STFWI_ERR_INVALID;
    if (!(grad_smooth_sigma >= 0.0)) return fail(h, STFWI_ERR_INVALID, "grad_smooth_sigma must be >= 0");
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    int radius = 0;
    if (grad_smooth_sigma > 0.0) {
        // fwi/loss.py:17-30: truncate = 3, radius = int(3 sigma + 0.5), normalised weights
        radius = (int)(3.0 * grad_smooth_sigma + 0.5);
        if (radius > POST_MAX_RADIUS)
            return fail(h, STFWI_ERR_INVALID, "grad_smooth_sigma %g needs a radius above %d", grad_smooth_sigma,
                        POST_MAX_RADIUS);
        std::vector<double> w(2 * radius + 1);
        double sum = 0.0;
        for (int k = -radius; k <= radius; ++k) {
            const double x = k / grad_smooth_sigma;
            w[k + radius] = std::exp(-0.5 * x * x);
            sum += w[k + radius];
        }
        for (double &v : w) v /= sum;
        CK(h, cudaMemcpyAsync(h->pw, w.data(), w.size() * 8, cudaMemcpyHostToDevice, st));
        CK(h, cudaStreamSynchronize(st));
    }
    if (source_taper) CK(h, cudaMemcpyAsync(h->ptaper, source_taper, (size_t)g.nd * 8, cudaMemcpyDefault, st));
    if (illumination) CK(h, cudaMemcpyAsync(h->pillum, illumination, (size_t)g.nd * 8, cudaMemcpyDefault, st));
    CK(h, cudaStreamSynchronize(st));
    h->post_sigma = grad_smooth_sigma;
    h->post_radius = radius;
    h->post_taper = source_taper != nullptr;
    h->post_illum = illumination != nullptr;
    return STFWI_OK;
}

stfwi_status stfwi_preconditioner(stfwi_handle *h, int32_t kind, int32_t component, double eps, double *out,
                                  void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if ((kind != STFWI_PRECOND_ILLUM && kind != STFWI_PRECOND_EPRECOND3) || component < 0 || component > 3 || !out ||
        !(eps >= 0.0))
        return fail(h, STFWI_ERR_INVALID, "bad preconditioner request");
    if (kind == STFWI_PRECOND_EPRECOND3 && h->rec_x_h.empty())
        return fail(h, STFWI_ERR_STATE, "eprecond3 needs receivers");
    cudaStream_t st = (cudaStream_t)stream;
    GraphKey key{2, (uint32_t)component, h->nshot};
    rc = run_graph(h, key, st, [&](cudaStream_t s) { return enqueue_forward(h, 0, component, s); });
    if (rc) return rc;
    h->stored = false;
    const Geo &g = h->g;
    const long long n = g.nd, np = (long long)g.nz * g.nx;
    const unsigned nb = (unsigned)((n + 255) / 256), npb = (unsigned)((np + 255) / 256);
    double *res;
    if (kind == STFWI_PRECOND_ILLUM) {
        // fwi/illumination.py:44-47: crop, H = 1/(Ws + eps max Ws), H / max H
        k_crop<<<nb, 256, 0, st>>>(g.nz_dom, g.nx_dom, g.nx, g.z0, g.pad, h->energy, h->ptmp);
        k_max_1block<<<1, 1024, 0, st>>>(n, h->ptmp, h->pmax);
        k_illum_inverse<<<nb, 256, 0, st>>>(n, h->ptmp, h->pmax, eps, h->pscr);
        res = h->pscr;
    } else {
        // fwi/preconditioning.py:65-139 + fwi/optim_lbfgsb.py:95-99: the
        // receiver line's orientation is the coordinate with the larger spread
        auto stdev = [](const std::vector<int> &v) {
            double m = 0, q = 0;
            for (int x : v) m += x;
            m /= (double)v.size();
            for (int x : v) q += (x - m) * (x - m);
            return std::sqrt(q / (double)v.size());
        };
        const auto &rx = h->rec_x_h, &rz = h->rec_z_h;
        const bool horiz = stdev(rx) >= stdev(rz);
        const double dx = h->d.dx, dz = h->d.dz;
        const double lmin = horiz ? *std::min_element(rx.begin(), rx.end()) * dx : *std::min_element(rz.begin(), rz.end()) * dz;
        const double lmax = horiz ? *std::max_element(rx.begin(), rx.end()) * dx : *std::max_element(rz.begin(), rz.end()) * dz;
        const double perp = horiz ? rz[0] * dz : rx[0] * dx;
        k_eprecond3_we<<<npb, 256, 0, st>>>(g.nz, g.nx, g.z0, g.pad, dx, dz, horiz ? 1 : 0, lmin, lmax, perp, h->energy,
                                            h->pscr);
        k_max_1block<<<1, 1024, 0, st>>>(np, h->pscr, h->pmax);
        k_eprecond3_inv<<<nb, 256, 0, st>>>(g.nz_dom, g.nx_dom, g.nx, g.z0, g.pad, h->pscr, h->pmax, eps, h->ptmp);
        res = h->ptmp;
    }
    k_max_1block<<<1, 1024, 0, st>>>(n, res, h->pmax + 1);
    k_scale_by_inverse_max<<<nb, 256, 0, st>>>(n, res, h->pmax + 1);
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(out, res, (size_t)n * 8, cudaMemcpyDefault, st));
    return STFWI_OK;
}

stfwi_status stfwi_project_velocity(int64_t n, double *vs, double *vp, double *rho, double K_margin, double vp_cap,
                                    double vs_floor, double rho_floor, void *stream)
{
    if (n < 0 || !vs || !vp || !rho || !(K_margin > -1.0)) {
        fprintf(stderr, "stfwi_project_velocity: invalid arguments\n");
        return STFWI_ERR_INVALID;
    }
    if (n == 0) return STFWI_OK;
    for (const double *ptr : {(const double *)vs, (const double *)vp, (const double *)rho}) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess ||
            (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();
            fprintf(stderr, "stfwi_project_velocity: the model arrays must be device memory\n");
            return STFWI_ERR_INVALID;
        }
    }
    // fwi/projections.py:37-48: r = (1 + K_margin) * 2/sqrt(3)
    const double r = (1.0 + K_margin) * (2.0 / std::sqrt(3.0));
    const int use_cap = (vp_cap > 0.0 && std::isfinite(vp_cap)) ? 1 : 0;
    k_project_velocity<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, vs, vp, rho, r, vp_cap,
                                                                                   use_cap, vs_floor, rho_floor);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "stfwi_project_velocity: %s\n", cudaGetErrorString(e));
        return STFWI_ERR_CUDA;
    }
    return STFWI_OK;
}

stfwi_status stfwi_profile(stfwi_handle *h, int32_t every)
{
    if (!h || every < 0) return STFWI_ERR_INVALID;
    CK(h, cudaStreamSynchronize(h->hs));
    drop_graphs(h);
    for (int k = 0; k < 4; ++k) {
        for (cudaEvent_t e : h->pev[k]) cudaEventDestroy(e);
        h->pev[k].clear();
        h->prof_ms[k] = 0;
        h->prof_cnt[k] = 0;
    }
    h->prof_every = every;
    if (every > 0) {
        const int ns = (h->g.nt + every - 1) / every;
        for (int k = 0; k < 4; ++k) {
            h->pev[k].resize(2 * (size_t)ns);
            for (auto &e : h->pev[k]) CK(h, cudaEventCreate(&e));
        }
    }
    return STFWI_OK;
}

stfwi_status stfwi_kernel_times(stfwi_handle *h, double *out)
{
    if (!h || !out) return STFWI_ERR_INVALID;
    CK(h, cudaStreamSynchronize(h->hs));
    for (int k = 0; k < 4; ++k) {
        out[2 * k] = h->prof_ms[k];
        out[2 * k + 1] = (double)h->prof_cnt[k];
        h->prof_ms[k] = 0;
        h->prof_cnt[k] = 0;
    }
    return STFWI_OK;
}

// `steps` forward then `steps` adjoint steps of the handle's current
// schedule, launched directly (not captured) on `st`, split into chains
// exactly as a captured pass would be (pass_chains); the timing passes of
// the autotuner
static stfwi_status enqueue_timing_steps(stfwi_handle *h, int steps, cudaStream_t st)
{
    const Geo &g = h->g;
    stfwi_status r;
    if ((r = zero_forward_state(h, st)) || (r = zero_adjoint_state(h, st))) return r;
    const int C = h->nchain_cur = pass_chains(h);
    if (C > 1 && (r = fork_chains(h, st))) return r;
    FwdOut o{};
    o.rec = h->rec; o.status = h->status; o.slots = h->slots;
    for (int n = 0; n < steps; ++n)
        for (int q = 0; q < C; ++q) fwd_step(h, n, o, chain_stream(h, st, q), C > 1 ? q : -1);
    const bool ex = h->snap != nullptr;
    for (int n = steps - 1; n >= 0; --n) {
        AdjIn ai{};
        ai.rec_adj = h->rec_adj; ai.row0 = h->row0; ai.slots = h->slots; ai.slot = 0;
        ai.accLr = h->accLr; ai.want_exact = ex && g.fs; ai.ping = n & 1;
        AdjOut ao{};
        ao.snap = h->snap; ao.slots = h->slots; ao.slot_in = 0; ao.slot_img = h->slots > 1 ? 1 : -1;
        ao.slot_next = -1; ao.accp = h->accp; ao.acc = h->acc; ao.want_exact = ex; ao.want_img = 0;
        ao.rec_adj = h->rec_adj; ao.ping = n & 1; ao.hist_tma = h->hist_tma ? 1 : 0;
        for (int q = 0; q < C; ++q) {
            cudaStream_t cs = chain_stream(h, st, q);
            const int part = C > 1 ? q : -1;
            switch (h->d.fd_order) {
            case 2: launch_adj_step<2>(h, n, ai, ao, cs, part); break;
            case 4: launch_adj_step<4>(h, n, ai, ao, cs, part); break;
            default: launch_adj_step<8>(h, n, ai, ao, cs, part); break;
            }
        }
    }
    if (C > 1 && (r = join_chains(h, st))) return r;
    return STFWI_OK;
}

stfwi_status stfwi_autotune(stfwi_handle *h, int32_t steps, int32_t *spg_out, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    const Geo &g = h->g;
    steps = std::max(2, std::min((int)steps, g.nt));
    CK(h, cudaStreamSynchronize((cudaStream_t)stream));
    cudaStream_t st = h->hs;
    // time `steps` forward and adjoint steps per candidate with a CUDA-event
    // pair around every kernel (the sampled-profile records, every step)
    const int saved_every = h->prof_every;
    std::vector<cudaEvent_t> saved[4];
    for (int k = 0; k < 4; ++k) {
        saved[k].swap(h->pev[k]);
        h->pev[k].resize(2 * (size_t)steps);
        for (auto &e : h->pev[k]) CK(h, cudaEventCreate(&e));
    }
    h->prof_every = 1;
    // shots per block up to 25: with boundary tiles dispatched first, large
    // groups (fewer, longer blocks per tile) can pay on grids with many
    // boundary tiles; and both tile heights (rows per thread 1, 2: 8- and
    // 16-row tiles)
    static const int cand[] = {1, 2, 3, 4, 5, 6, 8, 10, 13, 17, 25};
    double best[2][4];
    int pick[2][4];
    for (int q = 0; q < 2; ++q)
        for (int k = 0; k < 4; ++k) { best[q][k] = 1e300; pick[q][k] = h->spgk[k]; }
    const int ra0 = h->ra, rb0 = h->rb;
    stfwi_status r = STFWI_OK;
    for (int q = 0; q < 2 && !r; ++q) {
      if ((r = set_tiling(h, q + 1, q + 1))) break;
      for (int c : cand) {
        if (c > h->nshot) break;
        const int spg[4] = {c, c, c, c};
        set_groups(h, spg);
        // one chain here: the sampled timing (prof_every = 1) is on
        if ((r = enqueue_timing_steps(h, steps, st))) break;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            r = fail(h, STFWI_ERR_CUDA, "autotune pass with %d shots per block, %d-row tiles: %s", c, 8 * (q + 1),
                     cudaGetErrorString(e));
            break;
        }
        for (int k = 0; k < 4; ++k) {
            double ms = 0;
            for (int n = 1; n < steps; ++n) {   // step 0 warms up
                float e = 0.f;
                if (cudaEventElapsedTime(&e, h->pev[k][2 * n], h->pev[k][2 * n + 1]) == cudaSuccess) ms += e;
            }
            if (ms < best[q][k]) { best[q][k] = ms; pick[q][k] = c; }
        }
      }
    }
    cudaGetLastError();
    for (int k = 0; k < 4; ++k) {
        for (cudaEvent_t e : h->pev[k]) cudaEventDestroy(e);
        h->pev[k].swap(saved[k]);
    }
    h->prof_every = saved_every;
    if (r) {
        set_tiling(h, ra0, rb0);
        return r;
    }
    // fwd_vel, fwd_str and adj_a share a tiling (the receivers' tile lists):
    // the height with the lower sum of their best times; adj_b its own
    const double sa[2] = {best[0][0] + best[0][1] + best[0][2], best[1][0] + best[1][1] + best[1][2]};
    const int qa = sa[0] < sa[1] ? 0 : 1, qb = best[0][3] < best[1][3] ? 0 : 1;
    if ((r = set_tiling(h, qa + 1, qb + 1))) return r;
    int spg[4] = {pick[qa][0], pick[qa][1], pick[qa][2], pick[qb][3]};
    // stage 2: whole steps, split into chains as the passes will be.  The
    // per-kernel picks let a pass split only when they coincide; a uniform
    // grouping always does.  Time the picks and every uniform grouping and
    // keep the fastest.
    if (h->d.shot_group <= 0 && h->chains > 1) {
        // no sampled timing while timing whole steps (it would also keep
        // the passes in one chain)
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CK(h, cudaEventCreate(&e0));
        if (cudaEventCreate(&e1) != cudaSuccess) {
            cudaEventDestroy(e0);
            return fail(h, STFWI_ERR_CUDA, "autotune: cudaEventCreate failed");
        }
        const int keep_every = h->prof_every;
        h->prof_every = 0;
        double best_ms = 1e300;
        int keep[4] = {spg[0], spg[1], spg[2], spg[3]};
        for (int ci = -1; ci < (int)(sizeof(cand) / sizeof(cand[0])) && !r; ++ci) {
            int trial[4];
            if (ci < 0) {
                for (int k = 0; k < 4; ++k) trial[k] = spg[k];
            } else {
                if (cand[ci] > h->nshot) break;
                for (int k = 0; k < 4; ++k) trial[k] = cand[ci];
            }
            set_groups(h, trial);
            float ms = 0.f;
            for (int rep = 0; rep < 2 && !r; ++rep) {   // the first run warms up
                if (rep == 1 && cudaEventRecord(e0, st) != cudaSuccess) r = STFWI_ERR_CUDA;
                if (!r) r = enqueue_timing_steps(h, steps, st);
            }
            if (!r && (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                       cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                r = fail(h, STFWI_ERR_CUDA, "autotune: timing of whole steps failed");
            if (!r && ms < best_ms) {
                best_ms = ms;
                for (int k = 0; k < 4; ++k) keep[k] = trial[k];
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaGetLastError();
        h->prof_every = keep_every;
        if (r) return r;
        for (int k = 0; k < 4; ++k) spg[k] = keep[k];
    }
    for (int k = 0; k < 4; ++k) h->tuned[k] = spg[k];
    // a descriptor shot_group > 0 keeps its shots per block (the tile
    // shapes are still the tuned ones)
    if (h->d.shot_group > 0)
        for (int k = 0; k < 4; ++k) spg[k] = h->d.shot_group;
    set_groups(h, spg);
    drop_graphs(h);
    h->stored = false;   // the timing passes overwrote the state
    if (spg_out)
        for (int k = 0; k < 4; ++k) spg_out[k] = spg[k];
    return STFWI_OK;
}

stfwi_status stfwi_set_tile_rows(stfwi_handle *h, int32_t rows_a, int32_t rows_b)
{
    if (!h) return STFWI_ERR_INVALID;
    if (rows_a % NWARP || rows_b % NWARP)
        return fail(h, STFWI_ERR_INVALID, "tile rows (%d, %d): use 8 or 16", rows_a, rows_b);
    // the state and a kept history do not depend on the tiling
    return set_tiling(h, rows_a / NWARP, rows_b / NWARP);
}

stfwi_status stfwi_set_chains(stfwi_handle *h, int32_t chains)
{
    if (!h) return STFWI_ERR_INVALID;
    if (chains < 1 || chains > MAX_CHAINS)
        return fail(h, STFWI_ERR_INVALID, "chains %d outside [1, %d]", chains, MAX_CHAINS);
    if (chains != h->chains) {
        CK(h, cudaStreamSynchronize(h->hs));
        h->chains = chains;
        drop_graphs(h);   // the split is part of the captured graphs
    }
    return STFWI_OK;
}

stfwi_status stfwi_tile_rows(const stfwi_handle *h, int32_t *rows_out)
{
    if (!h || !rows_out) return STFWI_ERR_INVALID;
    rows_out[0] = h->tha;
    rows_out[1] = h->thb;
    return STFWI_OK;
}

stfwi_status stfwi_set_wait_limit(stfwi_handle *h, int64_t polls)
{
    if (!h) return STFWI_ERR_INVALID;
    const uint32_t v = polls < 0 ? WAIT3 : (uint32_t)std::min<int64_t>(polls, WAIT3);
    if (v != h->g.wait_polls) {
        h->g.wait_polls = v;
        drop_graphs(h);   // the limit is a kernel argument baked into the captured graphs
    }
    return STFWI_OK;
}

stfwi_status stfwi_check(stfwi_handle *h, void *stream)
{
    if (!h) return STFWI_ERR_INVALID;
    int v = 0;
    CK(h, cudaMemcpyAsync(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(h, cudaStreamSynchronize((cudaStream_t)stream));
    if (v & 1) return fail(h, STFWI_ERR_NONFINITE, "a receiver sample became non-finite (unstable dt or model?)");
    if (v & ST_TIMEOUT3) return fail(h, STFWI_ERR_TIMEOUT, "a tile copy did not complete within the wait limit");
    return STFWI_OK;
}


stfwi_status stfwi_forward_frames(stfwi_handle *h, uint32_t fields, float *frames, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if (!frames || fields == 0 || fields >= 32u) return fail(h, STFWI_ERR_INVALID, "no frames or bad field mask");
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    const int nf = popc5(fields);
    const size_t N = (size_t)g.nz * g.nx, sbytes = (size_t)h->nshot * nf * N * sizeof(float);
    float *stage = nullptr;
    if (cudaMallocAsync((void **)&stage, sbytes, st) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, STFWI_ERR_OOM, "no room for the %zu-byte frame staging buffer", sbytes);
    }
    rc = zero_forward_state(h, st);
    if (rc) { cudaFreeAsync(stage, st); return rc; }
    FwdOut o{};
    o.rec = h->rec;
    o.status = h->status;
    o.slots = h->slots;
    const dim3 grid((unsigned)((N + 255) / 256), h->nshot);
    for (int n = 0; n < g.nt; ++n) {
        fwd_step(h, n, o, st);
        k_frames_fwd<<<grid, 256, 0, st>>>(g, mat_of(h), h->F, fields, nf, stage);
        // frame n of every (shot, field) plane: rows of N floats, nt frames apart
        cudaError_t e = cudaMemcpy2DAsync(frames + (size_t)n * N, (size_t)g.nt * N * sizeof(float), stage,
                                          N * sizeof(float), N * sizeof(float), (size_t)h->nshot * nf,
                                          cudaMemcpyDefault, st);
        if (e != cudaSuccess) {
            cudaFreeAsync(stage, st);
            return fail(h, STFWI_ERR_CUDA, "frame copy: %s", cudaGetErrorString(e));
        }
    }
    cudaFreeAsync(stage, st);
    h->stored = false;
    CK(h, cudaGetLastError());
    return STFWI_OK;
}

stfwi_status stfwi_adjoint_frames(stfwi_handle *h, uint32_t fields, float *frames, float *src_wav_a, void *stream)
{
    stfwi_status rc = ready(h);
    if (rc) return rc;
    if (!frames || fields == 0 || fields >= 32u) return fail(h, STFWI_ERR_INVALID, "no frames or bad field mask");
    if (!src_wav_a) return fail(h, STFWI_ERR_INVALID, "src_wav_a is null");
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = h->g;
    const int nf = popc5(fields);
    int kex = -1, kez = -1;
    for (int b = 0, k = 0; b < 5; ++b)
        if (fields >> b & 1u) {
            if (b == 2) kex = k;
            if (b == 3) kez = k;
            ++k;
        }
    const size_t N = (size_t)g.nz * g.nx, sbytes = (size_t)h->nshot * nf * N * sizeof(float);
    float *stage = nullptr;
    if (cudaMallocAsync((void **)&stage, sbytes, st) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, STFWI_ERR_OOM, "no room for the %zu-byte frame staging buffer", sbytes);
    }
    rc = zero_adjoint_state(h, st);
    if (rc) { cudaFreeAsync(stage, st); return rc; }
    const int thr = 256;
    const unsigned nrb = (unsigned)((g.nshot * std::max(g.nrec, 1) + thr - 1) / thr);
    if (g.nrec > 0) k_inject_last<<<nrb, thr, 0, st>>>(g, h->rx, h->rz, h->rec_adj, h->A);
    const dim3 grid((unsigned)((N + 255) / 256), h->nshot);
    for (int n = g.nt - 1; n >= 0; --n) {
        const int ping = (g.nt - 1 - n) & 1;
        AdjIn ai{};
        ai.rec_adj = h->rec_adj; ai.row0 = h->row0; ai.slots = h->slots; ai.slot = 0;
        ai.accLr = h->accLr; ai.want_exact = 0; ai.ping = ping;
        AdjOut ao{};
        ao.snap = h->snap; ao.slots = h->slots; ao.slot_in = -1; ao.slot_img = -1; ao.slot_next = -1;
        ao.accp = h->accp; ao.acc = h->acc; ao.src_a = h->src_a; ao.rec_adj = h->rec_adj; ao.ping = ping;
        switch (h->d.fd_order) {
        case 2: launch_adj_step<2>(h, n, ai, ao, st); break;
        case 4: launch_adj_step<4>(h, n, ai, ao, st); break;
        default: launch_adj_step<8>(h, n, ai, ao, st); break;
        }
        k_frames_adj<<<grid, 256, 0, st>>>(g, mat_of(h), h->A, fields, nf, stage);
        if (g.nrec > 0 && n > 0 && (kex >= 0 || kez >= 0))
            k_frames_unpick<<<nrb, thr, 0, st>>>(g, h->rx, h->rz, h->rec_adj, n, kex, kez, nf, stage);
        cudaError_t e = cudaMemcpy2DAsync(frames + (size_t)n * N, (size_t)g.nt * N * sizeof(float), stage,
                                          N * sizeof(float), N * sizeof(float), (size_t)h->nshot * nf,
                                          cudaMemcpyDefault, st);
        if (e != cudaSuccess) {
            cudaFreeAsync(stage, st);
            return fail(h, STFWI_ERR_CUDA, "frame copy: %s", cudaGetErrorString(e));
        }
    }
    cudaFreeAsync(stage, st);
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(src_wav_a, h->src_a, (size_t)h->nshot * g.nt * 4, cudaMemcpyDefault, st));
    return STFWI_OK;
}

stfwi_status stfwi_imaging_condition(const stfwi_imaging_desc *d, const float *vs, const float *vp, const float *rho,
                                     const float *ex_hist, const float *ez_hist, const float *es_hist,
                                     const float *ua_hist, const float *va_hist, const float *vx_hist,
                                     const float *vz_hist, double *g_out, void *stream)
{
    if (!d || !vs || !vp || !rho || !ex_hist || !ez_hist || !es_hist || !ua_hist || !va_hist || !g_out) {
        fprintf(stderr, "stfwi_imaging_condition: null argument\n");
        return STFWI_ERR_INVALID;
    }
    if ((vx_hist == nullptr) != (vz_hist == nullptr)) {
        fprintf(stderr, "stfwi_imaging_condition: give both forward velocity histories or neither\n");
        return STFWI_ERR_INVALID;
    }
    if (d->nz_dom < 1 || d->nx_dom < 1 || d->pad < 0 || d->nt < 1 || !(d->dx > 0) || !(d->dz > 0) || !(d->dt > 0)) {
        fprintf(stderr, "stfwi_imaging_condition: bad descriptor\n");
        return STFWI_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nz = d->free_surface ? d->nz_dom + d->pad : d->nz_dom + 2 * d->pad, nx = d->nx_dom + 2 * d->pad;
    const long long N = (long long)nz * nx, nd = (long long)d->nz_dom * d->nx_dom;
    const int C = d->time_chunk > 0 ? d->time_chunk : 64;
    const bool rho_term = vx_hist != nullptr;
    // device copies of what is not device memory: the model, and chunks of
    // the histories (adjoint velocities with one frame on either side)
    const float *hist[7] = {ex_hist, ez_hist, es_hist, vx_hist, vz_hist, ua_hist, va_hist};
    bool dev[7];
    size_t stage_floats = 0;
    for (int k = 0; k < 7; ++k) {
        dev[k] = hist[k] ? device_resident(hist[k]) : true;
        if (!dev[k]) stage_floats += (size_t)(C + 2) * N;
    }
    const size_t model_floats = 3 * (size_t)nd;
    float *buf = nullptr;
    double *acc = nullptr, *gdev = nullptr;
    auto bail = [&](const char *what, cudaError_t e) {
        fprintf(stderr, "stfwi_imaging_condition: %s: %s\n", what, cudaGetErrorString(e));
        cudaGetLastError();
        if (buf) cudaFreeAsync(buf, st);
        if (acc) cudaFreeAsync(acc, st);
        if (gdev) cudaFreeAsync(gdev, st);
        return e == cudaErrorMemoryAllocation ? STFWI_ERR_OOM : STFWI_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMallocAsync((void **)&buf, (stage_floats + model_floats) * sizeof(float), st)) != cudaSuccess)
        return bail("staging", e);
    if ((e = cudaMallocAsync((void **)&acc, 3 * nd * sizeof(double), st)) != cudaSuccess) return bail("sums", e);
    if ((e = cudaMallocAsync((void **)&gdev, 6 * nd * sizeof(double), st)) != cudaSuccess) return bail("output", e);
    if ((e = cudaMemsetAsync(acc, 0, 3 * nd * sizeof(double), st)) != cudaSuccess) return bail("memset", e);
    float *mvs = buf + stage_floats, *mvp = mvs + nd, *mrho = mvp + nd;
    if ((e = cudaMemcpyAsync(mvs, vs, nd * 4, cudaMemcpyDefault, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(mvp, vp, nd * 4, cudaMemcpyDefault, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(mrho, rho, nd * 4, cudaMemcpyDefault, st)) != cudaSuccess)
        return bail("model copy", e);
    float *stage[7] = {nullptr};
    for (int k = 0, off = 0; k < 7; ++k)
        if (!dev[k]) { stage[k] = buf + (size_t)off * (C + 2) * N; ++off; }
    ImgArgs a{};
    a.nz = nz; a.nx = nx; a.nz_dom = d->nz_dom; a.nx_dom = d->nx_dom; a.z0 = d->free_surface ? 0 : d->pad;
    a.pad = d->pad; a.nt = d->nt; a.dt = d->dt; a.inv2dx = 1.0 / (2.0 * d->dx); a.inv2dz = 1.0 / (2.0 * d->dz);
    a.rho = mrho; a.acc = acc;
    for (int t0 = 0; t0 < d->nt; t0 += C) {
        const int t1 = std::min(t0 + C, d->nt);
        const int u0 = std::max(t0 - 1, 0), u1 = std::min(t1 + 1, d->nt);   // adjoint frames [u0, u1)
        const float *ptr[7];
        for (int k = 0; k < 7; ++k) {
            if (!hist[k]) { ptr[k] = nullptr; continue; }
            const int f0 = k >= 5 ? u0 : t0, f1 = k >= 5 ? u1 : t1;
            if (dev[k]) {
                ptr[k] = hist[k] + (size_t)f0 * N;
            } else {
                if ((e = cudaMemcpyAsync(stage[k], hist[k] + (size_t)f0 * N, (size_t)(f1 - f0) * N * 4,
                                         cudaMemcpyDefault, st)) != cudaSuccess)
                    return bail("history copy", e);
                ptr[k] = stage[k];
            }
        }
        a.ex = ptr[0]; a.ez = ptr[1]; a.es = ptr[2];
        a.vx = rho_term ? ptr[3] : nullptr; a.vz = rho_term ? ptr[4] : nullptr;
        a.ua = ptr[5]; a.va = ptr[6];
        a.t0 = t0; a.t1 = t1; a.ua0 = u0;
        k_imaging_hist<<<(unsigned)((nd + 127) / 128), 128, 0, st>>>(a);
    }
    k_imaging_chain<<<(unsigned)((nd + 255) / 256), 256, 0, st>>>(nd, mvs, mvp, mrho, acc, gdev);
    if ((e = cudaGetLastError()) != cudaSuccess) return bail("launch", e);
    if ((e = cudaMemcpyAsync(g_out, gdev, 6 * nd * sizeof(double), cudaMemcpyDefault, st)) != cudaSuccess)
        return bail("output copy", e);
    cudaFreeAsync(buf, st);
    cudaFreeAsync(acc, st);
    cudaFreeAsync(gdev, st);
    return STFWI_OK;
}

}  // extern "C"

// ================================================================ no-allocation misfit

// Residual preparation without any allocation, for callers that must not
// call cudaMalloc: an XLA custom call running inside a framework that has
// already reserved most of the device memory for its own pool (the JAX
// drivers of this workload run with 90 % preallocated), where a further
// cudaMalloc can fail or fragment the pool.  The only scratch it needs, one
// FP64 partial sum per trace, lives in this file-scope device array; every
// GPU that loads the library holds it until the process exits.
static constexpr int STFWI_NOALLOC_MAX_TRACES = 1 << 18;  // nshot * nrec <= 262144 (2 MiB)
static __device__ __align__(256) double g_noalloc_trace_sums[STFWI_NOALLOC_MAX_TRACES];

namespace {
std::mutex g_noalloc_mu;
// device address of the scratch per device, valid for the context it was
// looked up in (a reset device gets a new context and a fresh lookup)
struct NoallocSlot {
    void *ctx = nullptr;
    double *ptr = nullptr;
};
NoallocSlot g_noalloc_slot[256];

typedef int (*ctx_current_fn)(void **);
ctx_current_fn ctx_current()
{
    static ctx_current_fn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<ctx_current_fn>(p);
    }
    return fn;
}
}  // namespace

extern "C" stfwi_status stfwi_misfit_noalloc(int32_t nshot, int32_t nt, int32_t nrec, const float *pred,
                                             const float *obs, const stfwi_misfit_desc *m, float *rec_adj,
                                             double *misfit_out, void *stream)
{
    if (!pred || !obs || !m || !rec_adj || !misfit_out || nshot < 1 || nt < 1 || nrec < 1) {
        fprintf(stderr, "stfwi_misfit_noalloc: null pointer or empty size\n");
        return STFWI_ERR_INVALID;
    }
    if ((long long)nshot * nrec > STFWI_NOALLOC_MAX_TRACES) {
        fprintf(stderr, "stfwi_misfit_noalloc: %lld traces exceed the fixed scratch of %d traces\n",
                (long long)nshot * nrec, STFWI_NOALLOC_MAX_TRACES);
        return STFWI_ERR_INVALID;
    }
    if (m->component < 0 || m->component > 3 || m->nsos < 0 || m->nsos > MAX_SOS || (m->nsos > 0 && !m->sos)) {
        fprintf(stderr, "stfwi_misfit_noalloc: bad component %d or nsos %d\n", m->component, m->nsos);
        return STFWI_ERR_INVALID;
    }
    SosParams sp{};
    sp.nsos = m->nsos;
    for (int k = 0; k < m->nsos; ++k) {
        const double *c = m->sos + 6 * k;
        if (c[3] == 0.0) {
            fprintf(stderr, "stfwi_misfit_noalloc: sos section %d has a0 = 0\n", k);
            return STFWI_ERR_INVALID;
        }
        sp.c[k][0] = c[0] / c[3]; sp.c[k][1] = c[1] / c[3]; sp.c[k][2] = c[2] / c[3];
        sp.c[k][3] = c[4] / c[3]; sp.c[k][4] = c[5] / c[3];
    }
    // device address of the scratch, looked up once per device (and again
    // if the device's context changed, e.g. after cudaDeviceReset) with that
    // device current: the host-side symbol is only a stand-in
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return STFWI_ERR_CUDA;
    void *ctx = nullptr;
    ctx_current_fn cur = ctx_current();
    if (cur) cur(&ctx);
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoallocSlot &slot = g_noalloc_slot[dev];
        if (!slot.ptr || !ctx || slot.ctx != ctx) {
            double *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_trace_sums);
            if (e != cudaSuccess) {
                fprintf(stderr, "stfwi_misfit_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                slot = NoallocSlot{};
                return STFWI_ERR_CUDA;
            }
            // the lookup made the primary context current if it was not yet
            if (cur && !ctx) cur(&ctx);
            slot.ctx = ctx;
            slot.ptr = p;
        }
        scratch = slot.ptr;
    }
    Geo g{};
    g.nshot = nshot;
    g.nt = nt;
    g.nrec = nrec;
    cudaStream_t st = (cudaStream_t)stream;
    const int ntap = std::min(std::max(m->n_taper, 0), nt);
    const int nnorm = m->nshot_norm > 0 ? m->nshot_norm : nshot;
    const int n = nshot * nrec, thr = 128;
    k_misfit<<<(n + thr - 1) / thr, thr, 0, st>>>(g, m->component, ntap, sp, m->scale, nnorm, pred, obs, rec_adj,
                                                 scratch);
    k_misfit_reduce<<<(nshot + 127) / 128, 128, 0, st>>>(nshot, nrec, scratch, misfit_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "stfwi_misfit_noalloc: launch: %s\n", cudaGetErrorString(e));
        return STFWI_ERR_CUDA;
    }
    return STFWI_OK;
}
