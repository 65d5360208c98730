/*
 * stfwi.h -- C ABI of the B200 elastic velocity-strain solver.
 *
 * One handle = one padded grid + one shot batch on one CUDA device.  The
 * handle owns its device workspace (fields, C-PML memory strips, strain
 * history, gradient accumulators) and the batch's geometry.  Large inputs and
 * outputs are passed as plain pointers that may be host or device memory
 * (copies use cudaMemcpyDefault, so host pointers cost a transfer).  Calls
 * on one handle must come from one thread; every call is asynchronous on the
 * given stream unless it says otherwise.  Errors are status codes; a call
 * never aborts the process and never traps the GPU.  stfwi_last_error()
 * gives the message of the last failing call.
 *
 * The entry points replace the reference's Python functions
 * (paths relative to the reference project):
 *   stfwi_set_model + stfwi_forward  fwi/forward.py:119-501 (forward_jax) and
 *                                    :508-544 (build_forward_fn -> run_shot)
 *   stfwi_get_records                the (vx, vz, ex, ez) receiver tuple of
 *                                    forward_jax, fwi/forward.py:465-469
 *   stfwi_misfit                     fwi/gradient.py:139-156 (_shot_residual_prep
 *                                    and its jax.grad), fwi/loss.py:92-118
 *   stfwi_gradient(STFWI_GRAD_SRC)   fwi/adjoint_jax_kernel.py:61-483 (adjoint_jax)
 *   stfwi_gradient(STFWI_GRAD_EXACT) the 'ad' backend, fwi/gradient.py:106-132
 *   stfwi_gradient(STFWI_GRAD_IMAGING) the 'adjoint' backend's imaging,
 *                                    fwi/gradient.py:159-259, fwi/imaging.py:83-169
 *   stfwi_illumination               fwi/illumination.py:18-48 (Ws before cropping)
 *   stfwi_forward_frames             forward_jax return_vars '*_full' / return_wavefields
 *   stfwi_adjoint_frames             adjoint_jax(..., return_wavefields=True)
 *   stfwi_imaging_condition          fwi/imaging.py:83-169 (imaging_condition)
 */
#ifndef STFWI_H
#define STFWI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    STFWI_OK = 0,
    STFWI_ERR_INVALID = 1,     /* bad argument or descriptor (ValueError in the reference) */
    STFWI_ERR_UNSUPPORTED = 2, /* fd_order / src_type not supported (NotImplementedError) */
    STFWI_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    STFWI_ERR_OOM = 4,         /* workspace does not fit the memory budget */
    STFWI_ERR_NONFINITE = 5,   /* a receiver sample became NaN/Inf (unstable model or dt) */
    STFWI_ERR_STATE = 6,       /* call order: e.g. gradient before a storing forward */
    STFWI_ERR_TIMEOUT = 7      /* a kernel's bounded wait on a tile copy expired */
} stfwi_status;

typedef struct stfwi_handle stfwi_handle;

/* Grid, time and batch description (the static arguments of forward_jax). */
typedef struct {
    int32_t nz_dom, nx_dom; /* physical model size (rows z, columns x) */
    int32_t pad;            /* C-PML thickness in cells */
    int32_t fd_order;       /* 2, 4 or 8 */
    int32_t free_surface;   /* 1: free surface on top, PML on 3 sides */
    int32_t nt;             /* time steps */
    int32_t nrec;           /* receivers (shared by all shots) */
    int32_t max_shots;      /* shot batch capacity */
    double dx, dz, dt;      /* grid spacing [m], time step [s] */
    double fc;              /* source peak frequency, used by the PML profile */
    int32_t want_gradient;  /* 1: reserve the stress history + accumulators (g_Vs, g_Vp);
                               2: also keep the velocities in the history, for the density
                               gradient g_rho of both modes */
    int32_t shot_group;     /* shots per block (0: automatic) */
    double mem_budget_gb;   /* device memory the handle may use (0: 85% of free) */
    int32_t kernel_variant; /* must be 0 (the library has one stencil-kernel family; other values
                               return STFWI_ERR_UNSUPPORTED) */
    int32_t ckpt_interval;  /* gradient history: 0 = keep every step if it fits the budget, else
                               checkpoint the state every k steps and recompute each k-step
                               segment during the adjoint (k chosen to fit); k > 0 = that k */
} stfwi_desc;

/* source types */
#define STFWI_SRC_FORCE 0  /* vertical force into Vz (fwi/forward.py:366-367) */
#define STFWI_SRC_MOMENT 1 /* explosive moment into exx, ezz (fwi/forward.py:406-411) */

/* stfwi_forward flags */
#define STFWI_FWD_STORE 1u  /* keep the strain history a later stfwi_gradient needs */

/* stfwi_gradient modes (bit set) */
#define STFWI_GRAD_EXACT 1u   /* exact discrete gradient of the FP32 forward */
#define STFWI_GRAD_IMAGING 2u /* the reference's continuous imaging formula */
#define STFWI_GRAD_SRC 4u     /* source-wavelet adjoint (dot-product test) */

/* Residual preparation: misfit_k = scale/N * mean_{t,r}(F T (pred - obs))^2
 * on one receiver component; F = cascade of nsos biquads (b0 b1 b2 a0 a1 a2,
 * scipy 'sos' layout, normalised by a0), T = cosine end taper of n_taper
 * samples (fwi/filters.py).  N = nshot_norm when it is > 0, else the number
 * of shots of the call; the adjoint sources carry the same 1/N. */
typedef struct {
    int32_t component;  /* 0 vx, 1 vz, 2 exx, 3 ezz */
    int32_t n_taper;
    int32_t nsos;       /* 0: no filter; at most 16 sections */
    int32_t nshot_norm; /* 0: the call's own shot count; > 0: the total number of
                           shots across the ranks that share one loss (sharding) */
    double scale;
    const double *sos;  /* host pointer, [nsos][6] */
} stfwi_misfit_desc;

/* Device bytes stfwi_create allocates for d (with ckpt_interval = 0: the
 * every-step history). */
size_t stfwi_workspace_bytes(const stfwi_desc *d);
stfwi_status stfwi_create(const stfwi_desc *d, stfwi_handle **out);
void stfwi_destroy(stfwi_handle *h);
const char *stfwi_last_error(const stfwi_handle *h);

/* Model (nz_dom x nx_dom float32 each, z-major): builds the padded-grid
 * materials and C-PML profiles on the device. */
stfwi_status stfwi_set_model(stfwi_handle *h, const float *vs, const float *vp, const float *rho,
                             void *stream);

/* Receivers in physical-domain indices (host arrays of nrec). */
stfwi_status stfwi_set_receivers(stfwi_handle *h, int32_t nrec, const int32_t *rec_x,
                                 const int32_t *rec_z);

/* Shots: src = host [nshot][3] (x, z, type) in physical-domain indices;
 * wavelets = [nshot][nt] float32 (host or device). */
stfwi_status stfwi_set_shots(stfwi_handle *h, int32_t nshot, const int32_t *src,
                             const float *wavelets, void *stream);

/* Forward modelling of every shot of the batch in one launch per phase. */
stfwi_status stfwi_forward(stfwi_handle *h, uint32_t flags, void *stream);

/* Receiver traces of the last forward: [nshot][4][nt][nrec] (vx, vz, exx, ezz). */
stfwi_status stfwi_get_records(stfwi_handle *h, float *out, void *stream);

/* Misfit and adjoint sources from the last forward's traces.  obs =
 * [nshot][nt][nrec] float32 (host or device); misfit_out = [nshot] FP64
 * (host or device), per-shot terms whose sum is the reference's loss. */
stfwi_status stfwi_misfit(stfwi_handle *h, const float *obs, const stfwi_misfit_desc *m,
                          double *misfit_out, void *stream);

/* Explicit adjoint sources [nshot][4][nt][nrec] (replaces stfwi_misfit's). */
stfwi_status stfwi_set_adjoint_sources(stfwi_handle *h, const float *rec_adj, void *stream);

/* Adjoint sweep.  mode: STFWI_GRAD_* bits.  g_out: for each of EXACT then
 * IMAGING that is set, [3][nz_dom][nx_dom] FP64 = (dJ/dVs, dJ/dVp, dJ/drho)
 * summed over shots.  dJ/drho is filled by both modes when the handle was
 * created with want_gradient = 2 (the history then holds the velocities the
 * density term needs); with want_gradient = 1 both modes return it as 0.
 * src_wav_a: [nshot][nt] float32 when SRC is set. */
stfwi_status stfwi_gradient(stfwi_handle *h, uint32_t mode, double *g_out, float *src_wav_a,
                            void *stream);

/* Source illumination Ws = Sum_shots Sum_t field^2 of one component on the
 * padded grid, [nz_t][nx_t] FP64 (runs its own forward). */
stfwi_status stfwi_illumination(stfwi_handle *h, int32_t component, double *ws_out, void *stream);

/* Polls of a tile-copy wait before the kernel gives up, records
 * STFWI_ERR_TIMEOUT for stfwi_check and returns (no counterpart in the
 * reference).  polls < 0 restores the default (2^22); 0 makes every wait
 * give up at once, which is how the tests exercise the timeout path without
 * a GPU fault.  Values above the default are clamped to it. */
stfwi_status stfwi_set_wait_limit(stfwi_handle *h, int64_t polls);

/* Synchronises the stream and returns the device status word (0 = fine). */
stfwi_status stfwi_check(stfwi_handle *h, void *stream);

/* Sampled per-kernel timing (tracing).  With every > 0 the captured time
 * loops record a CUDA event pair around each kernel of every `every`-th
 * step; every = 0 turns it off.  Re-captures the graphs. */
stfwi_status stfwi_profile(stfwi_handle *h, int32_t every);

/* Sampled launch times of the passes run since the last call, as [4][2] =
 * (total ms, launches) for the kernels fwd_vel, fwd_str, adj_a, adj_b.
 * Synchronises the handle's stream; resets the sums. */
stfwi_status stfwi_kernel_times(stfwi_handle *h, double *out);

/* Tile-schedule autotuner (no counterpart in the reference): times `steps`
 * forward and adjoint steps of the handle's configuration for both tile
 * shapes (64 x 8 and 64 x 16 cells) and several numbers of shots per block
 * (1-25) with CUDA events around every kernel, and keeps the fastest: one
 * tile shape for fwd_vel, fwd_str and adj_a (they share the receivers' tile
 * lists), one for adj_b, and the shots per block of each of the four
 * stencil kernels (also across later stfwi_set_shots calls); spg_out [4]
 * (optional) receives the shots per block of fwd_vel, fwd_str, adj_a, adj_b,
 * stfwi_tile_rows the tile shapes.  A second stage times whole steps split
 * into chains as the passes will be (stfwi_set_chains) for those picks and
 * for each uniform grouping, and keeps the fastest.  Overwrites the fields
 * and history: call it before the forward whose history a gradient will
 * use.  A descriptor shot_group > 0 overrides the shots per block. */
stfwi_status stfwi_autotune(stfwi_handle *h, int32_t steps, int32_t *spg_out, void *stream);

/* Tile heights in rows (8 or 16; 16 and 16 until the autotuner has run):
 * rows_a for fwd_vel, fwd_str and adj_a, rows_b for adj_b.  Any other value
 * is STFWI_ERR_INVALID.  The fields and a kept history stay valid. */
stfwi_status stfwi_set_tile_rows(stfwi_handle *h, int32_t rows_a, int32_t rows_b);
/* rows_out [2]: the tile heights in use (rows_a, rows_b). */
stfwi_status stfwi_tile_rows(const stfwi_handle *h, int32_t *rows_out);

/* Chains a forward or adjoint pass may be split into (1-4, default 2; no
 * counterpart in the reference).  The shots never interact, so when all
 * four stencil kernels group the shots alike, a pass without checkpoint
 * segments and without sampled timing is recorded as `chains` independent
 * chains of launches over consecutive shot groups, on separate streams
 * joined at its end; their launches overlap on the GPU.  Traces are the
 * same bit for bit; the FP64 sums differ only in the order of their atomic
 * additions. */
stfwi_status stfwi_set_chains(stfwi_handle *h, int32_t chains);

/* Residual preparation that allocates nothing (no counterpart in the
 * reference): the same misfit and adjoint sources as stfwi_misfit, without a
 * handle, for callers that cannot call cudaMalloc -- e.g. a custom call made
 * from inside a framework that has reserved most of device memory for its own
 * pool, where one more allocation can fail or fragment that pool.  All
 * pointers are device memory:
 * pred [nshot][4][nt][nrec] (the layout stfwi_get_records returns), obs
 * [nshot][nt][nrec], rec_adj [nshot][4][nt][nrec] (written), misfit_out
 * [nshot] FP64 (written).  Its only scratch is a fixed device array of
 * 262144 FP64 per-trace sums (2 MiB, held by every GPU that loads the library
 * until exit): nshot * nrec above that limit returns STFWI_ERR_INVALID.  The
 * first call on a device (and the first after that device's context was
 * replaced, e.g. by cudaDeviceReset) looks the array up with
 * cudaGetSymbolAddress; make that first call before any stream capture on
 * the device.  Every slot of the array is written before it is read, and all
 * calls share it, so calls that overlap on the GPU race.  It calls no
 * cudaMalloc or cudaFree.  Errors are printed to stderr. */
stfwi_status stfwi_misfit_noalloc(int32_t nshot, int32_t nt, int32_t nrec, const float *pred,
                                  const float *obs, const stfwi_misfit_desc *m, float *rec_adj,
                                  double *misfit_out, void *stream);

/* Gradient post-processing applied on the device to every plane that
 * stfwi_gradient returns (fwi/gradient.py:266-277 _postprocess): Gaussian
 * smoothing with sigma grad_smooth_sigma (fwi/loss.py:17-30; 0 = none, at
 * most sigma 21), then the product with source_taper and with illumination
 * ([nz_dom][nx_dom] FP64, host or device, copied; null = none).  Stays set
 * for the following stfwi_gradient calls. */
stfwi_status stfwi_set_postprocess(stfwi_handle *h, double grad_smooth_sigma, const double *source_taper,
                                   const double *illumination, void *stream);

enum { STFWI_PRECOND_ILLUM = 0, STFWI_PRECOND_EPRECOND3 = 1 };

/* Gradient preconditioner from the forward energy Ws = sum_shots sum_t
 * field(component)^2 of the handle's model and shots, computed on the
 * device, written to out [nz_dom][nx_dom] FP64 (host or device), normalised
 * to max 1.  STFWI_PRECOND_ILLUM: 1 / (Ws + eps max Ws) on the physical grid
 * (fwi/illumination.py:18-48 compute_illumination_for_stage; the reference's
 * forward there injects forces, so set force shots to reproduce it).
 * STFWI_PRECOND_EPRECOND3: 1 / We with We the Plessix-Mulder energy of the
 * receiver line (fwi/preconditioning.py:65-139 eprecond3, as used by
 * fwi/optim_lbfgsb.py:51-100). */
stfwi_status stfwi_preconditioner(stfwi_handle *h, int32_t kind, int32_t component, double eps, double *out,
                                  void *stream);

/* Velocity feasibility projection in place on device FP64 arrays of n cells
 * (fwi/projections.py:67-117 project_velocity): Vp <= vp_cap (vp_cap <= 0:
 * no cap), Vs <= Vp / ((1 + K_margin) 2/sqrt(3)), Vs >= vs_floor, rho >=
 * rho_floor.  No handle; host pointers return STFWI_ERR_INVALID. */
stfwi_status stfwi_project_velocity(int64_t n, double *vs, double *vp, double *rho, double K_margin, double vp_cap,
                                    double vs_floor, double rho_floor, void *stream);

/* Full wavefield frames (bit set; frames come out in bit order). */
#define STFWI_FRAME_VX 1u  /* vx  (U)   forward; U_a adjoint */
#define STFWI_FRAME_VZ 2u  /* vz  (V)   forward; V_a adjoint */
#define STFWI_FRAME_EX 4u  /* exx       forward; ex_a adjoint */
#define STFWI_FRAME_EZ 8u  /* ezz       forward; ez_a adjoint */
#define STFWI_FRAME_ES 16u /* exz       forward; es_a adjoint */

/* Forward modelling that also returns full wavefields: the reference's
 * return_vars 'vx_full' .. 'es_full' and return_wavefields=True
 * (fwi/forward.py:122,148-155,449-463).  frames = [nshot][nfields][nt][nz_t][nx_t]
 * float32 (host or device), frame n = the state after step n, strains
 * recovered from the carried stresses.  The receiver traces are filled as by
 * stfwi_forward; no strain history is kept.  A device staging buffer of
 * nshot * nfields padded grids is allocated for the call (STFWI_ERR_OOM if it
 * does not fit). */
stfwi_status stfwi_forward_frames(stfwi_handle *h, uint32_t fields, float *frames, void *stream);

/* Adjoint sweep of the source-wavelet adjoint (STFWI_GRAD_SRC) that also
 * returns the adjoint wavefields: adjoint_jax(..., return_wavefields=True)
 * (fwi/adjoint_jax_kernel.py:69,91-93,470-483).  frames = [nshot][nfields]
 * [nt][nz_t][nx_t] float32 (host or device) of (U_a, V_a, ex_a, ez_a, es_a)
 * by STFWI_FRAME_* bits, in forward-time order: frame n = the carry out of
 * adjoint step n.  src_wav_a = [nshot][nt].  Adjoint sources come from
 * stfwi_set_adjoint_sources or stfwi_misfit. */
stfwi_status stfwi_adjoint_frames(stfwi_handle *h, uint32_t fields, float *frames, float *src_wav_a,
                                  void *stream);

/* The reference's imaging condition on histories the caller holds
 * (fwi/imaging.py:83-169 imaging_condition), without a handle. */
typedef struct {
    int32_t nz_dom, nx_dom, pad, free_surface, nt;
    int32_t time_chunk; /* frames per chunk of the time sums (0: 64) */
    double dx, dz, dt;
} stfwi_imaging_desc;

/* vs, vp, rho: [nz_dom][nx_dom] float32; ex, ez, es, ua, va (and optionally
 * vx, vz, both or neither): [nt][nz_t][nx_t] float32 histories of the forward
 * strains, adjoint velocities and forward velocities, host or device memory
 * (host histories are copied a chunk at a time).  g_out = [6][nz_dom][nx_dom]
 * FP64 (host or device): g_Vs, g_Vp, g_rho, g_lam, g_mu, g_rho_lame.  Time
 * sums in FP64.  Allocates its working buffers for the call; errors are
 * printed to stderr. */
stfwi_status stfwi_imaging_condition(const stfwi_imaging_desc *d, const float *vs, const float *vp,
                                     const float *rho, const float *ex_hist, const float *ez_hist,
                                     const float *es_hist, const float *ua_hist, const float *va_hist,
                                     const float *vx_hist, const float *vz_hist, double *g_out, void *stream);

/* Padded-grid shape of a descriptor. */
void stfwi_grid_shape(const stfwi_desc *d, int32_t *nz_t, int32_t *nx_t);

#ifdef __cplusplus
}
#endif
#endif
