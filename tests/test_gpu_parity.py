"""CUDA path vs the oracle and the reference's known answers (B200).

Tolerances (FP32 stencils against FP64 references):
* seismograms: rel-L2 <= 1e-5 on the 60-step dot-product cases
  (observed ~1e-7; bound from FP32 rounding growth over the steps);
* dot-product identity in FP32: |<Ls,y> - <s,L^T y>| / |<Ls,y>| <= 1e-5;
* Marmousi 5 shots x 400 steps: misfit rel <= 1e-6, g_Vs rel-L2 <= 1e-6
  against the reference's FP64 AD gradient and imaging gradient (measured
  3.7e-7, 3.0e-7, 2.8e-7).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _solver(nt, nrec, nshot, fd, fs, want_gradient=False, pad=C.PAD, nz=C.NZ, nx=C.NX, dx=C.DX,
            dz=C.DZ, dt=C.DT, fc=C.FC, **kw):
    from stfwi_b200 import Solver
    return Solver(nz, nx, dx, dz, dt, nt, fc, pad, nrec, nshot, fd_order=fd, free_surface=fs,
                  want_gradient=want_gradient, **kw)




@pytest.mark.parametrize("tiles", [(16, 16), (8, 8)])
@pytest.mark.parametrize("fd,fs,st", C.CONFIGS)
def test_forward_and_adjoint_vs_oracle(fd, fs, st, tiles):
    """The reference's dot-product case (test_adjoint_kernel.py) on the GPU:
    seismograms and the source adjoint against the FP64 oracle, and the
    dot-product identity of the FP32 kernels."""
    vs, vp, rho = C.model()
    sx, sz, rx, rz = C.acquisition(fs, st)
    s_in, ys = C.random_vectors()
    S = _solver(C.NT, len(rx), 1, fd, fs)
    S.set_tile_rows(*tiles)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots([sx], [sz], [st], s_in.astype(np.float32))
    S.forward()
    rec = S.records()[0]
    ref, _, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC,
                          C.PAD, s_in, fd, fs, st, d0_f32=True)
    for c in range(4):
        assert _rel(rec[c], ref[c]) < 1e-5, (c, _rel(rec[c], ref[c]))
    S.set_adjoint_sources(np.stack(ys)[None].astype(np.float32))
    src_a = S.gradient(exact=False, src=True)["src"][0]
    a = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                  fd_order=fd, free_surface=fs, src_type=st, d0_f32=True)
    assert _rel(src_a, a["src"]) < 1e-5, _rel(src_a, a["src"])
    lhs = sum(float(np.sum(rec[c].astype(np.float64) * ys[c])) for c in range(4))
    rhs = float(np.sum(s_in * src_a.astype(np.float64)))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)
    S.close()


@pytest.mark.parametrize("fd,fs,st", [(8, True, "force"), (8, True, "moment"), (4, False, "force"),
                                      (2, False, "moment")])
def test_exact_and_imaging_gradient_vs_oracle(fd, fs, st):
    """Model gradients of the GPU (FP32 stencils, FP64 sums) against the
    FP64 oracle on a small case: exact (AD) and imaging formula."""
    vs, vp, rho = C.model()
    nt = 120
    sx, sz, rx, rz = C.acquisition(fs, st)
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=nt,
               fc=C.FC, pad=C.PAD, fd_order=fd, free_surface=fs, d0_f32=True)
    obs = O.forward_batch(vs * 1.03, vp, rho, [sx], [sz], [st], src_wavelet=wav, **geo)[:, 0]
    kw = dict(src_x=[sx], src_z=[sz], src_wavelet=wav, observed=obs, src_types=[st], component=0,
              scale=1.0, invert="vs_vp", **geo)
    (gx_vs, gx_vp, _), loss = O.compute_gradient("ad", Vs=vs, Vp=vp, rho=rho, **kw)
    (gi_vs, gi_vp, _), _ = O.compute_gradient("adjoint", Vs=vs, Vp=vp, rho=rho, **kw)
    S = _solver(nt, len(rx), 1, fd, fs, want_gradient=True)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots([sx], [sz], [st], wav.astype(np.float32))
    S.forward(store=True)
    mis = S.misfit(obs.astype(np.float32), 0, 1.0)
    # the misfit is a sum of squared differences of nearly equal traces; its
    # FP32 error scales with |pred| / |pred - obs|
    rec = S.records()[0, 0].astype(np.float64)
    amp = float(np.linalg.norm(rec) / np.linalg.norm(rec - obs[0]))
    g = S.gradient(exact=True, imaging=True)
    errs = {"misfit": abs(mis.sum() / loss - 1),
            "exact_vs": _rel(g["exact"][0], gx_vs), "exact_vp": _rel(g["exact"][1], gx_vp),
            "img_vs": _rel(g["imaging"][0], gi_vs), "img_vp": _rel(g["imaging"][1], gi_vp)}
    print(f"fd{fd} fs={fs} {st}: amplification {amp:.1f} errors {errs}")
    tol = 2e-5 * max(amp, 1.0)
    assert all(e < tol for e in errs.values()), (tol, errs)
    S.close()


def test_marmousi_known_answers(known_answers):
    """Results_gradient/gradient_compare.npz: 5 shots, nt=400, fd8, free
    surface, exx misfit.  FP32 GPU against the reference's FP64 numbers."""
    K = known_answers
    nt, pad, fd = int(K["gc_nt"]), int(K["gc_pad"]), int(K["gc_fd_order"])
    dt, fc, comp = float(K["gc_dt"]), float(K["gc_f_c"]), int(K["gc_component"])
    nz, nx = K["Vs_true"].shape
    rx, rz = K["gc_rec_x"], K["gc_rec_z"]
    ns = len(K["gc_src_x"])
    wav = O.ricker(np.arange(nt) * dt, fc, 1.5 / fc).astype(np.float32)
    S = _solver(nt, len(rx), ns, fd, True, want_gradient=True, pad=pad, nz=nz, nx=nx, dx=20.0,
                dz=20.0, dt=dt, fc=fc)
    S.set_receivers(rx, rz)
    S.set_shots(K["gc_src_x"], K["gc_src_z"], "force", wav)
    S.set_model(K["Vs_true"], K["Vp_true"], K["rho_true"])
    S.forward()
    obs = S.records()[:, comp].copy()
    auto = 1.0 / (np.mean(obs.astype(np.float64) ** 2) + 1e-45)
    assert abs(auto / K["gc_auto_scale"] - 1) < 1e-4, (auto, K["gc_auto_scale"])
    S.set_model(K["Vs_init"], K["Vp_init"], K["rho_init"])
    S.forward(store=True)
    loss = S.misfit(obs, comp, float(K["gc_auto_scale"])).sum()
    assert abs(loss / K["gc_loss_AD"] - 1) < 1e-6, (loss, K["gc_loss_AD"])
    g = S.gradient(exact=True, imaging=True)
    e_ad = _rel(g["exact"][0], K["gc_g_Vs_AD"])
    e_hc = _rel(g["imaging"][0], K["gc_g_Vs_HC"])
    print(f"marmousi: loss rel {abs(loss / K['gc_loss_AD'] - 1):.3e}  g_Vs_AD rel-L2 {e_ad:.3e}  "
          f"g_Vs_HC rel-L2 {e_hc:.3e}")
    # measured on a B200: loss 3.7e-7, g_Vs_AD 3.0e-7, g_Vs_HC 2.8e-7 (FP32
    # stencils against the reference's FP64 numbers); bounds about 3x
    assert e_ad < 1e-6 and e_hc < 1e-6, (e_ad, e_hc)
    S.close()


def test_batch_of_shots_matches_single_shots():
    """A batch of 7 mixed force/moment shots (several shots per block, both
    pipeline stages in use) gives each shot's traces and the summed gradient
    of the single-shot runs."""
    vs, vp, rho = C.model()
    nt, fd, fs = 90, 8, True
    rx = np.arange(1, C.NX - 1, 3, dtype=np.int32)
    rz = np.ones_like(rx)
    sx = np.array([3, 7, 11, 15, 19, 23, 27])
    sz = np.array([2, 5, 3, 6, 2, 4, 3])
    types = ["force", "moment"] * 3 + ["force"]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    rng = np.random.default_rng(5)
    obs = rng.standard_normal((7, nt, len(rx))).astype(np.float32) * 1e-9
    S = _solver(nt, len(rx), 7, fd, fs, want_gradient=True, shot_group=2)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    S.forward(store=True)
    rec = S.records()
    mis = S.misfit(obs, 1, 1.0)
    g = S.gradient(exact=True)["exact"][0]
    S.close()
    gsum = np.zeros_like(g)
    for k in range(7):
        S1 = _solver(nt, len(rx), 1, fd, fs, want_gradient=True)
        S1.set_model(vs, vp, rho)
        S1.set_receivers(rx, rz)
        S1.set_shots(sx[k:k + 1], sz[k:k + 1], types[k:k + 1], wav)
        S1.forward(store=True)
        r1 = S1.records()[0]
        assert _rel(rec[k], r1) < 1e-6, (k, _rel(rec[k], r1))
        m1 = S1.misfit(obs[k:k + 1], 1, 1.0, nshot_norm=7)
        assert abs(m1[0] / mis[k] - 1) < 1e-6
        gsum += S1.gradient(exact=True)["exact"][0]
        S1.close()
    assert _rel(g, gsum) < 1e-5, _rel(g, gsum)


@pytest.mark.parametrize("ckpt,density", [(0, False), (7, False), (0, True), (7, True)])
def test_split_passes_equal_one_chain(ckpt, density):
    """With every kernel grouping the shots alike (shot_group 2: four groups
    of the 8 shots) a pass runs as 2, 3 or 4 independent chains over the
    groups on separate streams; with sampled kernel timing on, or one chain
    set, it runs as one.  With checkpoints every 7 steps the chains join
    around every checkpoint copy.  The traces agree bit for bit (each shot's
    arithmetic is the same) and the gradients to FP64 rounding (the order of
    the atomic FP64 sums)."""
    vs, vp, rho = C.model()
    nt, fd, fs = 90, 8, True
    rx = np.arange(1, C.NX - 1, 3, dtype=np.int32)
    rz = np.ones_like(rx)
    sx = np.array([3, 7, 11, 15, 19, 23, 27, 30])
    sz = np.array([2, 5, 3, 6, 2, 4, 3, 5])
    types = ["force", "moment"] * 4
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    obs = np.random.default_rng(6).standard_normal((8, nt, len(rx))).astype(np.float32) * 1e-9
    out = []
    for every, chains in ((7, 2), (0, 2), (0, 3), (0, 4), (0, 1)):
        S = _solver(nt, len(rx), 8, fd, fs, want_gradient=True, shot_group=2, ckpt_interval=ckpt,
                    density=density)
        S.set_model(vs, vp, rho)
        S.set_receivers(rx, rz)
        S.set_shots(sx, sz, types, wav)
        S.set_chains(chains)
        S.profile(every)
        S.forward(store=True)
        rec = S.records()
        mis = S.misfit(obs, 1, 1.0)
        g = S.gradient(exact=True, imaging=True)
        out.append((rec, mis, g["exact"][0], g["exact"][1], g["imaging"][0])
                   + ((g["exact"][2], g["imaging"][2]) if density else ()))
        S.close()
    for k in range(1, len(out)):
        assert np.array_equal(out[0][0], out[k][0]), k
        for a, b in zip(out[0][1:], out[k][1:]):
            assert _rel(a, b) < 1e-12, (k, _rel(a, b))
    S = _solver(nt, len(rx), 8, fd, fs)
    for bad in (0, 5, -1):
        with pytest.raises(ValueError):
            S.set_chains(bad)
    S.close()


def test_checkpointed_gradient_equals_store_all():
    """Checkpoint every k steps + recompute gives the gradient of the
    every-step history (the recompute is deterministic), for an explicit k
    that does not divide nt and for the k a small memory budget forces."""
    vs, vp, rho = C.model()
    nt, fd, fs = 100, 8, True
    rx = np.arange(1, C.NX - 1, 3, dtype=np.int32)
    rz = np.ones_like(rx)
    sx, sz, types = np.array([6, 20]), np.array([2, 5]), ["force", "moment"]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    obs = np.random.default_rng(3).standard_normal((2, nt, len(rx))).astype(np.float32) * 1e-9
    out = []
    for ck, budget in ((0, 0.0), (7, 0.0), (0, 0.06)):
        S = _solver(nt, len(rx), 2, fd, fs, want_gradient=True, ckpt_interval=ck,
                    mem_budget_gb=budget)
        S.set_model(vs, vp, rho)
        S.set_receivers(rx, rz)
        S.set_shots(sx, sz, types, wav)
        S.forward(store=True)
        mis = S.misfit(obs, 2, 1.0)
        g = S.gradient(exact=True, imaging=True)
        out.append((mis, g["exact"][0], g["exact"][1], g["imaging"][0]))
        S.close()
    for k in (1, 2):
        for a, b in zip(out[k], out[0]):
            assert _rel(a, b) < 1e-12, (k, _rel(a, b))


def _smooth_model(nz, nx, seed):
    """A heterogeneous model with structure at several scales (smoothed noise
    on a gradient), so that every tile sees different materials."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    zz = np.arange(nz)[:, None] / nz
    n1 = gaussian_filter(rng.standard_normal((nz, nx)), 4.0)
    n1 /= np.abs(n1).max()
    vp = 2200.0 + 900.0 * zz + 250.0 * n1
    vs = vp / 1.8 + 60.0 * gaussian_filter(rng.standard_normal((nz, nx)), 2.0)
    rho = 1900.0 + 250.0 * zz + 40.0 * n1
    return vs, vp, rho


@pytest.mark.parametrize("tiles", [(16, 16), (8, 8), (16, 8), (8, 16)])
@pytest.mark.parametrize("fd,fs", [(8, True), (8, False), (4, True), (2, False)])
def test_multi_tile_grid_vs_oracle(fd, fs, tiles):
    """A grid of several tiles in x and z (interior tiles without the C-PML
    fix-up, tile edges inside the stencil reach), with sources and receivers
    near tile edges: seismograms, misfit and the exact gradient against the
    FP64 oracle."""
    nz, nx, pad, nt = 70, 150, 10, 110
    dx = dz = 10.0
    dt, fc = 1.0e-3, 18.0
    vs, vp, rho = _smooth_model(nz, nx, 7)
    rx = np.arange(0, nx, 3, dtype=np.int32)
    rz = np.full_like(rx, 0 if fs else 3)
    rz[::4] = 31                      # a tile-row edge in z (tiles of 8 and 16 rows)
    # 44 + pad = 54: two columns below a 64-column tile edge; the second and
    # third sources sit inside interior tiles (rows 16-31 and 32-47, columns 64-127)
    sx = np.array([44, 54, 70])
    sz = np.array([0 if fs else 5, 22, 47])
    types = ["force", "moment", "force"]
    wav = O.ricker(np.arange(nt) * dt, fc, 1.5 / fc) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=nx, nz_dom=nz, dx=dx, dz=dz, dt=dt, nt=nt, fc=fc, pad=pad,
               fd_order=fd, free_surface=fs, d0_f32=True)
    obs = O.forward_batch(vs * 1.02, vp, rho, sx, sz, types, src_wavelet=wav, **geo)[:, 1]
    ref = O.forward_batch(vs, vp, rho, sx, sz, types, src_wavelet=wav, **geo)
    kw = dict(src_x=sx, src_z=sz, src_wavelet=wav, observed=obs, src_types=types, component=1,
              scale=1.0, invert="vs_vp", **geo)
    (gx_vs, gx_vp, _), loss = O.compute_gradient("ad", Vs=vs, Vp=vp, rho=rho, **kw)
    S = _solver(nt, len(rx), 3, fd, fs, want_gradient=True, pad=pad, nz=nz, nx=nx, dx=dx, dz=dz, dt=dt,
                fc=fc)
    S.set_tile_rows(*tiles)
    assert S.tile_rows() == tiles
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav.astype(np.float32))
    S.forward(store=True)
    rec = S.records()
    for k in range(3):
        for c in range(4):
            assert _rel(rec[k, c], ref[k, c]) < 1e-5, (k, c, _rel(rec[k, c], ref[k, c]))
    mis = S.misfit(obs.astype(np.float32), 1, 1.0)
    amp = float(np.linalg.norm(rec[:, 1]) / np.linalg.norm(rec[:, 1] - obs))
    g = S.gradient(exact=True)
    errs = {"misfit": abs(mis.sum() / loss - 1), "exact_vs": _rel(g["exact"][0], gx_vs),
            "exact_vp": _rel(g["exact"][1], gx_vp)}
    print(f"multi-tile fd{fd} fs={fs} tiles {tiles}: amplification {amp:.1f} errors {errs}")
    tol = 2e-5 * max(amp, 1.0)
    assert all(e < tol for e in errs.values()), (tol, errs)
    S.close()


def _density_case(fd, fs, st, big, nt):
    if big:
        nz, nx, pad, dx, dt, fc = 70, 150, 10, 10.0, 1.0e-3, 18.0
        vs, vp, rho = _smooth_model(nz, nx, 11)
        rx = np.arange(0, nx, 3, dtype=np.int32)
        rz = np.full_like(rx, 0 if fs else 3)
        sx, sz = np.array([54, 70]), np.array([22, 47])
        types = [st, "force"]
    else:
        nz, nx, pad, dx, dt, fc = C.NZ, C.NX, C.PAD, C.DX, C.DT, C.FC
        vs, vp, rho = C.model()
        sx0, sz0, rx, rz = C.acquisition(fs, st)
        sx, sz, types = np.array([sx0]), np.array([sz0]), [st]
    wav = O.ricker(np.arange(nt) * dt, fc, 1.5 / fc) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=nx, nz_dom=nz, dx=dx, dz=dx, dt=dt, nt=nt, fc=fc, pad=pad,
               fd_order=fd, free_surface=fs, d0_f32=True)
    obs = O.forward_batch(vs * 1.02, vp, rho * 1.01, sx, sz, types, src_wavelet=wav, **geo)[:, 1]
    return vs, vp, rho, sx, sz, types, wav, geo, obs


@pytest.mark.parametrize("fd,fs,st,big", [(8, True, "force", False), (8, True, "moment", False),
                                          (4, False, "force", False), (8, True, "moment", True)])
def test_density_gradient_vs_oracle(fd, fs, st, big):
    """invert='all': the exact g_rho (buoyancy, moment and free-surface terms
    through rho) and the imaging g_rho with its velocity term
    (fwi/imaging.py:145-154) against the FP64 oracle; g_Vs and g_Vp are the
    same with and without the velocity history."""
    nt = 110
    vs, vp, rho, sx, sz, types, wav, geo, obs = _density_case(fd, fs, st, big, nt)
    kw = dict(src_x=sx, src_z=sz, src_wavelet=wav, observed=obs, src_types=types, component=1,
              scale=1.0, invert="all", **geo)
    (gx_vs, gx_vp, gx_rho), loss = O.compute_gradient("ad", Vs=vs, Vp=vp, rho=rho, **kw)
    (gi_vs, gi_vp, gi_rho), _ = O.compute_gradient("adjoint", Vs=vs, Vp=vp, rho=rho, **kw)
    g = {}
    for density in (False, True):
        S = _solver(nt, len(geo["rec_x"]), len(sx), fd, geo["free_surface"], want_gradient=True,
                    pad=geo["pad"], nz=geo["nz_dom"], nx=geo["nx_dom"], dx=geo["dx"], dz=geo["dz"],
                    dt=geo["dt"], fc=geo["fc"], density=density)
        S.set_model(vs, vp, rho)
        S.set_receivers(geo["rec_x"], geo["rec_z"])
        S.set_shots(sx, sz, types, wav.astype(np.float32))
        S.forward(store=True)
        mis = S.misfit(obs.astype(np.float32), 1, 1.0)
        rec = S.records()[:, 1].astype(np.float64)
        amp = float(np.linalg.norm(rec) / np.linalg.norm(rec - obs))
        g[density] = S.gradient(exact=True, imaging=True)
        S.close()
    for k in ("exact", "imaging"):
        for c in (0, 1):
            assert _rel(g[True][k][c], g[False][k][c]) < 1e-12, (k, c)
    assert np.all(g[False]["exact"][2] == 0.0)
    errs = {"misfit": abs(mis.sum() / loss - 1), "exact_rho": _rel(g[True]["exact"][2], gx_rho),
            "img_rho": _rel(g[True]["imaging"][2], gi_rho), "exact_vs": _rel(g[True]["exact"][0], gx_vs)}
    print(f"density fd{fd} fs={fs} {st} big={big}: amplification {amp:.1f} errors {errs}")
    tol = 2e-5 * max(amp, 1.0)
    assert all(e < tol for e in errs.values()), (tol, errs)


def test_density_gradient_checkpointed_equals_store_all():
    """With the velocity history, checkpoint segments (k = 7, not dividing
    nt) give the every-step result: the imaging density term of a segment's
    last step reads the first output of the following segment."""
    nt = 100
    vs, vp, rho, sx, sz, types, wav, geo, obs = _density_case(8, True, "moment", True, nt)
    out = []
    for ck in (0, 7):
        S = _solver(nt, len(geo["rec_x"]), len(sx), 8, True, want_gradient=True, pad=geo["pad"],
                    nz=geo["nz_dom"], nx=geo["nx_dom"], dx=geo["dx"], dz=geo["dz"], dt=geo["dt"],
                    fc=geo["fc"], density=True, ckpt_interval=ck)
        S.set_model(vs, vp, rho)
        S.set_receivers(geo["rec_x"], geo["rec_z"])
        S.set_shots(sx, sz, types, wav.astype(np.float32))
        S.forward(store=True)
        S.misfit(obs.astype(np.float32), 1, 1.0)
        g = S.gradient(exact=True, imaging=True)
        out.append([g["exact"][2], g["imaging"][2], g["exact"][0]])
        S.close()
    for a, b in zip(out[1], out[0]):
        assert _rel(a, b) < 1e-12, _rel(a, b)


def test_tile_rows_are_checked():
    """Tile heights of 8 and 16 rows are accepted; other values are refused
    (ValueError) and leave the tiling unchanged."""
    S = _solver(10, 4, 1, 8, True)
    assert S.tile_rows() == (16, 16)
    for bad in ((12, 16), (16, 0), (24, 8), (32, 32), (-8, 16)):
        with pytest.raises(ValueError):
            S.set_tile_rows(*bad)
    assert S.tile_rows() == (16, 16)
    S.set_tile_rows(8, 16)
    assert S.tile_rows() == (8, 16)
    S.close()


def test_autotuned_schedule_gives_the_same_gradient():
    """stfwi_autotune picks the tile shapes and the shots per block of each
    kernel by timing; the gradient computed with the tuned schedule equals
    the default schedule's (the grouping only changes the summation order of
    a launch's shots)."""
    vs, vp, rho = C.model()
    nt, fd, fs = 90, 8, True
    rx = np.arange(1, C.NX - 1, 3, dtype=np.int32)
    rz = np.ones_like(rx)
    sx = np.array([3, 7, 11, 15, 19, 23, 27])
    sz = np.array([2, 5, 3, 6, 2, 4, 3])
    types = ["force", "moment"] * 3 + ["force"]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    obs = np.random.default_rng(5).standard_normal((7, nt, len(rx))).astype(np.float32) * 1e-9
    res = []
    for tune in (False, True):
        S = _solver(nt, len(rx), 7, fd, fs, want_gradient=True)
        S.set_model(vs, vp, rho)
        S.set_receivers(rx, rz)
        S.set_shots(sx, sz, types, wav)
        if tune:
            pick = S.autotune(steps=10)
            assert set(pick) == {"fwd_vel", "fwd_str", "adj_a", "adj_b"}
            assert all(v in (1, 2, 3, 4, 5, 6, 8, 10, 13, 17, 25) for v in pick.values()), pick
            assert all(r in (8, 16) for r in S.tile_rows()), S.tile_rows()
        S.forward(store=True)
        mis = S.misfit(obs, 1, 1.0)
        g = S.gradient(exact=True, imaging=True)
        res.append((mis, g["exact"][0], g["imaging"][0]))
        S.close()
    for a, b in zip(res[1], res[0]):
        assert _rel(a, b) < 1e-6, _rel(a, b)
    # a descriptor shot_group keeps its shots per block; the tile shapes are tuned
    S = _solver(nt, len(rx), 7, fd, fs, want_gradient=True, shot_group=2)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    assert set(S.autotune(steps=6).values()) == {2}
    S.close()


def test_config1_single_shot_gradient_vs_oracle():
    """The single-shot configuration at full size: 152 x 500 at 20 m, fd 4,
    20-cell C-PML with a free surface, 2000 steps of 1.5 ms, one Ricker (5 Hz)
    vertical force at 40 m depth and x = 5000 m, 250 receivers at 20 m depth
    recording vx and vz.  Observed data: the FP64 oracle on the seeded
    layered-fault model; start: that model smoothed (sigma 10 cells).  The
    GPU's traces, FP64 misfit and exact g_Vs on the start model against the
    FP64 oracle's."""
    from stfwi_b200 import models as Mo
    cfg = Mo.CONFIG1
    nz, nx, nt, dt, fc, pad, fd = cfg["nz"], cfg["nx"], cfg["nt"], cfg["dt"], cfg["fc"], cfg["pad"], cfg["fd_order"]
    true = Mo.layered_fault_model(nz, nx, seed=1)
    init = Mo.smooth_initial(*true, sigma=10.0)
    sx, sz, types, rx, rz = Mo.acquisition(cfg)
    wav = Mo.ricker(np.arange(nt) * dt, fc, 1.5 / fc)
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=nx, nz_dom=nz, dx=cfg["dx"], dz=cfg["dz"], dt=dt, nt=nt, fc=fc,
               pad=pad, fd_order=fd, free_surface=True, d0_f32=True)
    obs = O.forward_batch(*true, sx, sz, types, src_wavelet=wav, **geo)[:, 1]
    ref_rec = O.forward_batch(*init, sx, sz, types, src_wavelet=wav, **geo)
    (g_ref, _, _), loss = O.compute_gradient("ad", Vs=init[0], Vp=init[1], rho=init[2], src_x=sx, src_z=sz,
                                             src_wavelet=wav, observed=obs, src_types=types, component=1,
                                             scale=1.0, invert="vs", **geo)
    S = _solver(nt, len(rx), 1, fd, True, want_gradient=True, pad=pad, nz=nz, nx=nx, dx=cfg["dx"],
                dz=cfg["dz"], dt=dt, fc=fc)
    S.set_model(*init)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav.astype(np.float32))
    S.forward(store=True)
    rec = S.records()
    mis = S.misfit(obs.astype(np.float32), 1, 1.0)
    g = S.gradient(exact=True)["exact"][0]
    S.close()
    e_rec = max(_rel(rec[0, c], ref_rec[0, c]) for c in range(2))
    amp = float(np.linalg.norm(rec[0, 1]) / np.linalg.norm(rec[0, 1] - obs[0]))
    e_mis, e_g = abs(mis.sum() / loss - 1), _rel(g, g_ref)
    print(f"config 1 (fd4, 2000 steps): vx/vz traces rel-L2 {e_rec:.2e}, amplification {amp:.1f}, "
          f"misfit rel {e_mis:.2e}, g_Vs rel-L2 {e_g:.2e}")
    assert e_rec < 1e-5, e_rec
    tol = 2e-5 * max(amp, 1.0)
    assert e_mis < tol and e_g < tol, (e_mis, e_g, tol)
