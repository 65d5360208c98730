"""Extract the reference's own known answers into a committed test fixture.

Reads the result files that the reference ships (written by its scripts
compute_gradient_handcoded.py, compute_gradient.py and
compute_first_gradient.py) and stores, as float32 unless noted:

* the six Marmousi-II arrays those runs used (shared by all three files);
* ``gc_*``  Results_gradient/gradient_compare.npz: 5 shots, nt=400, fd8, free
  surface, force, exx, no filter -- FP64 loss_AD/loss_HC/auto_scale (float64),
  the exact gradient g_Vs_AD and the imaging gradient g_Vs_HC;
* ``gd_*``  Results_gradient/gradient_data.npz: same 5 shots, nt=2890, 3 Hz
  Butterworth + 10 % end taper, FP32 JAX run -- loss, auto_scale, raw g_vs;
* ``fg_*``  Results_first_gradient/first_gradient.npz: 34 shots, nt=2890,
  3 Hz + 10 % taper, sigma=1 smoothing -- FP64 losses, g_Vs_AD (with an
  illumination H_inv that the file does not store), g_Vs_HC and the
  eprecond3 multiplier it was scaled by.

Run from the repository root with the reference mounted:
    python tests/golden/make_reference_known_answers.py /path/to/reference
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_reference_known_answers.py <path to the reference project>")
ref = sys.argv[1]
gc = np.load(os.path.join(ref, "Results_gradient/gradient_compare.npz"))
gd = np.load(os.path.join(ref, "Results_gradient/gradient_data.npz"))
fg = np.load(os.path.join(ref, "Results_first_gradient/first_gradient.npz"), allow_pickle=True)

out = {}
for k in ("Vs_init", "Vp_init", "rho_init", "Vs_true", "Vp_true", "rho_true"):
    assert np.array_equal(gc[k], gd[k]) and np.array_equal(gc[k], fg[k])
    out[k] = gc[k].astype(np.float32)
for k in ("src_x", "src_z", "rec_x", "rec_z"):
    out["gc_" + k] = gc[k].astype(np.int32)
    out["fg_" + k] = fg[k].astype(np.int32)
for k in ("dx", "dz", "dt", "f_c", "auto_scale", "loss_AD", "loss_HC"):
    out["gc_" + k] = np.float64(gc[k])
for k in ("nt", "pad", "fd_order", "component", "free_surface"):
    out["gc_" + k] = np.int64(gc[k])
out["gc_g_Vs_AD"] = gc["g_Vs_AD"].astype(np.float32)
out["gc_g_Vs_HC"] = gc["g_Vs_HC"].astype(np.float32)
for k in ("dt", "f_c", "cutoff", "loss", "auto_scale"):
    out["gd_" + k] = np.float64(gd[k])
out["gd_nt"] = np.int64(gd["nt"])
out["gd_g_vs"] = gd["g_vs"].astype(np.float32)
for k in ("dt", "f_c", "cutoff", "auto_scale", "loss_AD", "loss_HC", "grad_smooth_sigma",
          "illumination_eps"):
    out["fg_" + k] = np.float64(fg[k])
out["fg_nt"] = np.int64(fg["nt"])
out["fg_g_Vs_AD"] = fg["g_Vs_AD"].astype(np.float32)
out["fg_g_Vs_HC"] = fg["g_Vs_HC"].astype(np.float32)
out["fg_illumination_eprecond3"] = fg["illumination_eprecond3"].astype(np.float32)
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_known_answers.npz")
np.savez_compressed(dst, **out)
print(dst, os.path.getsize(dst))
