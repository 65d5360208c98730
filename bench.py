#!/usr/bin/env python
"""Benchmark of the batched elastic forward + adjoint gradient on B200.

Workload (the batched-shot configuration): seeded 152 x 500 layered-fault
model at 20 m, 20-cell C-PML on three sides + free surface (172 x 540 padded
cells), fd_order 8, 50 shots every 200 m alternating vertical force and
explosive moment, 250 receivers, 2000 steps of 1.5 ms, Vz misfit after a
6th-order 3 Hz Butterworth low-pass (the first band of the multiscale
schedule) and a 10 % cosine end taper.

One step = one gradient evaluation: forward of every shot (keeping the strain
history), FP64 misfit + adjoint sources, adjoint sweep with the exact FP64
gradient accumulation.  Unit: fwd+adj cell-updates = shots x padded cells x
steps.  With N ranks every rank runs its own 50 shots (weak scaling) and the
gradient and misfit are summed with one NCCL all-reduce.

``--impl reference`` times the oracle port (the reference's algorithm
restated in C, FP32, OpenMP over shots) on the host cores instead, in its
tuned build (native ISA, FP contraction, every forward step kept): the
faster of the two CPU ports that the GPU line's ``cpu_baseline`` reports.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s fwd+adj"
UNIT = "Gcell/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="stfwi", choices=["stfwi", "reference"])
    p.add_argument("--nt", type=int, default=2000)
    p.add_argument("--shots", type=int, default=50)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-every", type=int, default=20)
    p.add_argument("--no-autotune", action="store_true", help="keep the default shots per block")
    p.add_argument("--shot-group", type=int, default=0,
                   help="shots per block of every kernel (0: autotuned)")
    p.add_argument("--chains", type=int, default=0,
                   help="chains a pass may be split into (stfwi_set_chains; 0: the library's default)")
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-vs-plain time-to-Vs-error measurement (N = 1 only)")
    return p.parse_args()


def workload(nt, shots):
    from stfwi_b200 import models as Mo
    cfg = dict(Mo.CONFIG2)
    cfg["nt"] = nt
    cfg["n_shots"] = shots
    return cfg


def config_json(cfg, n):
    return {"workload": f"batched gradient, {cfg['n_shots']} shots x {cfg['nz']}x{cfg['nx']} "
                        f"(+{cfg['pad']} C-PML, free surface) fd{cfg['fd_order']}, {cfg['nt']} steps",
            "model": "seeded layered-fault 152x500 @ 20 m",
            "shots_per_gpu": cfg["n_shots"], "nt": cfg["nt"], "fd_order": cfg["fd_order"],
            "padded_cells": (cfg["nz"] + cfg["pad"]) * (cfg["nx"] + 2 * cfg["pad"]),
            "misfit": "vz, 3 Hz Butterworth(6) + 10% taper, FP64",
            "gradient": "exact discrete (FP32 stencils; FP64 sums over steps and shot groups)",
            "l2": "inputs > L2: the strain history (91 GB) streams through HBM every step; a 256 MB buffer is also written between steps",
            "parallelism": f"shots x{n} ranks" if n > 1 else "shot batch, 1 GPU"}


# ----------------------------------------------------------------------------- clocks

class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3] not in ("", "[N/A]"))}


# ----------------------------------------------------------------------------- CPU (oracle port)

def cpu_gradient_rate(cfg, nshot, nt, threads=None, precision=32, ckpt=25):
    """fwd+adj cell-updates/s of the oracle port on a bounded sample of the
    workload: `nshot` shots x `nt` steps, one shot per OpenMP thread.

    precision 32: the port as written (FP32, every multiply and add rounded
    separately, portable x86-64-v2 code), checkpointed every `ckpt` steps
    with one recompute of each segment.  precision 'fast': the same FP32
    restatement built on this host with -march=native and FP contraction;
    with ckpt >= nt it keeps every step of its forward pass (no segment
    recompute), which is what the GPU path does."""
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    from stfwi_b200 import models as Mo
    if precision == "fast":
        O.lib_fast()   # built for this host before the clock starts
    vs, vp, rho = Mo.layered_fault_model(cfg["nz"], cfg["nx"], seed=1)
    sx, sz, types, rx, rz = Mo.acquisition(dict(cfg, n_shots=max(nshot, 2)))
    sx, sz, types = sx[:nshot], sz[:nshot], types[:nshot]
    wav = Mo.ricker(np.arange(nt) * cfg["dt"], cfg["fc"], 1.5 / cfg["fc"])
    rng = np.random.default_rng(0)
    rec_adj = rng.standard_normal((nshot, 4, nt, len(rx))) * 1e-12
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=cfg["nx"], nz_dom=cfg["nz"], dx=cfg["dx"], dz=cfg["dz"],
               dt=cfg["dt"], nt=nt, fc=cfg["fc"], pad=cfg["pad"], fd_order=cfg["fd_order"],
               free_surface=cfg["free_surface"], precision=precision)
    t0 = time.perf_counter()
    O.gradient_batch(vs, vp, rho, sx, sz, types, src_wavelet=wav, rec_adj=rec_adj, mode="gmat",
                     ckpt=ckpt, **geo)
    dt = time.perf_counter() - t0
    cells = (cfg["nz"] + cfg["pad"]) * (cfg["nx"] + 2 * cfg["pad"])
    return nshot * cells * nt / dt / 1e9, dt


def cpu_sample(cfg, ncores, nt=500):
    """Shots and steps of the CPU sample: one shot per core, and a step count
    whose store-all history (16 FP32 fields per cell and step) stays within a
    third of the host's free memory."""
    nshot = max(1, min(ncores, cfg["n_shots"]))
    cells = (cfg["nz"] + cfg["pad"]) * (cfg["nx"] + 2 * cfg["pad"])
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:  # pragma: no cover
        avail = 16e9
    per_step = nshot * cells * 16 * 4
    return nshot, int(max(20, min(nt, avail / 3 / per_step)))


def cpu_baselines(cfg, ncores):
    """Both CPU ports on the same sample; returns (faster, both)."""
    nshot, nt = cpu_sample(cfg, ncores)
    exact_v, exact_dt = cpu_gradient_rate(cfg, nshot, nt, threads=ncores, precision=32, ckpt=25)
    fast_v, fast_dt = cpu_gradient_rate(cfg, nshot, nt, threads=ncores, precision="fast", ckpt=nt)
    both = {"port_exact_rounding": {"value": exact_v, "seconds": exact_dt,
                                    "build": "FP32 as written, x86-64-v2, -ffp-contract=off, checkpoints "
                                             "every 25 steps with one recompute per segment"},
            "port_tuned": {"value": fast_v, "seconds": fast_dt,
                           "build": "FP32, -march=native, -ffp-contract=fast, store-all (no segment "
                                    "recompute)"}}
    best = "port_tuned" if fast_v >= exact_v else "port_exact_rounding"
    return nshot, nt, best, both


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg = workload(args.nt, args.shots)
    ncores = os.cpu_count() or 1
    # 200 steps a sample (about 5 s on 16 cores), so that warm-up plus timed
    # samples stay within a few minutes
    nshot, nt = cpu_sample(cfg, ncores, nt=200)
    from oracle import oracle as O
    O.lib_fast()
    vals = []
    for k in range(args.warmup + args.steps):
        v, dt = cpu_gradient_rate(cfg, nshot, nt, threads=ncores, precision="fast", ckpt=nt)
        if k >= args.warmup:
            vals.append((v, dt))
    value = float(np.mean([v for v, _ in vals]))
    ms = float(np.mean([d for _, d in vals])) * 1e3
    sample = (f"{nshot} shots x {nt} steps of the workload per step (oracle port, tuned build: FP32, "
              f"-march=native, FP contraction, one shot per thread, forward kept for every step, "
              f"adjoint with the exact gradient)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_json(cfg, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU

def kernel_bytes(cfg, nshot):
    """Algorithmic bytes per launch of each kernel (FP32 fields): every input
    read once and every output written once; materials once per launch."""
    nz, nx = cfg["nz"] + cfg["pad"], cfg["nx"] + 2 * cfg["pad"]
    cells = nz * nx
    phys = cfg["nz"] * cfg["nx"]
    mat = 4 * 4 * cells
    return {
        "fwd_vel": nshot * cells * (5 + 2) * 4 + mat,            # r ex ez es U V, w U V
        "fwd_str": nshot * (cells * (5 + 3) * 4 + phys * 3 * 4),  # r U V ex ez es, w ex ez es, w history
        "adj_a": nshot * cells * (5 + 2) * 4,                    # r exa eza esa Ua Va, w Ua Va
        "adj_b": nshot * (cells * (5 + 3) * 4 + phys * 3 * 4) + mat,  # r Ua Va exa eza esa, w 3, r history
    }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    torch.cuda.init()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from scipy.signal import butter
    from stfwi_b200 import Solver
    from stfwi_b200 import models as Mo

    cfg = workload(args.nt, args.shots)
    ns, nt = cfg["n_shots"], cfg["nt"]
    vs_t, vp_t, rho_t = Mo.layered_fault_model(cfg["nz"], cfg["nx"], seed=1)
    vs0, vp0, rho0 = Mo.smooth_initial(vs_t, vp_t, rho_t, 10.0)
    sx, sz, types, rx, rz = Mo.acquisition(cfg)
    sx = (sx + 3 * rank) % cfg["nx"]  # each rank its own shots
    wav = Mo.ricker(np.arange(nt) * cfg["dt"], cfg["fc"], 1.5 / cfg["fc"]).astype(np.float32)
    S = Solver(cfg["nz"], cfg["nx"], cfg["dx"], cfg["dz"], cfg["dt"], nt, cfg["fc"], cfg["pad"],
               len(rx), ns, fd_order=cfg["fd_order"], free_surface=cfg["free_surface"],
               want_gradient=True, shot_group=args.shot_group)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    comp = 1
    S.set_model(vs_t, vp_t, rho_t)
    S.forward()
    obs = torch.empty((ns, 4, nt, len(rx)), dtype=torch.float32, device="cuda")
    S.records(out=obs)
    obs = obs[:, comp].contiguous()
    scale = float(1.0 / (obs.double().pow(2).mean().item() + 1e-45))
    sos = butter(6, 3.0, fs=1.0 / cfg["dt"], output="sos")
    n_taper = int(0.1 * nt)
    S.set_model(vs0, vp0, rho0)
    # tile shapes and shots per block of each kernel, timed on this workload
    # (untimed set-up)
    schedule = None if args.no_autotune else S.autotune(steps=20)
    tile_rows = dict(zip(("fwd_vel,fwd_str,adj_a", "adj_b"), S.tile_rows()))
    if args.chains:
        S.set_chains(args.chains)
    mis_d = torch.zeros(ns, dtype=torch.float64, device="cuda")
    g_d = torch.zeros((1, 3, cfg["nz"], cfg["nx"]), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        S.forward(store=True)
        S.misfit(obs, comp, scale, sos, n_taper, nshot_norm=ns * world, out=mis_d, sync=False)
        S.gradient(exact=True, out=g_d, sync=False)
        if dist is not None:
            dist.all_reduce(g_d)
            dist.all_reduce(mis_d)

    for _ in range(max(args.warmup, 3)):
        step()
    S.check()

    def flush_l2():
        # the history (56 GB) already streams through HBM; flush anyway
        buf.zero_()

    buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot_ms = 0.0
    # STFWI_PROFILER_RANGE=1 marks the timed region for a profiler started
    # with its collection off (ncu --profile-from-start off)
    mark = os.environ.get("STFWI_PROFILER_RANGE") == "1"
    if mark:
        torch.cuda.cudart().cudaProfilerStart()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush_l2()
            ev0.record(stream)
            step()
            ev1.record(stream)
            ev1.synchronize()
            tot_ms += ev0.elapsed_time(ev1)
    if mark:
        torch.cuda.cudart().cudaProfilerStop()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    S.check()
    # per-kernel launch times in a separate pass: an event pair around each
    # launch of every profile_every-th step (the pairs sit inside the CUDA
    # graphs and add a few per cent, so the timed loop above runs without them)
    S.profile(args.profile_every)
    step()  # re-captures the graphs with the event pairs
    S.kernel_times()
    for _ in range(max(2, min(args.steps, 5))):
        flush_l2()
        step()
    torch.cuda.synchronize()
    S.check()
    ktimes = S.kernel_times()
    S.profile(0)
    clocks = clk.summary()
    t = torch.tensor([tot_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps
    cells = (cfg["nz"] + cfg["pad"]) * (cfg["nx"] + 2 * cfg["pad"])
    units = world * ns * cells * nt
    value = units / (ms_step * 1e-3) / 1e9

    # end to end through the public API with host buffers: model, observed
    # data and the result cross PCIe inside the timed region
    obs_h = obs.cpu().pin_memory()
    models_h = [np.ascontiguousarray(a) for a in (vs0, vp0, rho0)]
    g_h = np.zeros((1, 3, cfg["nz"], cfg["nx"]))
    mis_h = np.zeros(ns)

    def step_e2e():
        S.set_model(*models_h)
        S.forward(store=True)
        S.misfit(obs_h, comp, scale, sos, n_taper, nshot_norm=ns * world, out=mis_h, sync=False)
        S.gradient(exact=True, out=g_h, sync=True)
        return float(mis_h.sum())

    step_e2e()
    torch.cuda.synchronize()
    e_ms = 0.0
    for _ in range(args.steps):
        ev0.record(stream)
        step_e2e()
        ev1.record(stream)
        ev1.synchronize()
        e_ms += ev0.elapsed_time(ev1)
    te = torch.tensor([e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_val = units / (float(te.item()) / args.steps * 1e-3) / 1e9
    h2d = 3 * cfg["nz"] * cfg["nx"] * 4 + obs_h.numel() * 4
    d2h = g_h.nbytes + mis_h.nbytes

    # roofline of the dominant kernel from the sampled launch times of the
    # separate pass
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kb = kernel_bytes(cfg, ns)
    dom = max(ktimes, key=lambda k: ktimes[k][0])
    tot, cnt = ktimes[dom]
    avg_ms = tot / cnt if cnt else float("nan")
    achieved = kb[dom] / (avg_ms * 1e-3) / 1e9 if cnt and avg_ms > 0 else float("nan")
    # DRAM bytes of one launch of that kernel, from the committed ncu capture of
    # this workload (per-launch traffic does not depend on the step count)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic_50shots_fd8.json")) as fh:
            tr = json.load(fh)
        if ns == 50 and cfg["fd_order"] == 8:
            traffic = tr["kernels"][dom]["traffic_bytes"]
    except (OSError, KeyError, ValueError):
        pass
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": kb[dom],
            "kernels_ms_per_launch": {k: (v[0] / max(v[1], 1)) for k, v in ktimes.items()},
            "kernel_times": "one-chain pass sampled after the timed loop"}
    # the whole step against the same peak: the algorithmic bytes of all four
    # kernels per step, over the timed ms per step (the timed loop runs the
    # pass as two concurrent chains when the shots are grouped alike)
    step_bytes = nt * sum(kb.values())
    roof["step_achieved"] = step_bytes / (ms_step * 1e-3) / 1e9
    roof["step_frac"] = roof["step_achieved"] / peak
    # for context: the nominal HBM3e bandwidth of an HGX B200 (7.7 TB/s)
    roof["frac_of_nominal_7700"] = achieved / 7700.0
    roof["step_frac_of_nominal_7700"] = roof["step_achieved"] / 7700.0
    # stencil launches: 2 per forward step and 2 per adjoint step, once per
    # chain when the pass is split (every kernel with the same shots per
    # block: at most one chain per shot group); plus set-up, misfit, finalize
    spg = set(schedule.values()) if schedule else set()
    chains = min(args.chains or 2, -(-ns // spg.pop())) if len(spg) == 1 else 1
    launches = 4 * nt * chains + 6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ncores = os.cpu_count() or 1
        nsh, nts, best, both = cpu_baselines(cfg, ncores)
        cpu = {"value": both[best]["value"], "unit": UNIT, "cores": ncores, "kind": "port",
               "sample": f"{nsh} shots x {nts} steps of the workload, oracle port ({best}: "
                         f"{both[best]['build']}; {both[best]['seconds']:.1f} s)",
               "ports": both}
    S.close()
    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = learned_vs_plain()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config_json(cfg, world), shots_per_block=schedule, tile_rows=tile_rows,
                              tile_cols=64), "roofline": roof,
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": launches, "clocks": clocks,
                "misfit": float(mis_d.sum().item()),
                "learned_vs_plain": learned}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def learned_vs_plain(seeds=(5000, 5001, 5002, 5003)):
    """The metric's second half, after the timed region: wall time for the
    learned preconditioner (shipped U-Net, tcgen05 kernels) to reach the Vs
    relative-RMS error that plain illumination-preconditioned L-BFGS reaches
    in 20 iterations, over the plain method's time, on held-out seeded
    models (10 shots, 152 x 500, 3 Hz band; four models in lockstep)."""
    import torch
    try:
        from stfwi_b200.learned import UNet, padded_shape
        from stfwi_b200.learned import experiment as E
        from stfwi_b200.learned.unet import load_weights
        torch.cuda.empty_cache()
        h, w = padded_shape(152, 500)
        net = UNet(h, w)
        weights = os.path.join(ROOT, "stfwi_b200", "learned", "weights", "unet_152x500_3hz.npz")
        net.load_state_dict({"params": load_weights(weights), "h": h, "w": w})
        recs = E.evaluate(net, list(seeds), K=4, n_plain=20, log=lambda m: None)
        s = E.summarize(recs)
        return {"metric": "time to the plain method's Vs relative-RMS error, learned / plain",
                "median_time_ratio": s["median_time_ratio"], "mean_time_ratio": s["mean_time_ratio"],
                "models": s["models"], "reached_target": s["reached_target"],
                "learned_step_accepted": s["learned_step_accepted"],
                "plain_time_s": [r["plain_time_s"] for r in recs],
                "learned_time_s": [r["learned_time_s"] for r in recs],
                "target_vs_rel_rms": [r["target"] for r in recs],
                "config": {"workload": "held-out layered-fault models (seeds %d-%d), 152x500, 10 shots, "
                                       "3 Hz band, known Vp and density; plain = 20 L-BFGS iterations"
                                       % (seeds[0], seeds[-1])}}
    except Exception as e:  # the Gcell/s line stands on its own
        return {"error": f"{type(e).__name__}: {e}"}


if __name__ == "__main__":
    main()
