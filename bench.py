#!/usr/bin/env python
"""Throughput of the SH FWI gradient (forward + residual + adjoint with
correlation + energy preconditioning + conversion) on B200.

Workloads (--config; seeded synthetic models, no dataset exists for this path):
  c2 (default)  viscoelastic forward + adjoint gradient: NX=2000, NY=800,
                DH=0.25 m, FDORDER=8, L=3, NT=6000, one 40 Hz shot, 200
                receivers.  One step = one gradient (2 x NX x NY x NT updates).
  c1            elastic forward modelling: NX=500, NY=200, FDORDER=4, NT=2000,
                one 30 Hz shot, 96 receivers.  One step = NX x NY x NT updates.
  c4            uneven batch of 32 models (NX 256-2048, NY 128-512, FDORDER
                4/6/8, elastic / L=2, 8-32 shots each), one velocity and one
                stress launch per register class (body key) and step, tile
                shape picked by the autotuner;
                forward modelling; NT per model = 1.5 x diagonal traveltime
                (--nt-scale shortens all NTs alike).  Per-model throughput is
                reported beside the aggregate.
  c5            learned-preconditioner FWI: U-Net trained on solver-generated
                (gradient, energies, vs) -> pseudo-Hessian pairs, then 20 L-BFGS
                iterations of plain EPRECOND=1 FWI and of learned-preconditioned
                FWI on NX=1200, NY=400, 32 shots, L=3; value = GPU-seconds the
                learned method needs to reach the plain method's final misfit
                (within 1%) / the plain method's GPU-seconds (lower is better).
  c3            batched gradient of 64 shots in one launch per half-step:
                NX=1000, NY=300, FDORDER=8, L=2, NT=4000, 192 receivers, forward
                wavefield checkpointed every ceil(sqrt(NT)) steps with recompute
                (full storage would need 0.92 TB).  One step = 2 x NX x NY x NT x 64 updates; the
                recompute pass is extra work that is not counted.

  value  device-resident inputs (model and observed data already in HBM),
         through dsh_gradient_device; CUDA events on the launching stream
  e2e    the same metric through the public host API (dsh_set_model +
         dsh_gradient with host buffers): model and observed data copied in,
         gradients copied out, every step
Multi-GPU (torchrun): weak scaling, one distinct shot per rank, gradients
summed with one NCCL all-reduce per step (the shot-sum exchange).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dsh|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "denise-sh_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Gpt-updates/s"
UNIT = "Gpt/s"
FALLBACK_HBM_GBS = 6650.0


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dsh", choices=["dsh", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--train-models", type=int, default=200, help="c5 only: training models")
    ap.add_argument("--train-shots", type=int, default=8, help="c5 only: shots per training model")
    ap.add_argument("--epochs", type=int, default=12, help="c5 only: training epochs")
    ap.add_argument("--fwi-iters", type=int, default=20, help="c5 only: L-BFGS iterations")
    ap.add_argument("--net-cache", default=None, help="c5 only: .npz of trained U-Net weights (load if present, "
                                                      "else train and save)")
    ap.add_argument("--methods", default="learned,hessian,energy_src",
                    help="c5 only: preconditioners compared with plain (the first one gives `value`)")
    ap.add_argument("--targets", default="log_h_over_ws",
                    help="c5 only: comma list of network output modes (dsh.nn.TARGETS); the learned methods run "
                         "once per network, the first target's runs unsuffixed")
    ap.add_argument("--problem-seeds", default="6,7,8,9",
                    help="c5 only: comma list of FWI problem seeds (config5(seed)); value = median ratio")
    ap.add_argument("--nt-scale", type=float, default=1.0, help="c4 only: factor on every model's NT")
    ap.add_argument("--c4-models", type=int, default=32,
                    help="c4 only: the first K models of the batch (a small case for profiling)")
    ap.add_argument("--nt", type=int, default=None, help="time steps (default: the workload's NT)")
    ap.add_argument("--nx", type=int, default=2000, help="c2 only")
    ap.add_argument("--ny", type=int, default=800, help="c2 only")
    ap.add_argument("--shots", type=int, default=64, help="c3 only: shots per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--c3-steps", type=int, default=2,
                    help="c2 only: timed gradients of the 64-shot batched-gradient sub-measurement (0 = skip)")
    ap.add_argument("--c1-steps", type=int, default=5,
                    help="c2 only: timed forward passes of the 500x200 elastic sub-measurement (0 = skip)")
    ap.add_argument("--c5-small", type=int, default=1,
                    help="c2 only: 1 = add the reduced learned-vs-plain FWI sub-measurement (0 = skip)")
    ap.add_argument("--step-variant", type=int, default=-1,
                    help="pin the step-kernel variant (index into dsh.Engine.VARIANTS) instead of autotuning")
    ap.add_argument("--no-autotune", action="store_true",
                    help="c1-c3: keep the default kernel pair instead of timing the step-kernel variants "
                         "(for runs under a profiler)")
    ap.add_argument("--cpu-steps", type=int, default=24, help="time steps per pass in the CPU sample")
    ap.add_argument("--profile-steps", type=int, default=20)
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def kernels_hash():
    """sha256 of the step kernels' source (csrc/dsh_kernels.cuh): ties a
    recorded ncu traffic figure to the build it was measured on."""
    import hashlib

    with open(os.path.join(ROOT, "denise-sh_b200", "csrc", "dsh_kernels.cuh"), "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def bytes_per_point(l, nx, ny, fw, free_surf):
    """Algorithmic bytes per grid-point time step (each array touched once):
    state vy, sxy, syz and the 2L memory variables read and written; model
    parameters read once (elastic: 1/rho, uip, ujp; viscoelastic: 1/rho and
    the four factors muip, mujp, tausipjp, taus that every viscoelastic
    coefficient is a product of); forward pass: stored acceleration and
    strains written (12 B) and Ws R/W; adjoint: stored wavefield read (12 B)
    and g_u, g_rho, Wr R/W; plus CPML memory R/W on the strip points."""
    state = 8 * (3 + 2 * l)
    params = 12 if l == 0 else 20
    strips = 2 * fw * ny + (1 if free_surf else 2) * fw * nx
    cpml = 16.0 * strips / (nx * ny)
    fwd = state + params + 12 + 8 + cpml
    adj = state + params + 12 + 24 + cpml
    return fwd, adj


def kernel_bytes(l, store=True):
    """Per-point bytes a single launch must move (forward pass, with or
    without storage of acceleration, strains and the energy Ws)."""
    v = 8 + 8 + 4 + (4 if store else 0)    # vy R/W, sxy+syz R, 1/rho R, stored acceleration W
    params = 8 if l == 0 else 16           # uip, ujp | muip, mujp, tausipjp, taus
    s = 16 + 16 * l + 4 + params + (16 if store else 0)   # sxy/syz R/W, r/q R/W, vy R, params, strains W, Ws R/W
    return v, s


def kernel_bytes_adjoint(l):
    """Per-point bytes of the adjoint pass's velocity and stress launches:
    velocity vy R/W, sxy+syz R, 1/rho R, stored acceleration R, g_rho R/W;
    stress sxy/syz R/W, r/q R/W, vy R, parameters, stored strains R, g_u R/W,
    Wr R/W."""
    v = 8 + 8 + 4 + 4 + 8
    params = 8 if l == 0 else 16
    s = 16 + 16 * l + 4 + params + 8 + 8 + 8
    return v, s


def fused_bytes(l, store=True):
    """Per-point bytes of one fused step (each array once): vy, sxy, syz and
    the 2L memory variables read and written, model parameters read (1/rho,
    uip, ujp | 1/rho, muip, mujp, tausipjp, taus), and with storage the stored
    acceleration and strains written and Ws read and written."""
    return 8 * (3 + 2 * l) + (12 if l == 0 else 20) + (20 if store else 0)


def workload(name, nt=None, nx=2000, ny=800, shots=64):
    """(cfg, kind, label, fdorder) of a named workload."""
    from dsh import configs

    if name == "c4":   # the CPU sample of the uneven batch: its largest model, one shot
        ms = configs.config4()
        m = max(ms, key=lambda m: m["params"]["nx"] * m["params"]["ny"])
        m["params"].pop("max_shots")
        if nt:
            m["params"]["nt"] = nt
        return m, "forward", "uneven-batch-32-models", m["params"]["fdorder"]
    if name == "c1":
        cfg = configs.config1(**({"nt": nt} if nt else {}))
        return cfg, "forward", f"elastic-forward-500x200-fd4", 4
    if name == "c3":
        cfg = configs.config3(nshots=shots, **({"nt": nt} if nt else {}))
        return cfg, "gradient", f"batched-gradient-1000x300-fd8-L2-{shots}shots", 8
    cfg = configs.config2(nx=nx, ny=ny, **({"nt": nt} if nt else {}))
    return cfg, "gradient", f"visc-gradient-{nx}x{ny}-fd8-L3", 8


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="dsh_clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own functions (oracle/_ref, -O3 timing build)
# ---------------------------------------------------------------------------

def _cpu_sample(payload):
    """One bounded sample of the gradient on the CPU: `steps` forward steps
    with storage, residual, `steps` adjoint steps, eprecond.  Returns seconds."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cfg, steps, kind, gradient = payload
    devnull = os.open(os.devnull, os.O_WRONLY)      # the reference logs to stdout/stderr
    os.dup2(devnull, 1)
    os.dup2(devnull, 2)
    p = dict(cfg["params"])
    m = O.Model(nx=p["nx"], ny=p["ny"], nt=steps, dh=p["dh"], dt=p["dt"], vs=cfg["vs"], rho=cfg["rho"],
                qs=cfg["qs"], fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=p["l"],
                fl=p.get("fl", ()), fpml=p["fpml"], damping=p["damping"])
    o = O.Oracle(m, kind)
    sh = cfg["shots"][0]
    t0 = time.perf_counter()
    seis = o.forward(sh.srcpos, sh.recpos, store=gradient)
    if gradient:
        o.residual(seis * np.float32(0.9))
        o.adjoint()
        o.eprecond_scale()
    dt = time.perf_counter() - t0
    o.close()
    return dt


def cpu_workload(a):
    cfg, kind, label, fdo = workload(a.config, 16, a.nx, a.ny, 1)
    cfg = dict(cfg)
    cfg.pop("true", None)
    cfg["shots"] = cfg["shots"][:1]
    return cfg, kind == "gradient"


def run_cpu(nprocs, steps, a, repeats=1):
    """Times `repeats` rounds of nprocs concurrent samples; returns per-round seconds (max over processes)."""
    import multiprocessing as mp

    import oracle as O

    kind = "ref_fast" if O.available("ref_fast") else "port"
    cfg, gradient = cpu_workload(a)
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(nprocs) as pool:
        for _ in range(repeats):
            t = pool.map(_cpu_sample, [(cfg, steps, kind, gradient)] * nprocs)
            times.append(max(t))
    return times, ("reference" if kind == "ref_fast" else "port")


def reference_arm(a, rank, world):
    if rank != 0:
        return
    ncpu = os.cpu_count() or 1
    nprocs = max(1, min(ncpu, 32))
    cfg, wkind, label, fdo = workload(a.config, a.nt, a.nx, a.ny, a.shots)
    steps = 12 if wkind == "gradient" else 200
    p = cfg["params"]
    nx, ny, L = p["nx"], p["ny"], p["l"]
    passes = 2 if wkind == "gradient" else 1
    times, kind = run_cpu(nprocs, steps, a, repeats=a.warmup + a.steps)
    timed = times[a.warmup:]
    pts = passes * nx * ny * steps * nprocs
    val = pts * len(timed) / sum(timed) / 1e9
    what = f"{steps} forward (with storage) + {steps} adjoint steps" if passes == 2 else f"{steps} forward steps"
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * sum(timed) / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": label, "nx": nx, "ny": ny, "fdorder": fdo, "l": L,
                       "nt_sample": steps, "shots": nprocs},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nprocs, "kind": kind,
                             "sample": f"{what} of the {nx}x{ny} FD{fdo} L={L} {wkind} per process, "
                                       f"{nprocs} independent single-rank processes (one shot each)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------

def c1_sub(a, local):
    """Plain elastic forward modelling as its configuration states it:
    NX=500, NY=200, FDORDER 4, NT=2000, one shot, 96 receivers, through the
    device API with the step-kernel variant the autotuner picks for this grid
    (on a B200 the temporally blocked launches, four steps per launch).  CUDA
    events on the launching stream, three untimed passes first.  The state
    (1.2 MB) stays in L2 and shared memory, so the effective bandwidth below
    (the kernel pair's algorithmic 36 B per point and step over the measured
    time) is not bounded by HBM."""
    import torch

    import dsh
    from dsh import configs

    cfg = configs.config1()
    p, shots = cfg["params"], cfg["shots"]
    nx, ny, nt = p["nx"], p["ny"], p["nt"]
    eng = dsh.Engine(dsh.make_params(**p), device=local)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_model(cfg["vs"], cfg["rho"], None)
    variant, variant_ms = eng.autotune(shots, nsteps=64)
    seis = torch.empty(sum(sh.ntr for sh in shots) * nt, device="cuda", dtype=torch.float32)
    for _ in range(3):
        eng.forward_device(shots, seis.data_ptr())
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    e0.record(stream)
    for _ in range(a.c1_steps):
        eng.forward_device(shots, seis.data_ptr())
        launches += eng.stats()["kernel_launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    eng.close()
    ms = e0.elapsed_time(e1) / a.c1_steps
    gpt = nx * ny * nt / (ms / 1e3) / 1e9
    return {"workload": f"elastic-forward-{nx}x{ny}-fd4-nt{nt}", "steps": a.c1_steps, "warmup": 3,
            "gpt_per_s": gpt, "ms_per_forward": ms, "us_per_time_step": 1e3 * ms / nt,
            "step_variant": variant, "autotune_ms_per_step": variant_ms, "gpu_launches": launches,
            "effective_gbs": 36.0 * nx * ny * nt / (ms / 1e3) / 1e9,
            "l2": "state 1.2 MB: resident on chip; bytes counted algorithmically (kernel pair's 36 B/pt)",
            "clocks": clk}


def c5_small_sub(a, local):
    """The learned preconditioner against plain EPRECOND=1 L-BFGS on a reduced
    problem that fits the default run (the c5 configuration itself, 1200x400
    with 32 shots and a U-Net trained on 200 models, takes ~13 minutes and
    runs as --config c5): 160x80 elastic FDORDER 4, 8 shots, NT 600, a U-Net
    trained on solver-generated pairs of 16 models (seeds 100-115), FWI on a
    problem it has not seen (seed 41), up to 8 iterations each.  Reports the
    GPU-seconds each method needs to reach plain's final misfit (within 1 %)
    over plain's GPU-seconds, for the network and for its prior without the
    network (energy_src)."""
    import torch

    from dsh import configs, fwi
    from dsh import nn as dnn

    cfg = configs.config5(seed=41, nx=160, ny=80, nt=600, nshots=8, ntr=60)
    cfg["params"].update(fdorder=4, l=0, fl=())
    cfg["qs"] = None
    p = cfg["params"]
    t0 = time.time()
    models = list(configs.training_models(count=16, first_seed=100, nx=p["nx"], ny=p["ny"]))
    xs, ts = fwi.training_pairs(torch, models, p, cfg["shots"][::2])
    net = dnn.UNet(torch, seed=3)
    net.target = "log_h_over_ws"
    fwi.train(net, torch, xs, dnn.residual_targets(torch, xs, ts), p["ny"], p["nx"], epochs=25, batch=2, lr=2e-3)
    t_train = time.time() - t0
    clocks = Clocks(local)
    clocks.start()
    prob = fwi.Problem(cfg, test_shots=3)
    try:
        plain, _ = fwi.run(prob, 8, method="plain", eps_scale=0.02)
        target = plain[-1]["misfit"] * 1.01
        t_plain = plain[-1]["gpu_s"]
        learned, _ = fwi.run(prob, 8, method="learned", net=net, torch=torch, eps_scale=0.02, target_misfit=target)
        prior, _ = fwi.run(prob, 8, method="energy_src", eps_scale=0.02, target_misfit=target)
    finally:
        prob.close()
    clk = clocks.stop()
    ratio = lambda run: (None if fwi.time_to_reach(run, target) is None else fwi.time_to_reach(run, target) / t_plain)
    return {"workload": "learned-vs-plain-fwi-160x80-fd4-8shots-nt600 (reduced; the configuration is --config c5)",
            "metric": "GPU-seconds to plain's final misfit (within 1 %) / plain's GPU-seconds (lower is better)",
            "learned": ratio(learned), "energy_src_prior": ratio(prior),
            "plain": {"iterations": len(plain) - 1, "final_misfit": plain[-1]["misfit"], "gpu_s": t_plain},
            "training": {"models": 16, "epochs": 25, "wall_s": t_train}, "clocks": clk}


def c3_sub(a, local):
    """The batched multi-shot FWI gradient as the configuration states it:
    NX=1000, NY=300, FDORDER 8, L=2, NT=4000, 64 shots advanced in one launch
    per half-step, forward wavefield checkpointed every ceil(sqrt(NT)) = 64
    steps and recomputed segment by segment for the adjoint.  Inputs resident
    in HBM (observed data synthesised on the true model first); CUDA events on
    the launching stream; one untimed gradient first.  Reports FWI gradients/s
    (shots per second), Gpt/s counted over the two passes a gradient needs
    and over the three passes it executes (the recompute included), and the
    stress kernel's roofline."""
    import torch

    import dsh
    from dsh import configs

    nt = 4000
    every = math.ceil(math.sqrt(nt))
    cfg = configs.config3(nt=nt)
    p, shots = cfg["params"], cfg["shots"]
    nsh, nx, ny = len(shots), p["nx"], p["ny"]
    n = nx * ny
    eng = dsh.Engine(dsh.make_params(**p, max_shots=nsh, ckpt_every=every), device=local)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_model(cfg["true"], cfg["rho"], cfg["qs"])
    seis = torch.empty(sum(sh.ntr for sh in shots) * nt, device="cuda", dtype=torch.float32)
    eng.forward_device(shots, seis.data_ptr())
    eng.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
    gv = torch.empty(n, device="cuda", dtype=torch.float32)
    gr = torch.empty(n, device="cuda", dtype=torch.float32)
    eng.gradient_device(shots, seis.data_ptr(), gv.data_ptr(), gr.data_ptr())
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, ms_f, ms_a = 0, 0.0, 0.0
    e0.record(stream)
    for _ in range(a.c3_steps):
        eng.gradient_device(shots, seis.data_ptr(), gv.data_ptr(), gr.data_ptr())
        st = eng.stats()
        launches += st["kernel_launches"]
        ms_f += st["ms_forward"]
        ms_a += st["ms_adjoint"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = eng.stats()
    ms = e0.elapsed_time(e1) / a.c3_steps
    prof = eng.profile_step("forward_store", a.profile_steps)
    eng.close()
    # the same 64 shots advanced 8 at a time: 8 shots' stored forward wavefields
    # (115 GB) fit the device, so the engine keeps full storage and skips the
    # recomputed forward pass (two passes per gradient instead of three)
    eng8 = dsh.Engine(dsh.make_params(**p, max_shots=8), device=local)
    eng8.set_stream(stream.cuda_stream)
    eng8.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
    eng8.gradient_device(shots, seis.data_ptr(), gv.data_ptr(), gr.data_ptr())
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(a.c3_steps):
        eng8.gradient_device(shots, seis.data_ptr(), gv.data_ptr(), gr.data_ptr())
    f1.record(stream)
    torch.cuda.synchronize()
    ms8 = f0.elapsed_time(f1) / a.c3_steps
    st8 = eng8.stats()
    eng8.close()
    hbm, peak_kind = peaks()
    kv, ks = kernel_bytes(2, store=True)
    s_gbs = ks * n * nsh / (prof["s_step"] / 1e3) / 1e9
    v_gbs = kv * n * nsh / (prof["v_step"] / 1e3) / 1e9
    return {
        "workload": f"batched-gradient-{nx}x{ny}-fd8-L2-{nsh}shots-nt{nt}", "steps": a.c3_steps, "warmup": 1,
        "gradients_per_s": nsh / (ms / 1e3), "ms_per_gradient": ms,
        "gpt_per_s": 2.0 * n * nt * nsh / (ms / 1e3) / 1e9,
        "gpt_per_s_executed": 3.0 * n * nt * nsh / (ms / 1e3) / 1e9,
        "counting": "gpt_per_s: forward + adjoint pass (2 x NX x NY x NT x shots per gradient); "
                    "gpt_per_s_executed adds the recomputed forward pass of checkpointing",
        "checkpoint_interval": st["checkpoint_interval"], "storage_gb": st["storage_bytes"] / 1e9,
        "ms_forward_pass": ms_f / a.c3_steps, "ms_adjoint_and_recompute": ms_a / a.c3_steps,
        "gpu_launches": launches,
        "l2": f"inputs larger than L2 (state of {nsh} shots {(3 + 2 * 2) * n * 4 * nsh / 1e6:.0f} MB)",
        "roofline": {"bound": "hbm", "achieved": s_gbs, "peak": hbm, "unit": "GB/s", "frac": s_gbs / hbm,
                     "kernel": "s_step<8,2> (forward pass with storage, 64 slots)", "bytes_per_point": ks,
                     "ms_per_launch": prof["s_step"], "peak_source": peak_kind},
        "kernels_ms": prof, "v_step_gbs": v_gbs,
        "clocks": clk,
        "eight_at_a_time": {"shots_per_launch": 8, "checkpoint_interval": st8["checkpoint_interval"],
                            "storage_gb": st8["storage_bytes"] / 1e9, "ms_per_gradient": ms8,
                            "gradients_per_s": nsh / (ms8 / 1e3),
                            "gpt_per_s": 2.0 * n * nt * nsh / (ms8 / 1e3) / 1e9,
                            "note": "not the configuration's method (all 64 shots in one launch with "
                                    "checkpoints): the same gradient with 8 shots per launch and full "
                                    "storage, which fits at 8 shots and removes the recomputed pass"},
    }


def main():
    a = args_parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return

    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    import dsh

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if a.config == "c4":
        return bench_batch(a, rank, world, local)
    if a.config == "c5":
        return bench_learned(a, rank, world, local)
    cfg, wkind, label, fdo = workload(a.config, a.nt, a.nx, a.ny, a.shots)
    gradient = wkind == "gradient"
    p = cfg["params"]
    shots = cfg["shots"]
    nx, ny, nt, L = p["nx"], p["ny"], p["nt"], p["l"]
    if world > 1:   # distinct shots per rank (weak scaling): sources shifted along x
        moved = []
        for sh in shots:
            sp = sh.srcpos.copy()
            sp[0, 0] = 1 + (int(sp[0, 0]) - 1 + rank * (nx // (world + 1))) % nx
            moved.append(dsh.Shot(sp, sh.recpos))
        shots = moved
    nsh = len(shots)
    n = nx * ny
    ntr_all = sum(s.ntr for s in shots)
    # the batched gradient as its configuration states it: a checkpoint every
    # ceil(sqrt(NT)) steps (the engine's own choice would be sqrt(NT (3+2L)/3))
    extra = {"ckpt_every": math.ceil(math.sqrt(nt))} if a.config == "c3" else {}
    params = dsh.make_params(**p, max_shots=nsh, **extra)
    eng = dsh.Engine(params, device=local)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
    if a.step_variant >= 0:
        eng.set_step_variant(a.step_variant)
        variant, variant_ms = f"{dsh.Engine.VARIANTS[a.step_variant]} (pinned)", None
    elif a.no_autotune:          # profiling runs: a profiler's serialised timings would mislead the tuner
        variant, variant_ms = "kernel pair (autotuner skipped)", None
    else:
        variant, variant_ms = eng.autotune(shots, nsteps=min(64, nt))   # step-kernel variant for this grid

    seis = torch.empty(ntr_all * nt, device="cuda", dtype=torch.float32)
    if gradient:
        # observed data: synthesised by the engine on the true model, kept in HBM
        eng.set_model(cfg["true"], cfg["rho"], cfg["qs"])
        eng.forward_device(shots, seis.data_ptr())
    eng.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
    gv = torch.empty(n, device="cuda", dtype=torch.float32)
    gr = torch.empty(n, device="cuda", dtype=torch.float32)

    def allreduce():
        if world > 1 and gradient:
            with torch.cuda.stream(stream):
                dist.all_reduce(gv)
                dist.all_reduce(gr)

    def barrier():
        if world > 1:
            dist.barrier()

    def device_step():
        if gradient:
            l2 = eng.gradient_device(shots, seis.data_ptr(), gv.data_ptr(), gr.data_ptr())
        else:
            eng.forward_device(shots, seis.data_ptr())
            l2 = None
        allreduce()
        return l2

    for _ in range(a.warmup):
        device_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, ms_f, ms_a, l2 = 0, 0.0, 0.0, None
    ckpt = 0
    e0.record(stream)
    for _ in range(a.steps):
        l2 = device_step()
        st = eng.stats()
        launches += st["kernel_launches"]
        ms_f += st["ms_forward"]
        ms_a += st["ms_adjoint"]
        ckpt = st["checkpoint_interval"]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    storage = eng.stats()["storage_bytes"]
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    passes = 2 if gradient else 1
    pts_step = float(passes) * n * nt * nsh * world
    value = pts_step * a.steps / (ms / 1e3) / 1e9

    # --- e2e through the host API, every step: model (and observed data) in, gradients (or seismograms) out
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    vs_h, rho_h = pin(cfg["vs"]), pin(cfg["rho"])
    qs_h = pin(cfg["qs"]) if L else None
    obs_p = pin(seis.cpu().numpy()) if gradient else None
    seis_h = torch.empty(ntr_all * nt, dtype=torch.float32).pin_memory()
    gvs_h = torch.empty((ny, nx), dtype=torch.float32).pin_memory()
    grh_h = torch.empty((ny, nx), dtype=torch.float32).pin_memory()
    arr = dsh._shots_c(shots)

    def host_step():
        eng.set_model(vs_h, rho_h, qs_h)
        if gradient:
            l2c = C.c_double(0)
            rc = dsh.lib().dsh_gradient(eng.h, arr, nsh, obs_p.ctypes.data, gvs_h.data_ptr(), grh_h.data_ptr(),
                                        C.byref(l2c), None, None, None)
        else:
            rc = dsh.lib().dsh_forward(eng.h, arr, nsh, seis_h.data_ptr())
        if rc != 0:
            raise dsh.DshError(rc, "dsh_gradient" if gradient else "dsh_forward")

    host_step()
    torch.cuda.synchronize()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(a.steps):
        host_step()
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)
    t = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e2e = float(t.item())
    e2e_value = pts_step * a.steps / (ms_e2e / 1e3) / 1e9
    nsrc_all = sum(s.srcpos.shape[1] for s in shots)
    h2d = (5 if L else 2) * n * 4 + 8 * 4 * nsrc_all + 2 * 4 * ntr_all   # model fields, geometry
    if gradient:
        h2d += ntr_all * nt * 4                                          # observed data
        d2h = 2 * n * 4 + 8
    else:
        d2h = ntr_all * nt * 4

    # --- roofline: whole step and the dominant kernel
    hbm, peak_kind = peaks()
    bf, ba = bytes_per_point(L, nx, ny, p["fw"], p["free_surf"])
    if not gradient:
        bf -= 12 + 8                       # no storage, no energy in plain forward modelling
    step_bytes = n * nt * nsh * (bf + (ba if gradient else 0)) * a.steps
    step_gbs = step_bytes / ((ms_f + ms_a) / 1e3) / 1e9
    pname = "forward_store" if gradient else "forward"
    fused_ms = eng.profile_fused(pname, a.profile_steps)
    prof = eng.profile_step(pname, a.profile_steps)
    trec = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and a.config == "c2":
        # DRAM bytes of one launch from an ncu capture; reported only when the
        # capture was taken on the step kernels' current source
        try:
            rec = json.load(open(tpath))
            if rec.get("kernels_sha256") == kernels_hash():
                trec = rec
        except Exception:
            trec = {}
    if fused_ms is not None:        # one fused kernel per step: it is the dominant (only) step kernel
        ks = fused_bytes(L, store=gradient)
        kname = f"fs_step<{fdo},{L}> (fused velocity+stress, forward pass{' with storage' if gradient else ''})"
        kms = fused_ms
        prof["fs_step"] = fused_ms
        traffic = trec.get("fs_step_forward_store_bytes_per_launch")
        rooflines = {}
    else:
        # the stress kernels of the forward pass (with storage) and of the
        # adjoint pass launch once per step each; the dominant one is the
        # slower of the two
        kv, ks = kernel_bytes(L, store=gradient)
        rooflines = {"forward": {"kernel": f"s_step<{fdo},{L}> (forward pass{' with storage' if gradient else ''})",
                                 "bytes_per_point": ks, "ms_per_launch": prof["s_step"],
                                 "traffic": trec.get("s_step_forward_store_bytes_per_launch")}}
        if gradient:
            pa = eng.profile_step("adjoint", a.profile_steps)
            prof["v_step_adjoint"], prof["s_step_adjoint"] = pa["v_step"], pa["s_step"]
            rooflines["adjoint"] = {"kernel": f"s_step<{fdo},{L}> (adjoint pass with correlation)",
                                    "bytes_per_point": kernel_bytes_adjoint(L)[1], "ms_per_launch": pa["s_step"],
                                    "traffic": trec.get("s_step_adjoint_bytes_per_launch")}
        for r in rooflines.values():
            r["achieved"] = r["bytes_per_point"] * n * nsh / (r["ms_per_launch"] / 1e3) / 1e9
            r["frac"] = r["achieved"] / hbm
        dom = max(rooflines, key=lambda k: rooflines[k]["ms_per_launch"])
        kname, ks, kms = rooflines[dom]["kernel"], rooflines[dom]["bytes_per_point"], rooflines[dom]["ms_per_launch"]
        traffic = rooflines[dom]["traffic"]
    s_gbs = ks * n * nsh / (kms / 1e3) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        steps = a.cpu_steps
        times, kind = run_cpu(1, steps, a, repeats=1)
        what = f"{steps} forward (with storage) + {steps} adjoint steps" if gradient else f"{steps} forward steps"
        cpu = {"value": passes * nx * ny * steps / times[0] / 1e9, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"{what} of one shot of the same {nx}x{ny} FD{fdo} L={L} {wkind}, one core"}

    if rank == 0:
        state_mb = (3 + 2 * L) * n * 4 * nsh / 1e6
        if gradient and not ckpt:
            l2note = f"inputs larger than L2 (stored forward wavefield {3 * n * nt * 4 * nsh / 1e9:.0f} GB)"
        elif gradient:
            l2note = (f"inputs larger than L2 (wavefield state {state_mb:.0f} MB, checkpoints + recompute "
                      f"buffer {storage / 1e9:.1f} GB)")
        else:
            l2note = (f"state {state_mb:.1f} MB fits in L2: no flush between steps, "
                      f"bytes counted algorithmically")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{label}-nt{nt}", "nx": nx, "ny": ny, "nt": nt, "fdorder": fdo, "l": L,
                       "shots_per_gpu": nsh, "receivers": shots[0].ntr, "parallelism": f"shots{world}",
                       "step_variant": variant, "autotune_ms_per_step": variant_ms,
                       "checkpoint_interval": ckpt, "storage_gb": storage / 1e9, "l2": l2note},
            "roofline": {"bound": "hbm", "achieved": s_gbs, "peak": hbm, "unit": "GB/s", "frac": s_gbs / hbm,
                         "traffic": traffic, "kernel": kname, "bytes_per_point": ks, "ms_per_launch": kms,
                         "peak_source": peak_kind},
            "stress_kernel_rooflines": rooflines,
            "step_roofline": {"achieved": step_gbs, "frac": step_gbs / hbm, "bytes_per_point_fwd": bf,
                              "bytes_per_point_adj": ba if gradient else None,
                              "ms_forward_pass": ms_f / a.steps,
                              "ms_adjoint_pass": ms_a / a.steps if gradient else None},
            "kernels_ms": prof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e / a.steps},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        if gradient:
            line["gradients_per_s"] = world * nsh * a.steps / (ms / 1e3)
            line["l2_misfit"] = l2
    eng.close()
    if rank == 0:
        if a.config == "c2" and world == 1 and a.c3_steps > 0:
            del seis, gv, gr
            torch.cuda.empty_cache()
            line["c3"] = c3_sub(a, local)
        if a.config == "c2" and world == 1 and a.c1_steps > 0:
            line["c1"] = c1_sub(a, local)
        if a.config == "c2" and world == 1 and a.c5_small:
            line["c5_small"] = c5_small_sub(a, local)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def bench_batch(a, rank, world, local):
    """The uneven multi-model batch through dsh_batch (one launch per half-step)."""
    import numpy as np
    import torch
    import torch.distributed as dist

    import dsh
    from dsh import configs

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    models = configs.config4(nmodels=a.c4_models, nt_scale=a.nt_scale)
    if world > 1:   # weak scaling: every rank its own copy of the batch, sources shifted
        for m in models:
            nx = m["params"]["nx"]
            for sh in m["shots"]:
                sh.srcpos[0, 0] = 1 + (int(sh.srcpos[0, 0]) - 1 + rank * (nx // (world + 1))) % nx
    plist = [dsh.make_params(**m["params"]) for m in models]
    b = dsh.Batch(plist, device=local)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    for k, m in enumerate(models):
        b.set_model(k, m["vs"], m["rho"], m["qs"])
    shots = [m["shots"] for m in models]
    nseis = sum(sh.ntr * m["params"]["nt"] for m in models for sh in m["shots"])
    seis = torch.empty(max(nseis, 1), device="cuda", dtype=torch.float32)
    pts_model = [m["params"]["nx"] * m["params"]["ny"] * m["params"]["nt"] * len(m["shots"]) for m in models]
    pts = float(sum(pts_model))

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(a.warmup):
        b.forward_device(shots, seis.data_ptr())
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    model_ms = np.zeros(len(models))
    e0.record(stream)
    for _ in range(a.steps):
        b.forward_device(shots, seis.data_ptr())
        st = b.stats()
        launches += st["kernel_launches"]
        model_ms += st["model_ms"]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = pts * world * a.steps / (ms / 1e3) / 1e9

    # e2e: models in, seismograms out, through the host API every step
    import ctypes as C

    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() if x is not None else None
    host_models = [(pin(m["vs"]), pin(m["rho"]), pin(m["qs"])) for m in models]
    seis_h = torch.empty(max(nseis, 1), dtype=torch.float32).pin_memory()
    flat = [sh for g in shots for sh in g]
    arr = dsh._shots_c(flat)
    nsh = np.array([len(g) for g in shots], np.int32)

    def host_step():
        for k, (vs, rho, qs) in enumerate(host_models):
            b.set_model(k, vs, rho, qs)
        rc = dsh.lib().dsh_batch_forward(b.h, arr, nsh.ctypes.data, seis_h.data_ptr())
        if rc != 0:
            raise dsh.DshError(rc, "dsh_batch_forward")

    host_step()
    torch.cuda.synchronize()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(a.steps):
        host_step()
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)
    t = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e2e = float(t.item())
    e2e_value = pts * world * a.steps / (ms_e2e / 1e3) / 1e9
    h2d = sum((3 if m["qs"] is not None else 2) * m["params"]["nx"] * m["params"]["ny"] * 4 for m in models)
    h2d += sum(8 * 4 + 2 * 4 * sh.ntr for sh in flat)
    d2h = nseis * 4

    # roofline of the stress half-step (its class launches): algorithmic bytes of every model's points / autotuned time
    st = b.stats()
    hbm, peak_kind = peaks()
    sbytes = sum(kernel_bytes(m["params"]["l"], store=False)[1] * m["params"]["nx"] * m["params"]["ny"] *
                 len(m["shots"]) for m in models)
    s_ms = st["s_ms"][st["s_variant"]]
    s_gbs = sbytes / (s_ms / 1e3) / 1e9
    per_model = [{"model": m["name"], "nt": m["params"]["nt"], "shots": len(m["shots"]),
                  "gpt_s": pts_model[k] / (model_ms[k] / a.steps / 1e3) / 1e9,
                  "ms_done": model_ms[k] / a.steps} for k, m in enumerate(models)]
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        steps = max(a.cpu_steps, 48)
        times, kind = run_cpu(1, steps, a, repeats=1)
        cfg, _, _, fdo = workload("c4", 16)
        q = cfg["params"]
        cpu = {"value": q["nx"] * q["ny"] * steps / times[0] / 1e9, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"{steps} forward steps of one shot of the batch's largest model "
                         f"({q['nx']}x{q['ny']} FD{fdo} L={q['l']}), one core"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"uneven-batch-{len(models)}-models-forward", "models": len(models),
                       "shots": int(nsh.sum()), "nt_scale": a.nt_scale, "phases": st["phases"],
                       "tile_variant": {"v": dsh.Batch.VARIANTS[st["v_variant"]],
                                        "s": dsh.Batch.VARIANTS[st["s_variant"]]},
                       "autotune_ms": {"v": st["v_ms"], "s": st["s_ms"]},
                       "l2": f"wavefield state {sum((3 + 2 * m['params']['l']) * m['params']['nx'] * m['params']['ny'] * len(m['shots']) for m in models) * 4 / 1e9:.1f} GB, larger than L2",
                       "parallelism": f"models{world}"},
            "roofline": {"bound": "hbm", "achieved": s_gbs, "peak": hbm, "unit": "GB/s", "frac": s_gbs / hbm,
                         "traffic": None, "kernel": f"s_multi_k (one stress half-step: a launch per register class, {len(models)} models)",
                         "bytes": sbytes, "ms_per_launch": s_ms, "peak_source": peak_kind},
            "per_model": per_model,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e / a.steps},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def bench_learned(a, rank, world, local):
    """C5: training set from the solver, U-Net training, plain vs learned FWI."""
    import numpy as np
    import torch

    import dsh
    from dsh import configs, fwi
    from dsh import nn as dnn

    torch.cuda.set_device(local)
    if rank != 0:
        return
    cfg = configs.config5(**({"nt": a.nt} if a.nt else {}))
    p = dict(cfg["params"])
    ny, nx = p["ny"], p["nx"]
    ns = len(cfg["shots"])
    pick = sorted({int(round(k)) for k in np.linspace(0, ns - 1, min(a.train_shots, ns))})
    train_shots = [cfg["shots"][k] for k in pick]
    log = lambda r: print(json.dumps(r), file=sys.stderr, flush=True)
    t0 = time.time()
    targets = [t for t in a.targets.split(",") if t]
    nets = {t: dnn.UNet(torch, seed=0) for t in targets}
    for t, n in nets.items():
        n.target = t
    cache = {t: (f"{os.path.splitext(a.net_cache)[0]}_{t}.npz" if a.net_cache else None) for t in targets}
    gen_s = 0.0
    train_s, losses = {t: 0.0 for t in targets}, {t: [None] for t in targets}
    todo = [t for t in targets if not (cache[t] and os.path.exists(cache[t]))]
    for t in targets:
        if t not in todo:
            nets[t].load_state(dict(np.load(cache[t])))
    if todo:
        clock0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clock0[0].record()
        models = configs.training_models(count=a.train_models, first_seed=100, nx=nx, ny=ny)
        xs, ts = fwi.training_pairs(torch, models, p, train_shots, log=log)
        clock0[1].record()
        torch.cuda.synchronize()
        gen_s = clock0[0].elapsed_time(clock0[1]) / 1e3
        for t in todo:
            tt = dnn.residual_targets(torch, xs, ts) if t == "log_h_over_ws" else ts
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            losses[t] = fwi.train(nets[t], torch, xs, tt, ny, nx, epochs=a.epochs, batch=2, lr=1e-3, log=log)
            e1.record()
            torch.cuda.synchronize()
            train_s[t] = e0.elapsed_time(e1) / 1e3
            if cache[t]:
                np.savez(cache[t], **nets[t].state())
            del tt
        del xs, ts
    curve = lambda h: [[round(r["gpu_s"], 3), r["misfit"]] for r in h]
    runs = []
    for m in [x for x in a.methods.split(",") if x]:
        if m.startswith("learned"):
            runs += [(m if k == 0 else f"{m}@{t}", m, nets[t]) for k, t in enumerate(targets)]
        else:
            runs.append((m, m, None))
    seeds = [int(x) for x in a.problem_seeds.split(",") if x]
    per_seed = []
    clocks = Clocks(local)            # clocks over the FWI runs the ratios come from
    clocks.start()
    for seed in seeds:
        pcfg = configs.config5(seed=seed, **({"nt": a.nt} if a.nt else {}))
        prob = fwi.Problem(pcfg, test_shots=4)
        prob.observe()
        w0 = time.time()
        hp, _ = fwi.run(prob, a.fwi_iters, method="plain", log=log)
        w1 = time.time()
        target = hp[-1]["misfit"] * 1.01
        t_plain = hp[-1]["gpu_s"]
        res = {}
        for key, m, net in runs:
            ws = time.time()
            hl, _ = fwi.run(prob, a.fwi_iters, method=m, net=net, torch=torch, target_misfit=target, log=log)
            t = fwi.time_to_reach(hl, target)
            res[key] = {"final_misfit": hl[-1]["misfit"], "gpu_s_to_target": t, "gpu_s_total": hl[-1]["gpu_s"],
                        "ratio": (t / t_plain) if t is not None else None,
                        "wall_ratio": ((time.time() - ws) / (w1 - w0)) if t is not None else None,
                        "iterations": len(hl) - 1, "fallbacks": sum(1 for r in hl if r.get("fallback")),
                        "network_target": net.target if net is not None else None, "curve": curve(hl)}
        prob.close()
        per_seed.append({"seed": seed, "plain": {"final_misfit": hp[-1]["misfit"], "gpu_s": t_plain,
                                                 "iterations": len(hp) - 1, "curve": curve(hp)},
                         "methods": res})
    clk = clocks.stop()
    primary = a.methods.split(",")[0]

    def median_ratio(key, field="ratio"):
        v = sorted(float("inf") if r["methods"][key][field] is None else r["methods"][key][field] for r in per_seed)
        med = v[len(v) // 2] if len(v) % 2 else 0.5 * (v[len(v) // 2 - 1] + v[len(v) // 2])
        return None if med == float("inf") else med

    summary = {key: {"median_ratio": median_ratio(key), "ratios": [r["methods"][key]["ratio"] for r in per_seed]}
               for key, _, _ in runs}
    line = {
        "metric": "learned-vs-plain FWI: GPU-seconds to the plain method's final misfit (ratio)",
        "value": summary[primary]["median_ratio"], "method": primary,
        "unit": "ratio", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 solver, bf16 network", "data": "synthetic",
        "config": {"workload": f"learned-fwi-{nx}x{ny}-fd8-L3-{ns}shots-nt{p['nt']}", "fwi_iters": a.fwi_iters,
                   "train_models": a.train_models, "train_shots": len(train_shots), "epochs": a.epochs,
                   "network_targets": targets, "problem_seeds": seeds,
                   "unet": "4 levels, 32 base channels, bf16 weights/activations, fp32 accumulation",
                   "target": "plain final misfit x 1.01", "value": "median over the problem seeds",
                   "net_cache": bool(a.net_cache and gen_s == 0.0)},
        "summary": summary,
        "plain": per_seed[0]["plain"],
        "methods": per_seed[0]["methods"],
        "per_seed": per_seed[1:],
        "training": {"data_gpu_s": gen_s, "train_gpu_s": train_s,
                     "loss_first": {t: v[0] for t, v in losses.items()},
                     "loss_last": {t: v[-1] for t, v in losses.items()}},
        "e2e": {"value": median_ratio(primary, "wall_ratio"), "unit": "ratio (host wall-clock of the FWI runs)",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "wall_s": time.time() - t0,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
