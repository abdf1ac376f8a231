#!/usr/bin/env python
"""Throughput of the SH FWI gradient (forward + residual + adjoint with
correlation + energy preconditioning + conversion) on B200.

Workload: the viscoelastic forward + adjoint gradient configuration —
NX=2000, NY=800, DH=0.25 m, FDORDER=8, L=3, NT=6000, one 40 Hz shot, 200
receivers; seeded synthetic model (no dataset exists for this path).  One
step = one full gradient evaluation (2 x NX x NY x NT grid-point updates).

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
    ap.add_argument("--nt", type=int, default=6000)
    ap.add_argument("--nx", type=int, default=2000)
    ap.add_argument("--ny", type=int, default=800)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=24, help="time steps per pass in the CPU sample")
    ap.add_argument("--profile-steps", type=int, default=20)
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


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


def kernel_bytes(l):
    """Per-point bytes a single launch must move (forward pass with storage)."""
    v = 8 + 8 + 4 + 4                      # vy R/W, sxy+syz R, 1/rho R, stored acceleration W
    params = 8 if l == 0 else 16           # uip, ujp | muip, mujp, tausipjp, taus
    s = 16 + 16 * l + 4 + params + 8 + 8   # sxy/syz R/W, r/q R/W, vy R, params, strains W, Ws R/W
    return v, s


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

    cfg, steps, kind = payload
    devnull = os.open(os.devnull, os.O_WRONLY)      # the reference logs to stdout/stderr
    os.dup2(devnull, 1)
    os.dup2(devnull, 2)
    p = dict(cfg["params"])
    m = O.Model(nx=p["nx"], ny=p["ny"], nt=steps, dh=p["dh"], dt=p["dt"], vs=cfg["vs"], rho=cfg["rho"],
                qs=cfg["qs"], fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=p["l"], fl=p["fl"],
                fpml=p["fpml"], damping=p["damping"])
    o = O.Oracle(m, kind)
    sh = cfg["shots"][0]
    t0 = time.perf_counter()
    seis = o.forward(sh.srcpos, sh.recpos, store=True)
    o.residual(seis * np.float32(0.9))
    o.adjoint()
    o.eprecond_scale()
    dt = time.perf_counter() - t0
    o.close()
    return dt


def cpu_workload(nx, ny):
    from dsh import configs

    cfg = configs.config2(nt=16, nx=nx, ny=ny)
    cfg.pop("true", None)
    return cfg


def run_cpu(nprocs, steps, nx, ny, repeats=1):
    """Times `repeats` rounds of nprocs concurrent samples; returns per-round seconds (max over processes)."""
    import multiprocessing as mp

    import oracle as O

    kind = "ref_fast" if O.available("ref_fast") else "port"
    cfg = cpu_workload(nx, ny)
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(nprocs) as pool:
        for _ in range(repeats):
            t = pool.map(_cpu_sample, [(cfg, steps, kind)] * nprocs)
            times.append(max(t))
    return times, ("reference" if kind == "ref_fast" else "port")


def reference_arm(a, rank, world):
    if rank != 0:
        return
    ncpu = os.cpu_count() or 1
    nprocs = max(1, min(ncpu, 32))
    steps = 12
    nx, ny = a.nx, a.ny
    times, kind = run_cpu(nprocs, steps, nx, ny, repeats=a.warmup + a.steps)
    timed = times[a.warmup:]
    pts = 2.0 * nx * ny * steps * nprocs
    val = pts * len(timed) / sum(timed) / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * sum(timed) / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"visc-gradient-{nx}x{ny}-fd8-L3", "nx": nx, "ny": ny, "fdorder": 8, "l": 3,
                       "nt_sample": steps, "shots": nprocs},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nprocs, "kind": kind,
                             "sample": f"{steps} forward (with storage) + {steps} adjoint steps of the {nx}x{ny} "
                                       f"FD8 L=3 gradient per process, {nprocs} independent single-rank processes"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------

def main():
    a = args_parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    import dsh
    from dsh import configs

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cfg = configs.config2(nt=a.nt, nx=a.nx, ny=a.ny)
    p = cfg["params"]
    shots = cfg["shots"]
    if world > 1:   # one distinct shot per rank (weak scaling)
        sp = shots[0].srcpos.copy()
        sp[0, 0] = 1 + (int(sp[0, 0]) - 1 + rank * (p["nx"] // (world + 1))) % p["nx"]
        shots = [dsh.Shot(sp, shots[0].recpos)]
    nx, ny, nt, L = p["nx"], p["ny"], p["nt"], p["l"]
    n = nx * ny
    ntr = shots[0].ntr
    params = dsh.make_params(**p, max_shots=1)
    eng = dsh.Engine(params, device=local)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)

    # observed data: synthesised by the engine on the true model, kept in HBM
    obs = torch.empty(ntr * nt, device="cuda", dtype=torch.float32)
    eng.set_model(cfg["true"], cfg["rho"], cfg["qs"])
    eng.forward_device(shots, obs.data_ptr())
    eng.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
    gv = torch.empty(n, device="cuda", dtype=torch.float32)
    gr = torch.empty(n, device="cuda", dtype=torch.float32)

    def allreduce():
        if world > 1:
            with torch.cuda.stream(stream):
                dist.all_reduce(gv)
                dist.all_reduce(gr)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(a.warmup):
        eng.gradient_device(shots, obs.data_ptr(), gv.data_ptr(), gr.data_ptr())
        allreduce()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, ms_f, ms_a = 0, 0.0, 0.0
    e0.record(stream)
    for _ in range(a.steps):
        l2 = eng.gradient_device(shots, obs.data_ptr(), gv.data_ptr(), gr.data_ptr())
        st = eng.stats()
        launches += st["kernel_launches"]
        ms_f += st["ms_forward"]
        ms_a += st["ms_adjoint"]
        allreduce()
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
    pts_step = 2.0 * n * nt * world
    value = pts_step * a.steps / (ms / 1e3) / 1e9

    # --- e2e through the host API: model + observed data in, gradients out, every step
    obs_h = obs.cpu().numpy().reshape(ntr, nt).copy()
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    vs_h, rho_h, qs_h, obs_p = pin(cfg["vs"]), pin(cfg["rho"]), pin(cfg["qs"]), pin(obs_h)
    gvs_h = torch.empty((ny, nx), dtype=torch.float32).pin_memory()
    grh_h = torch.empty((ny, nx), dtype=torch.float32).pin_memory()
    L2v = []
    import ctypes as C

    def host_step():
        eng.set_model(vs_h, rho_h, qs_h)
        arr = dsh._shots_c(shots)
        l2c = C.c_double(0)
        rc = dsh.lib().dsh_gradient(eng.h, arr, 1, obs_p.ctypes.data, gvs_h.data_ptr(), grh_h.data_ptr(),
                                    C.byref(l2c), None, None, None)
        if rc != 0:
            raise dsh.DshError(rc, "dsh_gradient")
        L2v.append(l2c.value)

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
    h2d = (9 if L else 5) * n * 4 + ntr * nt * 4 + 8 * 4 + 2 * ntr * 4   # model fields, observed data, geometry
    d2h = 2 * n * 4 + 8

    # --- roofline: whole step (both passes) and the dominant kernel
    hbm, peak_kind = peaks()
    bf, ba = bytes_per_point(L, nx, ny, p["fw"], p["free_surf"])
    step_gbs = n * nt * (bf + ba) * a.steps / ((ms_f + ms_a) / 1e3) / 1e9
    prof = eng.profile_step("forward_store", a.profile_steps)
    kv, ks = kernel_bytes(L)
    s_gbs = ks * n / (prof["s_step"] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("s_step_forward_store_bytes_per_launch")
        except Exception:
            traffic = None

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        steps = a.cpu_steps
        times, kind = run_cpu(1, steps, nx, ny, repeats=1)
        cpu = {"value": 2.0 * nx * ny * steps / times[0] / 1e9, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"{steps} forward (with storage) + {steps} adjoint steps of the same {nx}x{ny} FD8 L=3 "
                         f"gradient, one core"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"visc-gradient-{nx}x{ny}-fd8-L3-nt{nt}", "nx": nx, "ny": ny, "nt": nt,
                       "fdorder": 8, "l": 3, "shots_per_gpu": 1, "receivers": ntr, "parallelism": f"shots{world}",
                       "l2": "inputs larger than L2 (stored forward wavefield " +
                             f"{3 * n * nt * 4 / 1e9:.0f} GB per shot)"},
            "gradients_per_s": world * a.steps / (ms / 1e3),
            "l2_misfit": l2,
            "roofline": {"bound": "hbm", "achieved": s_gbs, "peak": hbm, "unit": "GB/s", "frac": s_gbs / hbm,
                         "traffic": traffic, "kernel": "s_step<8,3> (forward pass with storage)",
                         "bytes_per_point": ks, "ms_per_launch": prof["s_step"], "peak_source": peak_kind},
            "step_roofline": {"achieved": step_gbs, "frac": step_gbs / hbm, "bytes_per_point_fwd": bf,
                              "bytes_per_point_adj": ba, "ms_forward_pass": ms_f / a.steps,
                              "ms_adjoint_pass": ms_a / a.steps},
            "kernels_ms": prof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e / a.steps},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
