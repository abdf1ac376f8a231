"""Generates the golden fixtures of this directory by running the REFERENCE's
own C functions (compiled in place by oracle/Makefile into
oracle/_ref/libdenise_ref.so) on small seeded inputs.

The reference ships no tests, golden vectors or example models, so these
fixtures pin parity: each .npz holds the inputs (model, sources, receivers,
observed data) and the reference's outputs (seismograms, residual, L2,
per-shot energies, preconditioned per-shot gradients, converted gradients,
Hessian diagonal, final wavefields).

    python tests/golden/make_golden.py        # needs the reference tree to build the oracle
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Model, Oracle, build  # noqa: E402

CASES = [
    # name, nx, ny, nt, fdorder, L, free_surf, fw, seed
    ("elastic_fd4_fs", 48, 32, 220, 4, 0, 1, 8, 11),
    ("elastic_fd2_pml", 40, 36, 200, 2, 0, 0, 6, 12),
    ("visc_fd8_L2", 56, 40, 220, 8, 2, 1, 10, 13),
    ("visc_fd6_L3_pml", 44, 40, 200, 6, 3, 0, 8, 14),
    ("elastic_fd12_fs", 52, 44, 200, 12, 0, 1, 10, 15),
    ("visc_fd10_L1", 48, 44, 180, 10, 1, 1, 8, 16),
]


def make_case(name, nx, ny, nt, fdo, L, fs, fw, seed):
    rng = np.random.default_rng(seed)
    dh = 0.5
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    dt = np.float32(2.0e-4)
    fl = (7.5, 30.0, 120.0)[:L]
    m = Model(nx=nx, ny=ny, nt=nt, dh=dh, dt=float(dt), vs=vs, rho=rho, qs=qs, fdorder=fdo, fw=fw, free_surf=fs,
              l=L, fl=fl, fpml=30.0, damping=float(vs.max()))
    src = np.zeros((8, 2), np.float32)
    src[:, 0] = [nx // 2, 2, 0, -0.010, 60.0, 1.0, 0, 3]
    src[:, 1] = [nx // 3, 3, 0, -0.012, 50.0, 0.5, 0, 3]
    ntr = 6
    rec = np.array([np.linspace(3, nx - 3, ntr).astype(np.int32), np.full(ntr, 1 if fs else 4, np.int32)])
    o = Oracle(m, "ref")
    seis = o.forward(src, rec, store=False)
    # observed data: same geometry on a perturbed model
    vs2 = vs.copy()
    vs2[3:9, nx // 2 - 8:nx // 2 + 8] *= 1.1
    m2 = Model(**{**m.__dict__, "vs": vs2})
    o.close()
    o2 = Oracle(m2, "ref")
    obs = o2.forward(src, rec)
    o2.close()
    o = Oracle(m, "ref")
    g = o.shot_gradient(src, rec, obs)
    gv, gr = o.convert(g["g_u"], g["g_rho"])
    vy, sxy, syz = o.field("vy"), o.field("sxy"), o.field("syz")   # adjoint end state
    o.close()
    o = Oracle(m, "ref")
    o.forward(src, rec, hessian=True)
    hv, hr = o.hessian_out()
    fwd_vy = o.field("vy")
    o.close()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), nx=nx, ny=ny, nt=nt, dh=dh, dt=dt, fdorder=fdo, l=L,
                        free_surf=fs, fw=fw, fl=np.array(fl, np.float32), fpml=np.float32(30.0),
                        damping=np.float32(vs.max()), vs=vs, rho=rho, qs=qs, srcpos=src, recpos=rec, obs=obs,
                        seis=g["seis"], res=g["res"], l2=g["l2"], Ws=g["Ws"], Wr=g["Wr"], We=g["We"],
                        g_u=g["g_u"], g_rho=g["g_rho"], g_vs=gv, g_rhoc=gr, hess_vs=hv, hess_rho=hr,
                        adj_vy=vy, adj_sxy=sxy, adj_syz=syz, fwd_vy=fwd_vy, seis_plain=seis)


if __name__ == "__main__":
    build()
    for c in CASES:
        make_case(*c)
        print("wrote", c[0])
