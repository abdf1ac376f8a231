"""Seeded synthetic workloads with the shapes, sizes and value ranges of the
five benchmark configurations (there is no public dataset for this path; the
reference ships no models or observed data, so every input is generated).

Each builder returns a dict with ``params`` (keyword arguments of
``dsh.make_params``), the model ``vs``, ``rho``, ``qs`` ([ny, nx] float32), an
optional ``true`` model used to synthesise observed data, and ``shots``.
Grid positions follow the reference: i = iround(x/DH), j = iround(y/DH)
(src/receiver.c:40-41, src/splitsrc.c:20-21); depth of row j is j*DH.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.ndimage import gaussian_filter

from . import Shot, point_source


def iround(x):
    return int(math.floor(x + 0.5))


def _layered(nx, ny, dh, vs_l=(150.0, 250.0, 400.0), rho_l=(1800.0, 1900.0, 2000.0), z=(30.0, 60.0)):
    depth = (np.arange(1, ny + 1) * dh)[:, None] * np.ones((1, nx))
    vs = np.where(depth < z[0], vs_l[0], np.where(depth < z[1], vs_l[1], vs_l[2])).astype(np.float32)
    rho = np.where(depth < z[0], rho_l[0], np.where(depth < z[1], rho_l[1], rho_l[2])).astype(np.float32)
    return vs, rho


def _noise(rng, shape, sigma_pts, amp):
    w = gaussian_filter(rng.standard_normal(shape), sigma_pts)
    return (amp * w / np.max(np.abs(w))).astype(np.float32)


def receivers_line(x0, dx, n, y, dh):
    ii = [iround((x0 + k * dx) / dh) for k in range(n)]
    jj = [iround(y / dh)] * n
    return np.array([ii, jj], np.int32)


def config1(nt=2000, seed=1):
    """Plain elastic forward: 500 x 200, DH=0.5, 3 layers + 5% Gaussian vs noise, FDORDER 4."""
    nx, ny, dh = 500, 200, 0.5
    rng = np.random.default_rng(seed)
    vs, rho = _layered(nx, ny, dh)
    vs = (vs * (1.0 + _noise(rng, (ny, nx), 2.0 / dh, 0.05))).astype(np.float32)
    fc = 30.0
    shots = [Shot(point_source(iround(125.0 / dh), iround(1.0 / dh), fc), receivers_line(77.5, 1.0, 96, 0.5, dh))]
    params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=2e-4, fdorder=4, maxrelerror=1, fw=20, free_surf=1, l=0,
                  damping=float(vs.max()), fpml=fc, eprecond=1)
    return dict(name="elastic-forward-500x200-fd4", params=params, vs=vs, rho=rho, qs=None, shots=shots)


def config2(nt=6000, seed=2, nx=2000, ny=800, dh=0.25):
    """Viscoelastic forward + adjoint gradient: 2000 x 800, DH=0.25, FDORDER 8, L=3, one 40 Hz shot,
    200 receivers.  vs = 100 + 400*norm(gaussian(white, 5 m)); rho = 1740 (1.8 vs/1000)^0.25
    (Gardner); Qs ~ U[20, 60].  Observed data come from the same model with a +10% vs blob."""
    rng = np.random.default_rng(seed)
    w = gaussian_filter(rng.standard_normal((ny, nx)), 5.0 / dh)
    w = (w - w.min()) / (w.max() - w.min())
    vs = (100.0 + 400.0 * w).astype(np.float32)
    rho = (1740.0 * (1.8 * vs / 1000.0) ** 0.25).astype(np.float32)
    qs = np.random.default_rng(seed + 1).uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    fc = 40.0
    true = vs.copy()
    yy, xx = np.mgrid[1:ny + 1, 1:nx + 1] * dh
    cx, cy, rad = nx * dh * 0.5, ny * dh * 0.35, min(nx, ny) * dh * 0.08
    blob = np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * rad ** 2))
    true = (vs * (1.0 + 0.10 * blob)).astype(np.float32)
    ntr = 200
    dxr = nx * dh / ntr
    shots = [Shot(point_source(iround(nx * dh / 2 / dh), iround(0.5 / dh), fc),
                  receivers_line(dxr / 2, dxr, ntr, dh, dh))]
    params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=1e-4, fdorder=8, maxrelerror=1, fw=20, free_surf=1, l=3,
                  fl=(fc / 4, fc, 4 * fc), damping=float(max(vs.max(), true.max())), fpml=fc, eprecond=1)
    return dict(name=f"visc-gradient-{nx}x{ny}-fd8-L3", params=params, vs=vs, rho=rho, qs=qs, true=true,
                shots=shots)


def config3(nt=4000, nshots=64, seed=4):
    """Batched multi-shot FWI gradient: 1000 x 300, DH=0.5, layered + 5-15 elliptical +-20% anomalies;
    start model = true model smoothed with a 10 m Gaussian; 64 shots 7.5 m apart, 192 receivers, L=2."""
    nx, ny, dh = 1000, 300, 0.5
    rng = np.random.default_rng(seed)
    vs, rho = _layered(nx, ny, dh)
    yy, xx = np.mgrid[1:ny + 1, 1:nx + 1] * dh
    true = vs.copy()
    for _ in range(int(rng.integers(5, 16))):
        cx, cy = rng.uniform(0, nx * dh), rng.uniform(5, ny * dh)
        a, b = rng.uniform(5, 30), rng.uniform(5, 30)
        s = rng.choice([-0.2, 0.2])
        inside = ((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0
        true = np.where(inside, true * (1 + s), true)
    true = true.astype(np.float32)
    start = gaussian_filter(true, 10.0 / dh).astype(np.float32)
    qs = np.full((ny, nx), 40.0, np.float32)
    fc = 30.0
    rec = receivers_line(10.0, 2.5, 192, 0.5, dh)
    shots = [Shot(point_source(iround((13.75 + 7.5 * k) / dh), iround(1.0 / dh), fc), rec) for k in range(nshots)]
    params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=2e-4, fdorder=8, maxrelerror=1, fw=20, free_surf=1, l=2,
                  fl=(fc / 4, 2 * fc), damping=float(true.max()), fpml=fc, eprecond=1)
    return dict(name="batched-gradient-1000x300-fd8-L2", params=params, vs=start, rho=rho, qs=qs, true=true,
                shots=shots)


def small_case(nx=64, ny=48, nt=150, fdorder=4, l=0, free_surf=1, fw=10, seed=0, nshots=1, ntr=8, dh=0.5):
    """Small randomised model for parity tests (oracle runs it in seconds)."""
    rng = np.random.default_rng(seed)
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    fc = 30.0
    dt = 0.5 * float(np.sqrt(2.0)) ** -1 * dh / (1.4 * 330.0)
    dt = float(np.float32(min(dt, 2e-4)))
    shots = []
    for s in range(nshots):
        ix = int(rng.integers(fw // 2 + 2, nx - fw // 2 - 2))
        rec_i = np.linspace(3, nx - 3, ntr).astype(int)
        rec_j = np.full(ntr, 1 if free_surf else 3)
        shots.append(Shot(point_source(ix, 2 + s % 3, fc), np.array([rec_i, rec_j], np.int32)))
    params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=dt, fdorder=fdorder, maxrelerror=1, fw=fw, free_surf=free_surf,
                  l=l, fl=(7.5, 30.0, 120.0, 240.0)[:l], damping=float(vs.max()), fpml=fc, eprecond=1)
    return dict(name="small", params=params, vs=vs, rho=rho, qs=qs, shots=shots)


def config4(seed=5, nmodels=32, nt_scale=1.0):
    """Uneven batch of independent models: NX ~ U[256, 2048], NY ~ U[128, 512], DH = 0.5 m,
    FDORDER from {4, 6, 8}, elastic / viscoelastic (L=2, Qs 40) half each, 8-32 shots per model
    with Ricker fc ~ U[20, 60] Hz, C1-style layered model with seeded +-5% vs perturbations.
    DT = 0.8 x the stability limit (dt_limit), NT = ceil(1.5 t_max / DT) with t_max the diagonal
    traveltime at the slowest velocity; ``nt_scale`` shortens every NT by the same factor.
    Returns a list of per-model dicts like the other builders."""
    from . import dt_limit

    rng = np.random.default_rng(seed)
    dh = 0.5
    models = []
    for k in range(nmodels):
        nx = int(rng.integers(256, 2049))
        ny = int(rng.integers(128, 513))
        fdo = int(rng.choice([4, 6, 8]))
        visc = k % 2 == 1
        nsh = int(rng.integers(8, 33))
        fc = float(rng.uniform(20.0, 60.0))
        vs, rho = _layered(nx, ny, dh)
        vs = (vs * (1.0 + _noise(rng, (ny, nx), 2.0 / dh, 0.05))).astype(np.float32)
        vmax, vmin = float(vs.max()), float(vs.min())
        dt = float(np.float32(0.8 * dt_limit(fdo, 1, dh, vmax)))
        tmax = math.hypot(nx * dh, ny * dh) / vmin
        nt = max(2, int(math.ceil(1.5 * tmax / dt * nt_scale)))
        l = 2 if visc else 0
        qs = np.full((ny, nx), 40.0, np.float32) if visc else None
        ntr = 48
        rec = receivers_line(nx * dh * 0.05, nx * dh * 0.9 / ntr, ntr, dh, dh)
        xs = np.linspace(0.1, 0.9, nsh) * nx * dh
        shots = [Shot(point_source(iround(x / dh), iround(1.0 / dh), fc), rec) for x in xs]
        params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=dt, fdorder=fdo, maxrelerror=1, fw=20, free_surf=1, l=l,
                      fl=(fc / 4, 2 * fc)[:l], damping=vmax, fpml=fc, eprecond=1, max_shots=nsh)
        models.append(dict(name=f"m{k}-{nx}x{ny}-fd{fdo}-L{l}", params=params, vs=vs, rho=rho, qs=qs,
                           shots=shots))
    return models


def _anomaly_model(rng, nx, ny, dh):
    """Layered C1-style background plus 5-15 elliptical +-20% vs anomalies."""
    vs, rho = _layered(nx, ny, dh)
    yy, xx = np.mgrid[1:ny + 1, 1:nx + 1] * dh
    true = vs.copy()
    for _ in range(int(rng.integers(5, 16))):
        cx, cy = rng.uniform(0, nx * dh), rng.uniform(5, ny * dh)
        a, b = rng.uniform(5, 30), rng.uniform(5, 30)
        s = rng.choice([-0.2, 0.2])
        inside = ((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0
        true = np.where(inside, true * (1 + s), true)
    return true.astype(np.float32), rho


def config5(seed=6, nx=1200, ny=400, nt=3000, nshots=32, ntr=240):
    """Learned-preconditioner FWI problem: NX=1200, NY=400, DH=0.5, L=3, FDORDER=8, DT=2e-4,
    NT=3000, 30 Hz Ricker; true model = layered background + elliptical anomalies, start model =
    true smoothed with a 10 m Gaussian; 32 shots along the surface, 240 receivers 2.5 m apart."""
    dh = 0.5
    rng = np.random.default_rng(seed)
    true, rho = _anomaly_model(rng, nx, ny, dh)
    start = gaussian_filter(true, 10.0 / dh).astype(np.float32)
    qs = np.full((ny, nx), 40.0, np.float32)
    fc = 30.0
    rec = receivers_line(nx * dh * 0.5 - (ntr - 1) * 1.25, 2.5, ntr, 0.5, dh) if ntr * 2.5 < nx * dh else \
        receivers_line(dh, nx * dh / ntr, ntr, 0.5, dh)
    xs = np.linspace(0.05, 0.95, nshots) * nx * dh
    shots = [Shot(point_source(iround(x / dh), iround(1.0 / dh), fc), rec) for x in xs]
    params = dict(nx=nx, ny=ny, nt=nt, dh=dh, dt=2e-4, fdorder=8, maxrelerror=1, fw=20, free_surf=1, l=3,
                  fl=(fc / 4, fc, 4 * fc), damping=float(true.max()), fpml=fc, eprecond=1, max_shots=nshots)
    return dict(name=f"learned-fwi-{nx}x{ny}-fd8-L3", params=params, vs=start, rho=rho, qs=qs, true=true,
                shots=shots)


def training_models(count=200, first_seed=100, nx=1200, ny=400):
    """Seeded random models of the batched-gradient generator (seeds first_seed ..) at the learned-FWI
    grid: (true, start) pairs, start = true smoothed with a 10 m Gaussian."""
    dh = 0.5
    for seed in range(first_seed, first_seed + count):
        rng = np.random.default_rng(seed)
        true, rho = _anomaly_model(rng, nx, ny, dh)
        yield seed, true, gaussian_filter(true, 10.0 / dh).astype(np.float32), rho
