"""Shared set-up of the finite-difference gradient checks (CPU oracle and
GPU): a 240 x 120 viscoelastic model (FDORDER 8, L = 3, CPML width 10, free
surface), one 60 Hz source at 1 m depth, 31 surface receivers, observed data
from a model with a slower-Q / faster-vs patch, and 8 random Gaussian bump
directions kept >= 2 CPML widths from the absorbing strips and >= 10 points
from the source and receivers."""
import numpy as np
from scipy.ndimage import gaussian_filter

NX, NY, NT, DH, DT, FW = 240, 120, 3000, 0.5, 1e-4, 10
FL = (15.0, 60.0, 240.0)


def models():
    rng = np.random.default_rng(5)
    vs0 = gaussian_filter(200 + 30 * rng.standard_normal((NY, NX)), 4).astype(np.float32)
    rho = np.full((NY, NX), 1800, np.float32)
    q0 = (30 + 100 * gaussian_filter(rng.standard_normal((NY, NX)), 6)).clip(15, 60).astype(np.float32)
    vst = vs0.copy()
    vst[50:70, 100:140] *= 1.05
    qt = q0.copy()
    qt[50:70, 100:140] *= 0.7
    return vs0, rho, q0, vst, qt


def geometry():
    src = np.zeros((8, 1), np.float32)
    src[:, 0] = [120, 2, 0, 0, 60.0, 1.0, 0, 3]
    rec = np.array([np.arange(30, 211, 6), np.ones(31, int)], np.int32)
    return src, rec


def params(l=3):
    return dict(nx=NX, ny=NY, nt=NT, dh=DH, dt=DT, fdorder=8, fw=FW, free_surf=1, l=l, fl=FL[:l], fpml=60.0,
                damping=260.0, eprecond=0)


def directions(n=8, amp=1.0, seed=11):
    yy, xx = np.mgrid[0:NY, 0:NX]
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cy, cx = rng.uniform(25, NY - 30), rng.uniform(35, NX - 35)
        s = rng.uniform(4, 8)
        out.append(np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s ** 2)) * rng.choice([-1, 1]) * amp)
    return out


def cosine(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
