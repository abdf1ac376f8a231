"""Finite-difference checks of the gradients on the CPU oracle (the FP64
restatement), on the set-up of tests/fdsetup.py.  They state, from the
oracle's own numbers, how closely each gradient follows central differences
of the misfit J = sum res^2; tests/test_gpu_fdcheck.py holds the GPU to the
same bounds.

* vs (the reference's gradient, src/denise.c:1589-1609 converted at
  :1743-1813): a zero-lag correlation of the forward strain rate with the
  back-propagated *stress*.  The Lagrangian of the velocity-stress update
  makes the stress multiplier (2/rho) times the adjoint *strain*; in an
  elastic medium that is the back-propagated stress divided by mu, so the
  reference's correlation is the derivative weighted by mu(x) (on the
  elastic FDORDER-8 variant of this set-up the FD / <g, d> ratios spread 5x
  across directions and dividing by mu brings 6 of 8 within 1.3x).  On this
  viscoelastic set-up the oracle gives cosine 0.9985 over the 8 directions
  with every sign right and ratios within a factor 1.7; the test asserts
  cosine >= 0.98 and the signs.
* Qs (no counterpart in the reference; dsh_get_gradient_q): formed from the
  adjoint strain itself and the exact tau-sensitivity of the discrete SLS
  update, it matches the finite differences in scale as well (ratio within
  a few percent of 1 on the dominant directions, cosine >= 0.999).
"""
import numpy as np
import pytest

import oracle as O
import fdsetup as F


def _model(vs, rho, qs):
    p = F.params()
    return O.Model(nx=p["nx"], ny=p["ny"], nt=p["nt"], dh=p["dh"], dt=p["dt"], vs=vs, rho=rho, qs=qs,
                   fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=p["l"], fl=p["fl"],
                   fpml=p["fpml"], damping=p["damping"], eprecond=0)


def _obs():
    vs0, rho, q0, vst, qt = F.models()
    src, rec = F.geometry()
    o = O.Oracle(_model(vst, rho, qt), "port", fp64=True)
    obs = o.forward(src, rec).astype(np.float32)
    o.close()
    return obs


def _J(vs, rho, qs, obs):
    src, rec = F.geometry()
    o = O.Oracle(_model(vs.astype(np.float32), rho, qs.astype(np.float32)), "port", fp64=True)
    o.forward(src, rec)
    _, l2 = o.residual(obs)
    o.close()
    return l2


def test_oracle_vs_gradient_vs_finite_differences():
    vs0, rho, q0, _, _ = F.models()
    src, rec = F.geometry()
    obs = _obs()
    o = O.Oracle(_model(vs0, rho, q0), "port", fp64=True)
    o.forward(src, rec, store=True)
    o.residual(obs)
    o.adjoint()
    gu = o.field("g_u", f64=True)
    o.close()
    gv = 2.0 * rho.astype(np.float64) * vs0 * (-F.DT * gu)            # denise.c:1743-1813, no preconditioning
    an, fd = [], []
    for d in F.directions():
        h = 0.5
        fd.append((_J(vs0 + h * d, rho, q0, obs) - _J(vs0 - h * d, rho, q0, obs)) / (2 * h))
        an.append(float(np.sum(gv * d)))
    cos = F.cosine(an, fd)
    raw = np.array(fd) / np.array(an)
    print("vs: cos", cos, "FD / <g, d>", raw, "spread", raw.max() / raw.min())
    assert cos >= 0.98
    assert np.all(np.sign(an) == np.sign(fd))


def test_oracle_q_gradient_vs_finite_differences():
    vs0, rho, q0, _, _ = F.models()
    src, rec = F.geometry()
    obs = _obs()
    o = O.Oracle(_model(vs0, rho, q0), "port", fp64=True, grad_q=True)
    o.forward(src, rec, store=True)
    o.residual(obs)
    o.adjoint()
    g = o.grad_q()
    o.close()
    an, fd = [], []
    for d in F.directions(amp=2.0):
        h = 0.5
        fd.append((_J(vs0, rho, q0 + h * d, obs) - _J(vs0, rho, q0 - h * d, obs)) / (2 * h))
        an.append(float(np.sum(g * d)))
    fd, an = np.array(fd), np.array(an)
    cos = F.cosine(an, fd)
    big = np.abs(fd) >= 0.1 * np.abs(fd).max()
    print("Qs: cos", cos, "FD / <g, d>", fd / an)
    assert cos >= 0.999
    assert np.all(np.abs(fd[big] / an[big] - 1.0) < 0.05)
