"""The GPU gradients against central differences of the GPU misfit, on the
set-up of tests/fdsetup.py (240 x 120, FDORDER 8, L = 3, CPML width 10; 8
Gaussian bump directions >= 2 CPML widths from the strips and >= 10 points
from source and receivers).  The bounds are the CPU oracle's own numbers
(tests/test_fdcheck_oracle.py, FP64 restatement of the same computation):

* vs, the reference's correlation gradient (src/denise.c:1589-1609, :1743-1813),
  which the GPU reproduces bit for bit: the oracle gives cosine 0.9985
  between the directional derivatives and the finite differences, every
  sign right; asserted here: cosine >= 0.98 and the signs;
* Qs (dsh_get_gradient_q, no counterpart in the reference): the oracle gives
  cosine 0.9999996 and FD / <g, d> within 5 % of 1 on every direction whose
  finite difference is >= 10 % of the largest; asserted here: cosine >= 0.999
  and the same 5 %.
The misfit J is the L2 value dsh_gradient returns (sum res^2, summed in
double on the device), evaluated by forward runs at +-h along each direction.
"""
import numpy as np
import pytest

import dsh
import fdsetup as F

pytestmark = pytest.mark.gpu


def _engine(grad_q=False):
    e = dsh.Engine(dsh.make_params(**F.params(), grad_q=int(grad_q)))
    return e


def _obs(e, src, rec):
    vs0, rho, q0, vst, qt = F.models()
    e.set_model(vst, rho, qt)
    return e.forward([dsh.Shot(src, rec)])


def test_vs_gradient_vs_finite_differences():
    vs0, rho, q0, _, _ = F.models()
    src, rec = F.geometry()
    shot = dsh.Shot(src, rec)
    with _engine() as e:
        obs = _obs(e, src, rec)

        def J(vs):
            e.set_model(vs.astype(np.float32), rho, q0)
            return e.gradient([shot], obs)["l2"]

        e.set_model(vs0, rho, q0)
        g = e.gradient([shot], obs)["g_vs"].astype(np.float64)
        an, fd = [], []
        for d in F.directions():
            h = 0.5
            fd.append((J(vs0 + h * d) - J(vs0 - h * d)) / (2 * h))
            an.append(float(np.sum(g * d)))
    cos = F.cosine(an, fd)
    print("vs: cos", cos, "FD / <g, d>", np.array(fd) / np.array(an))
    assert cos >= 0.98
    assert np.all(np.sign(an) == np.sign(fd))


def test_q_gradient_vs_finite_differences():
    vs0, rho, q0, _, _ = F.models()
    src, rec = F.geometry()
    shot = dsh.Shot(src, rec)
    with _engine(grad_q=True) as e:
        obs = _obs(e, src, rec)

        def J(q):
            e.set_model(vs0, rho, q.astype(np.float32))
            return e.gradient([shot], obs)["l2"]

        e.set_model(vs0, rho, q0)
        e.gradient([shot], obs)
        g = e.gradient_q().astype(np.float64)
        an, fd = [], []
        for d in F.directions(amp=2.0):
            h = 0.5
            fd.append((J(q0 + h * d) - J(q0 - h * d)) / (2 * h))
            an.append(float(np.sum(g * d)))
    fd, an = np.array(fd), np.array(an)
    cos = F.cosine(an, fd)
    big = np.abs(fd) >= 0.1 * np.abs(fd).max()
    print("Qs: cos", cos, "FD / <g, d>", fd / an)
    assert cos >= 0.999
    assert np.all(np.abs(fd[big] / an[big] - 1.0) < 0.05)
