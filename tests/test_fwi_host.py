"""Host-side optimisation steps of the FWI loop (include/dsh_fwi.h): the
L-BFGS two-loop recursion against a textbook numpy version, the parabolic
step length (src/calc_opt_step.c) and the bracketing line search
(src/line_search.c) on misfit curves with a known minimum."""
import ctypes as C

import numpy as np
import pytest

import dsh
from dsh import fwi


def _twoloop(S, Y, q):
    r = q.astype(np.float64).copy()
    k = len(S)
    if k == 0:
        return r
    rho = [1.0 / float(y @ s) if float(y @ s) != 0 else 0.0 for s, y in zip(S, Y)]
    al = [0.0] * k
    for i in range(k - 1, -1, -1):
        al[i] = rho[i] * float(S[i] @ r)
        r -= al[i] * Y[i]
    r *= float(Y[-1] @ S[-1]) / float(Y[-1] @ Y[-1])
    for i in range(k):
        b = rho[i] * float(Y[i] @ r)
        r += S[i] * (al[i] - b)
    return r


@pytest.mark.parametrize("count", [0, 1, 3, 5])
def test_lbfgs_direction_matches_two_loop(count):
    rng = np.random.default_rng(count)
    n = 500
    S = rng.standard_normal((count, n)).astype(np.float32)
    Y = (S * rng.uniform(0.5, 2.0, n) + 0.01 * rng.standard_normal((count, n))).astype(np.float32)
    q = rng.standard_normal(n).astype(np.float32)
    r = fwi.lbfgs_direction(S, Y, q)
    ref = _twoloop(S.astype(np.float64), Y.astype(np.float64), q)
    assert np.allclose(r, ref, rtol=1e-4, atol=1e-5 * np.abs(ref).max())


def test_lbfgs_satisfies_newest_secant_equation():
    """The L-BFGS inverse Hessian maps the newest gradient difference to the
    newest model difference: H y_k = s_k."""
    rng = np.random.default_rng(1)
    n = 40
    h = rng.uniform(1.0, 3.0, n)
    S = rng.standard_normal((5, n)).astype(np.float32)
    Y = (S * h).astype(np.float32)
    r = fwi.lbfgs_direction(S, Y, Y[-1])
    assert np.allclose(r, S[-1], rtol=1e-4, atol=1e-4)


def test_opt_step_parabola():
    L = lambda e: 3.0 + 2.0 * (e - 0.7) ** 2
    eps = np.array([0.0, 0.4, 1.2], np.float32)
    got = fwi.opt_step([L(e) for e in eps], eps)
    assert got == pytest.approx(0.7, rel=1e-4)
    # misfit still falling at the third step: take the third step
    eps = np.array([0.0, 0.2, 0.4], np.float32)
    assert fwi.opt_step([L(e) for e in eps], eps) == pytest.approx(0.4)
    # extremum beyond the third step is clipped to it
    L2 = lambda e: 3.0 - 0.1 * e + 0.01 * e * e
    assert fwi.opt_step([L2(e) for e in eps], eps) == pytest.approx(0.4)


@pytest.mark.parametrize("emin", [0.003, 0.02, 0.3])
def test_line_search_brackets_and_fits(emin):
    L = lambda e: 1.0 + (e - emin) ** 2 / emin ** 2
    eps, tests = fwi.line_search(lambda e: L(e), L(0.0), eps_scale=0.01, scalefac=2.0, stepmax=10)
    assert eps == pytest.approx(emin, rel=0.05)
    assert 2 <= tests <= 14


def test_line_search_gives_up_without_descent():
    eps, tests = fwi.line_search(lambda e: 1.0 + e, 1.0, eps_scale=0.01, scalefac=2.0, stepmax=4)
    assert eps == 0.0 and tests == 5


def test_line_search_terminates_on_non_finite_misfits():
    eps, tests = fwi.line_search(lambda e: float("nan"), 1.0, eps_scale=0.01, scalefac=2.0, stepmax=3)
    assert eps == 0.0 and tests == 4
