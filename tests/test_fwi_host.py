"""Host-side optimisation steps of the FWI loop (include/dsh_fwi.h): the
L-BFGS two-loop recursion against a textbook numpy version, the
conjugate-gradient direction against the reference's src/PCG.c (compiled into
the oracle) bit for bit and against the oracle's restatement for the beta
choices the reference does not compile, the parabolic step length
(src/calc_opt_step.c) and the bracketing line search (src/line_search.c) on
misfit curves with a known minimum."""
import ctypes as C

import numpy as np
import pytest

import dsh
import oracle as O
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


def _pcg_fields(seed, ny=37, nx=53, reset=False):
    """vs and rho descent directions [2][ny][nx] of two iterations and the
    previous search direction; with reset the new gradient is half the old
    one (Polak-Ribiere beta < 0)."""
    rng = np.random.default_rng(seed)
    old = rng.standard_normal((2, ny, nx)).astype(np.float32) * np.float32([[[3e-3]], [[4e2]]])
    new = (0.5 * old if reset else 0.7 * old + 0.4 * old.std() * rng.standard_normal((2, ny, nx))).astype(np.float32)
    if not reset:
        new[1] = 0.9 * old[1] + 0.2 * old[1].std() * rng.standard_normal((ny, nx)).astype(np.float32)
    d = (old + 0.1 * rng.standard_normal((2, ny, nx)) * old.std(axis=(1, 2), keepdims=True)).astype(np.float32)
    return new, old, d


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
@pytest.mark.parametrize("seed,reset", [(1, False), (2, False), (3, True)])
def test_pcg_direction_bit_identical_to_reference(seed, reset):
    new, old, d = _pcg_fields(seed, reset=reset)
    ny, nx = new.shape[1:]
    xm = lambda a: np.ascontiguousarray(a.transpose(0, 2, 1))     # the reference's x-major class order
    got, betas = fwi.pcg_direction(xm(new), xm(old), xm(d))
    ref = O.pcg(xm(new), xm(old), xm(d), nx, ny)
    assert np.array_equal(got.ravel(), ref)
    assert (betas >= 0).all()
    if reset:
        assert (betas == 0).all() and np.array_equal(got, xm(new))


@pytest.mark.parametrize("beta", ["fletcher_reeves", "polak_ribiere", "hestenes_stiefel", "dai_yuan"])
def test_pcg_direction_beta_choices_match_restatement(beta):
    new, old, d = _pcg_fields(4, ny=9, nx=13)
    got, betas = fwi.pcg_direction(new, old, d, beta=beta)
    ref, ref_b = O.pcg_port(new, old, d, 2, fwi.PCG_BETA[beta])
    assert np.array_equal(got.ravel(), ref) and np.array_equal(betas, ref_b)


def test_pcg_direction_zero_denominator_and_bad_arguments():
    new = np.ones((1, 10), np.float32)
    got, betas = fwi.pcg_direction(new, np.zeros_like(new), np.full_like(new, 5.0))   # g_old = 0: beta = 0
    assert betas[0] == 0 and np.array_equal(got, new)
    with pytest.raises(dsh.DshError):
        fwi.pcg_direction(np.ones((9, 4), np.float32), np.ones((9, 4), np.float32), np.ones((9, 4), np.float32))
    with pytest.raises(KeyError):
        fwi.pcg_direction(new, new, new, beta="newton")


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


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
@pytest.mark.parametrize("it,pointer,filled", [(2, 1, 1), (3, 2, 2), (6, 3, 5), (9, 5, 5), (1, 1, 1)])
def test_lbfgs_ring_matches_reference(it, pointer, filled):
    """dsh_lbfgs_ring against the reference's LBFGS.c compiled into the oracle:
    ring buffers of 5 slots, some empty, the newest pair anywhere in the ring
    (after wrap-around the reference's slot order differs from age order)."""
    rng = np.random.default_rng(it * 10 + pointer)
    nl, n = 5, 301
    y = np.zeros((nl, n), np.float32)
    s = np.zeros((nl, n), np.float32)
    for k in range(filled):
        s[k] = rng.standard_normal(n).astype(np.float32) * np.float32(1e-2)
        y[k] = (s[k] * np.float32(3.0) + rng.standard_normal(n).astype(np.float32) * np.float32(1e-3))
    q = rng.standard_normal(n).astype(np.float32)
    got_q, got_r = fwi.lbfgs_ring(it, y, s, q, pointer)
    ref_q, ref_r = O.lbfgs_ring(it, y, s, q, pointer, nl)
    assert np.array_equal(got_q, ref_q) and np.array_equal(got_r, ref_r)
    if it > 1:
        assert np.abs(got_r).max() > 0


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
def test_opt_step_ref_matches_reference():
    """dsh_opt_step_ref against calc_opt_step.c + solvelin.c compiled into the
    oracle, bit for bit: line-search triples (first step 0), convex and
    concave fits, clipping to the third step, negative extrema, and a singular
    system (two equal steps), which is non-finite in both; dsh_opt_step, the
    double solve the line search uses, agrees to float rounding."""
    rng = np.random.default_rng(11)
    for k in range(400):
        e = np.sort(rng.uniform(0, 1, 3)).astype(np.float32)
        if k % 2 == 0:
            e[0] = 0
        l2 = rng.uniform(0.5, 2.0, 3).astype(np.float32)
        got, ref = fwi.opt_step_ref(l2, e), O.opt_step(l2, e)
        assert got == ref or (np.isnan(got) and np.isnan(ref)), (l2, e)
        dbl = np.float32(fwi.opt_step(l2, e))
        assert abs(float(dbl) - float(got)) <= 1e-3 * max(1.0, abs(float(got))), (l2, e, dbl, got)
    e = np.array([0.0, 0.3, 0.3], np.float32)
    l2 = np.array([1.0, 0.8, 0.9], np.float32)
    got, ref = fwi.opt_step_ref(l2, e), O.opt_step(l2, e)
    assert (got == ref) or (np.isnan(got) and np.isnan(ref))


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
@pytest.mark.parametrize("filt_size", [4, 5, 2, 7, 0, -4])
def test_smooth_model_median_matches_reference(filt_size):
    """dsh_smooth_model_median against the reference's smooth_model.c with
    median.c compiled into the oracle (model files in a temporary directory):
    identical fields and the same grown FILT_SIZE, for even and odd sizes,
    with ties (a layered model) and edge replication."""
    rng = np.random.default_rng(abs(filt_size) + 3)
    ny, nx = 23, 31
    vs = rng.uniform(100, 400, (ny, nx)).astype(np.float32)
    vs[5:9, :] = np.float32(250.0)                       # ties inside windows
    rho = np.round(rng.uniform(1500, 2200, (ny, nx)) / 50).astype(np.float32) * np.float32(50)
    v, r, used = fwi.smooth_model_median(vs, rho, filt_size)
    if filt_size == 0:
        assert used == 0 and np.array_equal(v, vs) and np.array_equal(r, rho)
        return
    rv, rr, rfs = O.smooth_model(vs, rho, filt_size)
    assert used == rfs
    assert np.array_equal(v, rv) and np.array_equal(r, rr)
    assert not np.array_equal(v, vs)


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
def test_calc_mres_matches_reference():
    """dsh_calc_mres against src/calc_mres.c compiled into the oracle, bit for bit."""
    rng = np.random.default_rng(5)
    for ny, nx in [(1, 1), (17, 29), (200, 120)]:
        u0 = rng.uniform(100, 500, (ny, nx)).astype(np.float32)
        u = (u0 * rng.uniform(0.9, 1.1, (ny, nx))).astype(np.float32)
        assert fwi.calc_mres(u, u0) == O.calc_mres(u, u0)
    assert fwi.calc_mres(u0, u0) == 0.0
