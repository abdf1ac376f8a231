"""Misfit norms of the residual (calc_res.c LNORM 1..5, GRAD_FORM=2): the
oracle's restatement against the reference's own calc_res compiled into the
oracle (residual, misfit and the gradient it drives, bit for bit), and on the
GPU the engine's residual kernels (dsh_set_misfit) against the oracle's shot
loop.  LNORM=5 divides by trace norms: a trace whose norms underflow in float
gives NaN residuals in the reference and here alike; the engine then reports
the non-finite adjoint field instead of returning a NaN gradient."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import oracle_model

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


def _problem(seed, weak_trace=False, nshots=1):
    from test_gpu_parity import _case

    d, shots = _case(seed, nx=41, ny=33, nt=150, fdo=8, L=2, fs=1, fw=6, nshots=nshots)
    out = []
    for sh in shots:
        rec = sh.recpos.copy()
        rec[1] = 1 if not weak_trace else np.where(rec[1] == 0, 1, rec[1])
        out.append(dsh.Shot(sh.srcpos, rec))
    m = oracle_model(d)
    obs = []
    rng = np.random.default_rng(seed)
    for sh in out:
        o = O.Oracle(m, "port")
        s = o.forward(sh.srcpos, sh.recpos)
        o.close()
        obs.append((s * np.float32(0.6) + np.float32(1e-4) * rng.standard_normal(s.shape)).astype(np.float32))
    return d, m, out, obs


@ref_only
@pytest.mark.parametrize("lnorm", [1, 2, 3, 4, 5])
def test_port_residual_and_gradient_match_reference(lnorm):
    d, m, shots, obs = _problem(5)
    out = {}
    for kind in ("ref", "port"):
        o = O.Oracle(m, kind)
        out[kind] = o.shot_gradient(shots[0].srcpos, shots[0].recpos, obs[0], lnorm=lnorm)
        o.close()
    a, b = out["ref"], out["port"]
    for k in ("res", "g_u", "g_rho"):
        assert np.array_equal(a[k], b[k]), k
    assert a["l2"] == b["l2"]
    if lnorm in (1, 3, 4):
        assert a["l2"] == 0.0                     # the reference adds nothing for these norms
    if lnorm == 1:
        assert set(np.unique(a["res"])) <= {-1.0, 0.0, 1.0}


@ref_only
def test_global_correlation_nan_traces_match_reference():
    """A receiver deep in the model records ~1e-15: |syn|^3 |obs| underflows
    and the reference's LNORM=5 residual of that trace is NaN."""
    d, m, shots, obs = _problem(5, weak_trace=True)
    out = {}
    for kind in ("ref", "port"):
        o = O.Oracle(m, kind)
        out[kind] = o.shot_gradient(shots[0].srcpos, shots[0].recpos, obs[0], lnorm=5)
        o.close()
    assert np.isnan(out["ref"]["res"]).any()
    for k in ("res", "g_u", "g_rho"):
        assert np.array_equal(out["ref"][k], out["port"][k], equal_nan=True), k


def _oracle_loop(m, shots, obs, lnorm):
    su = np.zeros((m.ny, m.nx), np.float32)
    sr = np.zeros((m.ny, m.nx), np.float32)
    l2, terms = 0.0, 0
    for sh, ob in zip(shots, obs):
        o = O.Oracle(m, "port")
        g = o.shot_gradient(sh.srcpos, sh.recpos, ob, lnorm=lnorm)
        o.close()
        su, sr = su + g["g_u"], sr + g["g_rho"]
        l2 += g["l2"]
        terms += ob.size
    o = O.Oracle(m, "port")
    gv, gr = o.convert(su, sr)
    o.close()
    return gv, gr, l2, terms


@pytest.mark.gpu
@pytest.mark.parametrize("lnorm", [1, 3, 4, 5])
def test_engine_misfit_norms_match_oracle(lnorm):
    from test_gpu_parity import engine_from

    d, m, shots, obs = _problem(9 + lnorm, nshots=3)
    gv, gr, l2, terms = _oracle_loop(m, shots, obs, lnorm)
    with engine_from(d, max_shots=2) as e:
        e.set_misfit(lnorm)
        out = e.gradient(shots, obs)
        per_shot = e.shot_misfits(len(shots))
        e.set_misfit("l2")
        back = e.gradient(shots, obs)
    assert np.array_equal(out["g_vs"], gv) and np.array_equal(out["g_rho"], gr)
    if lnorm == 5:
        # float sum in the oracle vs double on the device: |terms| <= 1 per trace
        ntr = sum(s.ntr for s in shots)
        assert abs(out["l2"] - l2) <= terms * 2.0 ** -24 * ntr
        assert out["l2"] < 0 and per_shot.sum() == pytest.approx(out["l2"], rel=1e-12)
    else:
        assert out["l2"] == 0.0
    assert not np.array_equal(back["g_vs"], out["g_vs"])


@pytest.mark.gpu
def test_engine_global_correlation_nan_trace_is_reported():
    """The reference carries the NaN residual of an underflowing trace into
    its gradient; the engine's finite check of the back-propagated field
    reports it as DSH_ERR_UNSTABLE instead."""
    from test_gpu_parity import engine_from

    d, m, shots, obs = _problem(5, weak_trace=True)
    gv, _, _, _ = _oracle_loop(m, shots, obs, 5)
    assert np.isnan(gv).any()
    with engine_from(d) as e:
        e.set_misfit(5)
        with pytest.raises(dsh.DshError) as ei:
            e.gradient(shots, obs)
        assert ei.value.code == dsh.ERR_UNSTABLE
        e.set_misfit(2)
        assert np.isfinite(e.gradient(shots, obs)["g_vs"]).all()     # the context stays usable


@pytest.mark.gpu
def test_set_misfit_rejects_lnorm_6():
    from test_gpu_parity import engine_from

    d, _, _, _ = _problem(5)
    with engine_from(d) as e:
        for bad in (0, 6):
            with pytest.raises(dsh.DshError):
                e.set_misfit(bad)
