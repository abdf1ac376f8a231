"""The Qs gradient (dsh_get_gradient_q; no counterpart in the reference,
which computes no Q gradient) against the CPU oracle's restatement of the
same computation: per forward step the stress increment's derivative with
respect to tau (prepare_update_s.c:40-55 through tau = 2/Qs, readmod.c:99),
correlated in the adjoint pass with the back-propagated adjoint strain, then
the four-point tau average (av_tau.c:12) and tau = 2/Qs by the chain rule.
The oracle and the kernels use the same float expressions (no multiply-add
contraction) and the same double conversion, so one shot is bit-identical;
with several shots the device sums the float correlations over shots before
the conversion while the test sums converted per-shot oracle gradients, so
those agree to float rounding.  Its finite-difference check is in
tests/test_gpu_fdcheck.py."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import oracle_model

pytestmark = pytest.mark.gpu


def _case(seed, nx, ny, nt, fdo, L, fs, fw, nshots=1):
    rng = np.random.default_rng(seed)
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    d = dict(nx=nx, ny=ny, nt=nt, dh=0.5, dt=np.float32(2e-4), fdorder=fdo, fw=fw, free_surf=fs, l=L,
             fl=np.array((7.5, 30.0, 120.0, 240.0)[:L], np.float32), damping=np.float32(vs.max()),
             fpml=np.float32(30.0), vs=vs, rho=rho, qs=qs)
    shots = []
    for s in range(nshots):
        sp = dsh.point_source(int(rng.integers(3, nx - 2)), 2 + s % 3, 60.0)
        rec = np.array([rng.integers(1, nx + 1, 6), [1, 1, 2, ny, max(1, ny // 2), 3]], np.int32)
        shots.append(dsh.Shot(sp, rec))
    return d, shots


def _params(d, **kw):
    return dsh.make_params(nx=d["nx"], ny=d["ny"], nt=d["nt"], dh=d["dh"], dt=float(d["dt"]), fdorder=d["fdorder"],
                           fw=d["fw"], free_surf=d["free_surf"], l=d["l"], fl=tuple(float(x) for x in d["fl"]),
                           damping=float(d["damping"]), fpml=float(d["fpml"]), grad_q=1, **kw)


def _oracle_q(d, shots, obs):
    m = oracle_model(d)
    tot = None
    for sh, ob in zip(shots, obs):
        o = O.Oracle(m, "port", grad_q=True)
        o.forward(sh.srcpos, sh.recpos, store=True)
        o.residual(ob)
        o.adjoint()
        g = o.grad_q()
        o.close()
        tot = g if tot is None else tot + g
    return tot


def _obs(d, shots):
    m = oracle_model(d)
    out = []
    for sh in shots:
        o = O.Oracle(m, "port")
        out.append((o.forward(sh.srcpos, sh.recpos) * np.float32(0.7) + np.float32(1e-4)).astype(np.float32))
        o.close()
    return out


@pytest.mark.parametrize("fdo,L,fs", [(2, 1, 1), (4, 2, 0), (8, 3, 1), (12, 4, 0), (6, 3, 0)])
def test_q_gradient_one_shot_bit_identical(fdo, L, fs):
    d, shots = _case(300 + fdo + L, nx=41 + fdo, ny=33 + L, nt=160, fdo=fdo, L=L, fs=fs, fw=6)
    obs = _obs(d, shots)
    ref = _oracle_q(d, shots, obs).astype(np.float32)
    with dsh.Engine(_params(d)) as e:
        e.set_model(d["vs"], d["rho"], d["qs"])
        out = e.gradient(shots, obs)
        g = e.gradient_q()
    assert np.abs(ref).max() > 0
    assert np.array_equal(g, ref)
    assert np.isfinite(out["g_vs"]).all()


def test_q_gradient_checkpointed_and_multi_shot():
    d, shots = _case(77, nx=70, ny=48, nt=220, fdo=8, L=3, fs=1, fw=8, nshots=3)
    obs = _obs(d, shots)
    ref = _oracle_q(d, shots, obs)
    runs = {}
    for name, kw in (("full", {}), ("checkpointed", {"ckpt_every": 15}), ("two slots", {"max_shots": 2})):
        with dsh.Engine(_params(d, **kw)) as e:
            e.set_model(d["vs"], d["rho"], d["qs"])
            e.gradient(shots, obs)
            runs[name] = e.gradient_q()
    assert np.array_equal(runs["checkpointed"], runs["full"])
    assert np.array_equal(runs["two slots"], runs["full"])
    scale = np.abs(ref).max()
    assert np.abs(runs["full"].astype(np.float64) - ref).max() <= 1e-5 * scale


def test_q_gradient_leaves_vs_rho_gradients_unchanged():
    d, shots = _case(5, nx=50, ny=40, nt=150, fdo=4, L=2, fs=1, fw=6)
    obs = _obs(d, shots)
    outs = []
    for gq in (0, 1):
        p = _params(d)
        p.grad_q = gq
        with dsh.Engine(p) as e:
            e.set_model(d["vs"], d["rho"], d["qs"])
            outs.append(e.gradient(shots, obs))
            if not gq:
                with pytest.raises(dsh.DshError):
                    e.gradient_q()
    for k in ("g_vs", "g_rho"):
        assert np.array_equal(outs[0][k], outs[1][k])


def test_q_gradient_rejected_for_elastic_models():
    with pytest.raises(dsh.DshError):
        dsh.Engine(dsh.make_params(nx=40, ny=30, nt=10, dh=0.5, dt=1e-4, l=0, grad_q=1))
