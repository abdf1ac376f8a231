"""Parity with the CPU oracle at the full grid sizes of the benchmark
configurations.  Every grid keeps its NX x NY, FDORDER, L, receiver layout and
shot count; only NT is cut (to 300-400 steps) so that the oracle, which runs
the reference's loops on the host, finishes in well under a minute.  The
oracle's grid loops are threaded (each point is computed on its own, so the
thread count does not change a bit).

* 2000 x 800, FDORDER 8, L 3 (one-shot viscoelastic gradient): seismograms,
  Ws, Wr, the per-shot preconditioned g_u and g_rho and the converted g_vs,
  g_rho bit-identical to the oracle's shot loop (src/denise.c:1179-1346,
  :1493-1651), both with full storage and with checkpoint-and-recompute;
* 1000 x 300, FDORDER 8, L 2, 64 shots in one launch, checkpoints every
  ceil(sqrt(NT)) steps: slots 0 and 63 bit-identical to the oracle; the shot
  sum and conversion of all 64 slots equal the oracle's conversion of the
  per-shot fields summed in shot order;
* the uneven 32-model batch, one velocity and one stress launch per step for
  all 597 shots: the largest model (1659 x 458, FDORDER 8, L 2), first and
  last shot, and the first shot of the largest model of every other FDORDER /
  L class, bit-identical to the oracle's forward loop;
* 1200 x 400, FDORDER 8, L 3, 32 shots (the learned-preconditioner problem):
  slots 0 and 31 bit-identical, misfit within the float summation bound.

The misfit is summed in double on the device and in float by the reference;
it is compared within the float summation bound (n-1) 2^-24 (relative, all
terms non-negative)."""
import math

import numpy as np
import pytest

import dsh
import oracle as O
from dsh import configs

pytestmark = pytest.mark.gpu


def _omodel(p, vs, rho, qs):
    return O.Model(nx=p["nx"], ny=p["ny"], nt=p["nt"], dh=p["dh"], dt=p["dt"], vs=vs, rho=rho,
                   qs=qs if p["l"] else None, fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=p["l"],
                   fl=tuple(p.get("fl", ())), fpml=p["fpml"], damping=p["damping"])


def _same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not np.array_equal(a, b):
        bad = int(np.count_nonzero(a != b))
        scale = float(np.abs(b).max()) or 1.0
        raise AssertionError(f"{what}: {bad} of {a.size} values differ, max |diff| / max |ref| = "
                             f"{float(np.abs(a.astype(np.float64) - b).max()) / scale:.3e}")


def _l2_close(got, ref, nterms, what="l2"):
    assert abs(got - ref) <= max(nterms - 1, 1) * 2.0 ** -24 * abs(ref), (what, got, ref)


def _oracle_shot(m, shot, obs):
    o = O.Oracle(m, "port")
    try:
        return o.shot_gradient(shot.srcpos, shot.recpos, obs)
    finally:
        o.close()


def _oracle_convert(m, su, sr):
    o = O.Oracle(m, "port")
    try:
        return o.convert(su, sr)
    finally:
        o.close()


def test_c2_gradient_full_grid_vs_oracle():
    cfg = configs.config2(nt=400)
    p, sh = cfg["params"], cfg["shots"][0]
    runs = {}
    for name, extra in (("full", {}), ("checkpointed", {"ckpt_every": 20})):
        with dsh.Engine(dsh.make_params(**dict(p, **extra))) as e:
            if name == "full":
                e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
                obs = e.forward([sh])
            e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
            out = e.gradient([sh], obs, want_seis=True, want_energy=True)
            out["g_u"], out["g_rho_shot"] = e.field("g_u"), e.field("g_rho")
            out["ckpt"] = e.stats()["checkpoint_interval"]
        runs[name] = out
    assert runs["full"]["ckpt"] == 0 and runs["checkpointed"]["ckpt"] == 20
    m = _omodel(p, cfg["vs"], cfg["rho"], cfg["qs"])
    ref = _oracle_shot(m, sh, obs[0])
    gv, gr = _oracle_convert(m, ref["g_u"], ref["g_rho"])
    for name, out in runs.items():
        _same(out["seis"][0], ref["seis"], f"{name} seismograms")
        _same(out["Ws"][0], ref["Ws"], f"{name} Ws")
        _same(out["Wr"][0], ref["Wr"], f"{name} Wr")
        _same(out["g_u"], ref["g_u"], f"{name} per-shot g_u")
        _same(out["g_rho_shot"], ref["g_rho"], f"{name} per-shot g_rho")
        _same(out["g_vs"], gv, f"{name} g_vs")
        _same(out["g_rho"], gr, f"{name} g_rho")
        _l2_close(out["l2"], ref["l2"], obs[0].size, f"{name} l2")
    assert np.abs(gv).max() > 0


def test_c3_64_shot_launch_full_grid_vs_oracle():
    nt = 300
    cfg = configs.config3(nt=nt)
    p, shots = cfg["params"], cfg["shots"]
    assert len(shots) == 64
    every = math.ceil(math.sqrt(nt))
    with dsh.Engine(dsh.make_params(**dict(p, max_shots=64, ckpt_every=every))) as e:
        e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
        obs = e.forward(shots)
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        out = e.gradient(shots, obs, want_seis=True, want_energy=True)
        assert e.stats()["checkpoint_interval"] == every
        g_u = [e.field("g_u", shot=k) for k in range(64)]
        g_r = [e.field("g_rho", shot=k) for k in range(64)]
        shot_l2 = e.shot_misfits(64)
    m = _omodel(p, cfg["vs"], cfg["rho"], cfg["qs"])
    for k in (0, 63):
        ref = _oracle_shot(m, shots[k], obs[k])
        _same(out["seis"][k], ref["seis"], f"slot {k} seismograms")
        _same(out["Ws"][k], ref["Ws"], f"slot {k} Ws")
        _same(out["Wr"][k], ref["Wr"], f"slot {k} Wr")
        _same(g_u[k], ref["g_u"], f"slot {k} g_u")
        _same(g_r[k], ref["g_rho"], f"slot {k} g_rho")
        _l2_close(shot_l2[k], ref["l2"], obs[k].size, f"slot {k} l2")
    # the shot sum runs in shot order in float (src/denise.c:1689-1694)
    su = np.zeros_like(g_u[0])
    sr = np.zeros_like(g_r[0])
    for k in range(64):
        su = (su + g_u[k]).astype(np.float32)
        sr = (sr + g_r[k]).astype(np.float32)
    gv, gr = _oracle_convert(m, su, sr)
    _same(out["g_vs"], gv, "64-shot g_vs")
    _same(out["g_rho"], gr, "64-shot g_rho")
    assert out["l2"] == pytest.approx(float(np.sum(shot_l2)), rel=1e-12)


def test_c4_uneven_batch_full_grids_vs_oracle():
    models = configs.config4(nt_scale=0.02)
    assert len(models) == 32
    with dsh.Batch([dsh.make_params(**m["params"]) for m in models]) as b:
        for k, m in enumerate(models):
            b.set_model(k, m["vs"], m["rho"], m["qs"])
        out = b.forward([m["shots"] for m in models])
    size = [m["params"]["nx"] * m["params"]["ny"] for m in models]
    big = int(np.argmax(size))
    checks = [(big, 0), (big, len(models[big]["shots"]) - 1)]
    for fdo in (4, 6, 8):
        for L in (0, 2):
            ks = [k for k, m in enumerate(models)
                  if m["params"]["fdorder"] == fdo and m["params"]["l"] == L and k != big]
            if ks:
                checks.append((max(ks, key=lambda k: size[k]), 0))
    assert models[big]["params"]["nx"] == 1659 and models[big]["params"]["ny"] == 458
    for k, s in checks:
        m = models[k]
        o = O.Oracle(_omodel(m["params"], m["vs"], m["rho"], m["qs"]), "port")
        sh = m["shots"][s]
        ref = o.forward(sh.srcpos, sh.recpos)
        o.close()
        _same(out[k][s], ref, f"{m['name']} shot {s}")


def test_c5_32_shot_gradient_full_grid_vs_oracle():
    cfg = configs.config5(nt=300)
    p, shots = cfg["params"], cfg["shots"]
    assert len(shots) == 32 and p["max_shots"] == 32
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
        obs = e.forward(shots)
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        out = e.gradient(shots, obs, want_seis=True, want_energy=True)
        g_u = {k: e.field("g_u", shot=k) for k in (0, 31)}
        g_r = {k: e.field("g_rho", shot=k) for k in (0, 31)}
        shot_l2 = e.shot_misfits(32)
    m = _omodel(p, cfg["vs"], cfg["rho"], cfg["qs"])
    for k in (0, 31):
        ref = _oracle_shot(m, shots[k], obs[k])
        _same(out["seis"][k], ref["seis"], f"slot {k} seismograms")
        _same(out["Ws"][k], ref["Ws"], f"slot {k} Ws")
        _same(out["Wr"][k], ref["Wr"], f"slot {k} Wr")
        _same(g_u[k], ref["g_u"], f"slot {k} g_u")
        _same(g_r[k], ref["g_rho"], f"slot {k} g_rho")
        _l2_close(shot_l2[k], ref["l2"], obs[k].size, f"slot {k} l2")
