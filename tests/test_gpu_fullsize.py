"""The benchmark workloads at their full sizes, where the CPU oracle is too
slow for a whole gradient, checked through properties that do not depend on
the size:

* 500 x 200, FDORDER 4, NT 2000 (forward modelling): small enough for the
  oracle itself — the seismograms are bit-identical to it;
* 2000 x 800, FDORDER 8, L 3, NT 6000 (one-shot viscoelastic gradient):
  doubling the source amplitude and the observed data doubles every
  wavefield, so the eprecond-scaled gradient, a ratio of correlations, is
  unchanged and the misfit is 4x — up to rounding: a factor 2 commutes with
  every float operation except where values ahead of the wavefront underflow,
  and from there the two runs part at the last bit (relative L2 of the
  gradients ~1e-4 on a 300 x 200 case run by the oracle); the gradient with
  checkpoint-and-recompute equals the one with full storage bit for bit;
* 1000 x 300, FDORDER 8, L 2, NT 4000, 64 shots: the gradient is the same
  bit for bit whether the shots advance 64 or 16 at a time (each shot's
  fields are independent and the shot sum runs in shot order either way).
"""
import numpy as np
import pytest

import dsh
import oracle as O
from dsh import configs

pytestmark = pytest.mark.gpu


def test_full_size_forward_matches_oracle():
    cfg = configs.config1()
    p = cfg["params"]
    sh = cfg["shots"][0]
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["vs"], cfg["rho"], None)
        seis = e.forward([sh])[0]
    m = O.Model(nx=p["nx"], ny=p["ny"], nt=p["nt"], dh=p["dh"], dt=p["dt"], vs=cfg["vs"], rho=cfg["rho"], qs=None,
                fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=0, fl=(), fpml=p["fpml"],
                damping=p["damping"])
    o = O.Oracle(m, "port")
    ref = o.forward(sh.srcpos, sh.recpos)
    o.close()
    assert np.array_equal(seis, ref)


def _scaled(shot, factor):
    sp = shot.srcpos.copy()
    sp[5] *= np.float32(factor)                # amplitude row of the source table
    return dsh.Shot(sp, shot.recpos)


def test_full_size_gradient_scaling_and_checkpointing():
    cfg = configs.config2()
    p = cfg["params"]
    sh = cfg["shots"][0]
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
        obs = e.forward([sh])
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        g1 = e.gradient([sh], obs)
        g2 = e.gradient([_scaled(sh, 2.0)], [(o * np.float32(2.0)).astype(np.float32) for o in obs])
        full_ckpt = e.stats()["checkpoint_interval"]
    assert np.isfinite(g1["g_vs"]).all() and np.abs(g1["g_vs"]).max() > 0
    for k in ("g_vs", "g_rho"):
        a, b = g1[k].astype(np.float64), g2[k].astype(np.float64)
        rel = float(np.linalg.norm(a - b) / np.linalg.norm(a))
        assert rel < 1e-3, (k, rel)
    assert g2["l2"] == pytest.approx(4.0 * g1["l2"], rel=1e-5)
    # the same gradient under a memory budget that forces checkpoint-and-recompute
    with dsh.Engine(dsh.make_params(**dict(p, mem_budget=16 << 30))) as e:
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        gc = e.gradient([sh], obs)
        ckpt = e.stats()["checkpoint_interval"]
    assert full_ckpt == 0 and ckpt > 0
    assert np.array_equal(gc["g_vs"], g1["g_vs"]) and np.array_equal(gc["g_rho"], g1["g_rho"])


def test_full_size_64_shots_independent_of_batching():
    cfg = configs.config3()
    p = cfg["params"]
    shots = cfg["shots"]
    assert len(shots) == 64
    out = {}
    for per in (64, 16):
        with dsh.Engine(dsh.make_params(**dict(p, max_shots=per))) as e:
            e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
            obs = e.forward(shots)
            e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
            out[per] = e.gradient(shots, obs)
    assert np.array_equal(out[64]["g_vs"], out[16]["g_vs"]) and np.array_equal(out[64]["g_rho"], out[16]["g_rho"])
    assert out[64]["l2"] == pytest.approx(out[16]["l2"], rel=1e-12)
