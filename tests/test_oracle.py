"""The CPU oracle is pinned before it is trusted: the repository's C
restatement must reproduce, bit for bit, the golden fixtures that the
reference's own compiled functions produced (tests/golden/make_golden.py),
and — where the reference tree has been compiled here — match the reference
on further randomised cases across every FD order, relaxation count and
boundary setting."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, oracle_model

import oracle as O


def _port_run(d):
    m = oracle_model(d)
    o = O.Oracle(m, "port")
    g = o.shot_gradient(d["srcpos"], d["recpos"], d["obs"])
    gv, gr = o.convert(g["g_u"], g["g_rho"])
    adj = (o.field("vy"), o.field("sxy"), o.field("syz"))
    o.close()
    o = O.Oracle(m, "port")
    o.forward(d["srcpos"], d["recpos"], hessian=True)
    hv, hr = o.hessian_out()
    fwd_vy = o.field("vy")
    o.close()
    return g, gv, gr, adj, hv, hr, fwd_vy


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_restatement_matches_reference_golden(name):
    d = golden(name)
    g, gv, gr, adj, hv, hr, fwd_vy = _port_run(d)
    for key, val in [("seis", g["seis"]), ("res", g["res"]), ("Ws", g["Ws"]), ("Wr", g["Wr"]), ("We", g["We"]),
                     ("g_u", g["g_u"]), ("g_rho", g["g_rho"]), ("g_vs", gv), ("g_rhoc", gr), ("adj_vy", adj[0]),
                     ("adj_sxy", adj[1]), ("adj_syz", adj[2]), ("hess_vs", hv), ("hess_rho", hr), ("fwd_vy", fwd_vy)]:
        assert np.array_equal(val, d[key]), f"{name}: {key} differs from the reference"
    assert g["l2"] == float(d["l2"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_restatement_close_to_fp32(name):
    """FP32 error statement: the FP32 run against an FP64 run of the same
    stencil with the same (FP32) coefficients."""
    d = golden(name)
    m = oracle_model(d)
    o = O.Oracle(m, "port", fp64=True)
    s64 = o.forward(d["srcpos"], d["recpos"])
    o.close()
    rel = np.linalg.norm(d["seis_plain"].astype(np.float64) - s64) / np.linalg.norm(s64)
    assert rel < 1e-5, rel


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_gradient_error_statement(name):
    """The FP32 gradient (the reference's, which the GPU reproduces bit for
    bit) against the FP64 restatement's on the same inputs: relative L2
    below 1e-5 for seismograms and the preconditioned per-shot gradients
    (measured 0.5e-6 to 9.3e-6 for the gradients, about 2e-7 for the
    seismograms)."""
    d = golden(name)
    o = O.Oracle(oracle_model(d), "port", fp64=True)
    g = o.shot_gradient(d["srcpos"], d["recpos"], d["obs"])
    gu64, gr64 = o.field("g_u", f64=True), o.field("g_rho", f64=True)
    o.close()
    rel = lambda a, b: np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b)
    assert rel(d["seis"], g["seis"]) < 1e-6
    assert rel(d["g_u"], gu64) < 1e-5 and rel(d["g_rho"], gr64) < 1e-5


def _rand_model(seed, nx, ny, nt, fdo, L, fs, fw):
    rng = np.random.default_rng(seed)
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    return O.Model(nx=nx, ny=ny, nt=nt, dh=0.5, dt=2e-4, vs=vs, rho=rho, qs=qs, fdorder=fdo, fw=fw, free_surf=fs,
                   l=L, fl=(7.5, 30.0, 120.0, 240.0)[:L], fpml=30.0, damping=float(vs.max()))


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
@pytest.mark.parametrize("fdo", [2, 4, 6, 8, 10, 12])
@pytest.mark.parametrize("L", [0, 1, 4])
def test_restatement_matches_reference_random(fdo, L):
    m = _rand_model(100 + fdo + 10 * L, 37, 29, 90, fdo, L, fs=(fdo // 2) % 2, fw=7)
    src = np.zeros((8, 1), np.float32)
    src[:, 0] = [18, 2, 0, -0.01, 60.0, 1.0, 0, 3]
    rec = np.array([[4, 10, 20, 33], [1, 1, 5, 20]], np.int32)
    outs = {}
    for kind in ("ref", "port"):
        o = O.Oracle(m, kind)
        seis = o.forward(src, rec, store=True)
        obs = (seis * np.float32(0.7)).astype(np.float32)
        _, l2 = o.residual(obs)
        o.adjoint()
        o.eprecond_scale()
        outs[kind] = dict(seis=seis, l2=l2, gu=o.field("g_u"), gr=o.field("g_rho"), We=o.field("We"),
                          vy=o.field("vy"), hc=o.hc()[1:], cn=o.cnorm(),
                          pml=np.concatenate([o.pml(n) for n in O.PML[:12]]))
        if L:
            outs[kind]["r"] = o.field("r", L - 1)
            outs[kind]["sls"] = np.concatenate(o.sls())
        o.close()
    for k in outs["ref"]:
        assert np.array_equal(outs["ref"][k], outs["port"][k]), k


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
@pytest.mark.parametrize("ep", [0, 1, 3])
def test_restatement_eprecond_variants(ep):
    m = _rand_model(7, 44, 30, 100, 4, 0, fs=1, fw=6)
    m.eprecond = ep
    src = np.zeros((8, 1), np.float32)
    src[:, 0] = [20, 2, 0, -0.01, 60.0, 1.0, 0, 3]
    rec = np.array([[5, 15, 25, 35], [1, 1, 1, 1]], np.int32)
    outs = {}
    for kind in ("ref", "port"):
        o = O.Oracle(m, kind)
        obs = (o.forward(src, rec) * np.float32(0.5)).astype(np.float32)
        o.close()
        o = O.Oracle(m, kind)
        g = o.shot_gradient(src, rec, obs)
        outs[kind] = (g["We"], g["g_u"], g["g_rho"], g["Wr"])
        o.close()
    for a, b in zip(outs["ref"], outs["port"]):
        assert np.array_equal(a, b)
