"""The FWI loop's vector steps on the device (dsh_lbfgs_direction_device,
dsh_pcg_direction_device) against the host versions (dsh_lbfgs_direction,
dsh_pcg_direction, the latter pinned to the reference's PCG.c in
tests/test_fwi_host.py): the device sums every dot product in double over a
fixed partition while the host adds in vector order (double for L-BFGS,
float as the reference for PCG), so the results agree to float rounding, and
the device results are reproducible bit for bit."""
import numpy as np
import pytest

from dsh import fwi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("count", [0, 1, 3, 5])
def test_lbfgs_direction_device_matches_host(count):
    n = 1200 * 400                                  # the learned-FWI grid
    rng = np.random.default_rng(count)
    q = rng.standard_normal(n).astype(np.float32)
    S = (1e-3 * rng.standard_normal((count, n))).astype(np.float32)
    Y = (S * rng.uniform(0.5, 2.0, (count, 1)) + 1e-4 * rng.standard_normal((count, n))).astype(np.float32)
    host = fwi.lbfgs_direction(S, Y, q)
    St, Yt, qt = (torch.from_numpy(x).cuda() for x in (S, Y, q))
    dev = fwi.lbfgs_direction_device(torch, St if count else None, Yt if count else None, qt)
    dev2 = fwi.lbfgs_direction_device(torch, St if count else None, Yt if count else None, qt)
    torch.cuda.synchronize()
    d = dev.cpu().numpy()
    assert np.array_equal(d, dev2.cpu().numpy())
    if count == 0:
        assert np.array_equal(d, q)
    assert _rel(d, host) < 1e-5, _rel(d, host)


@pytest.mark.parametrize("beta", ["fletcher_reeves", "polak_ribiere", "hestenes_stiefel", "dai_yuan"])
def test_pcg_direction_device_matches_host(beta):
    n = 1200 * 400
    rng = np.random.default_rng(7)
    g_new = rng.standard_normal((2, n)).astype(np.float32)
    g_old = (0.8 * g_new + 0.3 * rng.standard_normal((2, n))).astype(np.float32)
    d_old = rng.standard_normal((2, n)).astype(np.float32)
    d_host, b_host = fwi.pcg_direction(g_new, g_old, d_old, beta)
    dt = torch.from_numpy(d_old.copy()).cuda()
    d_dev, b_dev = fwi.pcg_direction_device(torch, torch.from_numpy(g_new).cuda(), torch.from_numpy(g_old).cuda(),
                                            dt, beta)
    torch.cuda.synchronize()
    # the exact betas, in double: the device's double sums agree to float rounding;
    # the host adds in float in vector order as the reference does (error ~ sqrt(n) 2^-24)
    a, b, d = (x.astype(np.float64) for x in (g_new, g_old, d_old))
    num = {"fletcher_reeves": (a * a).sum(1), "polak_ribiere": (a * (a - b)).sum(1),
           "hestenes_stiefel": (-a * (a - b)).sum(1), "dai_yuan": (-a * a).sum(1)}[beta]
    den = {"fletcher_reeves": (b * b).sum(1), "polak_ribiere": (b * b).sum(1),
           "hestenes_stiefel": (d * (a - b)).sum(1), "dai_yuan": (d * (a - b)).sum(1)}[beta]
    exact = num / den
    if beta == "polak_ribiere":
        exact = np.maximum(exact, 0.0)
    assert np.allclose(b_dev.cpu().numpy(), exact, rtol=1e-6, atol=1e-9), (b_dev, exact)
    assert np.allclose(b_host, exact, rtol=1e-3, atol=1e-6), (b_host, exact)
    assert _rel(d_dev.cpu().numpy(), d_host) < 1e-3


def test_plain_fwi_with_device_vectors_follows_host_path():
    """The plain L-BFGS loop with the gradient kept in HBM and the two-loop
    recursion on the device takes the same steps as the host loop (the
    directions differ at float rounding only): step lengths and misfits
    within 1e-4 relative."""
    from dsh import configs

    cfg = configs.config5(seed=11, nx=160, ny=80, nt=500, nshots=6, ntr=60)
    cfg["params"].update(fdorder=4, l=0, fl=())
    cfg["qs"] = None
    prob = fwi.Problem(cfg, test_shots=2)
    try:
        host, _ = fwi.run(prob, 3, method="plain", eps_scale=0.02)
        dev, _ = fwi.run(prob, 3, method="plain", eps_scale=0.02, torch=torch, device_vectors=True)
    finally:
        prob.close()
    assert len(host) == len(dev)
    for a, b in zip(host, dev):
        if "eps" in a:       # the parabolic step follows the test misfits, which differ at rounding
            assert b["eps"] == pytest.approx(a["eps"], rel=1e-4)
        assert b["misfit"] == pytest.approx(a["misfit"], rel=1e-4)
    assert dev[-1]["misfit"] < 0.9 * dev[0]["misfit"]
