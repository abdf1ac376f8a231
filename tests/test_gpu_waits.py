"""Bounded waits: every wait of the engine, on the device and on the host,
has a limit, and running into it returns DSH_ERR_TIMEOUT (-6) with the
context still usable.  No wait is made to hang and nothing faults: the
limits are set so small that a healthy run reaches them.

* device: the persistent launch's grid barrier polls a generation word; with
  a limit of one poll, blocks that arrive before the last one give up, set
  the error bit and leave their time loop, and the call reports the expiry;
* host: the waits for the context's stream poll an event against a
  wall-clock limit; with 0.1 ms the first wait of a long forward pass
  expires and the call returns while the device finishes the pass.
After either, a call with the default limits gives exactly the seismograms
of a fresh context."""
import numpy as np
import pytest

import dsh
from dsh import configs

pytestmark = pytest.mark.gpu

TIMEOUT = -6


def _fresh(cfg, shots, **extra):
    with dsh.Engine(dsh.make_params(**dict(cfg["params"], **extra))) as e:
        e.set_model(cfg["vs"], cfg["rho"], cfg.get("qs") if cfg["params"].get("l") else None)
        return e.forward(shots)


def test_device_barrier_limit_expires_and_context_recovers():
    cfg = configs.config1(nt=300)            # 500 x 200: 100 tiles, one wave -> persistent launch
    shots = cfg["shots"]
    ref = _fresh(cfg, shots)
    with dsh.Engine(dsh.make_params(**cfg["params"])) as e:
        e.set_model(cfg["vs"], cfg["rho"], None)
        e.set_step_variant(3)
        e.set_wait_limits(device_polls=1)
        with pytest.raises(dsh.DshError) as ei:
            e.forward(shots)
        assert ei.value.code == TIMEOUT
        e.set_wait_limits()                  # defaults again
        out = e.forward(shots)
        assert np.array_equal(out[0], ref[0])
        e.set_step_variant(-1)
        assert np.array_equal(e.forward(shots)[0], ref[0])


def test_host_wait_limit_expires_and_context_recovers():
    cfg = configs.config2(nt=1500, nx=1000, ny=400, dh=0.5)
    shots = cfg["shots"]
    ref = _fresh(cfg, shots)
    with dsh.Engine(dsh.make_params(**cfg["params"])) as e:
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        e.set_wait_limits(host_seconds=1e-4)
        with pytest.raises(dsh.DshError) as ei:
            e.forward(shots)
        assert ei.value.code == TIMEOUT
        e.set_wait_limits()
        out = e.forward(shots)
    assert np.array_equal(out[0], ref[0])


def test_batch_host_wait_limit_expires_and_batch_recovers():
    cfg = configs.config1(nt=1200)
    models = [cfg, dict(cfg, params=dict(cfg["params"], nt=900))]
    shots = [cfg["shots"], cfg["shots"]]
    ref = [_fresh(m, s) for m, s in zip(models, shots)]
    with dsh.Batch([dsh.make_params(**m["params"]) for m in models]) as b:
        for k, m in enumerate(models):
            b.set_model(k, m["vs"], m["rho"], None)
        b.set_host_timeout(1e-4)
        with pytest.raises(dsh.DshError) as ei:
            b.forward(shots)
        assert ei.value.code == TIMEOUT
        b.set_host_timeout(0)
        out = b.forward(shots)
    for k in range(2):
        assert np.array_equal(out[k][0], ref[k][0])


def test_gemm_mbarrier_limit_expires_and_next_call_is_exact():
    """The tensor-core GEMM's pipeline waits (TMA producer, MMA issuer,
    epilogue) poll an mbarrier at most a run-time number of times.  With one
    poll they expire on a healthy run: the CTAs record DSH_NN_ERR_TIMEOUT,
    stop issuing, let the copies and multiply operations already issued
    finish, free their tensor memory and exit.  A following call with the
    default limit gives the exact product."""
    torch = pytest.importorskip("torch")
    from dsh import nn

    rng = np.random.default_rng(3)
    M, N, K = 512, 128, 2048
    A = torch.tensor(rng.standard_normal((M, K)), dtype=torch.float32).to(torch.bfloat16).cuda()
    B = torch.tensor(rng.standard_normal((N, K)), dtype=torch.float32).to(torch.bfloat16).cuda()
    ctx = nn.Ctx(torch)
    c = torch.zeros(M, N, device="cuda")
    try:
        nn.set_wait_limit(1)
        ctx.gemm(M, N, K, A, K, B, K, c32=c)
        torch.cuda.synchronize()
        assert int(ctx.err.item()) == TIMEOUT
    finally:
        nn.set_wait_limit(0)
    ctx.err.zero_()
    ctx.gemm(M, N, K, A, K, B, K, c32=c)
    ctx.check()
    ref = A.float() @ B.float().t()
    assert float((c - ref).abs().max()) <= 1e-5 * float(ref.abs().max())
