"""Uneven multi-model batches (dsh_batch): every model of a batch advanced by
one velocity and one stress launch per register class and step (or one
launch holding every body) must give exactly the seismograms of its own
single-model context, which the parity tests tie to the reference; every
tile-shape variant must agree bit for bit; the autotuner must report its
timings and pick the fastest."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import oracle_model

pytestmark = pytest.mark.gpu


def _model(seed, nx, ny, nt, fdo, L, nshots, pad_receiver=False):
    rng = np.random.default_rng(seed)
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32) if L else None
    dt = float(np.float32(0.8 * dsh.dt_limit(fdo, 1, 0.5, float(vs.max()) * 1.1)))
    p = dict(nx=nx, ny=ny, nt=nt, dh=0.5, dt=dt, fdorder=fdo, maxrelerror=1, fw=8, free_surf=1, l=L,
             fl=(7.5, 30.0)[:L], damping=float(vs.max()), fpml=30.0, eprecond=1, max_shots=nshots + 1)
    shots = []
    for s in range(nshots):
        sp = dsh.point_source(int(rng.integers(3, nx - 2)), 2 + s % 3, 45.0)
        rec_i = rng.integers(1, nx + 1, 6)
        rec_j = [1, 1, 2, ny, max(1, ny // 2), 0 if pad_receiver else 1]
        shots.append(dsh.Shot(sp, np.array([rec_i, rec_j], np.int32)))
    return dict(params=p, vs=vs, rho=rho, qs=qs, shots=shots)


def _batch_models():
    # uneven sizes (widths not multiples of 128, one wider than 128), FDORDER 4/6/8,
    # elastic and viscoelastic, different DT and NT, 1-4 shots, one model with a
    # receiver on the padding row (separate injection/sampling launch)
    return [_model(1, 70, 40, 90, 4, 0, 3), _model(2, 131, 33, 140, 8, 2, 2), _model(3, 50, 61, 120, 6, 2, 4),
            _model(4, 96, 24, 90, 8, 0, 1, pad_receiver=True), _model(5, 45, 45, 60, 6, 0, 2)]


def _single(m):
    with dsh.Engine(dsh.make_params(**m["params"])) as e:
        e.set_model(m["vs"], m["rho"], m["qs"])
        return e.forward(m["shots"])


def _run_batch(models, variant=None):
    with dsh.Batch([dsh.make_params(**m["params"]) for m in models]) as b:
        if variant is not None:
            b.set_variant(*variant)
        for k, m in enumerate(models):
            b.set_model(k, m["vs"], m["rho"], m["qs"])
        out = b.forward([m["shots"] for m in models])
        return out, b.stats()


def test_batch_matches_single_model_contexts():
    models = _batch_models()
    out, st = _run_batch(models)
    for m, seis in zip(models, out):
        ref = _single(m)
        assert len(seis) == len(ref)
        for a, b in zip(seis, ref):
            assert np.array_equal(a, b)
    assert st["phases"] == len({m["params"]["nt"] for m in models})
    assert st["point_updates"] == sum(m["params"]["nx"] * m["params"]["ny"] * m["params"]["nt"] * len(m["shots"])
                                      for m in models)
    # completion times follow NT
    nts = [m["params"]["nt"] for m in models]
    ms = st["model_ms"]
    assert ms[int(np.argmax(nts))] == pytest.approx(st["ms_total"])
    assert all(ms[i] <= ms[j] + 1e-6 for i in range(len(nts)) for j in range(len(nts)) if nts[i] < nts[j])


def test_batch_matches_reference_oracle():
    models = _batch_models()[:2]
    out, _ = _run_batch(models)
    for m, seis in zip(models, out):
        d = dict(m["params"], vs=m["vs"], rho=m["rho"], qs=m["qs"])
        d.pop("max_shots")
        mo = oracle_model(d)
        for sh, s_gpu in zip(m["shots"], seis):
            o = O.Oracle(mo, "port")
            ref = o.forward(sh.srcpos, sh.recpos)
            o.close()
            assert np.array_equal(s_gpu, ref)


@pytest.mark.parametrize("v", [0, 1, 2, 3])
@pytest.mark.parametrize("s", [0, 1, 2, 3])
def test_tile_variants_identical(v, s):
    models = _batch_models()
    base, _ = _run_batch(models, (0, 0))
    out, st = _run_batch(models, (v, s))
    assert (st["v_variant"], st["s_variant"]) == (v, s)
    for x, y in zip(out, base):
        for a, b in zip(x, y):
            assert np.array_equal(a, b)


def test_autotuner_times_every_variant():
    models = _batch_models()
    _, st = _run_batch(models)
    assert all(t > 0 for t in st["v_ms"]) and all(t > 0 for t in st["s_ms"])
    assert st["v_ms"][st["v_variant"]] == min(st["v_ms"])
    assert st["s_ms"][st["s_variant"]] == min(st["s_ms"])


def test_batch_reuse_and_fewer_shots():
    """A second run with other shot counts (one model skipped) rebuilds the
    block maps and still matches the single-model contexts."""
    models = _batch_models()
    with dsh.Batch([dsh.make_params(**m["params"]) for m in models]) as b:
        for k, m in enumerate(models):
            b.set_model(k, m["vs"], m["rho"], m["qs"])
        b.forward([m["shots"] for m in models])
        sub = [m["shots"][:1] for m in models]
        sub[2] = []
        out = b.forward(sub)
    for k, m in enumerate(models):
        if k == 2:
            assert out[k] == []
            continue
        ref = _single(dict(m, shots=m["shots"][:1]))
        assert np.array_equal(out[k][0], ref[0])


@pytest.mark.parametrize("var", ["DSH_MULTI_ARGS_DEVICE", "DSH_MULTI_MIXED"])
def test_other_launch_forms_in_subprocess(var):
    """Batches of up to 36 models pass their StepArgs in the kernels'
    parameter space and launch one kernel per register class; larger ones
    read them from a device array in one kernel holding every body.  With
    DSH_MULTI_ARGS_DEVICE=1 every batch takes the device-array path, with
    DSH_MULTI_MIXED=1 the parameter-space kernel holding every body (both
    read once per process, so in a child process): the same results bit for
    bit."""
    import os
    import subprocess
    import sys

    env = dict(os.environ, **{var: "1"})
    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-p', 'no:cacheprovider', '-m', 'gpu', 'tests/test_gpu_batch.py', "
            "'-k', 'not subprocess']))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
