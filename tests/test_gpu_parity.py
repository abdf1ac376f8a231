"""Parity of the CUDA path (through the C ABI) with the reference.

Bit-exact: seismograms, per-shot energies, preconditioned and converted
gradients, Hessian diagonal and final wavefields, against (a) the golden
fixtures that the reference's own compiled functions produced and (b) the CPU
oracle (the restatement pinned to those fixtures) on randomised cases over
every FD order, relaxation count, boundary setting, grid shapes that are not a
multiple of the 4-point vector width, and multi-shot batches.  The L2 misfit
is summed in double on the device while the reference adds its n terms one by
one in float, so it is compared within the float summation bound
(n-1)*2^-24 relative (non-negative terms)."""
import os

import numpy as np
import pytest

import dsh
import oracle as O
from conftest import GOLDEN_CASES, golden, oracle_model

pytestmark = pytest.mark.gpu

def l2_tol(nterms):
    return max(nterms - 1, 1) * 2.0 ** -24


def engine_from(d, max_shots=1, **kw):
    p = dsh.make_params(nx=int(d["nx"]), ny=int(d["ny"]), nt=int(d["nt"]), dh=float(d["dh"]), dt=float(d["dt"]),
                        fdorder=int(d["fdorder"]), fw=int(d["fw"]), free_surf=int(d["free_surf"]), l=int(d["l"]),
                        fl=tuple(float(x) for x in d["fl"]), damping=float(d["damping"]), fpml=float(d["fpml"]),
                        max_shots=max_shots, **kw)
    e = dsh.Engine(p)
    e.set_model(d["vs"], d["rho"], d["qs"] if int(d["l"]) else None)
    return e


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_forward(name):
    d = golden(name)
    shot = dsh.Shot(d["srcpos"], d["recpos"])
    with engine_from(d) as e:
        seis = e.forward([shot])[0]
        assert e.stats()["kernel_launches"] > 0
    assert np.array_equal(seis, d["seis_plain"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_gradient(name):
    d = golden(name)
    shot = dsh.Shot(d["srcpos"], d["recpos"])
    with engine_from(d) as e:
        out = e.gradient([shot], [d["obs"]], want_seis=True, want_energy=True)
        end = {k: e.field(k) for k in ("vy", "sxy", "syz")}
        We = e.field("We")
        gu, gr = e.field("g_u"), e.field("g_rho")
    assert np.array_equal(out["seis"][0], d["seis"])
    assert np.array_equal(out["Ws"][0], d["Ws"])
    assert np.array_equal(out["Wr"][0], d["Wr"])
    assert np.array_equal(We, d["We"])
    assert np.array_equal(gu, d["g_u"])
    assert np.array_equal(gr, d["g_rho"])
    assert np.array_equal(out["g_vs"], d["g_vs"])
    assert np.array_equal(out["g_rho"], d["g_rhoc"])
    for k in ("vy", "sxy", "syz"):
        assert np.array_equal(end[k], d["adj_" + k]), k
    assert abs(out["l2"] - float(d["l2"])) <= l2_tol(d["obs"].size) * float(d["l2"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_hessian(name):
    d = golden(name)
    shot = dsh.Shot(d["srcpos"], d["recpos"])
    with engine_from(d) as e:
        hv, hr = e.hessian_diag([shot])
        vy = e.field("vy")
    assert np.array_equal(hv, d["hess_vs"])
    assert np.array_equal(hr, d["hess_rho"])
    assert np.array_equal(vy, d["fwd_vy"])


def _case(seed, nx, ny, nt, fdo, L, fs, fw, nshots=1):
    rng = np.random.default_rng(seed)
    vs = (200.0 + 40.0 * rng.standard_normal((ny, nx))).clip(120, 320).astype(np.float32)
    rho = (1800.0 + 80.0 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    fl = (7.5, 30.0, 120.0, 240.0)[:L]
    d = dict(nx=nx, ny=ny, nt=nt, dh=0.5, dt=np.float32(2e-4), fdorder=fdo, fw=fw, free_surf=fs, l=L,
             fl=np.array(fl, np.float32), damping=np.float32(vs.max()), fpml=np.float32(30.0), vs=vs, rho=rho, qs=qs)
    shots = []
    for s in range(nshots):
        sp = np.zeros((8, 2), np.float32)
        sp[:, 0] = [int(rng.integers(2, nx)), 2 + s % 3, 0, -0.01, 60.0, 1.0, 0, 3]
        sp[:, 1] = [int(rng.integers(2, nx)), 1, 0, -0.012, 45.0, -0.5, 0, 3 if s % 2 == 0 else 1]
        rec = np.array([rng.integers(1, nx + 1, 5), [1, 1, 0, ny, max(1, ny // 2)]], np.int32)
        shots.append(dsh.Shot(sp, rec))
    return d, shots


def _oracle_gradient(d, shots, obs):
    """Reference shot loop on the CPU oracle: per-shot preconditioned gradients
    summed in shot order (denise.c:1689-1694), then converted."""
    m = oracle_model(d)
    su = np.zeros((m.ny, m.nx), np.float32)
    sr = np.zeros((m.ny, m.nx), np.float32)
    l2 = 0.0
    seis = []
    for sh, ob in zip(shots, obs):
        o = O.Oracle(m, "port")
        g = o.shot_gradient(sh.srcpos, sh.recpos, ob)
        su = su + g["g_u"]
        sr = sr + g["g_rho"]
        l2 += g["l2"]
        seis.append(g["seis"])
        o.close()
    o = O.Oracle(m, "port")
    gv, gr = o.convert(su, sr)
    o.close()
    return gv, gr, l2, seis


@pytest.mark.parametrize("fdo", [2, 4, 6, 8, 10, 12])
@pytest.mark.parametrize("L,fs", [(0, 1), (1, 0), (2, 1), (3, 0), (4, 1)])
def test_random_cases_vs_oracle(fdo, L, fs):
    d, shots = _case(1000 + 7 * fdo + L, nx=37 + fdo, ny=31 + L, nt=140, fdo=fdo, L=L, fs=fs, fw=6)
    m = oracle_model(d)
    o = O.Oracle(m, "port")
    seis_ref = o.forward(shots[0].srcpos, shots[0].recpos)
    o.close()
    obs = [(seis_ref * np.float32(0.6) + np.float32(1e-3)).astype(np.float32)]
    gv, gr, l2, seis = _oracle_gradient(d, shots, obs)
    with engine_from(d) as e:
        s_gpu = e.forward(shots)[0]
        out = e.gradient(shots, obs)
    assert np.array_equal(s_gpu, seis_ref)
    assert np.array_equal(out["g_vs"], gv)
    assert np.array_equal(out["g_rho"], gr)
    assert abs(out["l2"] - l2) <= l2_tol(obs[0].size) * abs(l2)


@pytest.mark.parametrize("L", [1, 2])
def test_high_q_models(L):
    """Weak attenuation (Qs 80-240, L*tau = 2L/Q down to 0.008): the
    relaxed-modulus products fipjp = muip*DT*(1+L*tau) that the stress kernel
    forms per point in the reference's float/double mix still match the
    oracle bit for bit."""
    d, shots = _case(900 + L, nx=45, ny=33, nt=140, fdo=8, L=L, fs=1, fw=6)
    d["qs"] = (d["qs"] * np.float32(4.0)).astype(np.float32)
    m = oracle_model(d)
    o = O.Oracle(m, "port")
    seis_ref = o.forward(shots[0].srcpos, shots[0].recpos)
    o.close()
    obs = [(seis_ref * np.float32(0.7)).astype(np.float32)]
    gv, gr, l2, _ = _oracle_gradient(d, shots, obs)
    with engine_from(d) as e:
        assert np.array_equal(e.forward(shots)[0], seis_ref)
        out = e.gradient(shots, obs)
    assert np.array_equal(out["g_vs"], gv) and np.array_equal(out["g_rho"], gr)


@pytest.mark.parametrize("max_shots", [1, 2, 5])
def test_multi_shot_batches(max_shots):
    d, shots = _case(77, nx=61, ny=45, nt=160, fdo=8, L=2, fs=1, fw=8, nshots=5)
    m = oracle_model(d)
    obs = []
    for sh in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sh.srcpos, sh.recpos) * np.float32(1.1)).astype(np.float32))
        o.close()
    gv, gr, l2, seis = _oracle_gradient(d, shots, obs)
    with engine_from(d, max_shots=max_shots) as e:
        fwd = e.forward(shots)
        out = e.gradient(shots, obs)
    for a, b in zip(fwd, seis):
        assert np.array_equal(a, b)
    assert np.array_equal(out["g_vs"], gv)
    assert np.array_equal(out["g_rho"], gr)
    assert abs(out["l2"] - l2) <= l2_tol(sum(o.size for o in obs)) * abs(l2)


def test_multi_shot_hessian_sum():
    """Per shot the Hessian is bit-exact; the reference chains one float
    accumulator through all shots while shots advance concurrently here, so
    the multi-shot sum agrees to float rounding."""
    d, shots = _case(78, nx=40, ny=36, nt=120, fdo=4, L=0, fs=1, fw=6, nshots=3)
    m = oracle_model(d)
    hv = np.zeros((m.ny, m.nx), np.float64)
    for sh in shots:
        with engine_from(d) as e:
            h1, _ = e.hessian_diag([sh])
        o = O.Oracle(m, "port")
        o.forward(sh.srcpos, sh.recpos, hessian=True)
        h_ref, _ = o.hessian_out()
        o.close()
        assert np.array_equal(h1, h_ref)
        hv += h1
    with engine_from(d, max_shots=3) as e:
        hs, _ = e.hessian_diag(shots)
    assert np.allclose(hs, hv, rtol=1e-5, atol=0)


@pytest.mark.parametrize("ep", [0, 3])
def test_eprecond_off_and_plessix_mulder(ep):
    """EPRECOND=0 (no energy scaling) is bit-exact; EPRECOND=3 (Plessix &
    Mulder receiver approximation, eprecond1.c:35-58) calls asinh, whose last
    bit may differ between CUDA and glibc, so it is compared to 1e-6."""
    d, shots = _case(79, nx=44, ny=30, nt=100, fdo=4, L=0, fs=1, fw=6)
    md = oracle_model(d)
    md.eprecond = ep
    o = O.Oracle(md, "port")
    obs = (o.forward(shots[0].srcpos, shots[0].recpos) * np.float32(0.5)).astype(np.float32)
    o.close()
    o = O.Oracle(md, "port")
    g = o.shot_gradient(shots[0].srcpos, shots[0].recpos, obs)
    gv0, gr0 = o.convert(g["g_u"], g["g_rho"])
    o.close()
    with engine_from(d, eprecond=ep) as e:
        out = e.gradient(shots, [obs])
    if ep == 0:
        assert np.array_equal(out["g_vs"], gv0)
        assert np.array_equal(out["g_rho"], gr0)
    else:
        assert np.allclose(out["g_vs"], gv0, rtol=1e-6, atol=1e-6 * np.abs(gv0).max())
        assert np.allclose(out["g_rho"], gr0, rtol=1e-6, atol=1e-6 * np.abs(gr0).max())


def test_unstable_model_reports_error():
    """DT far above the stability limit: the engine returns DSH_ERR_UNSTABLE
    (the reference aborts on a NaN probe, denise.c:1183-1185)."""
    d, shots = _case(80, nx=40, ny=32, nt=400, fdo=4, L=0, fs=1, fw=6)
    d["dt"] = np.float32(5e-3)
    with engine_from(d) as e:
        with pytest.raises(dsh.DshError) as ei:
            e.forward(shots)
        assert ei.value.code == -4
        # the context stays usable after the error
        d2 = dict(d)
    d2["dt"] = np.float32(2e-4)
    with engine_from(d2) as e:
        assert np.all(np.isfinite(e.forward(shots)[0]))


@pytest.mark.parametrize("nx,ny", [(70, 40), (500, 200), (1100, 300)])
def test_forward_persistent_and_pair_paths(nx, ny):
    """With DSH_PERSIST=1 (set for the GPU test run), plain forward modelling
    takes the one-launch persistent kernel when all tiles fit in one wave
    (70 x 40: 5 tiles, 500 x 200: 100 tiles whose completion flags order
    the neighbouring tiles) and the per-step kernel pair otherwise (1100 x
    300: 342 tiles); both are bit-identical to the oracle."""
    d, shots = _case(500 + nx, nx=nx, ny=ny, nt=90, fdo=8, L=2, fs=1, fw=10)
    rec = shots[0].recpos.copy()
    rec[1] = np.clip(rec[1], 1, ny)              # all receivers inside the grid: fused sampling lists
    shots = [dsh.Shot(shots[0].srcpos, rec)]
    m = oracle_model(d)
    o = O.Oracle(m, "port")
    ref = o.forward(shots[0].srcpos, shots[0].recpos)
    o.close()
    with engine_from(d) as e:
        seis = e.forward(shots)[0]
        st = e.stats()
    assert np.array_equal(seis, ref)
    tiles = ((nx + 127) // 128) * ((ny + 7) // 8)
    if tiles <= 148 and os.environ.get("DSH_PERSIST") == "1":
        assert st["kernel_launches"] <= 8      # one cooperative launch (+ counter, transpose)
    else:
        assert st["kernel_launches"] >= 2 * 90


def test_persistent_forward_in_subprocess():
    """The opt-in persistent kernel (DSH_PERSIST=1 is read once per process,
    so it runs in a child process): one cooperative launch for the whole
    forward pass, bit-identical to the oracle."""
    import subprocess
    import sys

    env = dict(os.environ, DSH_PERSIST="1")
    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-p', 'no:cacheprovider', '-m', 'gpu', "
            "'tests/test_gpu_parity.py::test_forward_persistent_and_pair_paths']))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]


def test_other_block_heights_in_subprocess():
    """The stress and velocity launches take 128 x 4-point blocks by default;
    8- and 2-row blocks (DSH_SROWS / DSH_VBROWS, read once per process, so in
    a child process) give the same results bit for bit: random cases,
    multi-shot batches and checkpointed gradients."""
    import subprocess
    import sys

    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-p', 'no:cacheprovider', '-m', 'gpu', "
            "'tests/test_gpu_parity.py::test_random_cases_vs_oracle', "
            "'tests/test_gpu_parity.py::test_multi_shot_batches', 'tests/test_gpu_checkpoint.py']))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for rows in (("8", "2"), ("2", "8")):
        env = dict(os.environ, DSH_SROWS=rows[0], DSH_VBROWS=rows[1])
        out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                             timeout=900)
        assert out.returncode == 0, rows + (out.stdout[-2000:] + out.stderr[-2000:],)


@pytest.mark.parametrize("mask", ["0", "1", "3"])
def test_l2_policies_in_subprocess(mask):
    """The stress kernel streams the memory variables (bit 0 of the L2 policy
    mask) and the model factors (bit 1) evict-first when the host finds that
    the velocity kernel's read set then stays in L2; the cache hints change no
    arithmetic.  Each mask forced through DSH_L2_STREAM (read once per
    process, so in a child process): random cases, multi-shot batches and
    checkpointed gradients bit-identical to the oracle."""
    import subprocess
    import sys

    env = dict(os.environ, DSH_L2_STREAM=mask)
    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-p', 'no:cacheprovider', '-m', 'gpu', "
            "'tests/test_gpu_parity.py::test_random_cases_vs_oracle', "
            "'tests/test_gpu_parity.py::test_multi_shot_batches', 'tests/test_gpu_checkpoint.py']))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                         timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]


def test_tma_velocity_kernel_in_subprocess():
    """The opt-in persistent velocity kernel whose stress taps the tensor-memory
    accelerator stages in shared memory (DSH_VTMA=1, read once per process, so
    in a child process): every FD order and relaxation count, multi-shot
    batches and checkpointed gradients stay bit-identical to the oracle."""
    import subprocess
    import sys

    env = dict(os.environ, DSH_VTMA="1")
    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-p', 'no:cacheprovider', '-m', 'gpu', "
            "'tests/test_gpu_parity.py::test_random_cases_vs_oracle', "
            "'tests/test_gpu_parity.py::test_multi_shot_batches', 'tests/test_gpu_checkpoint.py']))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]


def test_autotune_picks_a_variant_and_keeps_parity():
    """dsh_autotune times every applicable step-kernel variant and keeps the
    fastest; forward and gradient afterwards are still bit-identical."""
    d, shots = _case(611, nx=70, ny=40, nt=120, fdo=8, L=2, fs=1, fw=10)
    rec = shots[0].recpos.copy()
    rec[1] = np.clip(rec[1], 1, d["ny"])
    shots = [dsh.Shot(shots[0].srcpos, rec)]
    m = oracle_model(d)
    o = O.Oracle(m, "port")
    seis_ref = o.forward(shots[0].srcpos, shots[0].recpos)
    o.close()
    obs = [(seis_ref * np.float32(0.9)).astype(np.float32)]
    gv, gr, l2, _ = _oracle_gradient(d, shots, obs)
    with engine_from(d) as e:
        name, ms = e.autotune(shots, nsteps=40)
        assert name in dsh.Engine.VARIANTS
        assert ms["kernel pair"] > 0 and ms["fused step"] > 0 and ms["persistent launch"] > 0
        assert ms[name] == min(t for t in ms.values() if t > 0)
        assert np.array_equal(e.forward(shots)[0], seis_ref)
        out = e.gradient(shots, obs)
    assert np.array_equal(out["g_vs"], gv) and np.array_equal(out["g_rho"], gr)
