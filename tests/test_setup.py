"""Host-side coefficient generation of the product library (libdsh.so,
dsh_setup_*) against the CPU oracle: every coefficient the kernels consume must
be bit-identical to the reference's (the oracle restatement is itself pinned to
the reference's golden fixtures and, where compiled, to the reference)."""
import numpy as np
import pytest

import dsh
import oracle as O

KIND = "ref" if O.available("ref") else "port"


@pytest.mark.parametrize("fdo", [2, 4, 6, 8, 10, 12])
@pytest.mark.parametrize("err", [0, 1, 2, 3, 4])
def test_holberg(fdo, err):
    rng = np.random.default_rng(0)
    vs = rng.uniform(150, 300, (6, 8)).astype(np.float32)
    m = O.Model(nx=8, ny=6, nt=4, dh=0.5, dt=1e-4, vs=vs, rho=vs * 8, fdorder=fdo, maxrelerror=err, fw=2)
    o = O.Oracle(m, KIND)
    ref = o.hc()
    o.close()
    assert np.array_equal(dsh.holberg(fdo, err)[1:], ref[1:])


@pytest.mark.parametrize("nx,ny,fw,dh,dt,fpml,damp", [(60, 40, 10, 0.5, 2e-4, 30.0, 400.0),
                                                      (2000, 800, 20, 0.25, 1e-4, 40.0, 500.0),
                                                      (33, 47, 15, 1.0, 5e-4, 7.0, 3000.0),
                                                      (500, 200, 20, 0.5, 2e-4, 30.0, 150.0)])
def test_pml_profiles(nx, ny, fw, dh, dt, fpml, damp):
    vs = np.full((ny, nx), damp, np.float32)
    m = O.Model(nx=nx, ny=ny, nt=4, dh=dh, dt=dt, vs=vs, rho=vs, fw=fw, fpml=fpml, damping=damp)
    o = O.Oracle(m, KIND)
    mine = dsh.pml_profiles(nx, ny, fw, dh, dt, damp, fpml)
    for name in O.PML:
        assert np.array_equal(mine[name], o.pml(name)), name
    o.close()


@pytest.mark.parametrize("L", [0, 1, 2, 3, 4])
def test_model_coefficients(L):
    rng = np.random.default_rng(L)
    ny, nx = 23, 31
    vs = rng.uniform(100, 500, (ny, nx)).astype(np.float32)
    vs[3, 4] = 0.0                                  # zero-modulus branch of av_mue
    rho = rng.uniform(1500, 2200, (ny, nx)).astype(np.float32)
    qs = rng.uniform(20, 60, (ny, nx)).astype(np.float32)
    fl = (10.0, 40.0, 160.0, 320.0)[:L]
    m = O.Model(nx=nx, ny=ny, nt=4, dh=0.25, dt=1e-4, vs=vs, rho=rho, qs=qs, l=L, fl=fl, fw=3)
    o = O.Oracle(m, KIND)
    c = dsh.model_coefficients(vs, rho, qs, l=L, fl=fl, dt=1e-4)
    assert np.array_equal(c["uip"], o.field("uip"))
    assert np.array_equal(c["ujp"], o.field("ujp"))
    assert np.array_equal(c["cnorm"], o.cnorm())
    b = (1.0 / rho.astype(np.float64)).astype(np.float32)
    assert np.array_equal(c["brho"], b)
    if L:
        assert np.array_equal(c["fipjp"], o.field("fipjp"))
        assert np.array_equal(c["f"], o.field("f"))
        for k in range(L):
            assert np.array_equal(c["dip"][k], o.field("dip", k))
            assert np.array_equal(c["d"][k], o.field("d", k))
        for a, b2 in zip([c["bip"], c["bjm"], c["cip"], c["cjm"]], o.sls()):
            assert np.array_equal(a, b2)
    o.close()


@pytest.mark.parametrize("quellart", [1, 2, 4, 5, 6])
def test_wavelets(quellart):
    nt, dt = 700, 2e-4
    sp = np.zeros((8, 3), np.float32)
    sp[3] = [0.0, 0.004, -0.002]
    sp[4] = [30.0, 45.0, 12.5]
    sp[5] = [1.0, 0.5, 2.0]
    m = O.Model(nx=8, ny=8, nt=nt, dh=0.5, dt=dt, vs=np.full((8, 8), 200, np.float32),
                rho=np.full((8, 8), 1800, np.float32), quellart=quellart, fw=2)
    o = O.Oracle(m, KIND)
    ref = o.wavelet(sp)
    o.close()
    assert np.array_equal(dsh.wavelet(quellart, nt, dt, sp), ref)


def test_dt_limit():
    # the staggered scheme's stability bound: DH / (sqrt(2) * sum|hc| * vmax)
    hc = dsh.holberg(8, 1)
    expect = 0.25 / (np.sqrt(2.0) * np.abs(hc[1:]).astype(np.float64).sum() * 500.0)
    assert abs(dsh.dt_limit(8, 1, 0.25, 500.0) - expect) < 1e-12


def test_visc_base_binding_runs_on_cpu():
    """The host restatement the device coefficient kernel is checked against
    (dsh_setup_visc_base) is callable and gives tau = 2/Qs."""
    rng = np.random.default_rng(5)
    vs = rng.uniform(150, 400, (9, 11)).astype(np.float32)
    rho = rng.uniform(1800, 2100, (9, 11)).astype(np.float32)
    qs = rng.uniform(20, 60, (9, 11)).astype(np.float32)
    b = dsh.visc_base(vs, rho, qs, 3, (7.5, 30.0, 120.0), 2e-4)
    assert np.array_equal(b["taus"], (2.0 / qs.astype(np.float64)).astype(np.float32))
    assert np.all(b["muip"] > 0) and np.all(b["mujp"] > 0)
