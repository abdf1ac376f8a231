"""dsh_set_model forms the per-point model coefficients on the device: 1/rho,
the harmonic shear-modulus averages with the periodic one-rank neighbour
(src/av_mue.c:28-52, the zero-modulus branch included) and, for L > 0, tau =
2/Qs, its four-point average (src/av_tau.c:12) and the relaxed moduli
(src/prepare_update_s.c:40-47).  The fields must equal the host restatement
(csrc/dsh_setup.c, itself pinned bit for bit to the reference's
prepare_update_s / av_mue / av_tau compiled into the oracle by
tests/test_setup.py) bit for bit."""
import numpy as np
import pytest

import dsh

pytestmark = pytest.mark.gpu


def _model(seed, nx, ny):
    rng = np.random.default_rng(seed)
    vs = rng.uniform(100.0, 500.0, (ny, nx)).astype(np.float32)
    rho = rng.uniform(1500.0, 2500.0, (ny, nx)).astype(np.float32)
    qs = rng.uniform(20.0, 60.0, (ny, nx)).astype(np.float32)
    vs[3, 5] = 0.0                      # zero modulus at a point and at the periodic wrap
    vs[ny - 1, nx - 1] = 0.0
    rho[2, 7] = 0.0                     # 1/rho set to 0 below 1e-20
    return vs, rho, qs


@pytest.mark.parametrize("L", [0, 3])
@pytest.mark.parametrize("nx,ny", [(37, 29), (130, 64)])
def test_device_model_coefficients_equal_host(L, nx, ny):
    vs, rho, qs = _model(100 + L + nx, nx, ny)
    fl = (7.5, 30.0, 120.0)[:L]
    dt = 2e-4
    p = dsh.make_params(nx=nx, ny=ny, nt=10, dh=0.5, dt=dt, fdorder=4, fw=6, free_surf=1, l=L, fl=fl,
                        damping=500.0, fpml=30.0)
    with dsh.Engine(p) as e:
        e.set_model(vs, rho, qs if L else None)
        dev = {k: e.field(k) for k in ("brho", "uip", "ujp")}
        if L:
            dev.update({k: e.field(k) for k in ("muip", "mujp", "tausipjp", "taus")})
    host = dsh.model_coefficients(vs, rho, qs, l=0, fl=fl, dt=dt)
    for k in ("brho", "uip", "ujp"):
        assert np.array_equal(dev[k], host[k]), k
    if L:
        base = dsh.visc_base(vs, rho, qs, L, fl, dt)
        for k in ("muip", "mujp", "tausipjp", "taus"):
            assert np.array_equal(dev[k], base[k]), k
