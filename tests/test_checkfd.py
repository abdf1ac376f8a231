"""The FD grid check of a starting model (dsh_check_fd) against the
reference's checkfd_ssg_visc / checkfd_ssg_elastic compiled into the oracle:
the velocities, the stability limit and the recommended grid spacing it
reports are the same numbers (compared as the reference prints them, %e);
a DT above the limit and an absorbing frame wider than the grid are the
reference's two stops, reported as DSH_ERR_UNSTABLE and DSH_ERR_PARAM."""
import re

import numpy as np
import pytest

import dsh
import oracle as O

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


def _model(seed, nx, ny, l):
    rng = np.random.default_rng(seed)
    vs = rng.uniform(120, 480, (ny, nx)).astype(np.float32)
    rho = rng.uniform(1500, 2200, (ny, nx)).astype(np.float32)
    qs = rng.uniform(10, 80, (ny, nx)).astype(np.float32) if l else None
    return vs, rho, qs


def _report(text, key):
    pats = {"cmax": r"Vp_max= (\S+) m/s", "cmin": r"Vs_min=(\S+) m/s", "dtstab": r"timestep DT is (\S+) seconds",
            "dhstab": r"recommended value for DH is (\S+) meter"}
    return re.search(pats[key], text).group(1)


@ref_only
@pytest.mark.parametrize("l,fdo,mre,ts", [(3, 8, 1, 0.03), (2, 4, 0, 0.05), (1, 12, 3, 0.1), (0, 6, 1, 0.02),
                                          (0, 2, 2, 0.04), (4, 10, 4, 0.025)])
def test_check_fd_matches_reference(l, fdo, mre, ts):
    vs, rho, qs = _model(10 + l + fdo, 31, 23, l)
    fl = [4.0, 15.0, 45.0, 90.0][:l]
    dh = 0.5
    rc0, v0, _ = dsh.check_fd(vs, rho, qs, fl, dh=dh, dt=1e-6, ts=ts, fdorder=fdo, maxrelerror=mre, fw=12)
    dt = float(np.float32(0.9 * v0["dtstab"]))
    rc, v, warn = dsh.check_fd(vs, rho, qs, fl, dh=dh, dt=dt, ts=ts, fdorder=fdo, maxrelerror=mre, fw=12)
    assert rc0 == dsh.DSH_OK and rc == dsh.DSH_OK
    text = O.checkfd(vs, rho, qs, fl, dh, dt, ts, fdo, mre, 12)
    for key in ("cmin", "cmax", "dtstab", "dhstab"):
        assert "%e" % v[key] == _report(text, key), key
    assert bool(warn & 1) == bool(np.float32(dh) > v["dhstab"])      # the reference's warning condition
    if l == 0:
        assert v["cmax"] == vs.max() and v["cmin"] == vs.min()
    else:
        assert v["cmax"] > v["cmin"]          # dispersion of the SLS medium: faster at infinite frequency


def test_check_fd_stops_like_the_reference():
    vs, rho, qs = _model(3, 20, 15, 2)
    kw = dict(dh=0.5, ts=0.03, fdorder=8, maxrelerror=1)
    _, v, _ = dsh.check_fd(vs, rho, qs, (5.0, 30.0), dt=1e-6, fw=10, **kw)
    above = float(np.nextafter(np.float32(v["dtstab"]), np.float32(1)))
    assert dsh.check_fd(vs, rho, qs, (5.0, 30.0), dt=above, fw=10, **kw)[0] == dsh.ERR_UNSTABLE
    assert dsh.check_fd(vs, rho, qs, (5.0, 30.0), dt=float(v["dtstab"]), fw=10, **kw)[0] == dsh.DSH_OK
    assert dsh.check_fd(vs, rho, qs, (5.0, 30.0), dt=1e-6, fw=16, **kw)[0] == dsh.ERR_PARAM
    rc, _, warn = dsh.check_fd(vs, rho, qs, (5.0, 30.0), dt=1e-6, fw=8, **kw)
    assert rc == dsh.DSH_OK and warn & 2
    assert dsh.check_fd(vs, rho, None, (), dt=1e-6, fw=10, dh=0.5, ts=0.0, fdorder=8, maxrelerror=1)[0] == \
        dsh.ERR_PARAM
