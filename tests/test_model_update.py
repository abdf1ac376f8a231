"""The FWI model update (dsh_model_update) against the reference's
calc_mat_change_test.c compiled into the oracle, bit for bit: the step
lengths relative to the model and direction maxima, SCALERHO, the
INV_VS_ITER / INV_RHO_ITER delays and every bound (below VSLOWERLIM but
above 1e-6, above VSUPPERLIM, rho outside its limits, negative values)."""
import numpy as np
import pytest

import oracle as O
from dsh import fwi

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


def _fields(seed, nx, ny):
    rng = np.random.default_rng(seed)
    vs = rng.uniform(100, 500, (ny, nx)).astype(np.float32)
    vs[0, :3] = 0.0                                        # vacuum points the lower bound must not touch
    rho = rng.uniform(1500, 2300, (ny, nx)).astype(np.float32)
    d_vs = rng.standard_normal((ny, nx)).astype(np.float32)
    d_rho = rng.standard_normal((ny, nx)).astype(np.float32)
    return vs, rho, d_vs, d_rho


@ref_only
@pytest.mark.parametrize("eps_scale,scalerho,it,ivs,irho,limits", [
    (0.01, 1.0, 1, 0, 0, (0.0, 1e9, 0.0, 1e9)),
    (0.3, 0.5, 3, 0, 2, (150.0, 450.0, 1600.0, 2200.0)),        # every bound active
    (2.5, 1.0, 2, 0, 0, (50.0, 1e9, 0.0, 1e9)),                 # steps large enough to go negative
    (0.05, 2.0, 1, 2, 5, (0.0, 1e9, 0.0, 1e9)),                 # both parameters delayed
    (0.1, 1.0, 4, 3, 0, (120.0, 480.0, 1500.0, 2300.0)),
])
def test_model_update_matches_reference(eps_scale, scalerho, it, ivs, irho, limits):
    vs, rho, d_vs, d_rho = _fields(int(eps_scale * 100) + it, 29, 17)
    got = fwi.model_update(vs, rho, d_vs, d_rho, eps_scale, scalerho, it, ivs, irho, limits)
    ref = O.model_update(vs, rho, d_vs, d_rho, eps_scale, scalerho, it, ivs, irho, limits)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    vn, rn, eu, er = got
    if it < ivs:
        assert eu == 0 and np.array_equal(vn, vs)
    else:
        assert eu == np.float32(eps_scale) * (vs.max() / np.abs(d_vs).max())
    assert (vn >= 0).all() and (rn >= 0).all()
