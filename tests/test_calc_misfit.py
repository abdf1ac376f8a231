"""The FWI loop's reported misfit and data energy (dsh_calc_misfit,
dsh_calc_energy) against the reference's calc_misfit.c and calc_energy.c
compiled into the oracle, bit for bit: LNORM 2, 5 and 6 (and an LNORM that
adds nothing), running totals carried in from earlier shots, one trace and
many, zero traces (the LNORM=5 division by zero gives NaN in both)."""
import numpy as np
import pytest

import oracle as O
from dsh import fwi

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


def _traces(seed, ntr, ns):
    rng = np.random.default_rng(seed)
    obs = (rng.standard_normal((ntr, ns)) * 1e-3).astype(np.float32)
    syn = (obs * np.float32(0.8) + rng.standard_normal((ntr, ns)).astype(np.float32) * np.float32(2e-4))
    return obs, syn.astype(np.float32)


@ref_only
@pytest.mark.parametrize("lnorm", [2, 5, 6, 3])
@pytest.mark.parametrize("ntr,ns,l2_in", [(1, 50, 0.0), (17, 400, 0.0), (40, 1200, 3.5e-9)])
def test_calc_misfit_matches_reference(lnorm, ntr, ns, l2_in):
    obs, syn = _traces(ntr + ns + lnorm, ntr, ns)
    dt = 2e-4
    got = fwi.calc_misfit(obs, syn, lnorm, dt, l2_in)
    ref = O.calc_misfit(obs, syn, lnorm, dt, l2_in)
    assert got == ref
    if lnorm == 3:
        assert got == np.float32(l2_in)
    else:
        assert got != np.float32(l2_in)


@ref_only
@pytest.mark.parametrize("ntr,ns,e_in", [(1, 50, 0.0), (23, 800, 0.0), (64, 300, 1.25e-7)])
def test_calc_energy_matches_reference(ntr, ns, e_in):
    obs, _ = _traces(ntr * 3 + ns, ntr, ns)
    assert fwi.calc_energy(obs, 1e-4, e_in) == O.calc_energy(obs, 1e-4, e_in)


@ref_only
def test_zero_traces_like_the_reference():
    obs = np.zeros((3, 20), np.float32)
    syn = np.zeros((3, 20), np.float32)
    assert np.isnan(fwi.calc_misfit(obs, syn, 5, 1e-3)) and np.isnan(O.calc_misfit(obs, syn, 5, 1e-3))
    assert fwi.calc_misfit(obs, syn, 2, 1e-3) == O.calc_misfit(obs, syn, 2, 1e-3) == 0.0
    assert fwi.calc_energy(obs, 1e-3) == 0.0
