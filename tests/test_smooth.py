"""SPATFILTER=3 Gaussian gradient smoothing (src/gauss_filt.c): the C
restatement in the oracle against a float64 numpy transcription of the same
loop (filter-size rule, normalised kernel, edge replication), and the
library's C-ABI symbols; the GPU kernel is checked bit for bit against the
restatement in the GPU test below.  SPATFILTER=4 (src/gauss_filt_var.c,
kernel size following the local velocity): the host kernel tables plus a
float32 transcription of the device loop, and the GPU kernel, against the
reference's own gauss_filt_var compiled into the oracle, bit for bit."""
import numpy as np
import pytest

import dsh
import oracle as O


def _np_gauss(g, filt):
    hfs = abs(filt) // 2
    sigma = float(hfs // 2)
    s = 2.0 * sigma * sigma
    ii, jj = np.meshgrid(np.arange(-hfs, hfs + 1), np.arange(-hfs, hfs + 1))
    k = np.exp(-(ii * ii) / s - (jj * jj) / s)
    k /= k.sum()
    ny, nx = g.shape
    pad = np.pad(g.astype(np.float64), hfs, mode="edge")
    out = np.zeros((ny, nx))
    for a in range(2 * hfs + 1):
        for b in range(2 * hfs + 1):
            out += k[a, b] * pad[a:a + ny, b:b + nx]
    return out


def test_filter_size_rule():
    assert O.gauss_filter_size(0.5, 300.0, 30.0, 0.5) == 11      # round(10) -> 10 -> 11
    assert O.gauss_filter_size(0.25, 300.0, 30.0, 0.5) == 5
    assert O.gauss_filter_size(0.0, 300.0, 30.0, 0.5) == 0


@pytest.mark.parametrize("filt", [5, 9, 13])
def test_restatement_matches_float64_transcription(filt):
    g = np.random.default_rng(filt).standard_normal((37, 53)).astype(np.float32)
    out = O.gauss_filt(g, filt)
    ref = _np_gauss(g, filt)
    assert np.allclose(out, ref, rtol=1e-5, atol=1e-6)
    assert np.allclose(O.gauss_filt(np.ones((20, 30), np.float32), filt), 1.0, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("filt", [0, 5, 11, 21])
def test_gpu_smoothing_bit_identical(filt):
    import dsh

    g = np.random.default_rng(3).standard_normal((123, 257)).astype(np.float32)
    assert np.array_equal(dsh.smooth_gauss(g, filt), O.gauss_filt(g, filt) if filt else g)


def _var_case(seed, ny=40, nx=70):
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    vel = (gaussian_filter(80 * rng.random((ny, nx)), 3) + np.linspace(100, 900, ny)[:, None]).astype(np.float32)
    vel[:4, :] = 0.0                  # no smoothing where the depth length rounds to 0
    g = rng.standard_normal((ny, nx)).astype(np.float32)
    return g, vel


def _emulate_var(g, mp, pairs, w):
    """float32 transcription of the device loop over the host tables"""
    ny, nx = g.shape
    out = np.empty_like(g)
    for j in range(ny):
        for i in range(nx):
            k = mp[j, i]
            if k < 0:
                out[j, i] = g[j, i]
                continue
            hx, hz, off, s = pairs[k]
            conv = np.float32(0)
            q = off
            for ii in range(-hx, hx + 1):
                ic = min(max(i + ii, 0), nx - 1)
                for jj in range(-hz, hz + 1):
                    jc = min(max(j + jj, 0), ny - 1)
                    conv = np.float32(conv + np.float32(g[jc, ic] * w[q]))
                    q += 1
            out[j, i] = np.float32(conv / np.float32(s))
    return out


VAR_CASES = [(0.5, 0.8, 0.5, 60.0), (0.25, 0.6, 0.6, 80.0), (0.5, 0.4, 1.0, 50.0)]


@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
@pytest.mark.parametrize("dh,wd,wd1,fc", VAR_CASES)
def test_variable_gauss_tables_match_reference(dh, wd, wd1, fc):
    g, vel = _var_case(int(fc))
    ref = O.gauss_filt_var(g, vel, dh, wd, wd1, fc)
    mp, pairs, w = dsh.gauss_var_tables(vel, dh, wd, wd1, fc)
    assert len(pairs) >= 3 and (mp < 0).any()
    assert np.array_equal(_emulate_var(g, mp, pairs, w), ref)


@pytest.mark.gpu
@pytest.mark.skipif(not O.available("ref"), reason="reference build not present")
@pytest.mark.parametrize("dh,wd,wd1,fc", VAR_CASES)
def test_gpu_variable_gauss_bit_identical(dh, wd, wd1, fc):
    g, vel = _var_case(int(fc) + 1, ny=90, nx=130)
    ref = O.gauss_filt_var(g, vel, dh, wd, wd1, fc)
    assert np.array_equal(dsh.smooth_gauss_var(g, vel, dh, wd, wd1, fc), ref)
