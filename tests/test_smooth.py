"""SPATFILTER=3 Gaussian gradient smoothing (src/gauss_filt.c): the C
restatement in the oracle against a float64 numpy transcription of the same
loop (filter-size rule, normalised kernel, edge replication), and the
library's C-ABI symbols; the GPU kernel is checked bit for bit against the
restatement in the GPU test below."""
import numpy as np
import pytest

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
