"""Butterworth trace filtering of the multi-scale stages (src/timedomain_filt.c
with libcseife): the reference's own code (compiled into the oracle) against
a float64 transcription with scipy's lfilter of the same sections — including
the reference's off-by-one (its 1-based vector goes to 0-based libcseife: the
last sample comes back unfiltered, the highpass removes a zero lead-in
instead of the first sample); the GPU kernel against the reference bit for
bit (compat mode) and against the transcription of the intended filter."""
import math

import numpy as np
import pytest

import oracle as O

pytestmark_ref = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


def _sections(dt, fc, order, highpass):
    t0 = (1.0 / np.float32(fc)) / dt
    eps = 8.0 * math.atan(1.0) / t0
    secs = []
    if order % 2:
        g1 = (2 - eps) / (2 + eps)
        f = (eps / (2 + eps), eps / (2 + eps)) if not highpass else (2 / (2 + eps), -2 / (2 + eps))
        secs.append(([f[0], f[1], 0.0], [1.0, -g1, 0.0]))
    for j in range(1, order // 2 + 1):
        h = math.sin(2 * math.atan(1.0) * (2 * j - 1) / order)
        a = 1 - eps * h + eps * eps / 4
        b = -2 + eps * eps / 2
        c = 1 + eps * h + eps * eps / 4
        f0 = (eps * eps / 4 / c) if not highpass else 1 / c
        f = [f0, 2 * f0 if not highpass else -2 * f0, f0]
        secs.append((f, [1.0, b / c, a / c]))
    return secs


@pytestmark_ref
@pytest.mark.parametrize("order,method", [(4, 1), (5, 1), (4, 2), (3, 2)])
def test_reference_filter_matches_transcription(order, method):
    from scipy.signal import lfilter

    dt, fc = 2e-4, 60.0
    x = np.random.default_rng(order).standard_normal((6, 800)).astype(np.float32)
    got = O.timedomain_filt(x, dt, fc, order, method)
    ref = _transcription(x, dt, fc, order, method, compat=True)
    assert np.allclose(got, ref.astype(np.float32), rtol=1e-5, atol=1e-5 * np.abs(ref).max())
    assert np.array_equal(got[:, -1], x[:, -1])          # the reference leaves the last sample


def _transcription(x, dt, fc, order, method, compat):
    from scipy.signal import lfilter

    ref = x.astype(np.float64)
    n = ref.shape[1] - 1 if compat else ref.shape[1]
    y = ref[:, :n].copy()
    if method == 2 and not compat:
        y = y - y[:, :1]
    for b, a in _sections(np.float64(np.float32(dt)), fc, order, method == 2):
        y = lfilter(b, a, y, axis=1)
    out = ref.copy()
    out[:, :n] = y
    return out


@pytestmark_ref
@pytest.mark.gpu
@pytest.mark.parametrize("order,method", [(2, 1), (4, 1), (5, 2), (8, 2)])
def test_gpu_filter_bit_identical(order, method):
    import torch

    import dsh

    x = np.random.default_rng(10 + order).standard_normal((333, 1500)).astype(np.float32)
    ref = O.timedomain_filt(x, 1e-4, 45.0, order, method)
    d = torch.from_numpy(x).cuda()
    assert dsh.lib().dsh_timedomain_filt(d.data_ptr(), 333, 1500, 1e-4, 45.0, order, method, 1, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), ref)
    d = torch.from_numpy(x).cuda()
    assert dsh.lib().dsh_timedomain_filt(d.data_ptr(), 333, 1500, 1e-4, 45.0, order, method, 0, None) == 0
    torch.cuda.synchronize()
    intended = _transcription(x, 1e-4, 45.0, order, method, compat=False)
    assert np.allclose(d.cpu().numpy(), intended, rtol=1e-5, atol=1e-5 * np.abs(intended).max())
