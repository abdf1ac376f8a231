"""Gradient tapers (src/taper_grad.c after the shot sum, src/taper_grad_shot.c
per shot): the host coefficients against the reference's own functions
compiled into the oracle, bit for bit, for the vertical frame, the
horizontal ramp, the circular source tapers (erf and log shapes) and taper
files; the per-shot coefficient formula the engine evaluates on the device
against taper_grad_shot; on the GPU, dsh_taper_apply and the engine's
per-shot taper inside dsh_gradient against the reference."""
import ctypes as C

import numpy as np
import pytest

import dsh
import oracle as O

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")

NY, NX, DH = 40, 60, 0.5


def _grad(seed):
    return np.random.default_rng(seed).standard_normal((NY, NX)).astype(np.float32)


SRC = np.array([[10.0, 17.5, 24.0, 29.5], [1.0, 5.5, 12.0, 19.5]], np.float32)   # metres
REC = np.array([[3, 20, 33, 60], [1, 1, 2, 0]], np.int32)                          # one on the padding row

CASES = [
    (dsh.TAPER_VERTICAL, dict(gradt=(5, 15, 40, 55))),
    (dsh.TAPER_VERTICAL, dict(gradt=(0, 8, 30, 62))),
    (dsh.TAPER_HORIZONTAL, dict(gradt=(4, 12, 0, 0))),
    (dsh.TAPER_HORIZONTAL, dict(gradt=(1, 1, 0, 0))),
    (dsh.TAPER_SOURCES, dict(srtshape=1, srtradius=3.0, filtsize=2)),
    (dsh.TAPER_SOURCES, dict(srtshape=2, srtradius=2.2, filtsize=1)),
    (dsh.TAPER_SOURCES, dict(srtshape=1, srtradius=0.5, filtsize=0)),
    (dsh.TAPER_SOURCES, dict(srtshape=1, srtradius=40.0, filtsize=3)),
]


@ref_only
@pytest.mark.parametrize("sws,kw", CASES)
def test_taper_coefficients_bit_identical_to_reference(sws, kw):
    g = _grad(sws)
    ref, tc = O.taper(g, sws, DH, src_xy=SRC, recpos=REC, **kw)
    c, z = dsh.taper_coeff(sws, NX, NY, DH, src_xy=SRC, recpos=REC, **kw)
    assert np.array_equal(c, tc)
    assert np.array_equal(np.where(z, np.float32(0), g * c), ref)
    if sws == dsh.TAPER_VERTICAL:       # every interior source and receiver point zeroed
        assert z.sum() == SRC.shape[1] + 3


@ref_only
@pytest.mark.parametrize("sws", [dsh.TAPER_FILE_VS, dsh.TAPER_FILE_RHO])
def test_taper_from_file_values(sws):
    g = _grad(7)
    vals = np.random.default_rng(8).uniform(0, 2, NX * NY).astype(np.float32)
    ref, tc = O.taper(g, sws, DH, file_vals=vals)
    c, z = dsh.taper_coeff(sws, NX, NY, DH, file_vals=vals)
    assert not z.any() and np.array_equal(c, tc) and np.array_equal(g * c, ref)


def test_taper_rejects_bad_arguments():
    with pytest.raises(dsh.DshError):
        dsh.taper_coeff(4, NX, NY, DH)
    with pytest.raises(dsh.DshError):
        dsh.taper_coeff(dsh.TAPER_SOURCES, NX, NY, DH, srtshape=3, src_xy=SRC)
    with pytest.raises(dsh.DshError):
        dsh.taper_coeff(dsh.TAPER_FILE_VS, NX, NY, DH)


def _box(shape, radius, dh):
    L = dsh.lib()
    L.dsh_setup_taper_box.argtypes = [C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    L.dsh_setup_taper_norm.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    g, ijc = C.c_int(), C.c_int()
    assert L.dsh_setup_taper_box(shape, radius, dh, C.byref(g), C.byref(ijc), None) == 0
    m = np.zeros((g.value, g.value), np.float32)
    L.dsh_setup_taper_box(shape, radius, dh, C.byref(g), C.byref(ijc), m.ctypes.data)
    return m, ijc.value


def shot_taper(g, i1, j1, shape, radius, filt, dh):
    """The engine's per-shot taper (shot_sum_taper_kernel) in numpy float32:
    (min(1, box value) - minm) / maxm around source (i1, j1), 0 within filt."""
    ny, nx = g.shape
    m, ijc = _box(shape, radius, dh)
    G = m.shape[0]
    mn, mx = C.c_float(), C.c_float()
    dsh.lib().dsh_setup_taper_norm(nx, ny, G, ijc, m.ctypes.data, i1, j1, C.byref(mn), C.byref(mx))
    jj, ii = np.mgrid[1:ny + 1, 1:nx + 1]
    ix, iy = ii - i1 + ijc, jj - j1 + ijc
    inb = (ix >= 1) & (ix <= G) & (iy >= 1) & (iy <= G)
    mm = np.ones((ny, nx), np.float32)
    mm[inb] = m[iy[inb] - 1, ix[inb] - 1]
    ms = np.where(mm < 1, mm, np.float32(1)).astype(np.float32)
    c = (ms - np.float32(mn.value)) / np.float32(mx.value)
    z = (np.abs(ii - i1) <= filt) & (np.abs(jj - j1) <= filt)
    return np.where(z, np.float32(0), g * c)


@ref_only
@pytest.mark.parametrize("shape,radius,filt", [(1, 3.0, 2), (2, 2.2, 1), (1, 1.0, 0), (2, 6.0, 3), (1, 40.0, 1)])
def test_shot_taper_formula_matches_taper_grad_shot(shape, radius, filt):
    g = _grad(3)
    src = np.array([[10.0, 17.5, 24.0, 29.5, 1.0], [1.0, 5.5, 12.0, 19.5, 0.5]], np.float32)
    for k in range(1, src.shape[1] + 1):
        i1 = int(np.floor(src[0, k - 1] / np.float32(DH) + 0.5))
        j1 = int(np.floor(src[1, k - 1] / np.float32(DH) + 0.5))
        if i1 - filt < 1:     # the reference's writes left of column 1 alias other rows
            continue
        ref, _ = O.taper(g, 3, DH, srtshape=shape, srtradius=radius, filtsize=filt, src_xy=src, shot=k)
        assert np.array_equal(shot_taper(g, i1, j1, shape, radius, filt, DH), ref), (k, i1, j1)


@pytest.mark.gpu
@ref_only
@pytest.mark.parametrize("sws,kw", CASES[::2])
def test_taper_apply_on_gpu(sws, kw):
    import torch

    g = _grad(11 + sws)
    ref, _ = O.taper(g, sws, DH, src_xy=SRC, recpos=REC, **kw)
    c, z = dsh.taper_coeff(sws, NX, NY, DH, src_xy=SRC, recpos=REC, **kw)
    gd = torch.from_numpy(g).cuda()
    dsh.taper_apply(gd, c, z)
    assert np.array_equal(gd.cpu().numpy(), ref)


@pytest.mark.gpu
@ref_only
@pytest.mark.parametrize("shape,radius,filt", [(1, 3.0, 1), (2, 2.0, 2)])
def test_engine_shot_taper_matches_reference(shape, radius, filt):
    """dsh_gradient with the per-shot taper against the oracle's shot loop
    with the reference's taper_grad_shot applied to each shot's scaled
    gradients before the sum (src/denise.c:1681-1694)."""
    from conftest import oracle_model
    from test_gpu_parity import _case, engine_from

    d, shots = _case(77 + shape, nx=53, ny=35, nt=120, fdo=8, L=2, fs=1, fw=6, nshots=3)
    m = oracle_model(d)
    obs = []
    for sh in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sh.srcpos, sh.recpos) * np.float32(0.7)).astype(np.float32))
        o.close()
    su = np.zeros((m.ny, m.nx), np.float32)
    sr = np.zeros((m.ny, m.nx), np.float32)
    for sh, ob in zip(shots, obs):
        o = O.Oracle(m, "port")
        g = o.shot_gradient(sh.srcpos, sh.recpos, ob)
        o.close()
        i1, j1 = int(sh.srcpos[0, 0]), int(sh.srcpos[1, 0])
        assert i1 - filt >= 1
        xy = np.array([[i1 * d["dh"]], [j1 * d["dh"]]], np.float32)
        gr, _ = O.taper(g["g_rho"], 3, d["dh"], srtshape=shape, srtradius=radius, filtsize=filt, src_xy=xy, shot=1)
        gu, _ = O.taper(g["g_u"], 3, d["dh"], srtshape=shape, srtradius=radius, filtsize=filt, src_xy=xy, shot=1)
        su = su + gu
        sr = sr + gr
    o = O.Oracle(m, "port")
    gv_ref, gr_ref = o.convert(su, sr)
    o.close()
    with engine_from(d, max_shots=2) as e:         # two batches: 2 + 1 shots
        plain = e.gradient(shots, obs)
        e.set_shot_taper(shape, radius, filt)
        out = e.gradient(shots, obs)
        e.set_shot_taper(enable=False)
        again = e.gradient(shots, obs)
    assert np.array_equal(out["g_vs"], gv_ref) and np.array_equal(out["g_rho"], gr_ref)
    assert not np.array_equal(plain["g_vs"], out["g_vs"])
    assert np.array_equal(again["g_vs"], plain["g_vs"])
