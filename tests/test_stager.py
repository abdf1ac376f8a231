"""Asynchronous staging of observed SU data (dsh_stager, include/dsh_io.h):
batches read on the stager's thread equal dsh_read_su of the same files (the
reference's inseis values, tests/test_io.py), in order, across buffer reuse;
unreadable files and out-of-order calls are reported; on the GPU, a gradient
whose observed data come from the stager's device buffers equals the one
from host arrays."""
import numpy as np
import pytest

import dsh
from dsh import io


def _files(tmp_path, n, ns, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        ntr = 3 + k % 4
        sec = rng.standard_normal((ntr, ns)).astype(np.float32)
        rec = np.array([np.arange(1, ntr + 1) * 2, np.ones(ntr, int)], np.int32)
        path = str(tmp_path / f"shot{k}.su")
        io.write_su(path, sec, rec, xs=10.0 + k, ys=0.5, dh=0.5, dt=2e-4)
        out.append((path, ntr))
    return out


def test_batches_in_order_equal_read_su(tmp_path):
    ns = 120
    files = _files(tmp_path, 7, ns)
    batches = [files[0:2], files[2:3], files[3:6], files[6:7]]
    with io.Stager(2, 20 * ns, use_device=False) as st:
        for b in batches:
            st.submit([p for p, _ in b], [n for _, n in b], ns)
        for b in batches:
            got = st.acquire_host()
            ref = np.concatenate([io.read_su(p, n, ns).ravel() for p, n in b])
            assert np.array_equal(got, ref)
            st.release()


def test_more_batches_than_buffers_interleaved(tmp_path):
    ns = 64
    files = _files(tmp_path, 9, ns, seed=1)
    with io.Stager(3, 8 * ns, use_device=False) as st:
        for k, (p, n) in enumerate(files):
            st.submit([p], [n], ns)
            if k >= 2:                                      # consume while later batches are queued
                q, m = files[k - 2]
                assert np.array_equal(st.acquire_host(), io.read_su(q, m, ns).ravel())
                st.release()
        for q, m in files[-2:]:
            assert np.array_equal(st.acquire_host(), io.read_su(q, m, ns).ravel())
            st.release()


def test_errors_are_reported(tmp_path):
    ns = 32
    (p, n), = _files(tmp_path, 1, ns)
    with io.Stager(2, 100, use_device=False) as st:
        with pytest.raises(dsh.DshError):
            st.release()                                    # nothing acquired
        with pytest.raises(dsh.DshError):
            st.submit([p, p, p, p], [n] * 4, ns)            # larger than a buffer
        st.submit([str(tmp_path / "missing.su")], [n], ns)
        st.submit([p], [n], ns)
        with pytest.raises(dsh.DshError):
            st.acquire_host()                               # the unreadable file
        st.release()
        assert np.array_equal(st.acquire_host(), io.read_su(p, n, ns).ravel())
        with pytest.raises(dsh.DshError):
            st.acquire_host()                               # the previous batch is not released
        st.release()
        with pytest.raises(dsh.DshError):
            st.acquire_host()                               # nothing submitted


@pytest.mark.gpu
def test_gradient_with_staged_device_data(tmp_path):
    import torch

    from dsh import configs

    cfg = configs.config3(nt=150, nshots=4)
    p = dict(cfg["params"], max_shots=2)
    shots = cfg["shots"][:4]
    nt = p["nt"]
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["true"], cfg["rho"], cfg["qs"])
        obs = e.forward(shots)
        paths = []
        for k, (sh, o) in enumerate(zip(shots, obs)):
            path = str(tmp_path / f"obs{k}.su")
            io.write_su(path, o, sh.recpos, xs=float(sh.srcpos[0, 0]) * p["dh"], ys=float(sh.srcpos[1, 0]) * p["dh"],
                        dh=p["dh"], dt=p["dt"])
            paths.append(path)
        e.set_model(cfg["vs"], cfg["rho"], cfg["qs"])
        stream = torch.cuda.Stream()
        e.set_stream(stream.cuda_stream)
        ny, nx = p["ny"], p["nx"]
        gv = torch.empty(ny * nx, dtype=torch.float32, device="cuda")
        gr = torch.empty_like(gv)
        batches = [[0, 1], [2, 3]]
        with io.Stager(2, sum(s.ntr for s in shots) * nt) as st:
            for b in batches:
                st.submit([paths[k] for k in b], [shots[k].ntr for k in b], nt)
            for b in batches:
                ptr, n = st.acquire(stream.cuda_stream)
                assert n == sum(shots[k].ntr for k in b) * nt
                l2 = e.gradient_device([shots[k] for k in b], ptr, gv.data_ptr(), gr.data_ptr())
                st.release(stream.cuda_stream)
                stream.synchronize()
                host_obs = [io.read_su(paths[k], shots[k].ntr, nt) for k in b]
                e.set_stream(None)
                ref = e.gradient([shots[k] for k in b], host_obs)
                e.set_stream(stream.cuda_stream)
                assert np.array_equal(gv.cpu().numpy().reshape(ny, nx), ref["g_vs"])
                assert np.array_equal(gr.cpu().numpy().reshape(ny, nx), ref["g_rho"])
                assert l2 == ref["l2"]
        e.set_stream(None)
