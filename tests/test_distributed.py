"""Shot-parallel gradient across processes (CPU, gloo, world size 2): shot
partitioning, the all-reduce of gradients and misfit, the model broadcast and
the line search's scalar misfit all-reduce, and failure detection
when a rank dies before the collective (the survivor gets an error from a
short process-group timeout instead of hanging).  The per-rank gradient comes
from the CPU oracle, standing in for a GPU engine."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dsh.distributed import partition, shot_cost


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case():
    import oracle as O

    rng = np.random.default_rng(5)
    nx, ny, nt = 40, 30, 90
    vs = (200 + 30 * rng.standard_normal((ny, nx))).clip(120, 300).astype(np.float32)
    rho = (1800 + 60 * rng.standard_normal((ny, nx))).astype(np.float32)
    m = O.Model(nx=nx, ny=ny, nt=nt, dh=0.5, dt=2e-4, vs=vs, rho=rho, fdorder=4, fw=6, fpml=30.0,
                damping=float(vs.max()))
    shots = []
    for k in range(5):
        sp = np.zeros((8, 1), np.float32)
        sp[:, 0] = [6 + 7 * k, 2, 0, -0.01, 60.0, 1.0, 0, 3]
        rec = np.array([[4, 12, 20, 28, 36], [1, 1, 1, 1, 1]], np.int32)
        shots.append((sp, rec))
    obs = []
    for sp, rec in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sp, rec) * np.float32(0.7)).astype(np.float32))
        o.close()
    return m, shots, obs


def _local_gradient(m, shots, obs, idx):
    import oracle as O

    su = np.zeros((m.ny, m.nx), np.float32)
    sr = np.zeros((m.ny, m.nx), np.float32)
    l2 = 0.0
    for k in idx:
        o = O.Oracle(m, "port")
        g = o.shot_gradient(shots[k][0], shots[k][1], obs[k])
        su, sr, l2 = su + g["g_u"], sr + g["g_rho"], l2 + g["l2"]
        o.close()
    o = O.Oracle(m, "port")
    gv, gr = o.convert(su, sr)
    o.close()
    return {"g_vs": gv, "g_rho": gr, "l2": l2}


def _worker(rank, world, port, outdir, fail_rank):
    import datetime
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "denise-sh_b200"), os.path.join(root, "oracle")]
    import torch.distributed as dist

    from dsh.distributed import broadcast_model, distributed_gradient, distributed_misfit

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=8))
    m, shots, obs = _case()
    try:
        if rank == fail_rank:
            raise RuntimeError("injected failure before the collective")
        res = distributed_gradient(lambda idx: _local_gradient(m, shots, obs, idx), len(shots), (m.ny, m.nx),
                                   costs=[1.0] * len(shots))
        # rank 0's updated model reaches every rank in one broadcast
        vs_new = (m.vs * np.float32(1.01)).astype(np.float32) if rank == 0 else np.zeros_like(m.vs)
        rho_new = m.rho if rank == 0 else np.zeros_like(m.rho)
        bvs, brho, bqs = broadcast_model(vs_new, rho_new)
        # line-search misfit of three test shots: partitioned, one scalar all-reduce
        test = [0, 2, 4]
        mis = distributed_misfit(lambda idx: _local_gradient(m, shots, obs, idx)["l2"], test)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), g_vs=res.g_vs, g_rho=res.g_rho, l2=res.l2,
                 mine=np.array(res.my_shots), bvs=bvs, brho=brho, bqs_none=np.array(bqs is None), mis=mis)
    except Exception as e:   # noqa: BLE001 - report any failure to the parent
        with open(os.path.join(outdir, f"err{rank}.txt"), "w") as f:
            f.write(repr(e))
    finally:
        if rank != fail_rank:
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def test_partition_balances_and_is_deterministic():
    costs = [shot_cost(1000, 300, 4000, 2)] * 64
    parts = partition(costs, 8)
    assert sorted(sum(parts, [])) == list(range(64))
    assert all(len(p) == 8 for p in parts)
    assert parts == partition(costs, 8)
    uneven = [5.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    p2 = partition(uneven, 2)
    assert p2[0] == [0] and p2[1] == [1, 2, 3, 4, 5]


def test_two_ranks_match_single_process(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path), -1), nprocs=2, start_method="spawn")
    m, shots, obs = _case()
    ref = _local_gradient(m, shots, obs, list(range(len(shots))))
    outs = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    mine = sorted(np.concatenate([o["mine"] for o in outs]).tolist())
    assert mine == list(range(len(shots)))
    for o in outs:
        scale = np.abs(ref["g_vs"]).max()
        assert np.allclose(o["g_vs"], ref["g_vs"], rtol=1e-5, atol=1e-6 * scale)
        assert np.allclose(o["g_rho"], ref["g_rho"], rtol=1e-5, atol=1e-6 * np.abs(ref["g_rho"]).max())
        assert abs(float(o["l2"]) - ref["l2"]) <= 1e-12 * ref["l2"] + 1e-30
    assert np.array_equal(outs[0]["g_vs"], outs[1]["g_vs"])
    for o in outs:
        assert np.array_equal(o["bvs"], (m.vs * np.float32(1.01)).astype(np.float32))
        assert np.array_equal(o["brho"], m.rho) and bool(o["bqs_none"])
        ref_mis = _local_gradient(m, shots, obs, [0, 2, 4])["l2"]
        assert abs(float(o["mis"]) - ref_mis) <= 1e-12 * ref_mis


@pytest.mark.timeout(120)
def test_rank_failure_is_detected_not_hung(tmp_path):
    port = _free_port()
    try:
        mp.start_processes(_worker, args=(2, port, str(tmp_path), 1), nprocs=2, start_method="spawn")
    except Exception:
        pass
    err = (tmp_path / "err0.txt").read_text() if (tmp_path / "err0.txt").exists() else ""
    assert err, "surviving rank did not report the failed collective"
    assert (tmp_path / "err1.txt").exists()


def _case_visc():
    import oracle as O

    rng = np.random.default_rng(9)
    nx, ny, nt = 40, 30, 90
    vs = (200 + 30 * rng.standard_normal((ny, nx))).clip(120, 300).astype(np.float32)
    rho = (1800 + 60 * rng.standard_normal((ny, nx))).astype(np.float32)
    qs = rng.uniform(20, 60, (ny, nx)).astype(np.float32)
    m = O.Model(nx=nx, ny=ny, nt=nt, dh=0.5, dt=2e-4, vs=vs, rho=rho, qs=qs, fdorder=4, fw=6, fpml=30.0, l=2,
                fl=(7.5, 30.0), damping=float(vs.max()))
    shots = []
    for k in range(4):
        sp = np.zeros((8, 1), np.float32)
        sp[:, 0] = [6 + 9 * k, 2, 0, -0.01, 60.0, 1.0, 0, 3]
        shots.append((sp, np.array([[4, 14, 24, 34], [1, 1, 1, 1]], np.int32)))
    obs = []
    for sp, rec in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sp, rec) * np.float32(0.6)).astype(np.float32))
        o.close()
    return m, shots, obs


def _local_gradient_q(m, shots, obs, idx):
    import oracle as O

    out = _local_gradient(m, shots, obs, idx)
    gq = np.zeros((m.ny, m.nx), np.float64)
    for k in idx:
        o = O.Oracle(m, "port", grad_q=True)
        o.forward(shots[k][0], shots[k][1], store=True)
        o.residual(obs[k])
        o.adjoint()
        gq += o.grad_q()
        o.close()
    out["g_qs"] = gq
    return out


def _worker_q(rank, world, port, outdir):
    import datetime
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "denise-sh_b200"), os.path.join(root, "oracle")]
    import torch.distributed as dist

    from dsh.distributed import distributed_gradient

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=8))
    m, shots, obs = _case_visc()
    try:
        res = distributed_gradient(lambda idx: _local_gradient_q(m, shots, obs, idx), len(shots), (m.ny, m.nx),
                                   with_q=True)
        np.savez(os.path.join(outdir, f"q{rank}.npz"), g_qs=res.g_qs, g_vs=res.g_vs, mine=np.array(res.my_shots))
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_the_qs_gradient(tmp_path):
    """The Qs gradient travels in the same all-reduce as g_vs and g_rho: two
    gloo ranks, each with half of the shots, give the single-process sum."""
    port = _free_port()
    mp.start_processes(_worker_q, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    m, shots, obs = _case_visc()
    ref = _local_gradient_q(m, shots, obs, list(range(len(shots))))
    outs = [np.load(tmp_path / f"q{r}.npz") for r in range(2)]
    assert sorted(np.concatenate([o["mine"] for o in outs]).tolist()) == list(range(len(shots)))
    for o in outs:
        scale = np.abs(ref["g_qs"]).max()
        assert scale > 0
        assert np.allclose(o["g_qs"], ref["g_qs"], rtol=1e-5, atol=1e-6 * scale)
