"""Shot-parallel FWI gradients over several GPUs (one process per GPU).

The reference distributes one shot loop over MPI ranks and combines results
with MPI_Allreduce (src/denise.c:1689-1729, src/catseis.c:34).  Here every
rank owns whole shots: shots are assigned to ranks by a greedy cost model
(largest first onto the least loaded rank), each rank computes the summed
gradient of its shots with its own engine, and one all-reduce (NCCL on GPUs,
gloo on CPU) sums gradients and misfits.  No halo exchange exists: each grid
lives on one GPU.  The conversion to (vs, rho) is linear in the shot sums, so
summing converted per-rank gradients equals converting the global sum up to
float rounding.  Per iteration the updated model goes out from rank 0 in one
broadcast (broadcast_model) and the line search's test-shot misfits come back
in one scalar all-reduce per test step (distributed_misfit), as the reference
sums them over ranks (src/line_search.c:300-306).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np


def shot_cost(nx: int, ny: int, nt: int, l: int) -> float:
    """Relative cost of one shot: grid-point updates weighted by the
    viscoelastic memory-variable work (1 + 2L/3)."""
    return float(nx) * ny * nt * (1.0 + 2.0 * l / 3.0)


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of items to `world` ranks.
    Deterministic: ties broken by item index, then by rank index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += costs[k]
    for p in parts:
        p.sort()
    return parts


@dataclass
class GradientResult:
    g_vs: np.ndarray
    g_rho: np.ndarray
    l2: float
    my_shots: list[int]
    g_qs: np.ndarray | None = None


def distributed_gradient(local_gradient: Callable[[list[int]], dict], nshots: int, shape: tuple[int, int],
                         costs: Sequence[float] | None = None, group=None, device=None,
                         with_q: bool = False) -> GradientResult:
    """Sum of per-shot gradients over all ranks of `group`.

    local_gradient(indices) must return {"g_vs", "g_rho", "l2"} (and "g_qs",
    the Qs gradient, when with_q is set) for the given shot indices (e.g. a
    closure over dsh.Engine.gradient and Engine.gradient_q); a rank with no
    shots contributes zeros.  The Qs gradient is a plain sum over shots (no
    preconditioning), so it travels in the same all-reduce.  Every rank takes
    the same collective steps."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    parts = partition(costs if costs is not None else [1.0] * nshots, world)
    mine = parts[rank]
    if mine:
        out = local_gradient(mine)
        gv, gr, l2 = np.asarray(out["g_vs"], np.float32), np.asarray(out["g_rho"], np.float32), float(out["l2"])
        gq = np.asarray(out["g_qs"], np.float32) if with_q else None
    else:
        gv = np.zeros(shape, np.float32)
        gr = np.zeros(shape, np.float32)
        l2 = 0.0
        gq = np.zeros(shape, np.float32) if with_q else None
    if world == 1:
        return GradientResult(gv, gr, l2, mine, gq)
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() and dist.get_backend(group) == "nccl"
                                             else "cpu")
    parts_ = [gv.ravel(), gr.ravel()] + ([gq.ravel()] if with_q else [])
    buf = torch.from_numpy(np.concatenate(parts_)).to(dev)
    l2t = torch.tensor([l2], dtype=torch.float64, device=dev)
    dist.all_reduce(buf, group=group)
    dist.all_reduce(l2t, group=group)
    buf = buf.cpu().numpy()
    n = gv.size
    return GradientResult(buf[:n].reshape(shape), buf[n:2 * n].reshape(shape), float(l2t.item()), mine,
                          buf[2 * n:3 * n].reshape(shape) if with_q else None)


def _device(group, device):
    import torch
    import torch.distributed as dist

    if device is not None:
        return device
    return "cuda" if torch.cuda.is_available() and dist.get_backend(group) == "nccl" else "cpu"


def broadcast_model(vs: np.ndarray, rho: np.ndarray, qs: np.ndarray | None = None, src: int = 0, group=None,
                    device=None):
    """Rank src's model (vs, rho[, qs]) on every rank of `group`, in one
    broadcast of the concatenated fields; returns the received arrays."""
    import torch
    import torch.distributed as dist

    fields = [vs, rho] + ([qs] if qs is not None else [])
    shape = np.asarray(vs).shape
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return tuple(np.asarray(f, np.float32) for f in fields) + ((None,) if qs is None else ())
    buf = torch.from_numpy(np.concatenate([np.asarray(f, np.float32).ravel() for f in fields])).to(_device(group, device))
    dist.broadcast(buf, src=src, group=group)
    out = buf.cpu().numpy()
    n = int(np.prod(shape))
    arrs = [out[k * n:(k + 1) * n].reshape(shape).copy() for k in range(len(fields))]
    return tuple(arrs) + ((None,) if qs is None else ())


def distributed_misfit(local_misfit: Callable[[list[int]], float], indices: Sequence[int],
                       costs: Sequence[float] | None = None, group=None, device=None) -> float:
    """Sum over ranks of local_misfit(my share of `indices`) (e.g. the test
    shots of one line-search step): the shots are partitioned like the
    gradient's, a rank without shots contributes 0, one scalar all-reduce."""
    import torch
    import torch.distributed as dist

    idx = list(indices)
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    parts = partition(costs if costs is not None else [1.0] * len(idx), world)
    mine = [idx[k] for k in parts[rank]]
    val = float(local_misfit(mine)) if mine else 0.0
    if world == 1:
        return val
    t = torch.tensor([val], dtype=torch.float64, device=_device(group, device))
    dist.all_reduce(t, group=group)
    return float(t.item())
