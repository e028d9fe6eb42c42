"""One MP2 gradient shared among the GPUs of a job.

Every rank holds the same inputs (Cholesky vectors and orbitals), sets its
share with ``Context.set_partition(rank, world)`` and calls the gradient; the
library computes that rank's block pairs of occupied orbitals (the
independent (i, j) tiles of the backward, the bulk of the work) and returns
their energy, dE/dC and dE/deps.  ``allreduce_gradient`` then adds the
shares over the ranks, 3 + 2 N^2 + 2 N doubles at most, by
``torch.distributed.all_reduce`` (NCCL for CUDA tensors, gloo for host ones).
With ``Context.set_collectives(*nccl_collectives(device))`` the half
transforms and the transposed transforms are shared over occupied orbitals
as well: an all-gather of the MO vectors B after the forward transforms and
a reduce-scatter of Gamma before the transposed ones, in place on the
library's device buffers.
"""
from __future__ import annotations

import numpy as np

from . import capi

ENERGY_KEYS = ("ss_aa", "ss_bb", "os", "total")


class _DeviceArray:
    """count doubles of device memory at address ptr, for torch.as_tensor
    (zero copy, through the CUDA array interface)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def _device_tensor(ptr, count, device):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, count), device=device)


def nccl_collectives(device, group=None):
    """(allgather, reduce_scatter) for Context.set_collectives over an NCCL
    process group: in place on the library's buffer, on the library's
    stream (torch.distributed all_gather_into_tensor / reduce_scatter_tensor
    with the rank's chunk as input / output)."""
    import torch
    import torch.distributed as dist

    def run(ptr, count, stream, gather):
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        full = _device_tensor(ptr, world * count, device)
        mine = full[rank * count:(rank + 1) * count]
        with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=device)):
            if gather:
                dist.all_gather_into_tensor(full, mine, group=group)
            else:
                dist.reduce_scatter_tensor(mine, full, op=dist.ReduceOp.SUM, group=group)

    return (lambda p, c, st: run(p, c, st, True)), (lambda p, c, st: run(p, c, st, False))


def staged_collectives(device, group=None):
    """The same operations staged through host memory over a CPU process
    group (gloo): for ranks that share one GPU in tests, or jobs without
    NCCL.  The library's stream is synchronized before the copies."""
    import torch
    import torch.distributed as dist

    def run(ptr, count, stream, gather):
        torch.cuda.ExternalStream(stream, device=device).synchronize()
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        full = _device_tensor(ptr, world * count, device)
        host = full.cpu()
        if gather:
            parts = [torch.empty(count, dtype=torch.float64) for _ in range(world)]
            dist.all_gather(parts, host[rank * count:(rank + 1) * count].clone(), group=group)
            full.copy_(torch.cat(parts))
        else:
            dist.all_reduce(host, op=dist.ReduceOp.SUM, group=group)
            full[rank * count:(rank + 1) * count].copy_(host[rank * count:(rank + 1) * count])
        torch.cuda.synchronize(device)

    return (lambda p, c, st: run(p, c, st, True)), (lambda p, c, st: run(p, c, st, False))


def allreduce_gradient(g: capi.Gradient, group=None, device=None) -> capi.Gradient:
    """Sum of the ranks' partial gradients, on every rank.

    Works on the numpy results of ``Context.mp2_gradient`` (reduced as CPU
    tensors, so the process group needs a CPU backend such as gloo, or staged
    through ``device`` -- a CUDA device for NCCL -- and returned as numpy) and
    on the CUDA tensors of ``Context.mp2_gradient_torch`` (NCCL).  Timings in
    ``g.energy`` stay this rank's own."""
    import torch
    import torch.distributed as dist

    parts = [x for x in (g.dC_a, g.deps_a, g.dC_b, g.deps_b) if x is not None]
    on_torch = isinstance(g.dC_a, torch.Tensor)
    dev = g.dC_a.device if on_torch else torch.device(device if device is not None else "cpu")
    e = torch.tensor([float(g.energy[k]) for k in ENERGY_KEYS], dtype=torch.float64, device=dev)
    flat = torch.cat([e] + [(x if on_torch else torch.from_numpy(np.asarray(x))).reshape(-1).to(dev, torch.float64)
                            for x in parts])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    energy = dict(g.energy)
    for k, v in zip(ENERGY_KEYS, flat[:len(ENERGY_KEYS)].tolist()):
        energy[k] = v
    out, off = [], len(ENERGY_KEYS)
    for x in parts:
        n = int(np.prod(x.shape))
        piece = flat[off:off + n].reshape(tuple(x.shape))
        off += n
        if not on_torch:
            piece = piece.cpu().numpy().copy(order="F" if np.asarray(x).flags.f_contiguous and x.ndim == 2 else "C")
        out.append(piece)
    it = iter(out)
    dC_a = next(it)
    deps_a = next(it)
    dC_b = next(it) if g.dC_b is not None else None
    deps_b = next(it) if g.deps_b is not None else None
    return capi.Gradient(energy, dC_a, dC_b, deps_a, deps_b)
