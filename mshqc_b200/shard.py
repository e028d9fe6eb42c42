"""One MP2 gradient shared among the GPUs of a job.

Every rank holds the same inputs (Cholesky vectors and orbitals), sets its
share with ``Context.set_partition(rank, world)`` and calls the gradient; the
library computes that rank's block pairs of occupied orbitals (the
independent (i, j) tiles of the backward, the bulk of the work) and returns
their energy, dE/dC and dE/deps.  ``allreduce_gradient`` then adds the
shares over the ranks: the one exchange step of the path, 3 + 2 N^2 + 2 N
doubles at most, by ``torch.distributed.all_reduce`` (NCCL for CUDA tensors,
gloo for host ones).
"""
from __future__ import annotations

import numpy as np

from . import capi

ENERGY_KEYS = ("ss_aa", "ss_bb", "os", "total")


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
