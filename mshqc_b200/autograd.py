"""Differentiable CD-MP2 energy for PyTorch.

``mp2_energy(context, C, eps, nocc, ...)`` returns the CD-RMP2 (or, with beta
orbitals, CD-UMP2) correlation energy as a 0-d float64 tensor whose backward
gives the exact dE/dC and dE/deps from the library's backward pass
(mshqc_cd_mp2_gradient): Gamma^Q_ia = sum_jb t~_ij^ab B^Q_jb, then the
transposed half transforms.  Orbital energies enter only the denominators,
as in the reference (src/mp2/cholesky_rmp2.cc:135-151,
src/mp2/cholesky_ump2.cc:299-465).  The Cholesky vectors are fixed inputs of
the context (``context.set_vectors``), not differentiated.

An orbital-rotation gradient follows from autograd through any
parametrisation of C, e.g. C(kappa) = C0 @ torch.linalg.matrix_exp(-kappa).
"""
from __future__ import annotations

import torch

from . import capi

PRECISIONS = {"fp64": capi.FP64, "fp16x3": capi.FP16X3}


class CDMP2Energy(torch.autograd.Function):
    """forward(context, kind, precision, nocc_a, nocc_b, C_a, eps_a, C_b, eps_b) -> E."""

    @staticmethod
    def forward(fctx, context, kind, precision, nocc_a, nocc_b, C_a, eps_a, C_b, eps_b):
        context.set_orbitals(capi.ALPHA, C_a.detach(), eps_a.detach(), nocc_a)
        if kind == capi.UNRESTRICTED:
            context.set_orbitals(capi.BETA, C_b.detach(), eps_b.detach(), nocc_b)
        needs = any(fctx.needs_input_grad[5:])
        if needs:
            g = context.mp2_gradient_torch(kind, precision, device=C_a.device)
            e = g.energy["total"]
            if kind == capi.UNRESTRICTED:
                fctx.save_for_backward(g.dC_a, g.deps_a, g.dC_b, g.deps_b)
            else:
                fctx.save_for_backward(g.dC_a, g.deps_a)
        else:
            e = context.mp2_energy(kind, precision)["total"]
        fctx.kind = kind
        return torch.tensor(e, dtype=torch.float64, device=C_a.device)

    @staticmethod
    def backward(fctx, grad_e):
        saved = fctx.saved_tensors
        dC_a, de_a = saved[0] * grad_e, saved[1] * grad_e
        dC_b = de_b = None
        if fctx.kind == capi.UNRESTRICTED:
            dC_b, de_b = saved[2] * grad_e, saved[3] * grad_e
        return None, None, None, None, None, dC_a, de_a, dC_b, de_b


def mp2_energy(context: capi.Context, C: torch.Tensor, eps: torch.Tensor, nocc: int,
               C_b: torch.Tensor | None = None, eps_b: torch.Tensor | None = None,
               nocc_b: int | None = None, precision: str = "fp64") -> torch.Tensor:
    """Differentiable MP2 correlation energy.

    C: (N, N) float64 CUDA tensor C[mu, p] (first ``nocc`` columns occupied);
    eps: (N,).  With C_b / eps_b / nocc_b the unrestricted energy
    E_ss(aa) + E_ss(bb) + E_os is returned.  precision: "fp64" or "fp16x3"."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    for name, t in (("C", C), ("eps", eps)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64):
            raise ValueError(f"{name} must be a float64 CUDA tensor")
    kind = capi.UNRESTRICTED if C_b is not None else capi.RESTRICTED
    if kind == capi.UNRESTRICTED and (eps_b is None or nocc_b is None):
        raise ValueError("C_b needs eps_b and nocc_b")
    torch.cuda.current_stream(C.device).synchronize()
    return CDMP2Energy.apply(context, kind, PRECISIONS[precision], int(nocc),
                             int(nocc_b) if nocc_b is not None else 0, C, eps, C_b, eps_b)
