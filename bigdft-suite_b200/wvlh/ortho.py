"""Overlap matrix and orthonormalisation of the orbitals (FP64).

``overlap`` forms S = Psi Psi^T with the library's FP64 tensor-core kernel
(the reference's ``getOverlap``, ``wfn_opt/orthogonality.f90:2624-2697``).
``orthonormalize`` then applies either the Cholesky scheme (``cholesky``,
:2297-2430: S = L L^T, Psi <- L^-1 Psi) or the Loewdin scheme (``loewdin``,
:2431-2500: Psi <- S^-1/2 Psi), in FP64 on the device; the small dense
factorisations (norb x norb) use torch.linalg (cuSOLVER).
"""
import ctypes as C

from ._lib import WvlhError, check, lib


def overlap(ctx, psi, norb=None, K=None, ld=None, S=None):
    """psi: device tensor, either (norb, K) or flat with a row stride ld."""
    torch = ctx.torch
    if psi.dim() == 2:
        norb, K = psi.shape
        ld = psi.stride(0)
        if psi.stride(1) != 1:
            raise WvlhError("rows must be contiguous")
    if ld is None:
        ld = K
    prec = {torch.float32: 32, torch.float64: 64}.get(psi.dtype)
    if prec is None:
        raise WvlhError("psi must be float32 or float64")
    if S is None:
        S = torch.empty(norb, norb, dtype=torch.float64, device=psi.device)
    check(lib().wvlh_overlap(ctx.h, prec, int(norb), int(K), int(ld), C.c_void_p(psi.data_ptr()),
                             C.c_void_p(S.data_ptr())), "wvlh_overlap")
    return S


def orthonormalize(ctx, psi, method="cholesky"):
    """In place on a (norb, K) float64 device tensor; returns (psi, S)."""
    torch = ctx.torch
    S = overlap(ctx, psi)
    if method == "cholesky":
        L = torch.linalg.cholesky(S)
        psi.copy_(torch.linalg.solve_triangular(L, psi, upper=False))
    elif method == "loewdin":
        w, U = torch.linalg.eigh(S)
        psi.copy_((U * w.rsqrt()) @ U.T @ psi)
    else:
        raise WvlhError("method must be 'cholesky' or 'loewdin'")
    return psi, S
