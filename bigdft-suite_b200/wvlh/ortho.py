"""Overlap matrix and orthonormalisation of the orbitals (FP64).

``overlap`` forms S = Psi Psi^T with the library's FP64 tensor-core kernel
(the reference's ``getOverlap``, ``wfn_opt/orthogonality.f90:2624-2697``).
``orthonormalize`` then applies either the Cholesky scheme (``cholesky``,
:2297-2430: S = L L^T, Psi <- L^-1 Psi) or the Loewdin scheme (``loewdin``,
:2431-2500: Psi <- S^-1/2 Psi), in FP64 on the device: the psi-sized
product on the library's tensor-core panel apply (``panel_apply``), the
small dense factorisations (norb x norb) with torch.linalg (cuSOLVER).
``orthoconstraint`` is the gradient step that follows the Hamiltonian
(:375-625): Lagrange multipliers L = <psi_i|hpsi_j> on the same tensor-core
kernel, symmetrised and corrected for unequal occupations
(``lagrange_multiplier``, :293-369), then hpsi <- hpsi - L^T psi
(``subspace_update``, :254-271) on the panel apply.
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


def panel_apply(ctx, M, psi, out=None, alpha=1.0, beta=0.0, lower=False):
    """out = beta out + alpha M psi on the FP64 tensor-core kernel
    (wvlh_panel_apply): M (norb, norb) float64, psi and out (norb, K) float64
    device tensors with one row stride; out must not alias psi."""
    torch = ctx.torch
    norb, K = psi.shape
    if psi.dtype != torch.float64 or M.dtype != torch.float64 or M.shape != (norb, norb):
        raise WvlhError("panel_apply: FP64 M (norb, norb) and psi (norb, K)")
    if psi.stride(1) != 1:
        raise WvlhError("rows must be contiguous")
    M = M.contiguous()
    if out is None:
        out = torch.empty_like(psi)
    if out.stride() != psi.stride():
        raise WvlhError("out and psi must share one layout")
    check(lib().wvlh_panel_apply(ctx.h, int(norb), int(K), int(psi.stride(0)), C.c_void_p(M.data_ptr()),
                                 int(bool(lower)), float(alpha), C.c_void_p(psi.data_ptr()), float(beta),
                                 C.c_void_p(out.data_ptr())), "wvlh_panel_apply")
    return out


def orthonormalize(ctx, psi, method="cholesky", work=None):
    """In place on a (norb, K) float64 device tensor; returns (psi, S).

    Cholesky (orthogonality.f90:2297-2430): S = L L^T (dpotrf), L^-1
    (dtrtri) and psi <- L^-1 psi (dtrmm), the last on the library's
    tensor-core panel apply with the triangle's empty slices skipped.
    Loewdin (:2431-2500): S = U w U^T (dsyev), psi <- U w^-1/2 U^T psi on the
    same kernel.  The norb x norb factorisations use torch.linalg (cuSOLVER);
    work: an optional (norb, K) buffer for the product."""
    torch = ctx.torch
    S = overlap(ctx, psi)
    if method == "cholesky":
        L = torch.linalg.cholesky(S)
        eye = torch.eye(L.shape[0], dtype=L.dtype, device=L.device)
        M = torch.linalg.solve_triangular(L, eye, upper=False)
        lower = True
    elif method == "loewdin":
        w, U = torch.linalg.eigh(S)
        M = (U * w.rsqrt()) @ U.T
        lower = False
    else:
        raise WvlhError("method must be 'cholesky' or 'loewdin'")
    out = panel_apply(ctx, M, psi, out=work, lower=lower)
    psi.copy_(out)
    return psi, S


def subspace_matrix(ctx, psi, hpsi, L=None):
    """L[i, j] = <psi_i | hpsi_j> (FP64, norb x norb) of two (norb, K) device
    tensors with one dtype and row stride."""
    torch = ctx.torch
    if psi.dim() != 2 or hpsi.shape != psi.shape or psi.dtype != hpsi.dtype or psi.stride() != hpsi.stride():
        raise WvlhError("psi, hpsi: 2D tensors of one shape, dtype and layout")
    if psi.stride(1) != 1:
        raise WvlhError("rows must be contiguous")
    prec = {torch.float32: 32, torch.float64: 64}.get(psi.dtype)
    if prec is None:
        raise WvlhError("psi must be float32 or float64")
    norb, K = psi.shape
    if L is None:
        L = torch.empty(norb, norb, dtype=torch.float64, device=psi.device)
    check(lib().wvlh_subspace_matrix(ctx.h, prec, int(norb), int(K), int(psi.stride(0)),
                                     C.c_void_p(psi.data_ptr()), C.c_void_p(hpsi.data_ptr()),
                                     C.c_void_p(L.data_ptr())), "wvlh_subspace_matrix")
    return L


def lagrange_multiplier(L, occup, symm=True, correction=True):
    """In place on the (norb, norb) FP64 matrix L[i, j] = <psi_i|hpsi_j>, as the
    reference's lagrange_multiplier (orthogonality.f90:293-369) with real
    coefficients: its row loop symmetrises each pair (i < j) before either
    element is scaled, so the result is the symmetrised matrix followed by the
    occupation correction L[i, j] *= (f_i - f_j) / (2 f_i) (1/2 when |f_i| <=
    0.5) wherever f_i != f_j.  Returns (trace, asymm, mix): the trace, the
    largest (L_ij - L_ji)^2 and the largest squared coupling between states of
    different occupation."""
    import torch as _t
    f = _t.as_tensor(occup, dtype=_t.float64, device=L.device)
    trace = L.diagonal().sum()
    iu = _t.triu_indices(L.shape[0], L.shape[0], 1, device=L.device)
    d = L[iu[0], iu[1]] - L[iu[1], iu[0]]
    asymm = (d * d).max() if d.numel() else _t.zeros((), dtype=_t.float64, device=L.device)
    if symm:
        u = 0.5 * (L[iu[0], iu[1]] + L[iu[1], iu[0]])
        L[iu[0], iu[1]] = u
        L[iu[1], iu[0]] = u
    diff = f[:, None] != f[None, :]
    mix = (L * L)[diff].max() if bool(diff.any()) else _t.zeros((), dtype=_t.float64, device=L.device)
    if correction:
        fac = _t.where(f.abs()[:, None] > 0.5, 0.5 * (f[:, None] - f[None, :]) / f[:, None],
                       _t.full_like(L, 0.5))
        L.copy_(_t.where(diff, fac * L, L))
    return float(trace), float(asymm), float(mix)


def orthoconstraint(ctx, psi, hpsi, occup=None, symm=True, tr_min=False):
    """The orthogonality constraint on the gradient (orthoconstraint,
    orthogonality.f90:375-625) for real orbitals of one spin and k-point:
    L = <psi|hpsi>, lagrange_multiplier, hpsi -= L^T psi.  In place on hpsi;
    returns (L, trace, asymm, mix) (scprsum = occ x trace, occ = kwgt (3 -
    nspin) for the caller)."""
    torch = ctx.torch
    norb = psi.shape[0]
    if occup is None:
        occup = [2.0] * norb
    L = subspace_matrix(ctx, psi, hpsi)
    trace, asymm, mix = lagrange_multiplier(L, occup, symm=symm, correction=not tr_min)
    if psi.dtype == torch.float64 and hpsi.dtype == torch.float64 and psi.stride() == hpsi.stride():
        panel_apply(ctx, L.T.contiguous(), psi, out=hpsi, alpha=-1.0, beta=1.0)   # subspace_update
    else:
        hpsi.sub_(L.T.to(hpsi.dtype) @ psi)
    return L, trace, asymm, mix
