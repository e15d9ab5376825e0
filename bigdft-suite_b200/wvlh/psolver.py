"""Hartree potential on a periodic real-space grid (the reference's PSolver
with periodic boundary conditions, order-16 interpolating scaling functions):
wvlh_psolver_periodic on the device (cuFFT transforms, the library's kernel
multiply and energy reduction)."""
import ctypes as C

from ._lib import WvlhError, check, lib


def hartree_periodic(ctx, rho, h, offset=0.0, pot=None, energy=True):
    """rho: (n3, n2, n1) float64 device tensor (x fastest), h: (hx, hy, hz).
    Returns (pot, eh): the potential (a new tensor unless pot is given; pot
    may be rho itself when energy is False) and the Hartree energy
    0.5 sum(rho V) hx hy hz as a 0-d device tensor (None without energy)."""
    torch = ctx.torch
    if rho.dtype != torch.float64 or rho.dim() != 3 or not rho.is_contiguous():
        raise WvlhError("rho: contiguous 3D float64 device tensor (z, y, x)")
    if pot is None:
        pot = torch.empty_like(rho)
    if pot.shape != rho.shape or pot.dtype != torch.float64 or not pot.is_contiguous():
        raise WvlhError("pot: a tensor like rho")
    n = (C.c_int * 3)(rho.shape[2], rho.shape[1], rho.shape[0])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    eh = torch.empty((), dtype=torch.float64, device=rho.device) if energy else None
    check(lib().wvlh_psolver_periodic(ctx.h, n, hh, C.c_void_p(rho.data_ptr()), C.c_void_p(pot.data_ptr()),
                                      float(offset), C.c_void_p(eh.data_ptr()) if energy else None),
          "wvlh_psolver_periodic")
    return pot, eh
