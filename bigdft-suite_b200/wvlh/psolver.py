"""The potential from the density: the Hartree potential on a periodic
real-space grid (the reference's PSolver with periodic boundary conditions,
order-16 interpolating scaling functions; wvlh_psolver_periodic: cuFFT
transforms, the library's kernel multiply and energy reduction), the
exchange-correlation potential of the reference's default LDA (ixc = 1,
wvlh_xc_lda) and their sum with an external potential, the Kohn-Sham potential
of updatePotential (wvlh_ks_potential_periodic)."""
import ctypes as C

from ._lib import WvlhError, check, lib


def free_kernel_tables(n, h):
    """Host side of the free-BC kernel (no device work): (nf, rows, w) with
    nf the padded FFT lengths (N1, N2, N3), rows (89, N1/2+N2/2+N3/2+3) the
    1D cosine tables [C_x | C_y | C_z] per Gaussian and w the 89 weights."""
    import numpy as np
    nn = (C.c_int * 3)(*[int(v) for v in n])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    nf = (C.c_int * 3)()
    need = lib().wvlh_psolver_free_tables(nn, hh, nf, None, 0)
    if need < 0:
        check(-int(need), "wvlh_psolver_free_tables")
    tab = np.zeros(need)
    check(max(0, -int(lib().wvlh_psolver_free_tables(nn, hh, nf, tab.ctypes.data_as(C.c_void_p), need))),
          "wvlh_psolver_free_tables")
    return tuple(nf), tab[:-89].reshape(89, -1), tab[-89:]


def hartree_free(ctx, rho, h, pot=None, energy=True):
    """The Hartree potential with free (isolated) boundary conditions
    (wvlh_psolver_free); arguments and results as hartree_periodic."""
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
    check(lib().wvlh_psolver_free(ctx.h, n, hh, C.c_void_p(rho.data_ptr()), C.c_void_p(pot.data_ptr()),
                                  C.c_void_p(eh.data_ptr()) if energy else None), "wvlh_psolver_free")
    return pot, eh


def surface_kernel_table(n, h):
    """Host side of the surface-BC kernel (no device work): (N2, K), N2 the
    padded y length and K the (n3/2+1, N2/2+1, n1/2+1) Fourier table."""
    import numpy as np
    nn = (C.c_int * 3)(*[int(v) for v in n])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    N2 = C.c_int()
    need = lib().wvlh_psolver_surface_table(nn, hh, C.byref(N2), None, 0)
    if need < 0:
        check(-int(need), "wvlh_psolver_surface_table")
    tab = np.zeros(need)
    check(max(0, -int(lib().wvlh_psolver_surface_table(nn, hh, C.byref(N2), tab.ctypes.data_as(C.c_void_p), need))),
          "wvlh_psolver_surface_table")
    return N2.value, tab.reshape(n[2] // 2 + 1, N2.value // 2 + 1, n[0] // 2 + 1)


def wire_kernel_table(n, h):
    """Host side of the wire-BC kernel (no device work): ((Nx, Ny), K), the
    padded x and y lengths and the (n3/2+1, Ny/2+1, Nx/2+1) Fourier table."""
    import numpy as np
    nn = (C.c_int * 3)(*[int(v) for v in n])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    nf = (C.c_int * 2)()
    need = lib().wvlh_psolver_wire_table(nn, hh, nf, None, 0)
    if need < 0:
        check(-int(need), "wvlh_psolver_wire_table")
    tab = np.zeros(need)
    check(max(0, -int(lib().wvlh_psolver_wire_table(nn, hh, nf, tab.ctypes.data_as(C.c_void_p), need))),
          "wvlh_psolver_wire_table")
    return (nf[0], nf[1]), tab.reshape(n[2] // 2 + 1, nf[1] // 2 + 1, nf[0] // 2 + 1)


def _hartree_bc(ctx, fn, rho, h, pot, energy):
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
    check(getattr(lib(), fn)(ctx.h, n, hh, C.c_void_p(rho.data_ptr()), C.c_void_p(pot.data_ptr()),
                             C.c_void_p(eh.data_ptr()) if energy else None), fn)
    return pot, eh


def hartree_wire(ctx, rho, h, pot=None, energy=True):
    """The Hartree potential with wire boundary conditions (z periodic, x and
    y free; wvlh_psolver_wire); arguments and results as hartree_periodic."""
    return _hartree_bc(ctx, "wvlh_psolver_wire", rho, h, pot, energy)


def hartree_surface(ctx, rho, h, pot=None, energy=True):
    """The Hartree potential with surface boundary conditions (x, z periodic,
    y free; wvlh_psolver_surface); arguments and results as hartree_periodic."""
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
    check(lib().wvlh_psolver_surface(ctx.h, n, hh, C.c_void_p(rho.data_ptr()), C.c_void_p(pot.data_ptr()),
                                     C.c_void_p(eh.data_ptr()) if energy else None), "wvlh_psolver_surface")
    return pot, eh


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


def _check_rho(ctx, rho):
    torch = ctx.torch
    if rho.dtype != torch.float64 or not rho.is_contiguous() or not rho.is_cuda:
        raise WvlhError("rho: contiguous float64 device tensor")


def xc_lda(ctx, rho, vxc=None, accumulate=False, dvol=1.0, energy=True):
    """V_xc of the total density rho (any shape) for the Teter 1993 LDA
    (ixc = 1, spin-unpolarised): written into vxc (a new tensor unless given;
    added to it when accumulate).  Returns (vxc, energies), energies a
    (2,) device tensor (exc, evxc) = dvol * (sum eps rho, sum v_xc rho), or
    None without energy."""
    torch = ctx.torch
    _check_rho(ctx, rho)
    if vxc is None:
        if accumulate:
            raise WvlhError("accumulate needs vxc")
        vxc = torch.empty_like(rho)
    if vxc.shape != rho.shape or vxc.dtype != torch.float64 or not vxc.is_contiguous():
        raise WvlhError("vxc: a tensor like rho")
    en = torch.empty(2, dtype=torch.float64, device=rho.device) if energy else None
    check(lib().wvlh_xc_lda(ctx.h, rho.numel(), C.c_void_p(rho.data_ptr()), C.c_void_p(vxc.data_ptr()),
                            1 if accumulate else 0, float(dvol), C.c_void_p(en.data_ptr()) if energy else None),
          "wvlh_xc_lda")
    return vxc, en


def ks_potential_periodic(ctx, rho, h, vext=None, pot=None, energy=True, free=False):
    """pot = V_H[rho] + vext + V_xc[rho] on a periodic grid, or with free
    boundary conditions when free (rho: (n3, n2, n1) float64 device tensor,
    x fastest; vext None or a tensor like rho).  Returns (pot, energies),
    energies a (3,) device tensor (eh, exc, evxc), or None without energy."""
    torch = ctx.torch
    _check_rho(ctx, rho)
    if rho.dim() != 3:
        raise WvlhError("rho: (z, y, x) grid")
    if pot is None:
        pot = torch.empty_like(rho)
    for name, t in (("pot", pot), ("vext", vext)):
        if t is not None and (t.shape != rho.shape or t.dtype != torch.float64 or not t.is_contiguous()):
            raise WvlhError("%s: a tensor like rho" % name)
    n = (C.c_int * 3)(rho.shape[2], rho.shape[1], rho.shape[0])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    en = torch.empty(3, dtype=torch.float64, device=rho.device) if energy else None
    fn = "wvlh_ks_potential_free" if free else "wvlh_ks_potential_periodic"
    check(getattr(lib(), fn)(ctx.h, n, hh, C.c_void_p(rho.data_ptr()),
                             C.c_void_p(vext.data_ptr()) if vext is not None else None,
                             C.c_void_p(pot.data_ptr()), C.c_void_p(en.data_ptr()) if energy else None), fn)
    return pot, en


BC_CODES = {"periodic": 0, "free": 1, "surface": 2, "wire": 3}


def ks_potential(ctx, rho, h, bc="periodic", vext=None, pot=None, energy=True, rhocore=None):
    """The Kohn-Sham potential V_H + vext + V_xc and (eh, exc, evxc) for the
    boundary conditions bc ("periodic", "free", "surface": y free, "wire":
    x and y free), through wvlh_ks_potential_bc; rhocore: an optional core
    density for the nonlinear core correction (XC only)."""
    torch = ctx.torch
    _check_rho(ctx, rho)
    if rho.dim() != 3:
        raise WvlhError("rho: (z, y, x) grid")
    if bc not in BC_CODES:
        raise WvlhError("bc: one of %s" % sorted(BC_CODES))
    pot = torch.empty_like(rho) if pot is None else pot
    for name, t in (("pot", pot), ("vext", vext), ("rhocore", rhocore)):
        if t is not None and (t.shape != rho.shape or t.dtype != torch.float64 or not t.is_contiguous()):
            raise WvlhError("%s: a tensor like rho" % name)
    n = (C.c_int * 3)(rho.shape[2], rho.shape[1], rho.shape[0])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    en = torch.empty(3, dtype=torch.float64, device=rho.device) if energy else None
    check(lib().wvlh_ks_potential_bc(ctx.h, BC_CODES[bc], n, hh, C.c_void_p(rho.data_ptr()),
                                     C.c_void_p(rhocore.data_ptr()) if rhocore is not None else None,
                                     C.c_void_p(vext.data_ptr()) if vext is not None else None,
                                     C.c_void_p(pot.data_ptr()), C.c_void_p(en.data_ptr()) if energy else None),
          "wvlh_ks_potential_bc")
    return pot, en


def ks_potential_free(ctx, rho, h, vext=None, pot=None, energy=True):
    """ks_potential_periodic with free boundary conditions."""
    return ks_potential_periodic(ctx, rho, h, vext, pot, energy, free=True)


def xc_lsda(ctx, rho_up, rho_dn, vxc_up=None, vxc_dn=None, accumulate=False, dvol=1.0, energy=True):
    """Spin-polarised LDA (ixc = 1, nspin = 2) of the spin densities (two
    float64 device tensors of one shape): returns (vxc_up, vxc_dn, energies),
    energies a (2,) device tensor (exc, evxc) or None without energy."""
    torch = ctx.torch
    _check_rho(ctx, rho_up)
    _check_rho(ctx, rho_dn)
    if rho_up.shape != rho_dn.shape:
        raise WvlhError("rho_up and rho_dn must have one shape")
    if accumulate and (vxc_up is None or vxc_dn is None):
        raise WvlhError("accumulate needs vxc_up and vxc_dn")
    vxc_up = torch.empty_like(rho_up) if vxc_up is None else vxc_up
    vxc_dn = torch.empty_like(rho_dn) if vxc_dn is None else vxc_dn
    for t in (vxc_up, vxc_dn):
        if t.shape != rho_up.shape or t.dtype != torch.float64 or not t.is_contiguous():
            raise WvlhError("vxc: tensors like rho")
    en = torch.empty(2, dtype=torch.float64, device=rho_up.device) if energy else None
    check(lib().wvlh_xc_lsda(ctx.h, rho_up.numel(), C.c_void_p(rho_up.data_ptr()), C.c_void_p(rho_dn.data_ptr()),
                             C.c_void_p(vxc_up.data_ptr()), C.c_void_p(vxc_dn.data_ptr()), 1 if accumulate else 0,
                             float(dvol), C.c_void_p(en.data_ptr()) if energy else None), "wvlh_xc_lsda")
    return vxc_up, vxc_dn, en


def ks_potential_spin(ctx, rho_up, rho_dn, h, vext=None, free=False, pot_up=None, pot_dn=None, energy=True,
                      bc=None, rhocore=None):
    """The two Kohn-Sham potentials (nspin = 2) on a periodic grid, or with
    free boundary conditions when free (bc, one of BC_CODES, overrides free):
    returns (pot_up, pot_dn, energies), energies a (3,) device tensor (eh,
    exc, evxc) or None."""
    torch = ctx.torch
    for t in (rho_up, rho_dn):
        _check_rho(ctx, t)
    if rho_up.dim() != 3 or rho_dn.shape != rho_up.shape:
        raise WvlhError("rho_up, rho_dn: (z, y, x) grids of one shape")
    pot_up = torch.empty_like(rho_up) if pot_up is None else pot_up
    pot_dn = torch.empty_like(rho_up) if pot_dn is None else pot_dn
    for name, t in (("pot_up", pot_up), ("pot_dn", pot_dn), ("vext", vext), ("rhocore", rhocore)):
        if t is not None and (t.shape != rho_up.shape or t.dtype != torch.float64 or not t.is_contiguous()):
            raise WvlhError("%s: a tensor like rho" % name)
    n = (C.c_int * 3)(rho_up.shape[2], rho_up.shape[1], rho_up.shape[0])
    hh = (C.c_double * 3)(*[float(v) for v in h])
    en = torch.empty(3, dtype=torch.float64, device=rho_up.device) if energy else None
    code = BC_CODES[bc] if bc is not None else (1 if free else 0)
    check(lib().wvlh_ks_potential_spin(ctx.h, code, n, hh, C.c_void_p(rho_up.data_ptr()),
                                       C.c_void_p(rho_dn.data_ptr()),
                                       C.c_void_p(rhocore.data_ptr()) if rhocore is not None else None,
                                       C.c_void_p(vext.data_ptr()) if vext is not None else None,
                                       C.c_void_p(pot_up.data_ptr()), C.c_void_p(pot_dn.data_ptr()),
                                       C.c_void_p(en.data_ptr()) if energy else None), "wvlh_ks_potential_spin")
    return pot_up, pot_dn, en
