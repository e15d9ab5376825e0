"""Nonlocal pseudopotential projectors on the device.

Mirror of the reference's projector application for one set of orbitals on
one region (NonLocalHamiltonianApplication, bigdft/src/hpsiortho.f90:1044-1125,
through DFT_PSP_projectors_iter_apply, modules/psp_projectors.f90:585-712):
per atom, c = <p|psi> on the common points of the two key sets, hc = h c,
eproj += c . hc and hpsi += sum_i hc_i p_i.  The projector coefficients and
the coefficient matrices are given (the reference builds them from Gaussian
projectors and the HGH parameters); hgh_matrix builds an atom's matrix from
the HGH h_ij(l) blocks in the reference's projector order.
"""
import ctypes as C

import numpy as np

from ._lib import WvlhError, check, lib
from .batch import Region, _ptr


def hgh_matrix(hij, present):
    """The atom's coefficient matrix over its projectors, in the reference's
    order (apply_hij_coeff, orbitals/pseudopotentials.f90:1208-1292): l = 1..4,
    then i = 1..3 for the (i, l) present, then m = 1..2l-1.  hij[l-1][i-1][j-1]
    couples projectors (i, l, m) and (j, l, m) (same m); present[l-1][i-1] says
    whether projector (i, l) exists (the reference: h_ii(l) /= 0)."""
    idx = []
    for l in range(1, 5):
        for i in range(1, 4):
            if present[l - 1][i - 1]:
                for m in range(1, 2 * l):
                    idx.append((l, i, m))
    n = len(idx)
    h = np.zeros((n, n))
    for a, (l, i, m) in enumerate(idx):
        for b, (l2, j, m2) in enumerate(idx):
            if l == l2 and m == m2:
                h[a, b] = hij[l - 1][i - 1][j - 1]
    return h


class Projectors:
    """Projectors of several atoms against the orbitals of one region.

    atoms: sequence of (locreg, proj, h): the projectors' keys (a locreg of the
    same box), their coefficients (m vectors of the projector region's psi
    size, a 2D device float64 tensor or anything torch can take) and the m x m
    coefficient matrix (numpy)."""

    def __init__(self, ctx, psi_region, atoms):
        torch = ctx.torch
        self.ctx = ctx
        self.psi_region = psi_region
        self.regions = [Region(ctx, lr) for lr, _, _ in atoms]
        nproj, blocks, hs = [], [], []
        for reg, (lr, p, h) in zip(self.regions, atoms):
            p = torch.as_tensor(p, dtype=torch.float64, device=ctx.device).reshape(-1, reg.psi_size)
            h = np.ascontiguousarray(h, np.float64)
            if h.shape != (p.shape[0], p.shape[0]):
                raise WvlhError("h must be m x m for m projectors")
            nproj.append(p.shape[0])
            blocks.append(p.reshape(-1))
            hs.append(h.ravel())
        proj = torch.cat(blocks).contiguous() if blocks else torch.zeros(1, dtype=torch.float64, device=ctx.device)
        hcat = np.ascontiguousarray(np.concatenate(hs) if hs else np.zeros(1))
        regs = (C.c_void_p * max(1, len(self.regions)))(*[r.h for r in self.regions])
        np_arr = (C.c_int * max(1, len(nproj)))(*nproj)
        h = C.c_void_p()
        check(lib().wvlh_nlpsp_create(ctx.h, psi_region.h, len(self.regions), regs, np_arr, _ptr(proj),
                                      hcat.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)), "wvlh_nlpsp_create")
        self.h = h
        self.nproj = nproj

    def apply(self, psi, hpsi, eproj=None):
        """hpsi += V_nl psi for the rows of psi (2D float64 device tensors on
        the psi region's keys); returns eproj (FP64, one per row)."""
        torch = self.ctx.torch
        if psi.dtype != torch.float64 or hpsi.dtype != torch.float64 or psi.dim() != 2 or hpsi.shape != psi.shape:
            raise WvlhError("psi, hpsi: 2D float64 tensors of one shape")
        if psi.stride(1) != 1 or hpsi.stride(0) != psi.stride(0) or hpsi.stride(1) != 1:
            raise WvlhError("rows must be contiguous with one row stride")
        norb = psi.shape[0]
        if eproj is None:
            eproj = torch.empty(norb, dtype=torch.float64, device=psi.device)
        check(lib().wvlh_nlpsp_apply(self.h, norb, _ptr(psi), psi.stride(0), _ptr(hpsi), _ptr(eproj)),
              "wvlh_nlpsp_apply")
        return eproj

    def close(self):
        if getattr(self, "h", None):
            lib().wvlh_nlpsp_destroy(self.h)
            self.h = None
        for r in getattr(self, "regions", []):
            r.close()
        self.regions = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
