"""Batched local Hamiltonian over many orbitals and localisation regions.

The batch is the B200 form of the reference's orbital loop
(``LocalHamiltonianApplication``, ``bigdft/src/hpsiortho.f90:934-958``: for
each locreg, for each orbital, ``local_hamiltonian_ket``): all orbitals of all
regions go through one fused three-kernel launch sequence.  Coefficients of
orbital ``o`` are packed ``[psi_c | psi_f]`` (``nvctr_c + 7*nvctr_f`` values,
the reference's ``psi(nvctr_c+7*nvctr_f, norb)`` layout) starting at
``Batch.psi_offset(o)``; the potential of orbital ``o`` is an ISF grid (x
fastest) starting at ``pot_offset[o]``.
"""
import ctypes as C

import numpy as np

from ._lib import LocregDesc, OrbitalDesc, WvlhError, check, lib, require_cuda


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _fill_desc(d, L, keep):
    """wvlh_locreg of a Locreg; the key arrays are appended to keep."""
    d.n[:] = list(L.n)
    d.periodic[:] = list(L.periodic)
    d.hgrid[:] = list(L.hgrid)
    d.nseg_c, d.nseg_f = len(L.keyv_c), len(L.keyv_f)
    for nm in ("keyg_c", "keyv_c", "keyg_f", "keyv_f"):
        arr = np.ascontiguousarray(getattr(L, nm), np.int32)
        keep.append(arr)
        setattr(d, nm, arr.ctypes.data_as(C.POINTER(C.c_int32)))


class Context:
    """One device, one stream (the torch current stream at creation by default)."""

    def __init__(self, device=0, stream=None):
        torch = require_cuda()
        self.torch = torch
        self.device = device
        h = C.c_void_p()
        check(lib().wvlh_ctx_create(device, C.byref(h)), "wvlh_ctx_create")
        self.h = h
        s = stream if stream is not None else torch.cuda.current_stream(device)
        self.set_stream(s)

    def set_stream(self, stream):
        self.stream = stream
        check(lib().wvlh_ctx_set_stream(self.h, C.c_void_p(stream.cuda_stream)), "wvlh_ctx_set_stream")

    def synchronize(self):
        check(lib().wvlh_ctx_synchronize(self.h), "wvlh_ctx_synchronize")

    def close(self):
        if self.h:
            lib().wvlh_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    def __init__(self, ctx, locregs, orb_lr, pot_offset=None):
        self.ctx = ctx
        self.locregs = list(locregs)
        self.orb_lr = np.ascontiguousarray(orb_lr, np.int32)
        self.norb = len(self.orb_lr)
        descs = (LocregDesc * len(self.locregs))()
        self._keep = []
        for i, L in enumerate(self.locregs):
            _fill_desc(descs[i], L, self._keep)
        if pot_offset is None:
            po = None
            self.pot_offset = np.zeros(self.norb, np.int64)
        else:
            self.pot_offset = np.ascontiguousarray(pot_offset, np.int64)
            po = self.pot_offset.ctypes.data_as(C.POINTER(C.c_int64))
        h = C.c_void_p()
        rc = lib().wvlh_batch_create(ctx.h, len(self.locregs), descs, self.norb,
                                     self.orb_lr.ctypes.data_as(C.POINTER(C.c_int32)), po, C.byref(h))
        check(rc, "wvlh_batch_create")
        self.h = h
        self.psi_size = int(lib().wvlh_batch_psi_size(h))
        self.offsets = np.array([lib().wvlh_batch_psi_offset(h, o) for o in range(self.norb)], np.int64)

    def psi_offset(self, o):
        return int(self.offsets[o])

    def scratch_bytes(self, precision):
        return int(lib().wvlh_batch_scratch_bytes(self.h, precision))

    @property
    def pot_size(self):
        return int(max(self.pot_offset[o] + self.locregs[self.orb_lr[o]].nisf for o in range(self.norb)))

    @property
    def coarse_cells(self):
        return sum(self.locregs[l].coarse_cells for l in self.orb_lr)

    def locham(self, psi, pot, hpsi=None, ekin=None, epot=None, accumulate=False):
        """Device tensors; precision follows psi's dtype (float32 or float64)."""
        torch = self.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}.get(psi.dtype)
        if prec is None or pot.dtype != psi.dtype:
            raise WvlhError("psi and pot must both be float32 or float64")
        if psi.numel() < self.psi_size or pot.numel() < self.pot_size:
            raise WvlhError("psi/pot smaller than the batch layout")
        if hpsi is None:
            hpsi = torch.zeros_like(psi)
        if ekin is None:
            ekin = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        if epot is None:
            epot = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        rc = lib().wvlh_locham_batched(self.h, prec, _ptr(psi), _ptr(pot), _ptr(hpsi), _ptr(ekin), _ptr(epot),
                                       int(bool(accumulate)))
        check(rc, "wvlh_locham_batched")
        return hpsi, ekin, epot

    def autotune(self, psi, pot, hpsi=None, ekin=None, epot=None, reps=2):
        """Measure the plane kernels' block sizes on this batch's locham
        (wvlh_batch_autotune) and keep the fastest; returns (chosen,
        {block size: ms per call})."""
        torch = self.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}.get(psi.dtype)
        if prec is None or pot.dtype != psi.dtype:
            raise WvlhError("psi and pot must both be float32 or float64")
        if hpsi is None:
            hpsi = torch.empty_like(psi)
        if ekin is None:
            ekin = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        if epot is None:
            epot = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        chosen, n = C.c_int(), C.c_int()
        cand, ms = (C.c_int * 5)(), (C.c_double * 5)()
        check(lib().wvlh_batch_autotune(self.h, prec, _ptr(psi), _ptr(pot), _ptr(hpsi), _ptr(ekin), _ptr(epot),
                                        int(reps), C.byref(chosen), cand, ms, C.byref(n)), "wvlh_batch_autotune")
        return chosen.value, {int(cand[k]): float(ms[k]) for k in range(n.value)}

    def autotune_precond(self, x, rhs, cprec, ncong, reps=2):
        """Measure the plane kernels' block sizes on this batch's
        preconditioner (wvlh_batch_autotune_precond: ncong CG iterations per
        timed call; x is overwritten) and keep the fastest; returns (chosen,
        {block size: ms per call})."""
        torch = self.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}.get(x.dtype)
        if prec is None or rhs.dtype != x.dtype:
            raise WvlhError("x and rhs must both be float32 or float64")
        c = torch.as_tensor(cprec, dtype=torch.float64, device=x.device).contiguous()
        chosen, n = C.c_int(), C.c_int()
        cand, ms = (C.c_int * 5)(), (C.c_double * 5)()
        check(lib().wvlh_batch_autotune_precond(self.h, prec, int(ncong), _ptr(c), _ptr(x), _ptr(rhs), int(reps),
                                                C.byref(chosen), cand, ms, C.byref(n)),
              "wvlh_batch_autotune_precond")
        return chosen.value, {int(cand[k]): float(ms[k]) for k in range(n.value)}

    def block_sizes(self):
        """The CTA sizes the batch launches with (wvlh_batch_block_sizes):
        {"locham": {"plane": (fp32, fp64), "z": (fp32, fp64)}, "precond": ...}."""
        v = (C.c_int * 8)()
        check(lib().wvlh_batch_block_sizes(self.h, v), "wvlh_batch_block_sizes")
        return {"locham": {"plane": (v[0], v[1]), "z": (v[2], v[3])},
                "precond": {"plane": (v[4], v[5]), "z": (v[6], v[7])}}

    def locham_graph(self, psi, pot, hpsi, ekin, epot, accumulate=False):
        """Capture locham(psi, pot, hpsi, ekin, epot) into a CUDA graph; replay
        it with .launch() (the tensors must stay alive and in place)."""
        return LochamGraph(self, psi, pot, hpsi, ekin, epot, accumulate)

    def locham_host(self, psi, pot, hpsi, ekin, epot, precision):
        """Host buffers (numpy arrays or CPU tensors, ideally pinned)."""
        def addr(a):
            return C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)
        rc = lib().wvlh_locham_batched_host(self.h, precision, addr(psi), addr(pot), addr(hpsi), addr(ekin),
                                            addr(epot))
        check(rc, "wvlh_locham_batched_host")

    def locden(self, psi, hfac, rho):
        """rho[pot_offset[o] + r] += hfac[o] |psi_o(r)|^2 (rho FP64 device tensor, accumulated)."""
        torch = self.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}[psi.dtype]
        hf = torch.as_tensor(hfac, dtype=torch.float64, device=psi.device).contiguous()
        if rho.dtype != torch.float64 or rho.numel() < self.pot_size:
            raise WvlhError("rho must be a float64 tensor covering every density grid")
        check(lib().wvlh_locden_batched(self.h, prec, _ptr(psi), _ptr(hf), _ptr(rho)), "wvlh_locden_batched")
        self._keep_hf = hf
        return rho

    def precond(self, x, rhs, cprec, ncong, hist=None):
        """ncong CG iterations of the preconditioner for every orbital; x is
        overwritten with the result.  Returns x and the (ncong+1, norb)
        squared residual norms."""
        torch = self.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}[x.dtype]
        c = torch.as_tensor(cprec, dtype=torch.float64, device=x.device).contiguous()
        if hist is None:
            hist = torch.zeros(ncong + 1, self.norb, dtype=torch.float64, device=x.device)
        check(lib().wvlh_precond_batched(self.h, prec, int(ncong), _ptr(c), _ptr(x), _ptr(rhs), _ptr(hist)),
              "wvlh_precond_batched")
        self._keep_c = c
        return x, hist

    def locham_plain(self, psi, pot, hpsi=None, ekin=None, epot=None):
        """FP64, one kernel per 1D pass (the OpenCL backend's structure)."""
        torch = self.ctx.torch
        if psi.dtype != torch.float64 or pot.dtype != torch.float64:
            raise WvlhError("the plain path is FP64")
        if hpsi is None:
            hpsi = torch.zeros_like(psi)
        if ekin is None:
            ekin = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        if epot is None:
            epot = torch.empty(self.norb, dtype=torch.float64, device=psi.device)
        rc = lib().wvlh_locham_plain_batched(self.h, _ptr(psi), _ptr(pot), _ptr(hpsi), _ptr(ekin), _ptr(epot))
        check(rc, "wvlh_locham_plain_batched")
        return hpsi, ekin, epot

    def close(self):
        if getattr(self, "h", None):
            lib().wvlh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LochamGraph:
    """One packed-batch locham call captured as a CUDA graph (wvlh_locham_graph_create)."""

    def __init__(self, batch, psi, pot, hpsi, ekin, epot, accumulate=False):
        torch = batch.ctx.torch
        prec = {torch.float32: 32, torch.float64: 64}.get(psi.dtype)
        if prec is None or pot.dtype != psi.dtype or hpsi.dtype != psi.dtype:
            raise WvlhError("psi, pot and hpsi must share float32 or float64")
        self.batch = batch
        self._keep = (psi, pot, hpsi, ekin, epot)
        h = C.c_void_p()
        check(lib().wvlh_locham_graph_create(batch.h, prec, _ptr(psi), _ptr(pot), _ptr(hpsi), _ptr(ekin),
                                             _ptr(epot), int(bool(accumulate)), C.byref(h)),
              "wvlh_locham_graph_create")
        self.h = h

    def launch(self):
        check(lib().wvlh_graph_launch(self.h), "wvlh_graph_launch")

    def close(self):
        if getattr(self, "h", None):
            lib().wvlh_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Region:
    """A localisation region resident on the device: keys validated, decoded
    and uploaded once (wvlh_region_create), shared by every batch that
    names it."""

    def __init__(self, ctx, locreg):
        self.ctx = ctx
        self.locreg = locreg
        d = LocregDesc()
        keep = []
        _fill_desc(d, locreg, keep)
        h = C.c_void_p()
        check(lib().wvlh_region_create(ctx.h, C.byref(d), C.byref(h)), "wvlh_region_create")
        self.h = h
        self.psi_size = int(lib().wvlh_region_psi_size(h))
        self.grid_size = int(lib().wvlh_region_grid_size(h))

    def scratch_bytes(self, precision):
        """Fused-kernel scratch of one orbital of this region."""
        return int(lib().wvlh_region_scratch_bytes(self.h, precision))

    def close(self):
        if getattr(self, "h", None):
            lib().wvlh_region_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OrbitalBatch:
    """One launch over orbitals of any regions, each with its own device
    buffers (wvlh_batch_create_orbitals).  orbitals: sequence of
    (region, psi, hpsi, pot, rho) with tensors or None; the tables go to the
    context's arena, so launch before the next OrbitalBatch of the context."""

    def __init__(self, ctx, orbitals):
        self.ctx = ctx
        self.norb = len(orbitals)
        descs = (OrbitalDesc * self.norb)()
        self._keep = []
        dtype = None
        for i, (reg, psi, hpsi, pot, rho) in enumerate(orbitals):
            d = descs[i]
            d.region = reg.h.value
            for nm, t in (("psi", psi), ("hpsi", hpsi), ("pot", pot), ("rho", rho)):
                if t is not None:
                    self._keep.append(t)
                    setattr(d, nm, t.data_ptr())
            if psi is not None:
                if dtype is not None and psi.dtype != dtype:
                    raise WvlhError("all orbitals of a batch share one precision")
                dtype = psi.dtype
        self.dtype = dtype
        h = C.c_void_p()
        check(lib().wvlh_batch_create_orbitals(ctx.h, self.norb, descs, C.byref(h)), "wvlh_batch_create_orbitals")
        self.h = h

    @property
    def precision(self):
        torch = self.ctx.torch
        return {torch.float32: 32, torch.float64: 64}[self.dtype]

    def locham(self, ekin, epot, accumulate=False):
        """Hpsi of every orbital into its own hpsi; ekin/epot: device float64 (norb,)."""
        rc = lib().wvlh_locham_batched(self.h, self.precision, None, None, None, _ptr(ekin), _ptr(epot),
                                       int(bool(accumulate)))
        check(rc, "wvlh_locham_batched")

    def locden(self, hfac):
        """rho_o += hfac[o] |psi_o|^2 into each orbital's own rho; hfac device float64 (norb,)."""
        check(lib().wvlh_locden_batched(self.h, self.precision, None, _ptr(hfac), None), "wvlh_locden_batched")

    def close(self):
        if getattr(self, "h", None):
            lib().wvlh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scalar_products(ctx, ra, a, rb, b, out=None):
    """<a_i|b_j> (FP64, (na, nb)) between the rows of a on region ra's keys and
    the rows of b on region rb's keys, regions of the same box: the
    reference's wpdot (wavelib/scalprod.f90:3222) on the device.  a, b: 2D
    device tensors (float32 or float64, same dtype, unit column stride)."""
    torch = ctx.torch
    prec = {torch.float32: 32, torch.float64: 64}.get(a.dtype)
    if prec is None or b.dtype != a.dtype or a.dim() != 2 or b.dim() != 2:
        raise WvlhError("a and b must be 2D float32 or float64 tensors of one dtype")
    if a.stride(1) != 1 or b.stride(1) != 1:
        raise WvlhError("rows must be contiguous")
    na, nb = a.shape[0], b.shape[0]
    if out is None:
        out = torch.empty(na, nb, dtype=torch.float64, device=a.device)
    check(lib().wvlh_wpdot(ctx.h, prec, ra.h, na, _ptr(a), a.stride(0), rb.h, nb, _ptr(b), b.stride(0),
                           _ptr(out)), "wvlh_wpdot")
    return out
