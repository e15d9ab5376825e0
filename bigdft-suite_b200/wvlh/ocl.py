"""Python mirror of the reference's accelerator glue over the drop-in ABI.

BigDFT's Fortran host drives its OpenCL backend through
``bigdft/src/interface_ocl.f90``: it creates a context and an in-order queue
(``init_acceleration_OCL`` :20-41), allocates device buffers and uploads the
keys once (``allocate_data_OCL`` :43-190), then for every orbital writes
``psi_c``/``psi_f``, calls the composite entry point and reads the result back
(``local_hamiltonian_OCL`` :391-587, ``local_partial_density_OCL`` :908-1018,
``preconditionall_OCL`` :622-906).  This module does the same through
``libwvlh.so``'s ``ocl_*`` symbols, with the same names, argument meanings and
buffer roles, so a Fortran host can switch libraries without code changes.
"""
import ctypes as C

import numpy as np

from ._lib import WvlhError, lib

u32 = C.c_uint32
dbl = C.c_double


def _u(v):
    return C.byref(u32(int(v)))


class OclBuffer:
    def __init__(self, ctx, nbytes):
        self.h = C.c_void_p()
        self.nbytes = int(nbytes)
        lib().ocl_create_read_write_buffer_(C.byref(ctx), _u(max(nbytes, 8)), C.byref(self.h))
        if not lib().wvlh_mem_ptr(self.h):
            raise WvlhError("device buffer allocation failed")

    @property
    def ref(self):
        return C.byref(self.h)

    @property
    def ptr(self):
        return lib().wvlh_mem_ptr(self.h)

    def release(self):
        if self.h:
            lib().ocl_release_mem_object_(C.byref(self.h))


class OclQueue:
    """init_acceleration_OCL: one context and one in-order queue per process."""

    def __init__(self, device_index=0):
        L = lib()
        self.ctx = C.c_void_p()
        ndev = u32(0)
        L.ocl_create_gpu_context_(C.byref(self.ctx), C.byref(ndev))
        if not self.ctx:
            raise WvlhError("no CUDA device: the drop-in backend has no CPU path")
        L.ocl_build_programs_(C.byref(self.ctx))
        self.q = C.c_void_p()
        L.ocl_create_command_queue_id_(C.byref(self.q), C.byref(self.ctx), _u(device_index))
        self.buffers = []

    def buffer(self, nbytes):
        b = OclBuffer(self.ctx, nbytes)
        self.buffers.append(b)
        return b

    def write(self, buf, arr, asynchronous=False):
        arr = np.ascontiguousarray(arr)
        fn = lib().ocl_enqueue_write_buffer_async_ if asynchronous else lib().ocl_enqueue_write_buffer_
        fn(C.byref(self.q), buf.ref, _u(arr.nbytes), arr.ctypes.data_as(C.c_void_p))

    def read(self, buf, arr, asynchronous=False):
        fn = lib().ocl_enqueue_read_buffer_async_ if asynchronous else lib().ocl_enqueue_read_buffer_
        fn(C.byref(self.q), buf.ref, _u(arr.nbytes), arr.ctypes.data_as(C.c_void_p))

    def finish(self):
        lib().ocl_finish_(C.byref(self.q))

    def call(self, name, *args):
        lib().wvlh_get_last_error()  # reset the error slot left by any earlier call
        getattr(lib(), name)(C.byref(self.q), *args)
        err = lib().wvlh_get_last_error()
        if err:
            raise WvlhError("%s: %s" % (name, lib().wvlh_error_string(err).decode()))

    def close(self):
        for b in self.buffers:
            b.release()
        self.buffers = []
        if self.q:
            lib().ocl_clean_command_queue_(C.byref(self.q))
        if self.ctx:
            lib().ocl_clean_(C.byref(self.ctx))


class GpuPointers:
    """allocate_data_OCL (interface_ocl.f90:43-190): work buffers sized for the
    ISF grid, compressed psi buffers, keys uploaded once as 1-based uint32."""

    def __init__(self, q, lr):
        self.q, self.lr = q, lr
        n1b, n2b, n3b = lr.isf
        nw = n1b * n2b * n3b * 8
        nc, nf = max(lr.nvctr_c, 1), max(lr.nvctr_f, 1)
        self.psi_c, self.psi_f = q.buffer(nc * 8), q.buffer(7 * nf * 8)
        self.work1, self.work2, self.work3, self.d = (q.buffer(nw) for _ in range(4))
        self.rhopot = q.buffer(nw)
        self.keyg_c, self.keyv_c = q.buffer(max(len(lr.keyv_c), 1) * 8), q.buffer(max(len(lr.keyv_c), 1) * 4)
        self.keyg_f, self.keyv_f = q.buffer(max(len(lr.keyv_f), 1) * 8), q.buffer(max(len(lr.keyv_f), 1) * 4)
        if len(lr.keyv_c):
            q.write(self.keyg_c, lr.keyg_c.astype(np.uint32))
            q.write(self.keyv_c, lr.keyv_c.astype(np.uint32))
        if len(lr.keyv_f):
            q.write(self.keyg_f, lr.keyg_f.astype(np.uint32))
            q.write(self.keyv_f, lr.keyv_f.astype(np.uint32))
        self.psi_c_r, self.psi_f_r = q.buffer(nc * 8), q.buffer(7 * nf * 8)
        self.psi_c_b, self.psi_f_b = q.buffer(nc * 8), q.buffer(7 * nf * 8)
        self.psi_c_d, self.psi_f_d = q.buffer(nc * 8), q.buffer(7 * nf * 8)

    def dims(self):
        return (u32 * 3)(*self.lr.n)

    def periodic(self):
        return (u32 * 3)(*self.lr.periodic)

    def key_args(self):
        lr = self.lr
        return (_u(len(lr.keyv_c)), _u(lr.nvctr_c), self.keyg_c.ref, self.keyv_c.ref,
                _u(len(lr.keyv_f)), _u(lr.nvctr_f), self.keyg_f.ref, self.keyv_f.ref)


def local_hamiltonian_ocl(q, gp, psi, pot, kwgt_occ=None):
    """local_hamiltonian_OCL + finish_hamiltonian_OCL (interface_ocl.f90:391-620)
    for nspinor = 1: psi (norb, nvctr_c + 7 nvctr_f) float64, pot on the ISF grid.
    Returns hpsi, per-orbital (ekin, epot) and the occupation-weighted sums."""
    lr = gp.lr
    norb = psi.shape[0]
    hgrids = (dbl * 3)(*[0.5 * h for h in lr.hgrid])
    kpt = (dbl * 3)(0.0, 0.0, 0.0)
    q.write(gp.rhopot, np.ascontiguousarray(pot, np.float64), asynchronous=True)
    hpsi = np.empty_like(psi)
    ekinpot = np.zeros((norb, 2))
    epot = np.zeros((norb, 2))
    keep = []
    for o in range(norb):
        pc = np.ascontiguousarray(psi[o, :lr.nvctr_c])
        pf = np.ascontiguousarray(psi[o, lr.nvctr_c:])
        keep += [pc, pf]
        q.write(gp.psi_c, pc, asynchronous=True)
        if lr.nvctr_f:
            q.write(gp.psi_f, pf, asynchronous=True)
        ep = epot[o].ctypes.data_as(C.POINTER(dbl))
        ekp = ekinpot[o].ctypes.data_as(C.POINTER(dbl))
        q.call("ocl_fulllocham_generic_k_", gp.dims(), gp.periodic(), hgrids, kpt, *gp.key_args(),
               gp.psi_c.ref, gp.psi_f.ref, gp.psi_c.ref, gp.psi_f.ref, gp.rhopot.ref,
               gp.work1.ref, gp.work2.ref, gp.work3.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref,
               gp.d.ref, gp.d.ref, _u(1), ep, ekp)
        out_c = hpsi[o, :lr.nvctr_c]
        out_f = hpsi[o, lr.nvctr_c:]
        # read back into temporaries (async reads need contiguous host arrays)
        tc, tf = np.empty(lr.nvctr_c), np.empty(7 * lr.nvctr_f)
        q.read(gp.psi_c, tc)
        if lr.nvctr_f:
            q.read(gp.psi_f, tf)
        out_c[:] = tc
        out_f[:] = tf
    q.finish()
    ekin = ekinpot[:, 0] - epot[:, 0]
    w = np.ones(norb) if kwgt_occ is None else np.asarray(kwgt_occ)
    return hpsi, ekin, epot[:, 0], float((w * ekin).sum()), float((w * epot[:, 0]).sum())


def local_partial_density_ocl(q, gp, psi, hfac, rho_init=1e-20):
    """local_partial_density_OCL (interface_ocl.f90:908-1018): rho = rho_init +
    sum_o hfac_o |psi_o(r)|^2 on the ISF grid."""
    lr = gp.lr
    rho = np.full(lr.nisf, rho_init)
    q.write(gp.rhopot, rho)
    for o in range(psi.shape[0]):
        q.write(gp.psi_c, np.ascontiguousarray(psi[o, :lr.nvctr_c]))
        if lr.nvctr_f:
            q.write(gp.psi_f, np.ascontiguousarray(psi[o, lr.nvctr_c:]))
        h = dbl(float(hfac[o]))
        q.call("ocl_locden_generic_", gp.dims(), gp.periodic(), C.byref(h), *gp.key_args(),
               gp.psi_c.ref, gp.psi_f.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref, gp.rhopot.ref)
    q.read(gp.rhopot, rho)
    return rho


def preconditioner_ocl(q, gp, x, b, c, ncong):
    """ocl_preconditioner_generic_k for one orbital (interface_ocl.f90:759-830):
    x is the initial guess (overwritten by the result), b the right-hand side."""
    lr = gp.lr
    h = (dbl * 3)(*[0.5 * v for v in lr.hgrid])
    kpt = (dbl * 3)(0.0, 0.0, 0.0)
    cc = dbl(c)
    q.write(gp.psi_c, np.ascontiguousarray(x[:lr.nvctr_c]))
    q.write(gp.psi_f, np.ascontiguousarray(x[lr.nvctr_c:]))
    q.write(gp.psi_c_b, np.ascontiguousarray(b[:lr.nvctr_c]))
    q.write(gp.psi_f_b, np.ascontiguousarray(b[lr.nvctr_c:]))
    norms = np.zeros(2)
    q.call("ocl_preconditioner_generic_k_", gp.dims(), gp.periodic(), h, kpt, C.byref(cc), _u(ncong),
           *gp.key_args(), gp.psi_c.ref, gp.psi_f.ref, gp.psi_c.ref, gp.psi_f.ref,
           gp.psi_c_r.ref, gp.psi_f_r.ref, gp.psi_c_r.ref, gp.psi_f_r.ref,
           gp.psi_c_b.ref, gp.psi_f_b.ref, gp.psi_c_b.ref, gp.psi_f_b.ref,
           gp.psi_c_d.ref, gp.psi_f_d.ref, gp.psi_c_d.ref, gp.psi_f_d.ref,
           gp.d.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref, gp.d.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref,
           _u(1), norms.ctypes.data_as(C.POINTER(dbl)))
    out = np.empty_like(x)
    tc, tf = np.empty(lr.nvctr_c), np.empty(7 * lr.nvctr_f)
    q.read(gp.psi_c, tc)
    q.read(gp.psi_f, tf)
    out[:lr.nvctr_c], out[lr.nvctr_c:] = tc, tf
    return out


def signatures():
    """ctypes argtypes are left unset for the ocl_* symbols: every argument is a
    pointer, exactly like the Fortran caller passes them."""
    return None
