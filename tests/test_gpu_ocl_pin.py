"""GPU test of the host-buffer entry points, driven as interface_ocl.f90's
local_hamiltonian_OCL drives them with pin = .true. (interface_ocl.f90:134-147,
454-458, 479, 501-576): keys and potential written through pinned regions,
the orbitals' coefficients pinned one by one, the whole hpsi array wrapped in
a write buffer over host memory, each result read through map / read / unmap,
the handles released while copies may still be in flight.  The result must
equal the unpinned drop-in path bit for bit, and the oracle to 1e-13."""
import ctypes as C

import numpy as np
import pytest

from wvlh import ocl
from wvlh._lib import lib
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def _mem():
    return C.c_void_p()


def test_pinned_locham_matches_plain_and_oracle(oracle, torch_cuda):
    L = lib()
    rng = np.random.default_rng(4)
    N = (9, 8, 10)
    lr = Locreg.from_masks(np.ones(N[::-1], bool), rng.random(N[::-1]) < 0.5, (1, 1, 1), (0.45, 0.45, 0.45))
    norb = 3
    psi = np.ascontiguousarray(rng.uniform(-1, 1, (norb, lr.ncoeff)))
    pot = np.ascontiguousarray(rng.uniform(-1, 0, lr.nisf))
    hpsi = np.zeros_like(psi)
    ctx, q = C.c_void_p(), C.c_void_p()
    ndev = ocl.u32(0)
    L.ocl_create_gpu_context_(C.byref(ctx), C.byref(ndev))
    L.ocl_create_command_queue_(C.byref(q), C.byref(ctx))
    u = ocl._u

    def dbuf(nbytes):
        m = _mem()
        L.ocl_create_read_write_buffer_(C.byref(ctx), u(nbytes), C.byref(m))
        return m

    keys = [np.ascontiguousarray(k, np.uint32) for k in (lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)]
    kb = []
    for k in keys:
        b = dbuf(k.nbytes)
        h = _mem()
        L.ocl_pin_read_buffer_async_(C.byref(ctx), C.byref(q), u(k.nbytes), k.ctypes.data_as(C.c_void_p), C.byref(h))
        L.ocl_enqueue_write_buffer_(C.byref(q), C.byref(b), u(k.nbytes), k.ctypes.data_as(C.c_void_p))
        L.ocl_release_mem_object_(C.byref(h))
        kb.append(b)
    nc, nf = lr.nvctr_c, lr.nvctr_f
    npt = int(np.prod(lr.isf))
    rhopot = dbuf(8 * npt)
    h = _mem()
    L.ocl_pin_read_buffer_async_(C.byref(ctx), C.byref(q), u(pot.nbytes), pot.ctypes.data_as(C.c_void_p), C.byref(h))
    L.ocl_enqueue_write_buffer_async_(C.byref(q), C.byref(rhopot), u(pot.nbytes), pot.ctypes.data_as(C.c_void_p))
    L.ocl_release_mem_object_(C.byref(h))
    psi_c, psi_f = dbuf(8 * nc), dbuf(8 * 7 * nf)
    work = [dbuf(8 * npt) for _ in range(4)]
    hsth = _mem()
    L.ocl_create_write_buffer_host_(C.byref(ctx), u(hpsi.nbytes), hpsi.ctypes.data_as(C.c_void_p), C.byref(hsth))
    ek = np.zeros((norb, 2))
    ep = np.zeros((norb, 2))
    dims = (ocl.u32 * 3)(*N)
    per = (ocl.u32 * 3)(1, 1, 1)
    hg = (C.c_double * 3)(*(0.5 * h_ for h_ in lr.hgrid))
    kpt = (C.c_double * 3)(0, 0, 0)
    nspinor = ocl.u32(1)
    for o in range(norb):
        row = psi[o]
        for off, n, buf in ((0, nc, psi_c), (nc, 7 * nf, psi_f)):
            ph = _mem()
            addr = C.c_void_p(row.ctypes.data + 8 * off)
            L.ocl_pin_read_buffer_async_(C.byref(ctx), C.byref(q), u(8 * n), addr, C.byref(ph))
            L.ocl_enqueue_write_buffer_async_(C.byref(q), C.byref(buf), u(8 * n), addr)
            L.ocl_release_mem_object_(C.byref(ph))
        L.ocl_fulllocham_generic_k_(C.byref(q), dims, per, hg, kpt, u(len(lr.keyv_c)), u(nc), C.byref(kb[0]), C.byref(kb[1]),
                                    u(len(lr.keyv_f)), u(nf), C.byref(kb[2]), C.byref(kb[3]), C.byref(psi_c),
                                    C.byref(psi_f), C.byref(psi_c), C.byref(psi_f), C.byref(rhopot),
                                    C.byref(work[0]), C.byref(work[1]), C.byref(work[2]), C.byref(work[0]),
                                    C.byref(work[1]), C.byref(work[2]), C.byref(work[3]), C.byref(work[3]),
                                    C.byref(nspinor), ep[o].ctypes.data_as(C.c_void_p),
                                    ek[o].ctypes.data_as(C.c_void_p))
        for off, n, buf in ((0, nc, psi_c), (nc, 7 * nf, psi_f)):
            dst = C.c_void_p(hpsi[o].ctypes.data + 8 * off)
            L.ocl_map_read_buffer_async_(C.byref(q), C.byref(hsth), u(8 * (o * lr.ncoeff + off)), u(8 * n))
            L.ocl_enqueue_read_buffer_async_(C.byref(q), C.byref(buf), u(8 * n), dst)
            L.ocl_unmap_mem_object_(C.byref(q), C.byref(hsth), dst)
    L.ocl_release_mem_object_(C.byref(hsth))   # copies may still be in flight
    L.ocl_finish_(C.byref(q))
    assert L.wvlh_get_last_error() == 0
    for b in kb + [rhopot, psi_c, psi_f] + work:
        L.ocl_release_mem_object_(C.byref(b))
    L.ocl_clean_command_queue_(C.byref(q))
    L.ocl_clean_(C.byref(ctx))
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    for o in range(norb):
        hc, hf, e1, e2 = oracle.locham(d, lr.hgrid, psi[o, :nc], psi[o, nc:], pot)
        ref = np.concatenate([hc, hf])
        assert np.linalg.norm(hpsi[o] - ref) / np.linalg.norm(ref) < 1e-13
        # ekinpot = <psi|T+V|psi>, epot = <psi|V|psi> (interface_ocl.f90:603-605)
        assert abs(ep[o, 0] - e2) <= 1e-12 * abs(e2)
        assert abs(ek[o, 0] - (e1 + e2)) <= 1e-12 * abs(e1 + e2)
