"""The allocation-free local-Hamiltonian entry point (wvlh_locham_noalloc).

It serves callers that cannot call cudaMalloc (a host application whose
memory manager owns every device allocation, or a layer that must not grow
the device footprint by itself): its tables and scratch live in a fixed
static device array inside libwvlh.so.  These tests call it through the C ABI
twice in a row on the same inputs and compare both results with the
allocating batched entry point (wvlh_locham_batched), within the FP64 parity
tolerance used elsewhere (1e-13 relative on Hpsi, 1e-12 on energies), and
check that an oversized box is refused.  This file is named so that pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from wvlh._lib import lib
from wvlh.batch import Batch, Context
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def _i32(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int32))


def call_noalloc(torch, lr, psi, pot, prec, stream):
    dt = torch.float64 if prec == 64 else torch.float32
    h = torch.full_like(psi, float("nan"), dtype=dt)
    ek = torch.empty(1, dtype=torch.float64, device="cuda")
    ep = torch.empty(1, dtype=torch.float64, device="cuda")
    keep = [_i32(lr.keyg_c), _i32(lr.keyv_c), _i32(lr.keyg_f), _i32(lr.keyv_f)]
    n = (C.c_int * 3)(*lr.n)
    per = (C.c_int * 3)(*lr.periodic)
    hg = (C.c_double * 3)(*lr.hgrid)
    rc = lib().wvlh_locham_noalloc(prec, n, per, hg, len(lr.keyv_c), keep[0][1], keep[1][1], len(lr.keyv_f),
                                   keep[2][1], keep[3][1], C.c_void_p(psi.data_ptr()), C.c_void_p(pot.data_ptr()),
                                   C.c_void_p(h.data_ptr()), C.c_void_p(ek.data_ptr()), C.c_void_p(ep.data_ptr()),
                                   C.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    stream.synchronize()
    return h, ek.item(), ep.item()


@pytest.mark.parametrize("N,per,prec", [((12, 10, 11), (1, 1, 1), 64), ((9, 8, 10), (0, 0, 0), 64),
                                        ((16, 16, 16), (1, 1, 1), 32), ((10, 8, 12), (1, 0, 1), 64),
                                        ((11, 9, 8), (0, 0, 0), 32)])
def test_noalloc_matches_batched_entry_two_calls(N, per, prec):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(sum(N) + prec)
    mf = rng.random(N[::-1]) < 0.6
    lr = Locreg.from_masks(np.ones(N[::-1], bool), mf, per, (0.45, 0.4, 0.5))
    dt = torch.float64 if prec == 64 else torch.float32
    psi = torch.tensor(rng.uniform(-1, 1, lr.ncoeff), device="cuda", dtype=dt)
    pot = torch.tensor(rng.uniform(-1, 0, lr.nisf), device="cuda", dtype=dt)
    ctx = Context(0)
    b = Batch(ctx, [lr], [0])
    href, ekr, epr = b.locham(psi, pot)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    for _ in range(2):
        h, ek, ep = call_noalloc(torch, lr, psi, pot, prec, stream)
        tol = 1e-13 if prec == 64 else 1e-6
        assert ((h - href).norm() / href.norm()).item() < tol
        assert abs(ek - ekr.item()) <= 1e-12 * abs(ekr.item()) + (0 if prec == 64 else 1e-9)
        assert abs(ep - epr.item()) <= 1e-12 * abs(epr.item()) + (0 if prec == 64 else 1e-9)
    b.close()
    ctx.close()


def test_noalloc_rejects_oversized_box():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cap = lib().wvlh_noalloc_capacity()
    assert cap == 64 << 20
    N = (128, 128, 128)   # FP64 scratch of a 128^3 periodic box is far above the capacity
    m = np.ones(N[::-1], bool)
    lr = Locreg.from_masks(m, np.zeros_like(m), (1, 1, 1), (0.4, 0.4, 0.4))
    dummy = torch.zeros(8, device="cuda", dtype=torch.float64)
    e = torch.zeros(1, device="cuda", dtype=torch.float64)
    keep = [_i32(lr.keyg_c), _i32(lr.keyv_c)]
    rc = lib().wvlh_locham_noalloc(64, (C.c_int * 3)(*N), (C.c_int * 3)(1, 1, 1), (C.c_double * 3)(0.4, 0.4, 0.4),
                                   len(lr.keyv_c), keep[0][1], keep[1][1], 0, None, None,
                                   C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                   C.c_void_p(dummy.data_ptr()), C.c_void_p(e.data_ptr()), C.c_void_p(e.data_ptr()),
                                   None)
    assert rc == 6  # WVLH_ERR_TOO_LARGE
    lib().wvlh_get_last_error()
