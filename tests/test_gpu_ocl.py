"""GPU parity of the drop-in ocl_* entry points, driven the way
bigdft/src/interface_ocl.f90 drives the reference's OpenCL backend.

Integer (key) work must be bit-exact; FP64 results within 1e-13 relative L2
of the oracle."""
import ctypes as C

import numpy as np
import pytest

from wvlh import ocl
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


@pytest.fixture(scope="module")
def q(torch_cuda):
    qq = ocl.OclQueue(0)
    yield qq
    qq.close()


def make(N, per, seed, density=0.5):
    rng = np.random.default_rng(seed)
    mc = rng.random(N[::-1]) < 0.9
    mc[0, 0, :] = True
    mf = mc & (rng.random(N[::-1]) < density)
    return Locreg.from_masks(mc, mf, per, (0.45, 0.5, 0.4)), rng


def desc(oracle, lr):
    return oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)


@pytest.mark.parametrize("N,per", [((8, 9, 10), (1, 1, 1)), ((7, 6, 9), (0, 0, 0)), ((9, 8, 11), (1, 0, 1))])
def test_uncompress_compress_bit_exact(oracle, q, N, per):
    lr, rng = make(N, per, 1)
    gp = ocl.GpuPointers(q, lr)
    pc, pf = rng.uniform(-1, 1, lr.nvctr_c), rng.uniform(-1, 1, 7 * lr.nvctr_f)
    q.write(gp.psi_c, pc)
    q.write(gp.psi_f, pf)
    q.call("uncompress_d_", gp.dims(), *gp.key_args(), gp.psi_c.ref, gp.psi_f.ref, gp.work1.ref)
    psig = np.empty(8 * int(np.prod(lr.n)))
    q.read(gp.work1, psig)
    assert np.array_equal(psig, oracle.uncompress(desc(oracle, lr), pc, pf))
    q.call("compress_d_", gp.dims(), *gp.key_args(), gp.psi_c_b.ref, gp.psi_f_b.ref, gp.work1.ref)
    oc, of = np.empty(lr.nvctr_c), np.empty(7 * lr.nvctr_f)
    q.read(gp.psi_c_b, oc)
    q.read(gp.psi_f_b, of)
    assert np.array_equal(oc, pc) and np.array_equal(of, pf)


@pytest.mark.parametrize("N,per", [((8, 9, 10), (1, 1, 1)), ((7, 6, 9), (0, 0, 0)), ((9, 8, 11), (1, 0, 1))])
def test_fulllocham_matches_oracle(oracle, q, N, per):
    lr, rng = make(N, per, 2)
    gp = ocl.GpuPointers(q, lr)
    norb = 3
    psi = rng.uniform(-1, 1, (norb, lr.ncoeff))
    pot = rng.uniform(-1, 0, lr.nisf)
    hpsi, ekin, epot, esum, psum = ocl.local_hamiltonian_ocl(q, gp, psi, pot)
    d = desc(oracle, lr)
    for o in range(norb):
        hc, hf, ek, ep = oracle.locham(d, lr.hgrid, psi[o, :lr.nvctr_c], psi[o, lr.nvctr_c:], pot)
        assert rel(hpsi[o], np.concatenate([hc, hf])) < 1e-13
        assert abs(ekin[o] - ek) <= 1e-12 * abs(ek) and abs(epot[o] - ep) <= 1e-12 * abs(ep)


@pytest.mark.parametrize("N,per", [((8, 9, 10), (1, 1, 1)), ((7, 6, 9), (0, 0, 0))])
def test_locden_matches_oracle(oracle, q, N, per):
    lr, rng = make(N, per, 3)
    gp = ocl.GpuPointers(q, lr)
    psi = rng.uniform(-1, 1, (2, lr.ncoeff))
    hfac = np.array([2.0 / 0.3, 1.0 / 0.3])
    rho = ocl.local_partial_density_ocl(q, gp, psi, hfac)
    d = desc(oracle, lr)
    ref = np.full(lr.nisf, 1e-20)
    for o in range(2):
        ref = oracle.locden(d, psi[o, :lr.nvctr_c], psi[o, lr.nvctr_c:], hfac[o], ref)
    assert rel(rho, ref) < 1e-13


@pytest.mark.parametrize("N,per", [((8, 9, 10), (1, 1, 1)), ((7, 6, 9), (0, 0, 0))])
def test_preconditioner_matches_oracle(oracle, q, N, per):
    lr, rng = make(N, per, 4)
    gp = ocl.GpuPointers(q, lr)
    r = rng.uniform(-1, 1, lr.ncoeff)
    c = 0.7
    hf = [0.5 * h for h in lr.hgrid]
    s = oracle.precond_scal(hf, c)
    sc = np.concatenate([np.full(lr.nvctr_c, s[0]), np.tile(s[1:], lr.nvctr_f)])
    b = sc * r
    x0 = b.copy()
    out = ocl.preconditioner_ocl(q, gp, x0, b, c, 5)
    ref, _ = oracle.precond(desc(oracle, lr), hf, c, 5, x0, b)
    assert rel(out, ref) < 1e-12


def test_1d_passes_match_oracle(oracle, q):
    rng = np.random.default_rng(5)
    n, ndat = 12, 40
    buf_in, buf_out = q.buffer(8 * 4096), q.buffer(8 * 4096)
    cases = [("syn1d_d_", n, 2 * n, 2 * n, lambda x: oracle.syn_rot_per(n - 1, ndat, x)),
             ("ana1d_d_", n, 2 * n, 2 * n, lambda x: oracle.ana_rot_per(n - 1, ndat, x)),
             ("syngrow1d_d_", n, 2 * n, 2 * n + 14, lambda x: oracle.syn_grow_rot(n, ndat, x)),
             ("anashrink1d_d_", n, 2 * n + 14, 2 * n, lambda x: oracle.ana_shrink_rot(n, ndat, x)),
             ("magicfilter1d_d_", 2 * n, 2 * n, 2 * n, lambda x: oracle.convrot_n_per(2 * n - 1, ndat, x)),
             ("magicfilter1d_t_d_", 2 * n, 2 * n, 2 * n, lambda x: oracle.convrot_t_per(2 * n - 1, ndat, x)),
             ("magicfiltergrow1d_d_", 2 * n, 2 * n, 2 * n + 15, lambda x: oracle.mf_grow_rot(2 * n, ndat, x)),
             ("magicfiltershrink1d_d_", 2 * n, 2 * n + 15, 2 * n, lambda x: oracle.mf_shrink_rot(2 * n, ndat, x))]
    for name, narg, lin, lout, ref in cases:
        # the OpenCL layout is the transpose of the Fortran one on input:
        # in[p*ndat + j]  vs  Fortran x(p, j) = x[j*L + p]
        xf = rng.uniform(-1, 1, (ndat, lin))
        q.write(buf_in, np.ascontiguousarray(xf.T))
        q.call(name, ocl._u(narg), ocl._u(ndat), buf_in.ref, buf_out.ref)
        y = np.empty(ndat * lout)
        q.read(buf_out, y)
        yref = ref(xf.ravel()).reshape(lout, ndat).T      # Fortran out(ndat, q) -> [j][q]
        assert rel(y.reshape(ndat, lout), yref) < 1e-14, name


def test_1d_passes_match_reference_opencl_kernels(q):
    """The drop-in 1D kernels on the lines of tests/golden/opencl_kernels.npz,
    whose outputs replay the reference's own OpenCL kernels (syn1d, ana1d,
    syngrow1d, anashrink1d, magicfiltergrow1d, magicfiltershrink1d, kinetic1d;
    see tests/golden/make_opencl_kernels.py): FP64, to rounding."""
    from pathlib import Path
    gold = np.load(Path(__file__).resolve().parent / "golden" / "opencl_kernels.npz")
    buf_in, buf_out = q.buffer(8 * 4096), q.buffer(8 * 4096)
    wx, wy = q.buffer(8 * 4096), q.buffer(8 * 4096)
    one = ocl._u(1)
    for n in (8, 9, 13, 16, 24):
        x, yg, ym = gold["x_%d" % n], gold["yg_%d" % n], gold["ym_%d" % n]
        cases = [("syn1d_d_", n, x, "syn"), ("ana1d_d_", n, x, "ana"), ("syngrow1d_d_", n, x, "grow"),
                 ("anashrink1d_d_", n, yg, "shrink"), ("magicfiltergrow1d_d_", 2 * n, x, "mfgrow"),
                 ("magicfiltershrink1d_d_", 2 * n, ym, "mfshrink")]
        for name, narg, xin, key in cases:
            ref = gold["%s_%d" % (key, n)]
            q.write(buf_in, np.ascontiguousarray(xin))
            q.call(name, ocl._u(narg), one, buf_in.ref, buf_out.ref)
            y = np.empty(len(ref))
            q.read(buf_out, y)
            assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max(), (name, n)
        # kinetic1d: y = c x - K x / (2 h^2); with c = 0 and h = 1 the filter is -2 y
        ref = gold["kin_%d" % n]
        q.write(buf_in, np.ascontiguousarray(x))
        h, c0, e = C.c_double(1.0), C.c_double(0.0), C.c_double()
        q.call("kinetic1d_d_", ocl._u(2 * n), one, C.byref(h), C.byref(c0), buf_in.ref, buf_out.ref, wx.ref,
               wy.ref, C.byref(e))
        y = np.empty(2 * n)
        q.read(buf_out, y)
        assert np.abs(-2.0 * y - ref).max() <= 1e-14 * np.abs(ref).max(), ("kinetic1d_d_", n)


def test_dot_and_axpy(q):
    rng = np.random.default_rng(6)
    n = 100003
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    bx, by, bz = q.buffer(8 * n), q.buffer(8 * n), q.buffer(8 * n)
    q.write(bx, x)
    q.write(by, y)
    out = np.zeros(1)
    q.call("dot_d_", ocl._u(n), bx.ref, by.ref, bz.ref, bz.ref, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert abs(out[0] - x @ y) < 1e-12 * abs(x @ y) + 1e-12
    a = C.c_double(-0.5)
    q.call("axpy_d_", ocl._u(n), C.byref(a), bx.ref, by.ref, bz.ref)
    z = np.empty(n)
    q.read(bz, z)
    assert np.allclose(z, -0.5 * x + y, rtol=0, atol=1e-15)


def test_kpoint_spinors_report_unsupported(q):
    lr, _ = make((8, 8, 8), (1, 1, 1), 7)
    gp = ocl.GpuPointers(q, lr)
    from wvlh._lib import WvlhError
    e = np.zeros(2)
    with pytest.raises(WvlhError, match="unsupported"):
        q.call("ocl_fulllocham_generic_k_", gp.dims(), gp.periodic(), (C.c_double * 3)(0.2, 0.2, 0.2),
               (C.c_double * 3)(0.1, 0, 0), *gp.key_args(), gp.psi_c.ref, gp.psi_f.ref, gp.psi_c.ref, gp.psi_f.ref,
               gp.rhopot.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref, gp.work1.ref, gp.work2.ref, gp.work3.ref,
               gp.d.ref, gp.d.ref, ocl._u(2), e.ctypes.data_as(C.POINTER(C.c_double)),
               e.ctypes.data_as(C.POINTER(C.c_double)))
    from wvlh._lib import lib
    lib().wvlh_get_last_error()
