"""CPU oracle for the Daubechies-16 local-Hamiltonian path.

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use this module as the checker; the
product library never imports it.

``wvl_oracle.c`` restates the reference's FP64 CPU convolutions (Fortran,
``bigdft/src/orbitals/convolut_simple_per.f90`` and friends) and the
compositions of its OpenCL backend (``bigdft/src/OpenCL/*.c``); each C routine
cites the reference lines it follows.  Parity pins:

* the magic filter is checked against the reference's own C implementation
  (``bigdft/src/convolutions-c/MagicFilter_sse.c``) compiled into
  ``oracle/_ref`` (see ``Makefile``), and against golden vectors generated
  from it (``tests/golden``);
* the wavelet-basis kinetic operator against the reference's SSE C
  (``bigdft/src/orbitals/convolut_ib_sse.c``), also compiled into ``oracle/_ref``;
* synthesis and analysis (periodic and free) and the fine-grid kinetic filter
  against the arithmetic of the reference's OpenCL kernels, replayed from the
  kernel generators' source text into golden vectors
  (``tests/golden/make_opencl_kernels.py``);
* and by the reference's mathematical known-answer checks (orthonormality of
  DB16, analysis after synthesis = identity, magic-filter adjointness,
  kinetic symmetry, agreement of the fine-grid kinetic with the wavelet-basis
  ``ConvolkineticT`` filters, analytic Laplacian of a Gaussian).
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_MF = HERE / "_ref" / "libref_magicfilter.so"
REF_CONVIB = HERE / "_ref" / "libref_convib.so"

_lib = None

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
ip = C.POINTER(C.c_int)
dp = C.POINTER(C.c_double)


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.wo_num_segkeys.argtypes = [C.c_int, C.c_int, C.c_int, u8p, ip, ip]
        L.wo_segkeys.argtypes = [C.c_int, C.c_int, C.c_int, u8p, i32p, i32p]
        L.wo_uncompress.argtypes = [C.c_int] * 3 + [C.c_int, i32p, i32p, C.c_int, i32p, i32p, f64p, f64p, C.c_void_p, f64p]
        L.wo_compress.argtypes = [C.c_int] * 3 + [C.c_int, i32p, i32p, C.c_int, i32p, i32p, f64p, C.c_void_p, C.c_int, f64p, f64p]
        for nm in ("wo_ana_rot_per", "wo_syn_rot_per", "wo_convrot_n_per", "wo_convrot_t_per",
                   "wo_syn_grow_rot", "wo_ana_shrink_rot", "wo_mf_grow_rot", "wo_mf_shrink_rot"):
            getattr(L, nm).argtypes = [C.c_int, C.c_int, f64p, f64p]
        L.wo_kinetic_per_T.argtypes = [C.c_int] * 3 + [f64p, f64p, f64p, dp]
        L.wo_kinetic_generic.argtypes = [C.c_int] * 3 + [i32p, f64p, f64p, f64p, dp]
        L.wo_kinetic_wavelet.argtypes = [i32p, i32p, f64p, f64p, f64p, dp]
        L.wo_synthese_generic.argtypes = [i32p, i32p, f64p, f64p, f64p]
        L.wo_analyse_generic.argtypes = [i32p, i32p, f64p, f64p, f64p]
        L.wo_magic_generic.argtypes = [i32p, i32p, f64p, f64p, f64p]
        L.wo_magic_t_generic.argtypes = [i32p, i32p, f64p, f64p, f64p]
        L.wo_locham_per.argtypes = [C.c_int] * 3 + [f64p, C.c_int, i32p, i32p, C.c_int, i32p, i32p,
                                                    f64p, f64p, f64p, f64p, f64p, dp, dp]
        L.wo_locham_generic.argtypes = [i32p, i32p, f64p, C.c_int, i32p, i32p, C.c_int, i32p, i32p,
                                        f64p, f64p, f64p, f64p, f64p, dp, dp]
        L.wo_locden_generic.argtypes = [i32p, i32p, C.c_int, i32p, i32p, C.c_int, i32p, i32p,
                                        f64p, f64p, C.c_double, f64p]
        L.wo_precond_scal.argtypes = [f64p, C.c_double, f64p]
        L.wo_precond_generic.argtypes = [i32p, i32p, f64p, C.c_double, C.c_int,
                                         C.c_int, C.c_int, i32p, i32p, C.c_int, C.c_int, i32p, i32p,
                                         f64p, f64p, f64p]
        L.wo_overlap.argtypes = [C.c_int, C.c_int, f64p, f64p]
        L.wo_cholesky.argtypes = [C.c_int, f64p]
        L.wo_cholesky.restype = C.c_int
        L.wo_wpdot.argtypes = [C.c_int, i32p, i32p, C.c_int, i32p, i32p, f64p, f64p] * 2
        L.wo_wpdot.restype = C.c_double
        L.wo_mask_axpy.argtypes = [C.c_int, i32p, i32p, C.c_int, i32p, i32p, f64p, f64p] * 2 + [C.c_double]
        L.wo_apply_potential.argtypes = [C.c_size_t, f64p, f64p]
        L.wo_apply_potential.restype = C.c_double
        _lib = L
    return _lib


def threads(n):
    """Set the OpenMP thread count used by the oracle (for timing)."""
    os.environ["OMP_NUM_THREADS"] = str(n)


# ---------------------------------------------------------------- keys
def segkeys(mask):
    """mask[i3,i2,i1] (uint8) -> (keyg (nseg,2) int32 1-based, keyv (nseg,) int32)."""
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    n3, n2, n1 = (s - 1 for s in mask.shape)
    ms, mv = C.c_int(), C.c_int()
    lib().wo_num_segkeys(n1, n2, n3, mask, C.byref(ms), C.byref(mv))
    keyg = np.zeros((ms.value, 2), np.int32)
    keyv = np.zeros(ms.value, np.int32)
    if ms.value:
        lib().wo_segkeys(n1, n2, n3, mask, keyg, keyv)
    return keyg, keyv


def _k(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Desc:
    """Wavefunction descriptor: coarse counts N=(N1,N2,N3), per-dim periodicity,
    coarse and fine keys (1-based, as the reference)."""

    def __init__(self, N, periodic, keyg_c, keyv_c, keyg_f, keyv_f):
        self.N = np.asarray(N, np.int32)
        self.per = np.asarray(periodic, np.int32)
        self.keyg_c, self.keyv_c = _k(keyg_c), _k(keyv_c)
        self.keyg_f, self.keyv_f = _k(keyg_f), _k(keyv_f)
        self.nseg_c, self.nseg_f = len(self.keyv_c), len(self.keyv_f)
        self.nvctr_c = int((self.keyg_c[:, 1] - self.keyg_c[:, 0] + 1).sum()) if self.nseg_c else 0
        self.nvctr_f = int((self.keyg_f[:, 1] - self.keyg_f[:, 0] + 1).sum()) if self.nseg_f else 0

    @property
    def F(self):
        return np.where(self.per == 1, 2 * self.N, 2 * self.N + 14)

    @property
    def I(self):
        return np.where(self.per == 1, 2 * self.N, 2 * self.N + 29)

    def args(self):
        return (self.nseg_c, self.keyg_c, self.keyv_c, self.nseg_f, self.keyg_f, self.keyv_f)


def desc_from_masks(mask_c, mask_f, periodic):
    kc, vc = segkeys(mask_c)
    kf, vf = segkeys(mask_f)
    N = mask_c.shape[::-1]
    return Desc(N, periodic, kc, vc, kf, vf)


# ---------------------------------------------------------------- 1D passes
def _rot(fn, n, ndat, x, lout):
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(ndat * lout, np.float64)
    getattr(lib(), fn)(n, ndat, x, y)
    return y


def syn_rot_per(n, ndat, x):
    return _rot("wo_syn_rot_per", n, ndat, x, 2 * n + 2)


def ana_rot_per(n, ndat, x):
    return _rot("wo_ana_rot_per", n, ndat, x, 2 * n + 2)


def convrot_n_per(n1, ndat, x):
    return _rot("wo_convrot_n_per", n1, ndat, x, n1 + 1)


def convrot_t_per(n1, ndat, x):
    return _rot("wo_convrot_t_per", n1, ndat, x, n1 + 1)


def syn_grow_rot(N, ndat, x):
    return _rot("wo_syn_grow_rot", N, ndat, x, 2 * N + 14)


def ana_shrink_rot(N, ndat, x):
    return _rot("wo_ana_shrink_rot", N, ndat, x, 2 * N)


def mf_grow_rot(Lf, ndat, x):
    return _rot("wo_mf_grow_rot", Lf, ndat, x, Lf + 15)


def mf_shrink_rot(Lf, ndat, x):
    return _rot("wo_mf_shrink_rot", Lf, ndat, x, Lf)


# ---------------------------------------------------------------- 3D ops
def uncompress(d, psi_c, psi_f, scal=None):
    N = d.N
    out = np.empty(8 * int(np.prod(N)), np.float64)
    sc = None if scal is None else np.ascontiguousarray(scal, np.float64).ctypes.data
    lib().wo_uncompress(int(N[0]) - 1, int(N[1]) - 1, int(N[2]) - 1, *d.args(),
                        np.ascontiguousarray(psi_c, np.float64), np.ascontiguousarray(psi_f, np.float64), sc, out)
    return out


def compress(d, psig, scal=None, acc=False, psi_c=None, psi_f=None):
    N = d.N
    pc = np.zeros(d.nvctr_c) if psi_c is None else np.array(psi_c, np.float64)
    pf = np.zeros(7 * d.nvctr_f) if psi_f is None else np.array(psi_f, np.float64)
    sc = None if scal is None else np.ascontiguousarray(scal, np.float64).ctypes.data
    lib().wo_compress(int(N[0]) - 1, int(N[1]) - 1, int(N[2]) - 1, *d.args(),
                      np.ascontiguousarray(psig, np.float64), sc, int(acc), pc, pf)
    return pc, pf


def synthese(d, psig):
    n = int(np.prod(d.I))
    out, w = np.empty(n), np.empty(n)
    lib().wo_synthese_generic(d.N, d.per, np.ascontiguousarray(psig, np.float64), out, w)
    return out[: int(np.prod(d.F))]


def analyse(d, y):
    n = int(np.prod(d.I))
    out, w = np.empty(n), np.empty(n)
    lib().wo_analyse_generic(d.N, d.per, np.ascontiguousarray(y, np.float64), out, w)
    return out[: 8 * int(np.prod(d.N))]


def magic(d, x):
    n = int(np.prod(d.I))
    out, w = np.empty(n), np.empty(n)
    lib().wo_magic_generic(np.asarray(d.F, np.int32), d.per, np.ascontiguousarray(x, np.float64), out, w)
    return out


def magic_t(d, r):
    n = int(np.prod(d.I))
    out, w = np.empty(n), np.empty(n)
    lib().wo_magic_t_generic(np.asarray(d.F, np.int32), d.per, np.ascontiguousarray(r, np.float64), out, w)
    return out[: int(np.prod(d.F))]


def kinetic(d, hgrid_fine, x, y=None):
    F = d.F
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros_like(x) if y is None else np.array(y, np.float64)
    ek = C.c_double()
    lib().wo_kinetic_generic(int(F[0]), int(F[1]), int(F[2]), d.per,
                             np.asarray(hgrid_fine, np.float64), x, y, C.byref(ek))
    return y, ek.value


def kinetic_wavelet(d, hgrid_coarse, psig):
    y = np.zeros(8 * int(np.prod(d.N)))
    ek = C.c_double()
    lib().wo_kinetic_wavelet(d.N, d.per, np.asarray(hgrid_coarse, np.float64),
                             np.ascontiguousarray(psig, np.float64), y, C.byref(ek))
    return y, ek.value


def locham_per(d, hgrid, psi_c, psi_f, pot):
    """Fortran-chain periodic Hpsi (hpsi accumulated from zero)."""
    N = d.N
    hc, hf = np.zeros(d.nvctr_c), np.zeros(7 * d.nvctr_f)
    ek, ep = C.c_double(), C.c_double()
    lib().wo_locham_per(int(N[0]) - 1, int(N[1]) - 1, int(N[2]) - 1, np.asarray(hgrid, np.float64), *d.args(),
                        np.ascontiguousarray(psi_c, np.float64), np.ascontiguousarray(psi_f, np.float64),
                        np.ascontiguousarray(pot, np.float64), hc, hf, C.byref(ek), C.byref(ep))
    return hc, hf, ek.value, ep.value


def locham(d, hgrid, psi_c, psi_f, pot):
    """OpenCL-composition Hpsi for any per-dimension BC (hpsi overwritten)."""
    hc, hf = np.zeros(d.nvctr_c), np.zeros(7 * d.nvctr_f)
    ek, ep = C.c_double(), C.c_double()
    lib().wo_locham_generic(d.N, d.per, np.asarray(hgrid, np.float64), *d.args(),
                            np.ascontiguousarray(psi_c, np.float64), np.ascontiguousarray(psi_f, np.float64),
                            np.ascontiguousarray(pot, np.float64), hc, hf, C.byref(ek), C.byref(ep))
    return hc, hf, ek.value, ep.value


def locden(d, psi_c, psi_f, hfac, rho=None):
    n = int(np.prod(d.I))
    rho = np.zeros(n) if rho is None else np.array(rho, np.float64)
    lib().wo_locden_generic(d.N, d.per, *d.args(), np.ascontiguousarray(psi_c, np.float64),
                            np.ascontiguousarray(psi_f, np.float64), float(hfac), rho)
    return rho


def precond_scal(h_fine, c):
    s = np.empty(8)
    lib().wo_precond_scal(np.asarray(h_fine, np.float64), float(c), s)
    return s


def precond(d, h_fine, c, ncong, x, b):
    """ocl_preconditioner_generic: returns (x_out, rnorm[ncong+1])."""
    x = np.array(x, np.float64)
    b = np.array(b, np.float64)
    rn = np.zeros(ncong + 1)
    lib().wo_precond_generic(d.N, d.per, np.asarray(h_fine, np.float64), float(c), int(ncong),
                             d.nseg_c, d.nvctr_c, d.keyg_c, d.keyv_c, d.nseg_f, d.nvctr_f, d.keyg_f, d.keyv_f,
                             x, b, rn)
    return x, rn


def overlap(psi):
    """psi (norb, nvctr) row-major == (nvctr, norb) column-major -> S (norb,norb)."""
    psi = np.ascontiguousarray(psi, np.float64)
    norb, nv = psi.shape
    S = np.empty((norb, norb))
    lib().wo_overlap(nv, norb, psi, S)
    return S


def cholesky_lower(S):
    """Returns L (row-major numpy) with S = L L^T."""
    A = np.array(S, np.float64, order="C")
    info = lib().wo_cholesky(A.shape[0], A)  # operates column-major: A^T viewed
    if info:
        raise np.linalg.LinAlgError("not positive definite at %d" % info)
    return A.T.copy()


def wpdot(ka, a, kb, b):
    """<a|b> of two compressed vectors on different keys of one box, as the
    reference's wpdot (wavelib/scalprod.f90:3222) computes it with one thread.
    ka, kb: (keyg_c, keyv_c, keyg_f, keyv_f) 1-based; a, b: [c | f] vectors."""
    def parts(k, v):
        kgc, kvc, kgf, kvf = (np.ascontiguousarray(x, np.int32).ravel() for x in k)
        nvc = int(sum(kgc[1::2] - kgc[0::2] + 1)) if len(kvc) else 0
        v = np.ascontiguousarray(v, np.float64)
        fine = v[nvc:] if len(v) > nvc else np.zeros(7)
        return [len(kvc), _k(kgc), _k(kvc), len(kvf), _k(kgf), _k(kvf),
                v[:nvc] if nvc else np.zeros(1), np.ascontiguousarray(fine)]
    return lib().wo_wpdot(*parts(ka, a), *parts(kb, b))


def _parts(k, v):
    kgc, kvc, kgf, kvf = (np.ascontiguousarray(x, np.int32).ravel() for x in k)
    nvc = int(sum(kgc[1::2] - kgc[0::2] + 1)) if len(kvc) else 0
    return kgc, kvc, kgf, kvf, nvc


def mask_axpy(ka, a, kb, b, s):
    """a += s b on the points common to a's keys and b's keys, with the
    reference's pairing of segments (waxpy_mask_unpack over the masks of
    fill_wblas_segs, locregs/scalar_product.f90:953,1095).  a is updated in
    place (a contiguous float64 [c | f] vector)."""
    kgc, kvc, kgf, kvf, nva = _parts(ka, a)
    lgc, lvc, lgf, lvf, nvb = _parts(kb, b)
    b = np.ascontiguousarray(b, np.float64)
    ac = a[:nva] if nva else np.zeros(1)
    af = a[nva:] if len(a) > nva else np.zeros(7)
    bc = b[:nvb] if nvb else np.zeros(1)
    bf = np.ascontiguousarray(b[nvb:]) if len(b) > nvb else np.zeros(7)
    lib().wo_mask_axpy(len(kvc), _k(kgc), _k(kvc), len(kvf), _k(kgf), _k(kvf), ac, af,
                       len(lvc), _k(lgc), _k(lvc), len(lvf), _k(lgf), _k(lvf), bc, bf, float(s))


def nlpsp_apply(kw, psi, atoms):
    """Nonlocal projector application for the rows of psi on keys kw
    (NonLocalHamiltonianApplication, hpsiortho.f90:1044-1125): per atom
    (kp, proj, h) with proj (m, projector size) on keys kp and h (m, m),
    c_i = <p_i|psi> (wpdot pairing), hc = h c, eproj += c.hc and
    hpsi += sum_i hc_i p_i.  Returns (the added hpsi rows, eproj)."""
    psi = np.atleast_2d(np.asarray(psi, np.float64))
    out = np.zeros_like(psi)
    eproj = np.zeros(psi.shape[0])
    for o in range(psi.shape[0]):
        row = np.ascontiguousarray(out[o])
        for kp, proj, h in atoms:
            proj = np.atleast_2d(np.asarray(proj, np.float64))
            c = np.array([wpdot(kw, psi[o], kp, proj[i]) for i in range(proj.shape[0])])
            hc = np.asarray(h, np.float64) @ c
            eproj[o] += float(c @ hc)
            for i in range(proj.shape[0]):
                mask_axpy(kw, row, kp, proj[i], hc[i])
        out[o] = row
    return out, eproj


def lagrange_multiplier(lam, occup, symm=True, correction=True):
    """The reference's lagrange_multiplier (wfn_opt/orthogonality.f90:293-369)
    for real coefficients, loop for loop: lam is the Fortran lambda(i, j) =
    <psi_i|hpsi_j> as a numpy (norb, norb) array indexed [i, j]; modified in
    place.  Returns (trace, asymm, mix)."""
    norb = lam.shape[0]
    tol = 0.5
    asymm = mix = trace = 0.0
    for i in range(norb):
        trace += lam[i, i]
        for j in range(i + 1, norb):
            lij, lji = lam[i, j], lam[j, i]
            asymm = max(asymm, (lij - lji) ** 2)
            if symm:
                lij = lij + lji
                lam[i, j] = 0.5 * lij
                lam[j, i] = 0.5 * lij
        fi = occup[i]
        for j in range(norb):
            fj = occup[j]
            if fi != fj:
                mix = max(mix, lam[i, j] ** 2)
                if correction:
                    fac = 0.5 * ((fi - fj) / fi) if abs(fi) > tol else 0.5
                    lam[i, j] = fac * lam[i, j]
    return trace, asymm, mix


def orthoconstraint(psi, hpsi, occup, symm=True, tr_min=False):
    """orthoconstraint (orthogonality.f90:375-625) for real orbitals of one spin
    and k-point, rows of psi/hpsi the orbitals: lambda = psi hpsi^T
    (subspace_matrix, gemm('T','N')), lagrange_multiplier, then
    hpsi_j -= sum_i lambda(i, j) psi_i (subspace_update, gemm('N','N', -1)).
    Returns (new hpsi, lambda, trace, asymm, mix)."""
    lam = np.asarray(psi, np.float64) @ np.asarray(hpsi, np.float64).T
    tr, asy, mix = lagrange_multiplier(lam, occup, symm, not tr_min)
    return hpsi - lam.T @ psi, lam, tr, asy, mix


def isf_weights():
    """{m: w_m} for odd m = 1..15: the 16-point Lagrange interpolation weights
    at the midpoint of the odd offsets -15..15 (exact rationals), the odd taps
    ch(+-m) of the order-16 ISF two-scale filter (lazy_16.inc, ch(0) = 1)."""
    from fractions import Fraction
    odd = list(range(-15, 16, 2))
    w = {}
    for m in range(1, 16, 2):
        r = Fraction(1)
        for i in odd:
            if i != m:
                r *= Fraction(-i, m - i)
        w[m] = float(r)
    return w


def isf_fourier(n):
    """The order-16 ISF's Fourier transform at p = i 2 pi / (2 n), i = 0..n, as
    fourtrans_isf computes it (psolver/src/Build_Kernel.f90:202-262): odd i by
    the product of two-scale symbols H(p/2^j) until H is 1 to 1e-16, even i
    from i/2 by one more symbol.  H(p) = 1/2 + sum over odd m <= 15 of
    w_m cos(m p), w_m the 16-point Lagrange weights at the midpoint of the odd
    offsets (the lazy_16 filter)."""
    w = isf_weights()

    def H(p):
        return 0.5 + sum(w[m] * np.cos(m * p) for m in range(15, 0, -2))
    f = np.zeros(n + 1)
    f[0] = 1.0
    for i in range(1, n + 1):
        if i % 2 == 0:
            continue
        p = i * 2.0 * np.pi / (2.0 * n)
        v, q = 1.0, p
        while True:
            q *= 0.5
            hv = H(q)
            if abs(hv - 1.0) <= 1e-16:
                break
            v *= hv
        f[i] = v
        j, q = i, p
        while True:
            j *= 2
            if j > n:
                break
            f[j] = H(q) * f[j // 2]
            q *= 2.0
    return f


def psolver_periodic(rho, h, offset=0.0):
    """Hartree potential and energy of rho (n3, n2, n1; x fastest) on a
    periodic grid of spacings h, the reference's periodic PSolver restated
    with numpy FFTs (Periodic_Kernel, Build_Kernel.f90:16-197; P_multkernel_NO,
    PSolver_Base_new.f90:2515-2640: V^ = rho^ phi^x phi^y phi^z / (pi g^2),
    V^(0) = offset / h^3; scal = 1/N, createKernel.f90:299; energy
    0.5 sum(rho V) h^3, PSolver_Main.f90:403)."""
    rho = np.asarray(rho, np.float64)
    n3, n2, n1 = rho.shape
    L = (n1 * h[0], n2 * h[1], n3 * h[2])
    fx, fy, fz = isf_fourier(n1 // 2), isf_fourier(n2 // 2), isf_fourier(n3 // 2)
    k1 = np.arange(n1 // 2 + 1)
    p2 = np.minimum(np.arange(n2), n2 - np.arange(n2))
    p3 = np.minimum(np.arange(n3), n3 - np.arange(n3))
    g = ((k1 / L[0])[None, None, :] ** 2 + (p2 / L[1])[None, :, None] ** 2 + (p3 / L[2])[:, None, None] ** 2)
    fac = fx[None, None, k1] * fy[None, p2, None] * fz[p3, None, None]
    g[0, 0, 0] = 1.0
    z = np.fft.rfftn(rho) * fac / (np.pi * g)
    z[0, 0, 0] = offset / (h[0] * h[1] * h[2])
    V = np.fft.irfftn(z, s=rho.shape, axes=(0, 1, 2))
    return V, 0.5 * float((rho * V).sum()) * h[0] * h[1] * h[2]


def gequad():
    """(p, w): the 89-term expansion 1/r = sum w exp(-p r^2) on [1e-9, 1] of
    psolver/src/Build_Kernel.f90:1679-1873, from the generated filter header."""
    import re
    hdr = (HERE.parent / "bigdft-suite_b200" / "csrc" / "wvl_filters.h").read_text()
    out = []
    for name in ("WVL_GQ_P", "WVL_GQ_W"):
        body = re.search(r"#define %s_INIT \{(.*?)\}" % name, hdr, re.S).group(1)
        out.append(np.array([float(v) for v in body.replace("\\", " ").split(",")]))
    return out[0], out[1]


def isf_samples(itype=16, n_points=16):
    """(x, y), 2 itype n_points + 1 points: the order-16 ISF on [-15, 17] at
    spacing 1/16 by the cascade of scaling_function
    (psolver/src/scaling_function.f90:12-110; back_trans_16 :1232-1266): a unit
    value at x = 0 refined by doubling, even points kept, odd points the
    midpoint interpolation sum_j ch(2j+1) x(i-j), periodic on the current
    length (the support never reaches the wrap)."""
    ni, nd = 2 * itype, 2 * itype * n_points
    w = isf_weights()
    ch = {0: 1.0}
    for m, v in w.items():
        ch[m] = ch[-m] = v
    mm = itype + 2
    x = np.zeros(nd + 1)
    x[ni // 2 - 1] = 1.0
    nt = ni
    while True:
        nt *= 2
        half = nt // 2
        prev = x[:half].copy()
        y = np.zeros(nt)
        y[0::2] = prev
        for j in range(-mm // 2, mm // 2):
            c = ch.get(2 * j + 1, 0.0)
            if c:
                y[1::2] += c * np.roll(prev, j)      # prev[(i - j) mod half]
        x[:nt] = y
        if nt == nd:
            break
    a = np.arange(nd + 1) * ni / nd - (0.5 * ni - 1.0)
    return a, x


def gauss_conv_isf(p, h, n_range, xs, ys, itype=16):
    """k(i) = integral of phi(x - i) exp(-p h^2 x^2) dx (x in grid units), i =
    -n_range..n_range (index i + n_range), as gauss_conv_scf
    (psolver/src/Build_Kernel.f90:1597-1651): for a sharp Gaussian the
    exponent is first divided by 4^n_iter (n_iter = nint(log4(p h^2))), the
    Riemann sum over the ISF samples taken (terms past sqrt(634.7/p0)/h
    skipped, stopping after the first value below 1e-18), then n_iter
    two-scale steps k(i) <- 1/2 sum_j ch(j) k(2i - j) (scf_recursion_16,
    scaling_function.f90:1324-1356) bring it back to p."""
    dx = (2.0 * itype) / (len(xs) - 1)
    p0_cell = 1.0 / (h * h)
    n_iter = int(np.floor((np.log(p) - np.log(p0_cell)) / np.log(4.0) + 0.5))
    if n_iter <= 0:
        n_iter, p0 = 0, p
    else:
        p0 = p / 4.0 ** n_iter
    x_limit = np.sqrt(634.71369555645470 / p0) / h
    k = np.zeros(2 * n_range + 1)
    for i in range(n_range + 1):
        ab = xs - i
        m = np.abs(ab) < x_limit
        v = float(np.sum(ys[m] * np.exp(-p0 * (ab[m] * ab[m] * h ** 2))))
        k[n_range + i] = k[n_range - i] = v * dx
        if abs(v) < 1e-18:
            break
    w = isf_weights()
    ch = {0: 1.0}
    for mm, v in w.items():
        ch[mm] = ch[-mm] = v
    for _ in range(n_iter):
        k1 = k.copy()
        k[:] = 0.0
        for i in range(n_range + 1):
            tot = 0.0
            for j in range(-(itype + 2), itype + 3):
                ind = 2 * i - j
                if -n_range <= ind <= n_range and j in ch:
                    tot += ch[j] * k1[n_range + ind]
            if tot == 0.0:
                break
            k[n_range + i] = k[n_range - i] = 0.5 * tot
    return k


def free_kernel(n0, h, nfft):
    """The free-boundary Poisson kernel in Fourier space, as Free_Kernel
    (psolver/src/Build_Kernel.f90:985-1175) builds it: for each Gaussian of
    gequad, scaled to the box diagonal a (p / a^2, w / a), the three 1D
    ISF-Gaussian overlaps (gauss_conv_isf, n_range = max(n01, n02, n03, 32)
    points) cosine-transformed on the padded lengths nfft (gauconv_ffts
    :1184-1340: the symmetric sequence of min(n_range, n/2) values; the
    reference's centred layout multiplies each transform by (-1)^k, which only
    moves the origin of its convolution), summed from the last Gaussian to
    the first as k_x (k_z (k_y w)).  n0 = (n01, n02, n03), nfft = (N1, N2, N3);
    returns K of shape (N3/2+1, N2/2+1, N1/2+1), x fastest."""
    pg, wg = gequad()
    a = [h[d] * n0[d] for d in range(3)]
    a2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2]
    factor, factor2 = 1.0 / np.sqrt(a2), 1.0 / a2
    n_range = max(max(n0), 32)
    xs, ys = isf_samples()
    K = np.zeros((nfft[2] // 2 + 1, nfft[1] // 2 + 1, nfft[0] // 2 + 1))
    cosk = []
    for d in range(3):
        n = nfft[d]
        J = min(n_range, n // 2)
        kk = np.arange(n // 2 + 1)[:, None]
        jj = np.arange(1, J)[None, :]
        cosk.append((J, np.cos(2.0 * np.pi * ((kk * jj) % n) / n)))
    for g in range(len(pg) - 1, -1, -1):
        pgauss = pg[g] * factor2
        C = []
        for d in range(3):
            k = gauss_conv_isf(pgauss, h[d], n_range, xs, ys)
            J, cs = cosk[d]
            f = k[n_range:n_range + J]
            C.append(f[0] + 2.0 * (cs @ f[1:]))
        w = wg[g] * factor
        K += C[0][None, None, :] * (C[2][:, None, None] * (C[1][None, :, None] * w))
    return K


# closed 9-point Newton-Cotes weights (the composite rule of order 8 that
# calculates_green_opt integrates with: intorder 8, cpol(:, 8) times 8,
# psolver/src/Build_Kernel.f90:279-360, :734-864)
NC9 = np.array([989.0, 5888.0, -928.0, 10496.0, -4540.0, 10496.0, -928.0, 5888.0, 989.0]) * 4.0 / 14175.0


def _isf_fine():
    """The order-16 ISF sampled at 1/64 on [-15, 17] (scaling_function with
    2 * 16 * 64 intervals, as Surfaces_Kernel samples it)."""
    global _ISF_FINE
    try:
        return _ISF_FINE
    except NameError:
        _ISF_FINE = isf_samples(16, 64)
        return _ISF_FINE


def _two_scale_recursion(k, nr, n_iter, itype=16):
    """n_iter steps of k(i) <- 1/2 sum_j ch(j) k(2i - j) on k(-nr..nr) (index
    i + nr), stopping at the first zero sum (scf_recursion_16,
    scaling_function.f90:1324-1356)."""
    w = isf_weights()
    ch = {0: 1.0}
    for mm, v in w.items():
        ch[mm] = ch[-mm] = v
    i = np.arange(nr + 1)
    for _ in range(n_iter):
        k1 = k.copy()
        tot = np.zeros(nr + 1)
        for j in range(-(itype + 2), itype + 3):
            if j not in ch:
                continue
            ind = 2 * i - j
            ok = (ind >= -nr) & (ind <= nr)
            tot[ok] += ch[j] * k1[nr + ind[ok]]
        zero = np.nonzero(tot == 0.0)[0]
        if len(zero):
            tot[zero[0]:] = 0.0
        k[:] = 0.0
        k[nr:] = 0.5 * tot
        k[:nr + 1] = (0.5 * tot)[::-1]
    return k


def _segment_sums(xs, ys, izero, g, n_scf):
    """The composite Newton-Cotes integral of g(x) y(x) over each unit segment
    [j-1, j] from x = 0 (loop_integration of calculates_green_opt): returns a
    list, one sum per segment until the samples end."""
    out = []
    s = izero
    while s < n_scf:
        tot = 0.0
        for p in range(8):                       # 8 panels of 8 intervals at spacing 1/64
            idx = s + 8 * p + np.arange(9)
            tot += float(np.dot(NC9, ys[idx] * g(xs[idx])))
        out.append(tot)
        s += 64
    return out


def green_surface(n, mu, itype=16):
    """g(j), j = 0..n-1: the integral of phi(x - j) exp(-mu |x|) (mu > 0), as
    calculates_green_opt computes it (Build_Kernel.f90:734-864): mu divided by
    2^n_iter until it is <= 0.2, the integrals from each side accumulated
    segment by segment with exp(-+mu0) factors, then n_iter two-scale steps."""
    xs, ys = _isf_fine()
    n_scf = len(xs) - 1
    hres = 32.0 / n_scf
    n_iter, mu0 = 0, mu
    if mu > 0.2:
        n_iter = 1
        while mu / 2.0 ** n_iter > 0.2:
            n_iter += 1
        mu0 = mu / 2.0 ** n_iter
    nrec = 2 ** n_iter * n
    izero = int(np.argmax(xs >= 0.0))
    green = np.zeros(2 * nrec + 1)
    # the right half from x = 0: panels while 9 points and one more remain, then
    # the leftover points with the first weights (the tail is outside the support)
    gr, iv = 0.0, izero
    while iv < n_scf - 9:
        idx = iv + np.arange(9)
        gr += float(np.dot(NC9, ys[idx] * np.exp(-mu0 * xs[idx])))
        iv += 8
    idx = iv + np.arange(n_scf - iv)
    gr += float(np.dot(NC9[:len(idx)], ys[idx] * np.exp(-mu0 * xs[idx])))
    gright = hres * gr
    gleft = gright
    green[nrec] = gleft + gright
    sl = _segment_sums(xs, ys, izero, lambda x: np.exp(mu0 * x), n_scf)
    sr = _segment_sums(xs, ys, izero, lambda x: np.exp(-mu0 * x), n_scf)
    em, ep = np.exp(-mu0), np.exp(mu0)
    for ik in range(1, nrec + 1):
        lt = sl[ik - 1] if ik - 1 < len(sl) else 0.0
        rt = sr[ik - 1] if ik - 1 < len(sr) else 0.0
        gleft = em * (gleft + hres * np.exp(-mu0 * (ik - 1)) * lt)
        gright = ep * (gright - hres * np.exp(mu0 * (ik - 1)) * rt) if ik < len(sl) else 0.0
        green[nrec + ik] = green[nrec - ik] = gleft + gright
        if abs(gleft + gright) <= 1e-20:
            nrec_eff = ik
            break
    else:
        nrec_eff = nrec
    # the recursion runs on green(-nrec_eff..nrec_eff)
    k = green[nrec - nrec_eff:nrec + nrec_eff + 1].copy()
    k = _two_scale_recursion(k, nrec_eff, n_iter)
    out = np.zeros(n)
    m = min(n, nrec_eff)
    out[:m] = k[nrec_eff:nrec_eff + m]
    return out


def green_surface_mu0(n):
    """g(j), j = 0..n-1: the integral of phi(x) |x - j| (the k = 0 term),
    as calculates_green_opt_muzero (Build_Kernel.f90:867-953)."""
    xs, ys = _isf_fine()
    n_scf = len(xs) - 1
    hres = 32.0 / n_scf
    izero = int(np.argmax(xs >= 0.0))
    gr, iv = 0.0, izero
    while iv < n_scf - 9:
        idx = iv + np.arange(9)
        gr += float(np.dot(NC9, xs[idx] * ys[idx]))
        iv += 8
    idx = iv + np.arange(n_scf - iv)
    gr += float(np.dot(NC9[:len(idx)], xs[idx] * ys[idx]))
    gr1 = hres * gr
    gl1, gl0, gr0 = -gr1, 0.5, 0.5
    out = np.zeros(n)
    out[0] = 2.0 * gr1
    s0 = _segment_sums(xs, ys, izero, lambda x: np.ones_like(x), n_scf)
    s1 = _segment_sums(xs, ys, izero, lambda x: x, n_scf)
    for ik in range(1, n):
        c0 = hres * (s0[ik - 1] if ik - 1 < len(s0) else 0.0)
        c1 = hres * (s1[ik - 1] if ik - 1 < len(s1) else 0.0)
        gl0 += c0
        gl1 += c1
        gr0 -= c0
        gr1 -= c1
        out[ik] = ik * (gl0 - gr0) + gr1 - gl1
    return out


def surface_kernel(n0, h, N2):
    """The surface-BC kernel in Fourier space (x and z periodic, y free;
    Surfaces_Kernel, Build_Kernel.f90:279-731): for each in-plane frequency
    (k1, k3), mu = 2 pi h_y |g| and the 1D Green's function along y (-h_y /
    (2 mu) green_surface, or h_y / 2 green_surface_mu0 at mu = 0) on the
    box's n2 points, cosine-transformed on the padded length N2 (without the
    reference's centring sign (-1)^k).  n0 = (n1, n2, n3); returns K of shape
    (n3/2+1, N2/2+1, n1/2+1)."""
    n1, n2, n3 = n0
    nr = max(n2, 32)
    l1, l2, l3 = n1 // 2 + 1, N2 // 2 + 1, n3 // 2 + 1
    J = min(n2, N2 // 2)
    kk = np.arange(l2)[:, None]
    jj = np.arange(1, J)[None, :]
    cs = np.cos(2.0 * np.pi * ((kk * jj) % N2) / N2)
    K = np.zeros((l3, l2, l1))
    for k3 in range(l3):
        for k1 in range(l1):
            g1, g3 = k1 / (n1 * h[0]), k3 / (n3 * h[2])
            mu = h[1] * 2.0 * np.pi * np.sqrt(g1 * g1 + g3 * g3)
            if k1 == 0 and k3 == 0:
                v = 0.5 * h[1] * green_surface_mu0(nr)[:n2]
            else:
                v = -0.5 * h[1] / mu * green_surface(nr, mu)[:n2]
            K[k3, :, k1] = v[0] + 2.0 * (cs @ v[1:J])
    return K


def psolver_surface(rho, h, N2=None):
    """Hartree potential and energy of rho (n3, n2, n1; x fastest) with
    surface boundary conditions (x, z periodic; y free): rho zero-padded
    along y to N2 (default 2 n2), multiplied in Fourier space by
    surface_kernel, scaled by -4 pi h_y / (n1 N2 n3) (createKernel.f90:374),
    the first n2 planes of y kept; energy 0.5 sum(rho V) h^3."""
    rho = np.asarray(rho, np.float64)
    n3, n2, n1 = rho.shape
    N2 = 2 * n2 if N2 is None else N2
    K = surface_kernel((n1, n2, n3), h, N2)
    pad = np.zeros((n3, N2, n1))
    pad[:, :n2, :] = rho
    p2 = np.minimum(np.arange(N2), N2 - np.arange(N2))
    p3 = np.minimum(np.arange(n3), n3 - np.arange(n3))
    Kf = K[p3][:, p2]
    V = np.fft.irfftn(np.fft.rfftn(pad) * Kf, s=pad.shape, axes=(0, 1, 2))[:, :n2, :] * (-4.0 * np.pi * h[1])
    return V, 0.5 * float((rho * V).sum()) * h[0] * h[1] * h[2]


def wire_fits():
    """(p1, w1, p2, w2): the Gaussian fits of log r and K0(r) that the wire
    kernel is built from (psolver/src/gaussfit_wires.inc; 144 terms used),
    from the generated filter header."""
    import re
    hdr = (HERE.parent / "bigdft-suite_b200" / "csrc" / "wvl_filters.h").read_text()
    out = []
    for name in ("WVL_WIRE_P1", "WVL_WIRE_W1", "WVL_WIRE_P2", "WVL_WIRE_W2"):
        body = re.search(r"#define %s_INIT \{(.*?)\}" % name, hdr, re.S).group(1)
        out.append(np.array([float(v) for v in body.replace("\\", " ").split(",")])[:144])
    return tuple(out)


def wire_kernel(n0, h, Nx, Ny):
    """The wire-BC kernel in Fourier space (z periodic, x and y free;
    Wires_Kernel, Build_Kernel.f90:2244-2364): for each z frequency the 2D
    Green's function of the plane as a sum of separable Gaussians, each
    through the ISF overlaps and cosine transforms of the free kernel on the
    padded lengths (Nx, Ny): at k_z = 0 log(mu0 r) (p1, w1, mu0 =
    1/sqrt((h_x (n_x + 32))^2 + (h_y (n_y + 32))^2)) and -log(mu0) added at
    k = 0; otherwise -K0(mu r), mu = 2 pi k_z / (n_z h_z) (p2, -w2).
    n0 = (n_x, n_y, n_z); returns K of shape (n_z/2+1, Ny/2+1, Nx/2+1)."""
    nx, ny, nz = n0
    p1, w1, p2, w2 = wire_fits()
    nr = max(nx, ny, 32)
    xs, ys = isf_samples()
    cos = []
    for n in (Nx, Ny):
        J = min(nr, n // 2)
        kk = np.arange(n // 2 + 1)[:, None]
        jj = np.arange(1, J)[None, :]
        cos.append((J, np.cos(2.0 * np.pi * ((kk * jj) % n) / n)))
    K = np.zeros((nz // 2 + 1, Ny // 2 + 1, Nx // 2 + 1))
    for kz in range(nz // 2 + 1):
        if kz == 0:
            mu = 1.0 / np.sqrt((h[0] * (nx + 32)) ** 2 + (h[1] * (ny + 32)) ** 2)
            alpha, w = p1, w1
        else:
            mu = 2.0 * np.pi / nz * kz / h[2]
            alpha, w = p2, -w2
        for k in range(144):
            C = []
            for d, (J, cs) in enumerate(cos):
                f = gauss_conv_isf(alpha[k] * mu * mu, h[d], nr, xs, ys)[nr:nr + J]
                C.append(f[0] + 2.0 * (cs @ f[1:]))
            K[kz] += (w[k] * C[0])[None, :] * C[1][:, None]
        if kz == 0:
            K[0, 0, 0] -= Nx * Ny * np.log(mu)
    return K


def psolver_wire(rho, h, nfft=None):
    """Hartree potential and energy of rho (n_z, n_y, n_x; x fastest) with
    wire boundary conditions (z periodic, x and y free): rho zero-padded in
    x and y to (Nx, Ny) (default twice), multiplied in Fourier space by
    wire_kernel, scaled by -2 h_x h_y / (Nx Ny n_z) (createKernel.f90:502),
    the first (n_y, n_x) kept; energy 0.5 sum(rho V) h^3."""
    rho = np.asarray(rho, np.float64)
    nz, ny, nx = rho.shape
    Nx, Ny = (2 * nx, 2 * ny) if nfft is None else nfft
    K = wire_kernel((nx, ny, nz), h, Nx, Ny)
    pad = np.zeros((nz, Ny, Nx))
    pad[:, :ny, :nx] = rho
    py = np.minimum(np.arange(Ny), Ny - np.arange(Ny))
    pz = np.minimum(np.arange(nz), nz - np.arange(nz))
    Kf = K[pz][:, py]
    V = np.fft.irfftn(np.fft.rfftn(pad) * Kf, s=pad.shape, axes=(0, 1, 2))[:, :ny, :nx] * (-2.0 * h[0] * h[1])
    return V, 0.5 * float((rho * V).sum()) * h[0] * h[1] * h[2]


def psolver_free(rho, h, nfft=None):
    """Hartree potential and energy of rho (n3, n2, n1; x fastest) with free
    boundary conditions: rho zero-padded to nfft (default twice each
    dimension), multiplied in Fourier space by free_kernel, scaled by
    h1 h2 h3 / (N1 N2 N3) (createKernel.f90:439), the first n0 points kept;
    energy 0.5 sum(rho V) h^3 (PSolver_Main.f90:403)."""
    rho = np.asarray(rho, np.float64)
    n3, n2, n1 = rho.shape
    if nfft is None:
        nfft = (2 * n1, 2 * n2, 2 * n3)
    K = free_kernel((n1, n2, n3), h, nfft)
    N1, N2, N3 = nfft
    pad = np.zeros((N3, N2, N1))
    pad[:n3, :n2, :n1] = rho
    p2 = np.minimum(np.arange(N2), N2 - np.arange(N2))
    p3 = np.minimum(np.arange(N3), N3 - np.arange(N3))
    Kf = K[p3][:, p2]
    vol = h[0] * h[1] * h[2]
    V = np.fft.irfftn(np.fft.rfftn(pad) * Kf, s=pad.shape, axes=(0, 1, 2))[:n3, :n2, :n1] * vol
    return V, 0.5 * float((rho * V).sum()) * vol


# Goedecker-Teter-Hutter Pade fit of the Ceperley-Alder LDA (Phys. Rev. B 54,
# 1703 (1996), paramagnetic parameters; ixc = 1 of the reference, ABINIT's
# xcspol, libABINIT/src/abi_xc_lowlevel/abi_xcspol.F90:105-112): eps_xc(rs) =
# -(a0 + a1 rs + a2 rs^2 + a3 rs^3) / (b1 rs + b2 rs^2 + b3 rs^3 + b4 rs^4),
# rs = (3 / (4 pi rho))^(1/3).
TETER_A = (0.4581652932831429, 2.217058676663745, 0.7405551735357053, 0.01968227878617998)
TETER_B = (1.0, 4.504130959426697, 1.110667363742916, 0.02359291751427506)
RS_FAC = 0.6203504908994000     # (3 / (4 pi))^(1/3), abi_drivexc.F90:134


def xc_lda(rho):
    """(eps_xc, v_xc) of the total density rho (any shape), spin-unpolarised
    (abi_xcspol nspden = 1, :229-250: exc = -n1/d1, vxc = exc - rs/3 d exc/d rs).
    rs follows abi_drivexc (:213-224, rs = rsfac sign(|rho|^(-1/3), rho)); the
    reference's abi_invcb reaches |rho|^(-1/3) by a Pade iteration stopped at a
    relative residual of 1e-12, the oracle takes the cube root directly."""
    rho = np.asarray(rho, np.float64)
    a0, a1, a2, a3 = TETER_A
    b1, b2, b3, b4 = TETER_B
    rs = RS_FAC * np.sign(rho) * np.abs(rho) ** (-1.0 / 3.0)
    n1 = a0 + rs * (a1 + rs * (a2 + rs * a3))
    d1 = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)))
    eps = -n1 / d1
    dn1 = a1 + rs * (2.0 * a2 + rs * (3.0 * a3))
    dd1 = b1 + rs * (2.0 * b2 + rs * (3.0 * b3 + rs * (4.0 * b4)))
    deps = -(dn1 + eps * dd1) / d1
    return eps, eps - rs / 3.0 * deps


# ferromagnetic - paramagnetic differences of the fit's parameters (same
# paper; abi_xcspol.F90:113-116), the spin interpolation's alpha and
# fact = 1 / (2^(4/3) - 2) (:107, :176)
TETER_DA = (0.119086804055547, 0.6157402568883345, 0.1574201515892867, 0.003532336663397157)
TETER_DB = (0.0, 0.2673612973836267, 0.2052004607777787, 0.004200005045691381)
TETER_ALPHA = 1.0 - 1.0e-6


def xc_lsda(rho_up, rho_dn):
    """(eps_xc, v_up, v_dn) of a spin-polarised density (abi_xcspol
    nspden = 2, order 1, :355-395): zeta = 2 rho_up / rho - 1 (abi_drivexc
    :226-233), the parameters interpolated with f(zeta) = ((1 + a z)^(4/3) +
    (1 - a z)^(4/3) - 2) / (2^(4/3) - 2), v_up/dn = v_para - (zeta -/+ 1)
    d eps / d zeta."""
    up = np.asarray(rho_up, np.float64)
    dn = np.asarray(rho_dn, np.float64)
    rho = up + dn
    zet = 2.0 * up / rho - 1.0
    rs = RS_FAC * np.sign(rho) * np.abs(rho) ** (-1.0 / 3.0)
    fact = 1.0 / (2.0 ** (4.0 / 3.0) - 2.0)
    zp, zm = 1.0 + zet * TETER_ALPHA, 1.0 - zet * TETER_ALPHA
    zp3, zm3 = zp ** (1.0 / 3.0), zm ** (1.0 / 3.0)
    fxc = (zp * zp3 + zm * zm3 - 2.0) * fact
    a = [TETER_A[i] + fxc * TETER_DA[i] for i in range(4)]
    b = [TETER_B[i] + fxc * TETER_DB[i] for i in range(4)]
    n1 = a[0] + rs * (a[1] + rs * (a[2] + rs * a[3]))
    d1 = rs * (b[0] + rs * (b[1] + rs * (b[2] + rs * b[3])))
    eps = -n1 / d1
    dn1 = a[1] + rs * (2.0 * a[2] + rs * (3.0 * a[3]))
    dd1 = b[0] + rs * (2.0 * b[1] + rs * (3.0 * b[2] + rs * (4.0 * b[3])))
    vp = eps - rs / 3.0 * (-(dn1 + eps * dd1) / d1)
    dfdz = 4.0 / 3.0 * TETER_ALPHA * (zp3 - zm3) * fact
    dn1df = TETER_DA[0] + rs * (TETER_DA[1] + rs * (TETER_DA[2] + rs * TETER_DA[3]))
    dd1df = rs * (TETER_DB[0] + rs * (TETER_DB[1] + rs * (TETER_DB[2] + rs * TETER_DB[3])))
    dedz = dfdz * (-(dn1df + eps * dd1df) / d1)
    return eps, vp - (zet - 1.0) * dedz, vp - (zet + 1.0) * dedz


def ks_potential_spin(rho_up, rho_dn, h, vext=None, free=False, rhocore=None):
    """updatePotential for nspin = 2 (bigdft/src/modules/rhopotential.f90:
    87-120): V_H of the total density (XC_potential leaves the total in the
    first half, xc_energy_new :902-908), pot_sigma = (V_H + V_ext) + V_xc,sigma.
    Returns (pot_up, pot_dn, (eh, exc, evxc)), evxc = dvol sum_sigma v rho."""
    up = np.asarray(rho_up, np.float64)
    dn = np.asarray(rho_dn, np.float64)
    tot = up + dn
    vh, eh = _hartree_bc(tot, h, free)
    hc = 0.0 if rhocore is None else 0.5 * np.asarray(rhocore, np.float64)   # half the core on each spin
    eps, vu, vd = xc_lsda(up + hc, dn + hc)
    base = vh if vext is None else vh + np.asarray(vext, np.float64)
    dvol = h[0] * h[1] * h[2]
    return (base + vu, base + vd,
            (eh, float((eps * ((up + hc) + (dn + hc))).sum()) * dvol, float((vu * up + vd * dn).sum()) * dvol))


def _hartree_bc(rho, h, bc):
    """V_H for a boundary condition: False / "periodic", True / "free",
    "surface" or "wire"."""
    bc = {False: "periodic", True: "free"}.get(bc, bc)
    return {"periodic": psolver_periodic, "free": psolver_free, "surface": psolver_surface,
            "wire": psolver_wire}[bc](rho, h)


def ks_potential_free(rho, h, vext=None):
    """ks_potential_periodic with the free-boundary Hartree potential."""
    return ks_potential_periodic(rho, h, vext, free=True)


def ks_potential_periodic(rho, h, vext=None, free=False, rhocore=None):
    """The Kohn-Sham potential of a periodic box from the total density, as
    updatePotential (bigdft/src/modules/rhopotential.f90:29-125) builds it for
    nspin = 1 and ixc = 1: XC_potential (xcPSolver/xcenergy.f90:428; energies
    xc_energy_new, orbitals/xc.f90:763-925: exc = dvol sum eps rho, evxc =
    dvol sum v_xc rho), H_potential with V_ext summed in (offset 0), then
    rhov += V_xc.  Returns (pot, (eh, exc, evxc))."""
    rho = np.asarray(rho, np.float64)
    vh, eh = _hartree_bc(rho, h, free)
    # a core density joins the valence one for XC only; evxc keeps the valence
    # part (substract_from_vexcu, xcPSolver/xcenergy.f90:850-882)
    rx = rho if rhocore is None else rho + np.asarray(rhocore, np.float64)
    eps, vxc = xc_lda(rx)
    dvol = h[0] * h[1] * h[2]
    pot = (vh if vext is None else vh + np.asarray(vext, np.float64)) + vxc   # H_potential's sum, then the axpy
    return pot, (eh, float((eps * rx).sum()) * dvol, float((vxc * rho).sum()) * dvol)


# ---------------------------------------------------------------- reference pin
def ref_magicfilter():
    """ctypes handle to the reference's own C magic filter, or None."""
    if not REF_MF.exists():
        return None
    L = C.CDLL(str(REF_MF))
    for nm in ("magicfilter1d_naive_", "magicfilter1d_t_naive_", "magicfilter1d_sse_", "magicfilter1d_t_sse_"):
        getattr(L, nm).argtypes = [C.POINTER(C.c_uint), C.POINTER(C.c_uint), f64p, f64p]
    return L


def ref_convib():
    """ctypes handle to the reference's own SSE wavelet-basis kinetic
    operator (bigdft/src/orbitals/convolut_ib_sse.c), or None."""
    if not REF_CONVIB.exists():
        return None
    return C.CDLL(str(REF_CONVIB))


_FINE_X = ("convolut_ib_sse_fx_wss_", "convolut_ib_sse_fx_sws_wws_", "convolut_ib_sse_fx_ssw_wsw_",
           "convolut_ib_sse_fx_sww_www_")
_FINE_YZ = ("convolut_ib_sse_fy_sws_", "convolut_ib_sse_fy_wss_wws_", "convolut_ib_sse_fy_ssw_sww_",
            "convolut_ib_sse_fy_wsw_www_", "convolut_ib_sse_fz_ssw_", "convolut_ib_sse_fz_wss_wsw_",
            "convolut_ib_sse_fz_sws_sww_", "convolut_ib_sse_fz_wws_www_")


def ref_kinetic_sse(n, hgrid, cprecr, x_c, x_f, nfl, nfu, ibc, ibf):
    """The reference's FP32 SSE kinetic operator (c + T) in the wavelet
    basis, called as Convolkinetic_SSE does (convolut_ib_optim.f90:868-903):
    coarse->coarse (convolut_ib_sse_cxyz_) and fine->fine (the _fx/_fy/_fz
    functions, in that order), filters a, b, c, e (the tables of
    ConvolkineticT, :962-1046) scaled by -1/(2 h^2) for an isotropic coarse
    spacing h.  x_c: (n3+1, n2+1, n1+1) float32; x_f: (nfu3-nfl3+1,
    nfu2-nfl2+1, nfu1-nfl1+1, 7) float32; ibc / ibf: make_bounds triples
    (ibyz, ibxz, ibxy) as (.., .., 2) int32 arrays.  Returns (y_c, y_f)."""
    L = ref_convib()
    n1, n2, n3 = (int(v) for v in n)
    sc = -0.5 / (hgrid * hgrid)
    a = np.zeros(29)
    e = np.zeros(29)
    cc = np.zeros(29)
    b = np.zeros(29)
    for l in range(15):
        a[14 + l] = a[14 - l] = _filter_table("WVL_KIN")[l]
        e[14 + l] = e[14 - l] = _filter_table("WVL_KIN_E")[l]
    kc = _filter_table("WVL_KIN_C")
    for l in range(-14, 15):
        cc[l + 14] = kc[l + 14]
        b[l + 14] = kc[-l + 14]
    fa, fb, fc, fe = (np.ascontiguousarray(v * sc, np.float32) for v in (a, b, cc, e))
    x_c = np.ascontiguousarray(x_c, np.float32)
    x_f = np.ascontiguousarray(x_f, np.float32)
    y_c = np.zeros_like(x_c)
    y_f = np.zeros_like(x_f)
    ii = lambda v: C.byref(C.c_int(int(v)))
    cp = C.byref(C.c_float(cprecr))
    P = lambda arr: arr.ctypes.data_as(C.c_void_p)
    ibc = [np.ascontiguousarray(v, np.int32) for v in ibc]
    ibf = [np.ascontiguousarray(v, np.int32) for v in ibf]
    L.convolut_ib_sse_cxyz_(ii(n1), ii(n2), ii(n3), P(ibc[0]), P(ibc[1]), P(ibc[2]), cp, P(x_c), P(y_c), P(fa))
    lim = [ii(nfl[0]), ii(nfu[0]), ii(nfl[1]), ii(nfu[1]), ii(nfl[2]), ii(nfu[2])]
    for nm in _FINE_X:
        getattr(L, nm)(ii(n1), ii(n2), ii(n3), P(ibf[0]), cp, *lim, P(x_f), P(y_f), P(fa), P(fb), P(fc), P(fe))
    for nm in _FINE_YZ:
        ib = ibf[1] if "_fy_" in nm else ibf[2]
        getattr(L, nm)(ii(n1), ii(n2), ii(n3), P(ib), *lim, P(x_f), P(y_f), P(fa), P(fb), P(fc), P(fe))
    return y_c, y_f


def _filter_table(name):
    """A coefficient table of the generated filter header (parsed from the
    reference sources at build time), as float64."""
    import re
    hdr = (HERE.parent / "bigdft-suite_b200" / "csrc" / "wvl_filters.h").read_text()
    m = re.search(r"#define %s_AT\(i\) (.*)" % name, hdr)
    return [float(v) for v in re.findall(r"\(([-+]?\d[\d.eE+-]*)\)", m.group(1))]
