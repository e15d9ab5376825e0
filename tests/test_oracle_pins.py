"""Pins of the CPU oracle (the checker of every GPU parity test).

The reference stores no golden vectors for this path (its conv_check tests
recompute CPU references from random inputs), so the oracle is pinned by:
  * the reference's own C magic filter (bigdft/src/convolutions-c/MagicFilter_sse.c)
    compiled into oracle/_ref, bit-exact, and golden vectors generated from it;
  * the mathematical identities the reference relies on (DB16 orthonormality,
    analysis o synthesis = identity, magic-filter adjointness);
  * two independent formulations of the kinetic operator that the reference
    ships (the fine-grid 29-tap filter of convolut_kinetic_per_T and the
    wavelet-basis a/b/c/e filters of ConvolkineticT) agreeing to 1e-15;
  * the reference's Fortran chain (daub_to_isf_locham + isf_to_daub_kinetic)
    and its OpenCL composition (ocl_fulllocham_generic) agreeing;
  * an analytic known answer: the kinetic energy of a Gaussian;
  * the reference's OpenCL periodic synthesis, analysis and fine-grid kinetic
    kernels (OpenCL/Wavelet_Generator.cpp, Kinetic_Generator.cpp), whose
    multiply-add statements tests/golden/make_opencl_kernels.py replays from
    the generators' source text into tests/golden/opencl_kernels.npz.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from conftest import REFERENCE

GOLD = Path(__file__).resolve().parent / "golden"


def test_filter_header_matches_reference_sources():
    if not (REFERENCE / "bigdft").exists():
        pytest.skip("reference tree not present")
    import importlib.util
    gen = Path(__file__).resolve().parents[1] / "bigdft-suite_b200" / "csrc" / "gen_filters.py"
    spec = importlib.util.spec_from_file_location("gen_filters", gen)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    text = m.render(m.parse(REFERENCE))
    assert text == gen.with_name("wvl_filters.h").read_text()


def _filters():
    hdr = (Path(__file__).resolve().parents[1] / "bigdft-suite_b200" / "csrc" / "wvl_filters.h").read_text()
    import re
    out = {}
    for name in ("WVL_CH", "WVL_CG", "WVL_MF", "WVL_KIN", "WVL_KIN_C", "WVL_KIN_E"):
        body = re.search(r"#define %s_INIT \{(.*?)\}" % name, hdr, re.S).group(1)
        out[name] = np.array([float(v) for v in body.replace("\\", " ").split(",")])
    return out


def test_db16_orthonormality():
    f = _filters()
    ch, cg = f["WVL_CH"], f["WVL_CG"]
    assert abs(ch.sum() - np.sqrt(2)) < 1e-15
    assert abs(cg.sum()) < 1e-15
    for k in range(-7, 8):
        a = sum(ch[l] * ch[l + 2 * k] for l in range(16) if 0 <= l + 2 * k < 16)
        b = sum(cg[l] * cg[l + 2 * k] for l in range(16) if 0 <= l + 2 * k < 16)
        c = sum(ch[l] * cg[l + 2 * k] for l in range(16) if 0 <= l + 2 * k < 16)
        assert abs(a - (k == 0)) < 2e-15 and abs(b - (k == 0)) < 2e-15 and abs(c) < 2e-15


def test_magic_filter_and_kinetic_moments():
    f = _filters()
    assert abs(f["WVL_MF"].sum() - 1.0) < 1e-14
    k = f["WVL_KIN"]
    full = np.concatenate([k[:0:-1], k])
    l = np.arange(-14, 15)
    assert abs(full.sum()) < 1e-14                  # annihilates constants
    assert abs((full * l * l).sum() - 2.0) < 1e-12  # second derivative of x^2 / 2


def test_ana_after_syn_is_identity(oracle):
    rng = np.random.default_rng(3)
    for n, ndat in ((7, 5), (11, 3), (15, 2)):
        x = rng.uniform(-1, 1, (ndat, 2 * n + 2))
        y = oracle.syn_rot_per(n, ndat, x.ravel()).reshape(2 * n + 2, ndat).T.copy()
        z = oracle.ana_rot_per(n, ndat, y.ravel()).reshape(2 * n + 2, ndat).T
        assert np.abs(z - x).max() < 1e-15
    for N in (4, 9, 20):
        x = rng.uniform(-1, 1, (3, 2 * N))
        y = oracle.syn_grow_rot(N, 3, x.ravel()).reshape(2 * N + 14, 3).T.copy()
        z = oracle.ana_shrink_rot(N, 3, y.ravel()).reshape(2 * N, 3).T
        assert np.abs(z - x).max() < 1e-15


def test_magic_filter_adjoint(oracle):
    rng = np.random.default_rng(4)
    for L in (16, 23, 40):
        a, b = rng.uniform(-1, 1, L), rng.uniform(-1, 1, L)
        assert abs(oracle.convrot_n_per(L - 1, 1, a) @ b - a @ oracle.convrot_t_per(L - 1, 1, b)) < 1e-13
        bb = rng.uniform(-1, 1, L + 15)
        assert abs(oracle.mf_grow_rot(L, 1, a) @ bb - a @ oracle.mf_shrink_rot(L, 1, bb)) < 1e-13


def _ref_mf(oracle, fn, x, n, ndat):
    R = oracle.ref_magicfilter()
    y = np.zeros(n * ndat)
    getattr(R, fn)(C.byref(C.c_uint(n)), C.byref(C.c_uint(ndat)), np.ascontiguousarray(x), y)
    return y


def test_magic_filter_bit_exact_vs_reference_c(oracle):
    if oracle.ref_magicfilter() is None:
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    rng = np.random.default_rng(5)
    for n, ndat in ((16, 4), (24, 12), (64, 8)):
        x = rng.uniform(-1, 1, n * ndat)
        assert np.array_equal(oracle.convrot_n_per(n - 1, ndat, x), _ref_mf(oracle, "magicfilter1d_naive_", x, n, ndat))
        assert np.array_equal(oracle.convrot_t_per(n - 1, ndat, x), _ref_mf(oracle, "magicfilter1d_t_naive_", x, n, ndat))
        # the reference's SSE kernel sums in another order: agreement at rounding
        # level (its do-while loop assumes n > 16 and ndat a multiple of 4)
        if n > 16 and ndat % 4 == 0:
            sse = _ref_mf(oracle, "magicfilter1d_sse_", x, n, ndat)
            assert np.abs(oracle.convrot_n_per(n - 1, ndat, x) - sse).max() < 1e-15


def test_magic_filter_golden_vectors(oracle):
    g = np.load(GOLD / "magicfilter_ref.npz")
    for key in ("n", "t"):
        x, n, ndat, y = g["x_" + key], int(g["n"]), int(g["ndat"]), g["y_" + key]
        f = oracle.convrot_n_per if key == "n" else oracle.convrot_t_per
        assert np.array_equal(f(n - 1, ndat, x), y)


@pytest.mark.parametrize("per", [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
def test_fine_kinetic_matches_wavelet_basis_filters(oracle, per):
    rng = np.random.default_rng(6)
    N = (9, 8, 10)
    mc = np.ones(N[::-1], np.uint8)
    mf = np.zeros(N[::-1], np.uint8)
    mf[2:7, 1:6, 3:8] = 1
    d = oracle.desc_from_masks(mc, mf, per)
    pc, pf = rng.uniform(-1, 1, d.nvctr_c), rng.uniform(-1, 1, 7 * d.nvctr_f)
    h = (0.45, 0.5, 0.4)
    psig = oracle.uncompress(d, pc, pf)
    TX, ek = oracle.kinetic(d, [0.5 * v for v in h], oracle.synthese(d, psig))
    y1 = oracle.analyse(d, TX)
    y2, ek2 = oracle.kinetic_wavelet(d, h, psig)
    assert np.abs(y1 - y2).max() / np.abs(y1).max() < 1e-14
    assert abs(ek - ek2) / abs(ek) < 1e-14


def test_fortran_chain_matches_opencl_composition(oracle):
    rng = np.random.default_rng(7)
    N = (8, 9, 10)
    mc = np.ones(N[::-1], np.uint8)
    mf = np.zeros(N[::-1], np.uint8)
    mf[1:8, 2:6, 0:5] = 1
    d = oracle.desc_from_masks(mc, mf, (1, 1, 1))
    pc, pf = rng.uniform(-1, 1, d.nvctr_c), rng.uniform(-1, 1, 7 * d.nvctr_f)
    pot = rng.uniform(-2, 0, int(np.prod(d.I)))
    a = oracle.locham_per(d, (0.45, 0.45, 0.45), pc, pf, pot)
    b = oracle.locham(d, (0.45, 0.45, 0.45), pc, pf, pot)
    ref = np.concatenate([a[0], a[1]])
    got = np.concatenate([b[0], b[1]])
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-14
    assert abs(a[2] - b[2]) < 1e-12 * abs(a[2]) and abs(a[3] - b[3]) < 1e-12 * abs(a[3])


def test_compress_uncompress_roundtrip_bit_exact(oracle):
    rng = np.random.default_rng(8)
    N = (7, 6, 5)
    mc = rng.random(N[::-1]) < 0.7
    mf = mc & (rng.random(N[::-1]) < 0.5)
    d = oracle.desc_from_masks(mc.astype(np.uint8), mf.astype(np.uint8), (1, 1, 1))
    pc, pf = rng.uniform(-1, 1, d.nvctr_c), rng.uniform(-1, 1, 7 * d.nvctr_f)
    rc, rf = oracle.compress(d, oracle.uncompress(d, pc, pf))
    assert np.array_equal(rc, pc) and np.array_equal(rf, pf)


def test_gaussian_kinetic_energy_known_answer(oracle):
    # <f|-1/2 Lap|f>/<f|f> = 3/(4 s^2) for f = exp(-r^2/(2 s^2)); the wavelet
    # representation is built like the reference's libconv check
    # (tests/libs/wrappers/libconv.f90: isf_to_daub of an analytic function).
    s, n, h = 1.0, 32, 0.25   # box = 8 sigma: periodic images negligible
    d = oracle.desc_from_masks(np.ones((n,) * 3, np.uint8), np.ones((n,) * 3, np.uint8), (1, 1, 1))
    hf = 0.5 * h
    x = np.arange(2 * n) * hf
    c = n * h / 2
    g = np.exp(-(x - c) ** 2 / (2 * s * s))
    f = (g[:, None, None] * g[None, :, None] * g[None, None, :]).ravel()
    y = oracle.magic_t(d, f)                      # ISF values -> fine scaling coefficients
    psig = oracle.analyse(d, y)
    pc, pf = oracle.compress(d, psig)
    _, _, ekin, _ = oracle.locham(d, (h, h, h), pc, pf, np.zeros(int(np.prod(d.I))))
    norm = pc @ pc + pf @ pf
    assert abs(ekin / norm - 3 / (4 * s * s)) / (3 / (4 * s * s)) < 1e-6


def test_isf_weights_match_reference_lazy16():
    """The order-16 ISF two-scale filter the Poisson kernels use is computed
    from the 16-point Lagrange formula; it equals the reference's table
    (psolver/src/lazy_16.inc, ch(-18..18)) to its printed digits."""
    src = REFERENCE / "psolver" / "src" / "lazy_16.inc"
    if not src.exists():
        pytest.skip("reference tree not present")
    import re
    import oracle
    body = re.search(r"dimension\(-m:m\)\s*::\s*ch\s*=\s*\(/(.*?)/\)", src.read_text(), re.S).group(1)
    vals = [float(v.replace("D", "e").replace("d", "e")) for v in re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[dDeE][-+]?\d+)?",
                                                                            body.replace("&", " "))]
    assert len(vals) == 37
    ch = dict(zip(range(-18, 19), vals))
    w = oracle.isf_weights()
    assert ch[0] == 1.0
    for m in range(-18, 19):
        want = 1.0 if m == 0 else (w[abs(m)] if m % 2 and abs(m) <= 15 else 0.0)
        assert abs(ch[m] - want) <= 1e-17 + 1e-15 * abs(want)


def _ellipsoid(N, frac, shift=(0.0, 0.0, 0.0)):
    idx = np.meshgrid(*[np.arange(v) for v in N[::-1]], indexing="ij")
    r2 = np.zeros(N[::-1])
    for ax, n, s in zip(idx, N[::-1], shift[::-1]):
        r2 += ((ax - (n - 1) / 2.0 - s) / (frac * n)) ** 2
    return r2 <= 1.0


@pytest.mark.parametrize("N,fc,ff,cprecr", [((12, 10, 14), 0.6, 0.35, 0.0), ((16, 13, 11), 0.55, 0.3, 0.7)])
def test_wavelet_kinetic_matches_reference_sse(oracle, N, fc, ff, cprecr):
    """The oracle's wavelet-basis kinetic operator (the a, b, c, e filters of
    ConvolkineticT) against the reference's own SSE implementation of it,
    convolut_ib_sse.c (compiled where it lies into oracle/_ref), on a free
    region with irregular coarse and fine masks: coarse->coarse on a coarse
    input, fine->fine on a fine input, (c + T) x.  The reference computes in
    FP32: agreement to 2e-6 of the largest output."""
    if oracle.ref_convib() is None:
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    from wvlh.keys import Locreg, make_bounds
    mc = _ellipsoid(N, fc)
    mf = _ellipsoid(N, ff, (0.5, -0.5, 0.3)) & mc
    lr = Locreg.from_masks(mc, mf, (0, 0, 0), (0.45, 0.45, 0.45))
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    rng = np.random.default_rng(sum(N))
    # FP32-representable inputs, so both sides see the same numbers
    pc = rng.uniform(-1, 1, lr.nvctr_c).astype(np.float32).astype(np.float64)
    pf = rng.uniform(-1, 1, 7 * lr.nvctr_f).astype(np.float32).astype(np.float64)
    fz, fy, fx = np.nonzero(mf)
    nfl, nfu = (fx.min(), fy.min(), fz.min()), (fx.max(), fy.max(), fz.max())

    def ib(m):
        return [np.stack([b.lo, b.hi], axis=-1) for b in make_bounds(m)]

    def dense(c, f):
        """coarse (n3+1, n2+1, n1+1) and fine (.., .., .., 7) arrays from compressed values"""
        xc = np.zeros(N[::-1])
        xc[mc] = c                      # keys run x fastest, like C order of (i3, i2, i1)
        xf = np.zeros(N[::-1] + (7,))
        xf[mf] = f.reshape(-1, 7)
        return xc, xf[nfl[2]:nfu[2] + 1, nfl[1]:nfu[1] + 1, nfl[0]:nfu[0] + 1]

    n = tuple(v - 1 for v in N)
    h = lr.hgrid[0]
    zc, zf = np.zeros_like(pc), np.zeros_like(pf)
    for part in ("coarse", "fine"):
        c, f = (pc, zf) if part == "coarse" else (zc, pf)
        y, _ = oracle.kinetic_wavelet(d, lr.hgrid, oracle.uncompress(d, c, f))
        yc, yf = oracle.compress(d, y)
        xc, xf = dense(c, f)
        rc, rf = oracle.ref_kinetic_sse(n, h, cprecr, xc, xf, nfl, nfu, ib(mc), ib(mf))
        if part == "coarse":
            got, want = rc[mc], yc + cprecr * c
        else:
            full = np.zeros(N[::-1] + (7,), np.float32)
            full[nfl[2]:nfu[2] + 1, nfl[1]:nfu[1] + 1, nfl[0]:nfu[0] + 1] = rf
            got, want = full[mf].ravel(), yf + cprecr * f
        assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max(), part


def test_syn_ana_kinetic_match_reference_opencl_kernels(oracle):
    """The oracle's synthesis and analysis, periodic (syn_rot_per /
    ana_rot_per, convolut_simple_per.f90) and free (syn_grow_rot /
    ana_shrink_rot), its free-BC magic filters (mf_grow_rot / mf_shrink_rot)
    and its fine-grid kinetic filter (the x part of
    wo_kinetic_generic on a line) against the reference's OpenCL
    syn1dKernel_d / ana1dKernel_d / syngrow1dKernel_d / anashrink1dKernel_d /
    magicfiltergrow1dKernel_d / magicfiltershrink1dKernel_d / kinetic1dKernel_d
    arithmetic on the same
    lines (golden file), to FP64 rounding; with the reference tree present the
    golden file is re-derived first."""
    gold = np.load(GOLD / "opencl_kernels.npz")
    have_ref = (REFERENCE / "bigdft").exists()
    if have_ref:
        import importlib.util
        spec = importlib.util.spec_from_file_location("mk", GOLD / "make_opencl_kernels.py")
        mk = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mk)
        text = (REFERENCE / "bigdft/src/OpenCL/Wavelet_Generator.cpp").read_text()
        ana, (syn, start) = mk.ana_program(text), mk.syn_program(text)
        kin = mk.kin_program((REFERENCE / "bigdft/src/OpenCL/Kinetic_Generator.cpp").read_text())
        grow, gstart = mk.syn_program(text, "filter_grow(tmp1,tmp2)")
        mtext = (REFERENCE / "bigdft/src/OpenCL/MagicFilter_Generator.cpp").read_text()
        mf_fwd, mf_rev = mk.mf_program(mtext, "filter(tmp)"), mk.mf_program(mtext, "filter_reverse(tmp)")
    L = oracle.lib()
    for n in (8, 9, 13, 16, 24):
        x = gold["x_%d" % n]
        if have_ref:
            assert np.array_equal(mk.ana_line(ana, x), gold["ana_%d" % n])
            assert np.array_equal(mk.syn_line(syn, start, x), gold["syn_%d" % n])
            assert np.array_equal(mk.kin_line(kin, x), gold["kin_%d" % n])
            assert np.array_equal(mk.syngrow_line(grow, gstart, x), gold["grow_%d" % n])
            assert np.array_equal(mk.anashrink_line(ana, gold["yg_%d" % n]), gold["shrink_%d" % n])
            assert np.array_equal(mk.mfgrow_line(mf_fwd, x), gold["mfgrow_%d" % n])
            assert np.array_equal(mk.mfshrink_line(mf_rev, gold["ym_%d" % n]), gold["mfshrink_%d" % n])
        assert np.abs(oracle.ana_rot_per(n - 1, 1, x) - gold["ana_%d" % n]).max() < 1e-15
        assert np.abs(oracle.syn_rot_per(n - 1, 1, x) - gold["syn_%d" % n]).max() < 1e-15
        # free BC: n coarse points grow to 2n + 14 fine ones and shrink back
        assert np.abs(oracle.syn_grow_rot(n, 1, x) - gold["grow_%d" % n]).max() < 1e-15
        assert np.abs(oracle.ana_shrink_rot(n, 1, gold["yg_%d" % n]) - gold["shrink_%d" % n]).max() < 1e-15
        # free-BC magic filter: 2n fine points grow by 15 and shrink back
        assert np.abs(oracle.mf_grow_rot(2 * n, 1, x) - gold["mfgrow_%d" % n]).max() < 1e-15
        assert np.abs(oracle.mf_shrink_rot(2 * n, 1, gold["ym_%d" % n]) - gold["mfshrink_%d" % n]).max() < 1e-15
        # kinetic of a line of 2n points: a (2n, 1, 1) periodic box with unit
        # spacing adds -1/2 conv along x (the one-point y and z lines add 0)
        y, e = np.zeros(2 * n), C.c_double()
        L.wo_kinetic_generic(2 * n, 1, 1, np.ones(3, np.int32), np.ones(3), np.ascontiguousarray(x), y, C.byref(e))
        assert np.abs(-2.0 * y - gold["kin_%d" % n]).max() < 1e-14 * np.abs(gold["kin_%d" % n]).max()
