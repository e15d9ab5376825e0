"""CPU checks of the oracle's periodic Poisson solver (PSolver, periodic BC,
order-16 ISF): the ISF Fourier factors and the solution of an analytic
problem.  V = exp(cos x') exp(cos y') exp(cos z') (x' = 2 pi x / L) has the
analytic density rho = -lap V / (4 pi); the solver must return V minus its
mean (offset 0) to high order in h."""
import numpy as np
import pytest


def test_isf_fourier_factors(oracle):
    f = oracle.isf_fourier(32)
    assert f[0] == 1.0
    assert np.all(f > 0) and np.all(np.diff(f) <= 1e-15)     # smooth low-pass, monotone
    assert abs(f[1] - 1.0) < 1e-12                            # order 16: flat near 0
    assert 0.4 < f[32] < 0.6                                   # about 1/2 at the Nyquist frequency


def analytic(n, L):
    ax = [np.arange(m) * (L[i] / m) for i, m in enumerate(n)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    th = [2 * np.pi * x / L[0], 2 * np.pi * y / L[1], 2 * np.pi * z / L[2]]
    f = [np.exp(np.cos(t)) for t in th]
    d2 = [f[i] * (2 * np.pi / L[i]) ** 2 * (np.sin(th[i]) ** 2 - np.cos(th[i])) for i in range(3)]
    V = f[0] * f[1] * f[2]
    lap = d2[0] * f[1] * f[2] + f[0] * d2[1] * f[2] + f[0] * f[1] * d2[2]
    return V, -lap / (4 * np.pi)


def test_analytic_potential_high_order(oracle):
    """Errors fall with the order of the ISF family (16) as the grid refines:
    the oracle's normalisation (4 pi, 1/N, the ISF factors) is the physical one."""
    L = (10.0, 9.0, 8.0)
    errs = []
    for m in (32, 64):
        n = (m, m, m)
        V, rho = analytic(n, L)
        h = tuple(L[i] / n[i] for i in range(3))
        got, eh = oracle.psolver_periodic(rho, h)
        exact = V - V.mean()
        errs.append(np.abs(got - exact).max() / np.abs(exact).max())
        assert abs(eh - 0.5 * (rho * exact).sum() * np.prod(h)) <= 1e-7 * abs(eh)
    assert errs[0] < 1e-8 and errs[1] < 1e-12
    assert np.log2(errs[0] / errs[1]) > 12            # order of convergence


def test_uneven_grid_and_offset(oracle):
    L = (10.0, 9.0, 8.0)
    n = (48, 40, 36)
    V, rho = analytic(n, L)
    h = tuple(L[i] / n[i] for i in range(3))
    got, _ = oracle.psolver_periodic(rho, h)
    exact = V - V.mean()
    assert np.abs(got - exact).max() <= 1e-9 * np.abs(exact).max()
    # offset: the k = 0 term sets the mean of the potential to offset / volume
    got2, _ = oracle.psolver_periodic(rho, h, offset=3.0)
    assert abs(got2.mean() - 3.0 / np.prod(L)) <= 1e-12


def ps_check_periodic():
    """The periodic case of the reference's PS_Check test
    (psolver/tests/PS_Check.f90:29-113, test_functions_new with f_exp_cosine of
    frequency 2, psolver/tests/functions.f90:505-590, fill_functions_arrays
    :411-434; atlab/src/f_functions.f90:435-455, 591-665): a 64^3 box of side
    10 bohr, x = (i - 1) h - L/2, V = -4 pi f(x) f(y) f(z) with
    f = exp(cos(2 pi x / L)), rho = lap(f(x) f(y) f(z)), offset = sum(V) h^3.
    Arrays (z, y, x)."""
    n, L = 64, 10.0
    h = L / n
    x = np.arange(n) * h - 0.5 * L
    r = 2 * np.pi * x / L
    f = np.exp(np.cos(r))
    f2 = (2 * np.pi / L) ** 2 * (np.sin(r) ** 2 - np.cos(r)) * f
    rho = (f2[None, None, :] * f[None, :, None] * f[:, None, None] + f[None, None, :] * f2[None, :, None] * f[:, None, None]
           + f[None, None, :] * f[None, :, None] * f2[:, None, None])
    V = -4 * np.pi * f[None, None, :] * f[None, :, None] * f[:, None, None]
    return rho, V, (h, h, h), float(V.sum()) * h ** 3


# psolver/tests/PS_Check.ref.yaml:224-233 (periodic, 64^3): the Hartree energy,
# the largest difference from the analytic potential and the potential at
# (28, 28, 38), 1-based (x, y, z)
PS_CHECK_EH = 3.075484915324e04
PS_CHECK_INF = 9.890754881781e-12
PS_CHECK_V = -1.771130164828e02


def test_reference_ps_check_periodic_golden(oracle):
    rho, V, h, off = ps_check_periodic()
    pot, eh = oracle.psolver_periodic(rho, h, offset=off)
    assert abs(eh - PS_CHECK_EH) <= 5e-13 * PS_CHECK_EH      # all 13 printed digits
    assert abs(pot[37, 27, 27] - PS_CHECK_V) <= 5e-13 * abs(PS_CHECK_V)
    assert np.abs(pot - V).max() <= 2 * PS_CHECK_INF          # the same accuracy as the reference's run


def xc_test_density(n=100000):
    """The density of the reference's XC test (bigdft/tests/libs/xc/test_xc.f90:
    gauss, :187-215, spin-unpolarised, ABINIT kind): 1e-20 everywhere
    (xc_init_rho), a Gaussian over points 5..n-5, the 1e-20 floor
    (xc_clean_rho), normalised by the sum of the first n values.  xc_getvxc
    with nspden = 1 takes rho as the spin-up density: the total is 2 rho."""
    rho = np.full(2 * n, 1e-20)
    sigma = 1.0 / (n * 0.25)
    j = np.arange(5, n - 5 + 1)
    rho[j - 1] = np.exp(-((sigma * (n // 2 - j)) ** 2)) / n
    rho[j - 1 + n] = rho[j - 1]
    rho[rho < 1e-20] = 1e-20
    return rho[:n] / rho[:n].sum()


# bigdft/tests/libs/xc/xc.ref.yaml:2 (ixc 1, nosp): the sum of eps_xc over the test density
XC_REF_IXC1_NOSP = -2766.214885143616


def test_reference_xc_golden(oracle):
    eps, _ = oracle.xc_lda(2.0 * xc_test_density())
    assert abs(eps.sum() - XC_REF_IXC1_NOSP) <= 1e-12 * abs(XC_REF_IXC1_NOSP)


def test_xc_potential_is_the_density_derivative(oracle):
    """v_xc = d(rho eps_xc)/d rho (central differences, relative step 1e-5)."""
    rho = np.geomspace(1e-8, 1e2, 61)
    eps, v = oracle.xc_lda(rho)
    d = 1e-5 * rho
    ep, _ = oracle.xc_lda(rho + d)
    em, _ = oracle.xc_lda(rho - d)
    fd = ((rho + d) * ep - (rho - d) * em) / (2 * d)
    assert np.abs(fd - v).max() <= 1e-8 * np.abs(v).max()
    assert np.all(eps < 0) and np.all(v < eps)      # bound, and v_xc = eps + rho d eps/d rho < eps


def test_xc_high_density_limit_is_slater_exchange(oracle):
    """As rs -> 0 the fit tends to the exchange energy -(3/4)(3/(2 pi))^(2/3) / rs
    (a0 of the fit) and v_xc to 4/3 of it."""
    rs = 1e-6
    rho = 3.0 / (4 * np.pi * rs ** 3)
    eps, v = oracle.xc_lda(np.array([rho]))
    ex = -0.75 * (3 / (2 * np.pi)) ** (2.0 / 3.0) / rs
    assert abs(eps[0] / ex - 1) < 1e-5 and abs(v[0] / (4.0 / 3.0 * ex) - 1) < 1e-5


def test_ks_potential_is_the_sum_of_its_parts(oracle):
    rng = np.random.default_rng(3)
    n = (32, 24, 20)
    h = (0.3, 0.35, 0.4)
    rho = rng.uniform(1e-3, 1.0, n)
    vext = rng.uniform(-1, 1, n)
    pot, (eh, exc, evxc) = oracle.ks_potential_periodic(rho, h, vext)
    vh, eh0 = oracle.psolver_periodic(rho, h)
    eps, vxc = oracle.xc_lda(rho)
    assert np.array_equal(pot, (vh + vext) + vxc) and eh == eh0
    dv = np.prod(h)
    assert abs(exc - (eps * rho).sum() * dv) <= 1e-12 * abs(exc)
    assert abs(evxc - (vxc * rho).sum() * dv) <= 1e-12 * abs(evxc)


def ps_check_free():
    """The free-BC case of the reference's PS_Check test (psolver/tests/
    PS_Check.f90:29-113; test_functions_new case 'F', functions.f90:552-563):
    a 57 x 48 x 63 box of side 10 bohr per dimension, x = (i - 1) h - L/2, a
    unit Gaussian rho = exp(-r^2) / pi^(3/2) (a_gauss = 1) and its analytic
    potential erf(r) / r.  Arrays (z, y, x)."""
    from math import erf
    n = (57, 48, 63)
    h = tuple(10.0 / m for m in n)
    ax = [np.arange(n[d]) * h[d] - 0.5 * n[d] * h[d] for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    r2 = x * x + y * y + z * z
    r = np.sqrt(r2)
    rho = np.exp(-r2) / (np.pi * np.sqrt(np.pi))
    verf = np.vectorize(erf)
    V = np.where(r > 1e-15, verf(r) / np.where(r > 0, r, 1.0), 2.0 / np.sqrt(np.pi))
    return rho, V, h


# psolver/tests/PS_Check.ref.yaml:46-56 (free BC, 57 x 48 x 63): the Hartree
# energy, the largest difference from the analytic potential, where it lies
# (1-based x, y, z) and the potential there
PS_FREE_EH = 3.989422803962e-01
PS_FREE_INF = 3.365174805481e-10
PS_FREE_AT = (30, 25, 33)
PS_FREE_V = 1.123137867733e00


def test_isf_cascade_samples(oracle):
    """The cascade reproduces the interpolating scaling function: phi(k) =
    delta_k at the integers, phi(1/2) = w_1, unit integral, support [-15, 15]."""
    x, y = oracle.isf_samples()
    assert len(x) == 513 and x[0] == -15.0 and x[-1] == 17.0
    ints = (x == np.round(x))
    assert np.array_equal(y[ints], (x[ints] == 0).astype(float))
    assert y[15 * 16 + 8] == oracle.isf_weights()[1]
    assert abs(y.sum() / 16 - 1.0) < 1e-14
    assert np.all(y[x > 15] == 0)


def test_reference_ps_check_free_golden(oracle):
    rho, V, h = ps_check_free()
    pot, eh = oracle.psolver_free(rho, h)
    assert abs(eh - PS_FREE_EH) <= 5e-13 * PS_FREE_EH                   # all 13 printed digits
    i1, i2, i3 = (v - 1 for v in PS_FREE_AT)
    assert abs(pot[i3, i2, i1] - PS_FREE_V) <= 5e-13 * PS_FREE_V
    d = np.abs(pot - V)
    assert abs(d.max() - PS_FREE_INF) <= 1e-3 * PS_FREE_INF            # the same deviation ...
    assert np.unravel_index(d.argmax(), d.shape) == (i3, i2, i1)        # ... at the same point


def test_free_solution_independent_of_padding(oracle):
    """The zero-padded convolution is exact for any FFT length >= twice the
    box: the reference's FFT sizes (fourier_dim) and the doubled box agree."""
    rng = np.random.default_rng(7)
    rho = rng.uniform(0, 1, (12, 10, 9))
    h = (0.3, 0.25, 0.2)
    a, ea = oracle.psolver_free(rho, h)
    b, eb = oracle.psolver_free(rho, h, nfft=(24, 24, 30))
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max() and abs(ea - eb) <= 1e-13 * abs(ea)


def test_free_kernel_host_tables_match_oracle(oracle):
    """The library's host construction of the free kernel (no device work)
    equals the oracle's Free_Kernel restatement."""
    from wvlh.psolver import free_kernel_tables
    n = (57, 48, 63)
    h = tuple(10.0 / m for m in n)
    nf, rows, w = free_kernel_tables(n, h)
    assert all(v >= 2 * m and v % 2 == 0 for v, m in zip(nf, n))
    l1, l2, l3 = nf[0] // 2 + 1, nf[1] // 2 + 1, nf[2] // 2 + 1
    K = np.zeros((l3, l2, l1))
    for g in range(88, -1, -1):
        cx, cy, cz = rows[g, :l1], rows[g, l1:l1 + l2], rows[g, l1 + l2:]
        K += cx[None, None, :] * (cz[:, None, None] * (cy[None, :, None] * w[g]))
    ref = oracle.free_kernel(n, h, nf)
    assert np.abs(K - ref).max() <= 1e-13 * np.abs(ref).max()


def xc_test_density_spin(n=100000, delta=500):
    """The spin densities of the reference's XC test with nspin = 2
    (test_xc.f90:gauss): spin-up and spin-down Gaussians over points
    5..n-5, centred delta points either side of n/2, the 1e-20 floor, the
    pair normalised to one.  The value xc.ref.yaml prints for ixc 1 (scol)
    is reproduced with delta = 500 (n/200); the test program as committed
    has the offset line commented out (delta = 0, which gives -2239.706)."""
    rho = np.full(2 * n, 1e-20)
    sigma = 1.0 / (n * 0.25)
    j = np.arange(5, n - 5 + 1)
    rho[j - 1] = np.exp(-((sigma * (n // 2 - j + delta)) ** 2)) / 2 / n
    rho[j - 1 + n] = np.exp(-((sigma * (n // 2 - j - delta)) ** 2)) / 2 / n
    rho[rho < 1e-20] = 1e-20
    rho = rho / rho.sum()
    return rho[:n], rho[n:]


# bigdft/tests/libs/xc/xc.ref.yaml:2 (ixc 1, scol): sum of eps_xc, spin-polarised
XC_REF_IXC1_SCOL = -2240.035817927920


def test_reference_xc_spin_golden(oracle):
    up, dn = xc_test_density_spin()
    eps, _, _ = oracle.xc_lsda(up, dn)
    assert abs(eps.sum() - XC_REF_IXC1_SCOL) <= 1e-12 * abs(XC_REF_IXC1_SCOL)
    z = 2 * up / (up + dn) - 1
    assert z.min() < -0.05 and z.max() > 0.05        # a polarised density: the spin terms count


def test_lsda_unpolarised_limit_is_the_lda(oracle):
    rho = np.geomspace(1e-8, 1e2, 41)
    eps, vu, vd = oracle.xc_lsda(rho / 2, rho / 2)
    e0, v0 = oracle.xc_lda(rho)
    assert np.array_equal(eps, e0) and np.array_equal(vu, v0) and np.array_equal(vd, v0)


def test_lsda_potentials_are_the_spin_derivatives(oracle):
    """v_sigma = d(rho eps)/d rho_sigma (central differences, step 1e-6 rho)."""
    rng = np.random.default_rng(2)
    up = rng.uniform(1e-4, 1.0, 50)
    dn = rng.uniform(1e-4, 1.0, 50)
    eps, vu, vd = oracle.xc_lsda(up, dn)

    def E(u, d):
        return (u + d) * oracle.xc_lsda(u, d)[0]
    hu, hd = 1e-6 * up, 1e-6 * dn
    fu = (E(up + hu, dn) - E(up - hu, dn)) / (2 * hu)
    fd = (E(up, dn + hd) - E(up, dn - hd)) / (2 * hd)
    assert np.abs(fu - vu).max() <= 1e-7 * np.abs(vu).max()
    assert np.abs(fd - vd).max() <= 1e-7 * np.abs(vd).max()


def test_lsda_ferromagnetic_exchange_limit(oracle):
    """Fully polarised at high density: exchange scales by 2^(1/3)."""
    rs = 1e-6
    rho = 3.0 / (4 * np.pi * rs ** 3)
    e1, _, _ = oracle.xc_lsda(np.array([rho]), np.array([rho * 1e-12]))
    e0, _ = oracle.xc_lda(np.array([rho]))
    assert abs(e1[0] / e0[0] - 2 ** (1.0 / 3.0)) < 1e-4


def test_ks_potential_spin_is_the_sum_of_its_parts(oracle):
    rng = np.random.default_rng(4)
    n = (24, 20, 16)
    h = (0.3, 0.35, 0.4)
    up = rng.uniform(1e-3, 1.0, n)
    dn = rng.uniform(1e-3, 1.0, n)
    vext = rng.uniform(-1, 1, n)
    pu, pd, (eh, exc, evxc) = oracle.ks_potential_spin(up, dn, h, vext)
    vh, eh0 = oracle.psolver_periodic(up + dn, h)
    eps, vu, vd = oracle.xc_lsda(up, dn)
    assert np.array_equal(pu, (vh + vext) + vu) and np.array_equal(pd, (vh + vext) + vd) and eh == eh0
    dv = np.prod(h)
    assert abs(evxc - (vu * up + vd * dn).sum() * dv) <= 1e-12 * abs(evxc)


def ps_check_surface():
    """The surface-BC case of the reference's PS_Check test (x and z
    periodic, y free; test_functions_new case 'S', functions.f90:541-546,
    f_functions.f90:395-486): a 32 x 64 x 48 box of side 10 bohr per
    dimension, x = (i - 1) h - L/2, f = exp(cos(2 pi x / L)) along x and z, the
    shrunk Gaussian exp(-tan(pi y / L)^2) exp(-50 y^2 / L^2) along y,
    V = -f(x) f(y) f(z) and rho = lap(f f f) / (4 pi).  Arrays (z, y, x)."""
    n = (32, 64, 48)
    h = tuple(10.0 / m for m in n)
    ax = [np.arange(n[d]) * h[d] - 0.5 * n[d] * h[d] for d in range(3)]

    def expcos(x, L):
        r = 2 * np.pi * x / L
        f = np.exp(np.cos(r))
        return f, (2 * np.pi / L) ** 2 * (np.sin(r) ** 2 - np.cos(r)) * f

    def shrunk(x, L):
        r = np.pi * x / L
        y = np.tan(r)
        g = np.exp(-y ** 2)
        g1 = -2 * np.pi * g * y / (L * np.cos(r) ** 2)
        g2 = 2 * np.pi ** 2 * (2 * y ** 6 + y ** 4 - 2 * y ** 2 - 1) / L ** 2 * g
        a = 50.0 / L ** 2
        e = np.exp(-a * x * x)
        return g * e, g2 * e + g * (-2 * a + 4 * a * a * x * x) * e + 2 * g1 * (-2 * a * x * e)
    fx, fx2 = expcos(ax[0], 10.0)
    fy, fy2 = shrunk(ax[1], 10.0)
    fz, fz2 = expcos(ax[2], 10.0)

    def prod(a, b, c):
        return a[None, None, :] * b[None, :, None] * c[:, None, None]
    rho = (prod(fx2, fy, fz) + prod(fx, fy2, fz) + prod(fx, fy, fz2)) / (4 * np.pi)
    return rho, -prod(fx, fy, fz), h


# psolver/tests/PS_Check.ref.yaml:398-406 (surface BC, 32 x 64 x 48): the
# Hartree energy, the largest deviation from the analytic potential, where it
# lies (1-based x, y, z) and the potential there
PS_SURF_EH = 2.969431884210e01
PS_SURF_INF = 5.449589889578e-10
PS_SURF_AT = (17, 58, 25)
PS_SURF_V = -1.455736584652e-06


def test_reference_ps_check_surface_golden(oracle):
    rho, V, h = ps_check_surface()
    pot, eh = oracle.psolver_surface(rho, h)
    assert abs(eh - PS_SURF_EH) <= 5e-13 * PS_SURF_EH                    # all 13 printed digits
    i1, i2, i3 = (v - 1 for v in PS_SURF_AT)
    assert abs(pot[i3, i2, i1] - PS_SURF_V) <= 1e-14                      # the potential is O(1)
    d = np.abs(pot - V)
    assert abs(d.max() - PS_SURF_INF) <= 1e-4 * PS_SURF_INF
    # the deviation peaks at the reference's point or its mirror in y (the test is symmetric in y)
    j3, j2, j1 = np.unravel_index(d.argmax(), d.shape)
    assert (j3, j1) == (i3, i1) and j2 in (i2, rho.shape[1] - i2)


def test_surface_green_functions(oracle):
    """The 1D Green's functions tend to their continuum forms away from the
    ISF support: exp(-mu j) * (integral of phi e^(mu x)) and |j|."""
    g = oracle.green_surface(40, 0.3)
    assert np.all(np.diff(g[20:]) < 0) and abs(g[30] / g[29] - np.exp(-0.3)) < 1e-12
    g0 = oracle.green_surface_mu0(40)
    assert np.abs(np.diff(g0[20:]) - 1.0).max() < 1e-12        # slope 1 outside the support


def test_surface_solution_independent_of_padding(oracle):
    rng = np.random.default_rng(9)
    rho = rng.uniform(0, 1, (8, 10, 12))
    h = (0.3, 0.25, 0.35)
    a, ea = oracle.psolver_surface(rho, h)
    b, eb = oracle.psolver_surface(rho, h, N2=26)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max() and abs(ea - eb) <= 1e-13 * abs(ea)


def test_surface_kernel_host_table_matches_oracle(oracle):
    from wvlh.psolver import surface_kernel_table
    n = (10, 12, 8)
    h = (0.3, 0.35, 0.4)
    N2, K = surface_kernel_table(n, h)
    assert N2 >= 2 * n[1] and N2 % 2 == 0
    ref = oracle.surface_kernel(n, h, N2)
    assert np.abs(K - ref).max() <= 1e-13 * np.abs(ref).max()


def ps_check_wire():
    """The wire-BC case of the reference's PS_Check test (z periodic, x and
    y free; fill_functions_arrays_wires, psolver/tests/functions.f90:437-467):
    a 51 x 55 x 64 box of side 10 bohr per dimension, rho = exp(-2 (x^2 + y^2))
    on centred coordinates.  Arrays (z, y, x)."""
    n = (51, 55, 64)
    h = tuple(10.0 / m for m in n)
    x = np.arange(n[0]) * h[0] - 0.5 * n[0] * h[0]
    y = np.arange(n[1]) * h[1] - 0.5 * n[1] * h[1]
    r2 = x[None, None, :] ** 2 + y[None, :, None] ** 2
    return np.broadcast_to(np.exp(-2.0 * r2), (n[2], n[1], n[0])).copy(), h


# psolver/tests/PS_Check.ref.yaml:569-578 (wire BC, 51 x 55 x 64): the Hartree
# energy and the potential at (26, 28, 1), 1-based (x, y, z)
PS_WIRE_EH = 7.121112829810e00
PS_WIRE_AT = (26, 28, 1)
PS_WIRE_V = 1.939819652123e00


def test_reference_ps_check_wire_golden(oracle):
    rho, h = ps_check_wire()
    pot, eh = oracle.psolver_wire(rho, h)
    assert abs(eh - PS_WIRE_EH) <= 5e-13 * PS_WIRE_EH                    # all 13 printed digits
    i1, i2, i3 = (v - 1 for v in PS_WIRE_AT)
    assert abs(pot[i3, i2, i1] - PS_WIRE_V) <= 5e-13 * PS_WIRE_V


def test_wire_kernel_host_table_matches_oracle(oracle):
    from wvlh.psolver import wire_kernel_table
    n = (10, 12, 8)
    h = (0.3, 0.35, 0.4)
    (Nx, Ny), K = wire_kernel_table(n, h)
    assert Nx >= 2 * n[0] and Ny >= 2 * n[1]
    ref = oracle.wire_kernel(n, h, Nx, Ny)
    assert np.abs(K - ref).max() <= 1e-12 * np.abs(ref).max()


def test_kernel_table_entry_points_reject_bad_grids():
    """The host-only table builders validate their arguments like the device
    entry points: at least 2 points per dimension, positive spacings."""
    from wvlh._lib import WvlhError
    from wvlh.psolver import free_kernel_tables, surface_kernel_table, wire_kernel_table
    for fn in (free_kernel_tables, surface_kernel_table, wire_kernel_table):
        with pytest.raises(WvlhError):
            fn((1, 8, 8), (0.3, 0.3, 0.3))
        with pytest.raises(WvlhError):
            fn((8, 8, 8), (0.3, 0.0, 0.3))


@pytest.mark.parametrize("n", [(11, 10, 9), (9, 13, 7)])
def test_odd_periodic_sizes_host_tables_match_oracle(oracle, n):
    """Odd lengths along the periodic axes (x and z for surfaces, z for
    wires): the half-spectrum and folded frequencies stay consistent."""
    from wvlh.psolver import surface_kernel_table, wire_kernel_table
    h = (0.31, 0.27, 0.35)
    N2, K = surface_kernel_table(n, h)
    ref = oracle.surface_kernel(n, h, N2)
    assert np.abs(K - ref).max() <= 1e-13 * np.abs(ref).max()
    (Nx, Ny), K = wire_kernel_table(n, h)
    ref = oracle.wire_kernel(n, h, Nx, Ny)
    assert np.abs(K - ref).max() <= 1e-12 * np.abs(ref).max()


def test_core_density_enters_xc_only(oracle):
    """The nonlinear core correction: V_xc and E_xc see rho + rho_core, V_H
    and int rho V_xc the valence density alone (XC_potential with rhocore,
    substract_from_vexcu)."""
    rng = np.random.default_rng(6)
    n, h = (20, 16, 18), (0.3, 0.35, 0.32)
    rho = rng.uniform(1e-3, 0.5, n)
    core = rng.uniform(0.0, 0.3, n)
    pot, (eh, exc, evxc) = oracle.ks_potential_periodic(rho, h, rhocore=core)
    vh, eh0 = oracle.psolver_periodic(rho, h)
    eps, vxc = oracle.xc_lda(rho + core)
    dv = np.prod(h)
    assert np.array_equal(pot, vh + vxc) and eh == eh0
    assert abs(exc - (eps * (rho + core)).sum() * dv) <= 1e-12 * abs(exc)
    assert abs(evxc - (vxc * rho).sum() * dv) <= 1e-12 * abs(evxc)
    # spin-unpolarised limit of the spin variant with the core split evenly
    pu, pd, (eh2, exc2, evxc2) = oracle.ks_potential_spin(rho / 2, rho / 2, h, rhocore=core)
    assert np.abs(pu - pot).max() <= 1e-13 * np.abs(pot).max() and np.array_equal(pu, pd)
    assert abs(exc2 - exc) <= 1e-12 * abs(exc) and abs(evxc2 - evxc) <= 1e-12 * abs(evxc)
