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
