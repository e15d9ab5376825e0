"""GPU parity of the periodic Poisson solver (wvlh_psolver_periodic: cuFFT and
the library's ISF kernel multiply) with the oracle's numpy restatement of the
reference's periodic PSolver: potential within 1e-13 of its magnitude, the
Hartree energy within 1e-12, on random and analytic densities."""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.psolver import hartree_periodic

from test_psolver_rule import analytic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,h", [((32, 32, 32), (0.3, 0.3, 0.3)), ((48, 40, 36), (0.21, 0.25, 0.27)),
                                 ((96, 96, 96), (0.225, 0.225, 0.225))])
def test_matches_oracle_random_density(oracle, torch_cuda, wctx, n, h):
    torch = torch_cuda
    rng = np.random.default_rng(n[0])
    rho = rng.uniform(-1, 1, n[::-1])
    ref, eref = oracle.psolver_periodic(rho, h, offset=0.5)
    pot, eh = hartree_periodic(wctx, torch.tensor(rho, device="cuda"), h, offset=0.5)
    got = pot.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(eh.item() - eref) <= 1e-12 * abs(eref)


def test_analytic_and_in_place(oracle, torch_cuda, wctx):
    torch = torch_cuda
    L = (10.0, 9.0, 8.0)
    n = (64, 64, 64)
    V, rho = analytic(n, L)
    h = tuple(L[i] / n[i] for i in range(3))
    t = torch.tensor(rho, device="cuda")
    pot, eh = hartree_periodic(wctx, t, h)
    exact = V - V.mean()
    assert np.abs(pot.cpu().numpy() - exact).max() <= 1e-12 * np.abs(exact).max()
    # deterministic
    pot2, eh2 = hartree_periodic(wctx, t, h)
    assert torch.equal(pot, pot2) and torch.equal(eh, eh2)
    # in place without the energy; refused with it
    with pytest.raises(WvlhError):
        hartree_periodic(wctx, t, h, pot=t, energy=True)
    hartree_periodic(wctx, t, h, pot=t, energy=False)
    assert torch.equal(t, pot)


def test_rejects_odd_or_small_grids(torch_cuda, wctx):
    torch = torch_cuda
    for shape in ((16, 16, 15), (8, 16, 16)):
        with pytest.raises(WvlhError):
            hartree_periodic(wctx, torch.zeros(shape, dtype=torch.float64, device="cuda"), (0.3, 0.3, 0.3))
