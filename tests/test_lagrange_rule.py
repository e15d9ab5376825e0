"""CPU checks of the Lagrange-multiplier step (orthoconstraint,
wfn_opt/orthogonality.f90:375-625): the oracle's loop restatement of
lagrange_multiplier (:293-369) against the closed form the library uses
(symmetrise, then scale couplings between unequal occupations), and the
properties of the constrained gradient."""
import numpy as np
import pytest
import torch

from wvlh.ortho import lagrange_multiplier


@pytest.mark.parametrize("seed,occ", [(0, "equal"), (1, "mixed"), (2, "small"), (3, "equal")])
def test_closed_form_matches_reference_loop(oracle, seed, occ):
    rng = np.random.default_rng(seed)
    n = 9
    lam = rng.uniform(-1, 1, (n, n))
    f = {"equal": np.full(n, 2.0), "mixed": rng.choice([2.0, 1.0, 0.0], n),
         "small": rng.choice([2.0, 0.3, 0.0], n)}[occ]
    for symm in (True, False):
        for corr in (True, False):
            ref = lam.copy()
            r = oracle.lagrange_multiplier(ref, f, symm, corr)
            got = torch.tensor(lam)
            g = lagrange_multiplier(got, f, symm=symm, correction=corr)
            assert np.allclose(got.numpy(), ref, rtol=0, atol=1e-15)
            assert np.allclose(g, r, rtol=1e-15, atol=1e-15)


def test_constrained_gradient_orthogonal_to_orbitals(oracle):
    rng = np.random.default_rng(4)
    norb, K = 6, 200
    q, _ = np.linalg.qr(rng.standard_normal((K, norb)))
    psi = q.T                                  # orthonormal rows
    A = rng.standard_normal((K, K))
    hpsi = psi @ (A + A.T)                     # H psi for a symmetric H
    g, lam, tr, asy, mix = oracle.orthoconstraint(psi, hpsi, np.full(norb, 2.0))
    # equal occupations and symmetric H: the gradient is orthogonal to every orbital
    assert np.abs(psi @ g.T).max() <= 1e-10
    assert asy <= 1e-20 and mix == 0.0
    assert abs(tr - np.trace(psi @ hpsi.T)) <= 1e-10
