"""CPU checks of the oracle's nonlocal projector application (the reference's
NonLocalHamiltonianApplication, hpsiortho.f90:1044-1125): scalar products and
updates through the masks of common segments (locregs/scalar_product.f90:
953-1187), h applied per atom, eproj = sum c.hc.

* Projectors inside a convex wavefunction region: the masks are the plain
  common grid points, so c, the update and eproj equal dense-grid algebra.
* For symmetric h the operator is symmetric and eproj = <psi|V_nl psi>.
* hgh_matrix lays the HGH blocks out in the reference's projector order.
"""
import numpy as np
import pytest

from wvlh.keys import segkeys

from test_wpdot_rule import dense


def sphere(N, c, r):
    z, y, x = np.meshgrid(*[np.arange(n) for n in N[::-1]], indexing="ij")
    return (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r


def case(rng, N, natoms, m=4):
    """psi on the full box (coarse) with a fine ellipsoid; projectors on balls."""
    full = np.ones(N[::-1], bool)
    fine = sphere(N, [n / 2 for n in N], min(N) * 0.4)
    kw = segkeys(full) + segkeys(fine)
    atoms = []
    for _ in range(natoms):
        c = rng.uniform(2, np.array(N) - 2)
        pc = sphere(N, c, rng.uniform(2, 4))
        pf = pc & sphere(N, c, 1.8)
        kp = segkeys(pc) + segkeys(pf)
        proj = rng.uniform(-1, 1, (m, int(pc.sum() + 7 * pf.sum())))
        h = rng.uniform(-1, 1, (m, m))
        atoms.append((kp, proj, h + h.T))
    psi = rng.uniform(-1, 1, (2, int(full.sum() + 7 * fine.sum())))
    return kw, psi, atoms, fine


@pytest.mark.parametrize("seed", range(4))
def test_projectors_inside_region_are_dense_algebra(oracle, seed):
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(9, 14, 3))
    kw, psi, atoms, fine = case(rng, N, 3)
    out, ep = oracle.nlpsp_apply(kw, psi, atoms)
    for o in range(psi.shape[0]):
        wc, wf = dense(kw, psi[o], N)
        dc, df = np.zeros_like(wc), np.zeros_like(wf)
        e = 0.0
        for kp, proj, h in atoms:
            P = [dense(kp, p, N) for p in proj]
            c = np.array([(pc * wc).sum() + (pf * wf).sum() for pc, pf in P])
            hc = h @ c
            e += c @ hc
            for (pc, pf), s in zip(P, hc):
                dc += s * pc
                df += s * pf
        gc, gf = dense(kw, out[o], N)
        # the update lands on the wavefunction's points only
        assert np.abs(gc - dc).max() <= 1e-12 and np.abs(gf - df * fine[..., None]).max() <= 1e-12
        assert abs(ep[o] - e) <= 1e-11 * max(1.0, abs(e))


def test_symmetric_operator_and_energy_identity(oracle):
    rng = np.random.default_rng(7)
    N = (11, 10, 12)
    kw, psi, atoms, _ = case(rng, N, 4)
    out, ep = oracle.nlpsp_apply(kw, psi, atoms)
    # eproj = <psi | V_nl psi> (the update and the energy use the same c and h)
    for o in range(2):
        assert abs(ep[o] - psi[o] @ out[o]) <= 1e-11 * max(1.0, abs(ep[o]))
    # <phi | V psi> = <V phi | psi> for symmetric h
    assert abs(psi[0] @ out[1] - out[0] @ psi[1]) <= 1e-11 * max(1.0, abs(psi[0] @ out[1]))


def test_projector_partly_outside_region_sees_common_points_only(oracle):
    rng = np.random.default_rng(3)
    N = (12, 12, 12)
    ball = sphere(N, (6, 6, 6), 4.5)           # convex wavefunction region
    kw = segkeys(ball) + segkeys(np.zeros(N, bool))
    pc = sphere(N, (9.5, 6, 6), 3.0)           # straddles the region's edge
    kp = segkeys(pc) + segkeys(np.zeros(N, bool))
    proj = rng.uniform(-1, 1, (1, int(pc.sum())))
    psi = rng.uniform(-1, 1, (1, int(ball.sum())))
    out, ep = oracle.nlpsp_apply(kw, psi, [(kp, proj, np.array([[2.0]]))])
    wc, _ = dense(kw, psi[0], N)
    pcd, _ = dense(kp, proj[0], N)
    c = (wc * pcd).sum()
    gc, _ = dense(kw, out[0], N)
    assert np.abs(gc - 2.0 * c * pcd * ball).max() <= 1e-12
    assert abs(ep[0] - 2.0 * c * c) <= 1e-11 * max(1.0, 2 * c * c)


def test_hgh_matrix_order():
    from wvlh.nlpsp import hgh_matrix
    hij = np.zeros((4, 3, 3))
    hij[0] = [[1.0, 0.5, 0.0], [0.5, 2.0, 0.0], [0.0, 0.0, 0.0]]   # s: two projectors
    hij[1] = [[3.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]]   # p: one radial, 3 m
    present = [[True, True, False], [True, False, False], [False] * 3, [False] * 3]
    h = hgh_matrix(hij, present)
    assert h.shape == (5, 5)
    assert np.allclose(h[:2, :2], [[1.0, 0.5], [0.5, 2.0]])
    assert np.allclose(h[2:, 2:], 3.0 * np.eye(3))
    assert np.allclose(h[:2, 2:], 0.0)
