"""GPU parity of the periodic Poisson solver (wvlh_psolver_periodic: cuFFT and
the library's ISF kernel multiply) with the oracle's numpy restatement of the
reference's periodic PSolver: potential within 1e-13 of its magnitude, the
Hartree energy within 1e-12, on random and analytic densities; grid lengths
with prime factors 2, 3, 5, 7 and 11 and a long axis of 250 points."""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.psolver import hartree_periodic

from test_psolver_rule import analytic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,h", [((32, 32, 32), (0.3, 0.3, 0.3)), ((48, 40, 36), (0.21, 0.25, 0.27)),
                                 ((96, 96, 96), (0.225, 0.225, 0.225)),
                                 ((50, 30, 20), (0.3, 0.28, 0.26)),      # factors 5 and 3
                                 ((250, 16, 18), (0.1, 0.3, 0.3)),       # a long axis
                                 ((28, 42, 22), (0.3, 0.3, 0.3))])       # factors 7 and 11
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


def test_reference_ps_check_periodic_golden(torch_cuda, wctx):
    """The reference's own PS_Check periodic run (64^3, exp-cosine density):
    the Hartree energy and the potential at (28, 28, 38) to its 13 printed
    digits, the analytic potential to the reference's accuracy."""
    from test_psolver_rule import PS_CHECK_EH, PS_CHECK_INF, PS_CHECK_V, ps_check_periodic
    torch = torch_cuda
    rho, V, h, off = ps_check_periodic()
    pot, eh = hartree_periodic(wctx, torch.tensor(rho, device="cuda"), h, offset=off)
    got = pot.cpu().numpy()
    assert abs(eh.item() - PS_CHECK_EH) <= 5e-13 * PS_CHECK_EH
    assert abs(got[37, 27, 27] - PS_CHECK_V) <= 5e-13 * abs(PS_CHECK_V)
    assert np.abs(got - V).max() <= 2 * PS_CHECK_INF


def test_xc_lda_matches_oracle_on_reference_test_density(oracle, torch_cuda, wctx):
    from test_psolver_rule import xc_test_density
    from wvlh.psolver import xc_lda
    torch = torch_cuda
    rho = 2.0 * xc_test_density()
    eps, v = oracle.xc_lda(rho)
    t = torch.tensor(rho, device="cuda")
    vxc, en = xc_lda(wctx, t, dvol=1.0)
    got = vxc.cpu().numpy()
    assert np.abs(got - v).max() <= 1e-14 * np.abs(v).max()
    e = en.cpu().numpy()
    assert abs(e[0] - (eps * rho).sum()) <= 1e-13 * abs(e[0])
    assert abs(e[1] - (v * rho).sum()) <= 1e-13 * abs(e[1])
    # accumulate, and in place
    acc = torch.full_like(t, 0.25)
    xc_lda(wctx, t, vxc=acc, accumulate=True, energy=False)
    assert np.abs(acc.cpu().numpy() - (0.25 + v)).max() <= 1e-14 * np.abs(v).max()
    t2 = t.clone()
    _, en2 = xc_lda(wctx, t2, vxc=t2)
    assert torch.equal(t2, vxc) and torch.equal(en2, en)


@pytest.mark.parametrize("n,h,ext", [((32, 32, 32), (0.3, 0.3, 0.3), True), ((48, 40, 36), (0.21, 0.25, 0.27), False),
                                     ((96, 96, 96), (0.225, 0.225, 0.225), True)])
def test_ks_potential_matches_oracle(oracle, torch_cuda, wctx, n, h, ext):
    from wvlh.psolver import ks_potential_periodic
    torch = torch_cuda
    rng = np.random.default_rng(sum(n))
    rho = rng.uniform(1e-4, 0.5, n[::-1])
    vext = rng.uniform(-2, 2, n[::-1]) if ext else None
    ref, (eh, exc, evxc) = oracle.ks_potential_periodic(rho, h, vext)
    pot, en = ks_potential_periodic(wctx, torch.tensor(rho, device="cuda"), h,
                                    vext=torch.tensor(vext, device="cuda") if ext else None)
    got = pot.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    e = en.cpu().numpy()
    for a, b in zip(e, (eh, exc, evxc)):
        assert abs(a - b) <= 1e-12 * abs(b)
    # deterministic
    pot2, en2 = ks_potential_periodic(wctx, torch.tensor(rho, device="cuda"), h,
                                      vext=torch.tensor(vext, device="cuda") if ext else None)
    assert torch.equal(pot, pot2) and torch.equal(en, en2)


def test_ks_potential_rejects_aliasing(torch_cuda, wctx):
    from wvlh.psolver import ks_potential_periodic
    torch = torch_cuda
    t = torch.full((16, 16, 16), 0.1, dtype=torch.float64, device="cuda")
    with pytest.raises(WvlhError):
        ks_potential_periodic(wctx, t, (0.3, 0.3, 0.3), pot=t)
    v = torch.zeros_like(t)
    with pytest.raises(WvlhError):
        ks_potential_periodic(wctx, t, (0.3, 0.3, 0.3), vext=v, pot=v)


def test_reference_ps_check_free_golden(torch_cuda, wctx):
    """The reference's PS_Check free-BC run (57 x 48 x 63 unit Gaussian): the
    Hartree energy and the potential at its largest-deviation point to the 13
    printed digits, the same deviation from the analytic potential."""
    from test_psolver_rule import PS_FREE_AT, PS_FREE_EH, PS_FREE_INF, PS_FREE_V, ps_check_free
    from wvlh.psolver import hartree_free
    torch = torch_cuda
    rho, V, h = ps_check_free()
    pot, eh = hartree_free(wctx, torch.tensor(rho, device="cuda"), h)
    got = pot.cpu().numpy()
    i1, i2, i3 = (v - 1 for v in PS_FREE_AT)
    assert abs(eh.item() - PS_FREE_EH) <= 5e-13 * PS_FREE_EH
    assert abs(got[i3, i2, i1] - PS_FREE_V) <= 5e-13 * PS_FREE_V
    assert abs(np.abs(got - V).max() - PS_FREE_INF) <= 1e-3 * PS_FREE_INF


@pytest.mark.parametrize("n,h", [((9, 10, 12), (0.3, 0.25, 0.2)), ((33, 40, 28), (0.35, 0.3, 0.4)),
                                 ((64, 64, 64), (0.225, 0.225, 0.225))])
def test_free_matches_oracle(oracle, torch_cuda, wctx, n, h):
    from wvlh.psolver import hartree_free
    torch = torch_cuda
    rng = np.random.default_rng(sum(n))
    rho = rng.uniform(-1, 1, n[::-1])
    ref, eref = oracle.psolver_free(rho, h)
    t = torch.tensor(rho, device="cuda")
    pot, eh = hartree_free(wctx, t, h)
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(eh.item() - eref) <= 1e-12 * abs(eref)
    # deterministic; the padded buffer's zeros survive repeated solves
    pot2, eh2 = hartree_free(wctx, t, h)
    assert torch.equal(pot, pot2) and torch.equal(eh, eh2)
    # in place without the energy; refused with it
    with pytest.raises(WvlhError):
        hartree_free(wctx, t, h, pot=t, energy=True)
    hartree_free(wctx, t, h, pot=t, energy=False)
    assert torch.equal(t, pot)


def test_ks_potential_free_matches_oracle(oracle, torch_cuda, wctx):
    from wvlh.psolver import ks_potential_free
    torch = torch_cuda
    n, h = (40, 36, 44), (0.3, 0.3, 0.3)
    rng = np.random.default_rng(11)
    rho = rng.uniform(1e-4, 0.5, n[::-1])
    vext = rng.uniform(-2, 2, n[::-1])
    ref, (eh, exc, evxc) = oracle.ks_potential_free(rho, h, vext)
    pot, en = ks_potential_free(wctx, torch.tensor(rho, device="cuda"), h, vext=torch.tensor(vext, device="cuda"))
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    for a, b in zip(en.cpu().numpy(), (eh, exc, evxc)):
        assert abs(a - b) <= 1e-12 * abs(b)


def test_xc_lsda_matches_oracle_on_reference_test_density(oracle, torch_cuda, wctx):
    from test_psolver_rule import xc_test_density_spin
    from wvlh.psolver import xc_lsda
    torch = torch_cuda
    up, dn = xc_test_density_spin()
    eps, vu, vd = oracle.xc_lsda(up, dn)
    tu, td = torch.tensor(up, device="cuda"), torch.tensor(dn, device="cuda")
    gu, gd, en = xc_lsda(wctx, tu, td)
    scale = max(np.abs(vu).max(), np.abs(vd).max())
    assert np.abs(gu.cpu().numpy() - vu).max() <= 1e-14 * scale
    assert np.abs(gd.cpu().numpy() - vd).max() <= 1e-14 * scale
    e = en.cpu().numpy()
    assert abs(e[0] - (eps * (up + dn)).sum()) <= 1e-13 * abs(e[0])
    assert abs(e[1] - (vu * up + vd * dn).sum()) <= 1e-13 * abs(e[1])
    # in place
    xc_lsda(wctx, tu, td, vxc_up=tu, vxc_dn=td, energy=False)
    assert torch.equal(tu, gu) and torch.equal(td, gd)


@pytest.mark.parametrize("free", [False, True])
def test_ks_potential_spin_matches_oracle(oracle, torch_cuda, wctx, free):
    from wvlh.psolver import ks_potential_spin
    torch = torch_cuda
    n, h = (32, 28, 36), (0.3, 0.32, 0.28)
    rng = np.random.default_rng(21 + free)
    up = rng.uniform(1e-4, 0.4, n[::-1])
    dn = rng.uniform(1e-4, 0.4, n[::-1])
    vext = rng.uniform(-1, 1, n[::-1])
    ru, rd, (eh, exc, evxc) = oracle.ks_potential_spin(up, dn, h, vext, free=free)
    pu, pd, en = ks_potential_spin(wctx, torch.tensor(up, device="cuda"), torch.tensor(dn, device="cuda"), h,
                                   vext=torch.tensor(vext, device="cuda"), free=free)
    scale = max(np.abs(ru).max(), np.abs(rd).max())
    assert np.abs(pu.cpu().numpy() - ru).max() <= 1e-13 * scale
    assert np.abs(pd.cpu().numpy() - rd).max() <= 1e-13 * scale
    for a, b in zip(en.cpu().numpy(), (eh, exc, evxc)):
        assert abs(a - b) <= 1e-12 * abs(b)
    t = torch.tensor(up, device="cuda")
    with pytest.raises(WvlhError):
        ks_potential_spin(wctx, t, t.clone(), h, pot_up=t)


def test_reference_ps_check_surface_golden(torch_cuda, wctx):
    """The reference's PS_Check surface-BC run (32 x 64 x 48): the Hartree
    energy to its 13 printed digits, the potential at the printed point, the
    same deviation from the analytic potential."""
    from test_psolver_rule import PS_SURF_AT, PS_SURF_EH, PS_SURF_INF, PS_SURF_V, ps_check_surface
    from wvlh.psolver import hartree_surface
    torch = torch_cuda
    rho, V, h = ps_check_surface()
    pot, eh = hartree_surface(wctx, torch.tensor(rho, device="cuda"), h)
    got = pot.cpu().numpy()
    i1, i2, i3 = (v - 1 for v in PS_SURF_AT)
    assert abs(eh.item() - PS_SURF_EH) <= 5e-13 * PS_SURF_EH
    assert abs(got[i3, i2, i1] - PS_SURF_V) <= 1e-14
    assert abs(np.abs(got - V).max() - PS_SURF_INF) <= 1e-4 * PS_SURF_INF


@pytest.mark.parametrize("n,h", [((12, 10, 8), (0.3, 0.25, 0.35)), ((32, 24, 40), (0.3, 0.35, 0.28))])
def test_surface_matches_oracle(oracle, torch_cuda, wctx, n, h):
    from wvlh.psolver import hartree_surface
    torch = torch_cuda
    rng = np.random.default_rng(sum(n) + 1)
    rho = rng.uniform(-1, 1, n[::-1])
    ref, eref = oracle.psolver_surface(rho, h)
    t = torch.tensor(rho, device="cuda")
    pot, eh = hartree_surface(wctx, t, h)
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(eh.item() - eref) <= 1e-12 * abs(eref)
    pot2, eh2 = hartree_surface(wctx, t, h)
    assert torch.equal(pot, pot2) and torch.equal(eh, eh2)
    with pytest.raises(WvlhError):
        hartree_surface(wctx, t, h, pot=t, energy=True)
    hartree_surface(wctx, t, h, pot=t, energy=False)
    assert torch.equal(t, pot)


def test_reference_ps_check_wire_golden(torch_cuda, wctx):
    """The reference's PS_Check wire-BC run (51 x 55 x 64): the Hartree
    energy and the potential at the printed point to their 13 digits."""
    from test_psolver_rule import PS_WIRE_AT, PS_WIRE_EH, PS_WIRE_V, ps_check_wire
    from wvlh.psolver import hartree_wire
    torch = torch_cuda
    rho, h = ps_check_wire()
    pot, eh = hartree_wire(wctx, torch.tensor(rho, device="cuda"), h)
    i1, i2, i3 = (v - 1 for v in PS_WIRE_AT)
    assert abs(eh.item() - PS_WIRE_EH) <= 5e-13 * PS_WIRE_EH
    assert abs(pot.cpu().numpy()[i3, i2, i1] - PS_WIRE_V) <= 5e-13 * PS_WIRE_V


def test_wire_matches_oracle(oracle, torch_cuda, wctx):
    from wvlh.psolver import hartree_wire
    torch = torch_cuda
    n, h = (10, 12, 8), (0.3, 0.35, 0.4)
    rng = np.random.default_rng(13)
    rho = rng.uniform(-1, 1, n[::-1])
    ref, eref = oracle.psolver_wire(rho, h)
    t = torch.tensor(rho, device="cuda")
    pot, eh = hartree_wire(wctx, t, h)
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(eh.item() - eref) <= 1e-12 * abs(eref)
    pot2, eh2 = hartree_wire(wctx, t, h)
    assert torch.equal(pot, pot2) and torch.equal(eh, eh2)


@pytest.mark.parametrize("n", [(11, 10, 9), (9, 13, 7)])
def test_surface_and_wire_odd_periodic_sizes(oracle, torch_cuda, wctx, n):
    from wvlh.psolver import hartree_surface, hartree_wire
    torch = torch_cuda
    h = (0.31, 0.27, 0.35)
    rng = np.random.default_rng(sum(n) + 7)
    rho = rng.uniform(-1, 1, n[::-1])
    t = torch.tensor(rho, device="cuda")
    for fn, ref_fn in ((hartree_surface, oracle.psolver_surface), (hartree_wire, oracle.psolver_wire)):
        ref, eref = ref_fn(rho, h)
        pot, eh = fn(wctx, t, h)
        assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
        assert abs(eh.item() - eref) <= 1e-12 * abs(eref)


@pytest.mark.parametrize("bc", ["surface", "wire", "free", "periodic"])
def test_ks_potential_every_boundary_condition(oracle, torch_cuda, wctx, bc):
    """updatePotential's step for each of the reference's boundary
    conditions, nspin = 1 and 2, against the oracle."""
    from wvlh.psolver import ks_potential, ks_potential_spin
    torch = torch_cuda
    n, h = (16, 18, 20), (0.3, 0.32, 0.28)
    rng = np.random.default_rng(len(bc))
    up = rng.uniform(1e-4, 0.4, n[::-1])
    dn = rng.uniform(1e-4, 0.4, n[::-1])
    vext = rng.uniform(-1, 1, n[::-1])
    tu, td, tv = (torch.tensor(a, device="cuda") for a in (up, dn, vext))
    ref, (eh, exc, evxc) = oracle.ks_potential_periodic(up + dn, h, vext, free=bc)
    pot, en = ks_potential(wctx, tu + td, h, bc=bc, vext=tv)
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    for a, b in zip(en.cpu().numpy(), (eh, exc, evxc)):
        assert abs(a - b) <= 1e-12 * abs(b)
    ru, rd, refs = oracle.ks_potential_spin(up, dn, h, vext, free=bc)
    pu, pd, en2 = ks_potential_spin(wctx, tu, td, h, vext=tv, bc=bc)
    scale = max(np.abs(ru).max(), np.abs(rd).max())
    assert np.abs(pu.cpu().numpy() - ru).max() <= 1e-13 * scale
    assert np.abs(pd.cpu().numpy() - rd).max() <= 1e-13 * scale
    for a, b in zip(en2.cpu().numpy(), refs):
        assert abs(a - b) <= 1e-12 * abs(b)


@pytest.mark.parametrize("bc", ["periodic", "free"])
def test_ks_potential_with_core_density(oracle, torch_cuda, wctx, bc):
    from wvlh.psolver import ks_potential, ks_potential_spin
    torch = torch_cuda
    n, h = (16, 18, 20), (0.3, 0.32, 0.28)
    rng = np.random.default_rng(40 + len(bc))
    up = rng.uniform(1e-4, 0.4, n[::-1])
    dn = rng.uniform(1e-4, 0.4, n[::-1])
    core = rng.uniform(0.0, 0.3, n[::-1])
    tu, td, tc = (torch.tensor(a, device="cuda") for a in (up, dn, core))
    ref, refs = oracle.ks_potential_periodic(up + dn, h, free=bc, rhocore=core)
    pot, en = ks_potential(wctx, tu + td, h, bc=bc, rhocore=tc)
    assert np.abs(pot.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    for a, b in zip(en.cpu().numpy(), refs):
        assert abs(a - b) <= 1e-12 * abs(b)
    ru, rd, refs2 = oracle.ks_potential_spin(up, dn, h, free=bc, rhocore=core)
    pu, pd, en2 = ks_potential_spin(wctx, tu, td, h, bc=bc, rhocore=tc)
    scale = max(np.abs(ru).max(), np.abs(rd).max())
    assert np.abs(pu.cpu().numpy() - ru).max() <= 1e-13 * scale
    assert np.abs(pd.cpu().numpy() - rd).max() <= 1e-13 * scale
    for a, b in zip(en2.cpu().numpy(), refs2):
        assert abs(a - b) <= 1e-12 * abs(b)
