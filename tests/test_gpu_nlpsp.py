"""GPU parity of the nonlocal projector application (wvlh_nlpsp_apply) with the
oracle's restatement of the reference's (NonLocalHamiltonianApplication,
hpsiortho.f90:1044-1125; masks of locregs/scalar_product.f90:953-1187):
hpsi and eproj in FP64 within 1e-13 of their magnitude, on convex regions
(the projector-inside-wavefunction case) and on random key sets (the
reference's segment pairing), with overlapping atoms and up to 29 projectors
per atom."""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.batch import Region
from wvlh.keys import Locreg
from wvlh.nlpsp import Projectors

pytestmark = pytest.mark.gpu


def sphere(N, c, r):
    z, y, x = np.meshgrid(*[np.arange(n) for n in N[::-1]], indexing="ij")
    return (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r


def keys(lr):
    return (lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)


def atoms_on_balls(rng, N, natoms, m):
    out = []
    for a in range(natoms):
        c = rng.uniform(2, np.array(N) - 2)
        pc = sphere(N, c, rng.uniform(2.5, 4.5))
        pf = pc & sphere(N, c, 2.0)
        lr = Locreg.from_masks(pc, pf, (0, 0, 0), (0.45, 0.45, 0.45))
        mm = m[a % len(m)]
        h = rng.uniform(-1, 1, (mm, mm))
        out.append((lr, rng.uniform(-1, 1, (mm, lr.ncoeff)), h + h.T))
    return out


def run(torch, wctx, lw, psi, hpsi0, atoms):
    nl = Projectors(wctx, Region(wctx, lw), [(lr, torch.tensor(p, device="cuda"), h) for lr, p, h in atoms])
    tp = torch.tensor(psi, device="cuda")
    th = torch.tensor(hpsi0, device="cuda")
    ep = nl.apply(tp, th)
    return th.cpu().numpy(), ep.cpu().numpy(), nl


def check(oracle, lw, psi, hpsi0, atoms, got, gep):
    ref, rep = oracle.nlpsp_apply(keys(lw), psi, [(keys(lr), p, h) for lr, p, h in atoms])
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(got - (hpsi0 + ref)).max() <= 1e-13 * scale
    assert np.abs(gep - rep).max() <= 1e-13 * max(1.0, np.abs(rep).max())


@pytest.mark.parametrize("seed,m", [(0, (4,)), (1, (1, 9)), (2, (13, 5, 3)), (3, (29,))])
def test_projectors_match_oracle_convex(oracle, torch_cuda, wctx, seed, m):
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(14, 22, 3))
    full = np.ones(N[::-1], bool)
    lw = Locreg.from_masks(full, sphere(N, [n / 2 for n in N], min(N) * 0.4), (0, 0, 0), (0.45, 0.45, 0.45))
    atoms = atoms_on_balls(rng, N, 5, m)            # balls overlap one another
    psi = rng.uniform(-1, 1, (3, lw.ncoeff))
    hpsi0 = rng.uniform(-1, 1, (3, lw.ncoeff))
    got, gep, _ = run(torch_cuda, wctx, lw, psi, hpsi0, atoms)
    check(oracle, lw, psi, hpsi0, atoms, got, gep)


@pytest.mark.parametrize("seed", [4, 5])
def test_projectors_match_oracle_random_keys(oracle, torch_cuda, wctx, seed):
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(10, 16, 3))
    m = rng.random(N[::-1]) < 0.7
    lw = Locreg.from_masks(m, m & (rng.random(N[::-1]) < 0.5), (0, 0, 0), (0.45, 0.45, 0.45))
    atoms = []
    for a in range(3):
        pm = rng.random(N[::-1]) < 0.4
        lr = Locreg.from_masks(pm, pm & (rng.random(N[::-1]) < 0.4), (0, 0, 0), (0.45, 0.45, 0.45))
        h = rng.uniform(-1, 1, (3, 3))
        atoms.append((lr, rng.uniform(-1, 1, (3, lr.ncoeff)), h + h.T))
    psi = rng.uniform(-1, 1, (2, lw.ncoeff))
    hpsi0 = np.zeros_like(psi)
    got, gep, _ = run(torch_cuda, wctx, lw, psi, hpsi0, atoms)
    check(oracle, lw, psi, hpsi0, atoms, got, gep)


def test_projectors_deterministic_and_row_stride(torch_cuda, wctx):
    torch = torch_cuda
    rng = np.random.default_rng(9)
    N = (16, 15, 17)
    full = np.ones(N[::-1], bool)
    lw = Locreg.from_masks(full, full & sphere(N, (8, 7, 8), 5.0), (0, 0, 0), (0.45, 0.45, 0.45))
    atoms = atoms_on_balls(rng, N, 4, (6,))
    nl = Projectors(wctx, Region(wctx, lw), atoms)
    base = torch.tensor(rng.uniform(-1, 1, (4, lw.ncoeff + 5)), device="cuda")
    psi = base[:, :lw.ncoeff]                       # row stride above the vector length
    h1 = torch.zeros(4, lw.ncoeff + 5, dtype=torch.float64, device="cuda")[:, :lw.ncoeff]
    h2 = torch.zeros(4, lw.ncoeff + 5, dtype=torch.float64, device="cuda")[:, :lw.ncoeff]
    e1 = nl.apply(psi, h1)
    e2 = nl.apply(psi, h2)
    assert torch.equal(h1, h2) and torch.equal(e1, e2)
    # eproj = <psi | V_nl psi> for symmetric h
    for o in range(4):
        assert abs(e1[o].item() - (psi[o] * h1[o]).sum().item()) <= 1e-12 * max(1.0, abs(e1[o].item()))


def test_projectors_reject_bad_input(torch_cuda, wctx):
    rng = np.random.default_rng(1)
    N = (10, 10, 10)
    full = np.ones(N[::-1], bool)
    lw = Locreg.from_masks(full, full, (0, 0, 0), (0.45, 0.45, 0.45))
    pm = sphere(N, (5, 5, 5), 3)
    lr = Locreg.from_masks(pm, pm, (0, 0, 0), (0.45, 0.45, 0.45))
    with pytest.raises(WvlhError):      # more than 32 projectors on one atom
        Projectors(wctx, Region(wctx, lw), [(lr, rng.uniform(-1, 1, (33, lr.ncoeff)), np.eye(33))])
    other = Locreg.from_masks(np.ones((11, 10, 10), bool), np.zeros((11, 10, 10), bool), (0, 0, 0),
                              (0.45, 0.45, 0.45))
    with pytest.raises(WvlhError):      # projector keys of another box
        Projectors(wctx, Region(wctx, lw), [(other, rng.uniform(-1, 1, (1, other.ncoeff)), np.eye(1))])
