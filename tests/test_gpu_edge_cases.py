"""Edge cases of the batched entry points on the GPU: malformed keys and
boxes are refused with their error codes and leave the context usable; the
smallest boxes, a zero orbital, a region without fine cells and a batch of
mixed boundary conditions give the oracle's results."""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.batch import Batch
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def oracle_locham(oracle, lr, psi, pot):
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    hc, hf, ek, ep = oracle.locham(d, lr.hgrid, psi[:lr.nvctr_c], psi[lr.nvctr_c:], pot)
    return np.concatenate([hc, hf]), ek, ep


def region(N, per, dens, seed):
    rng = np.random.default_rng(seed)
    mc = np.ones(N[::-1], bool)
    mf = rng.random(N[::-1]) < dens
    return Locreg.from_masks(mc, mf, per, (0.45, 0.4, 0.5)), rng


def gpu_locham(torch, wctx, lr, psi, pot, dtype):
    b = Batch(wctx, [lr], [0])
    tp = torch.zeros(b.psi_size, dtype=dtype, device="cuda")
    tp[:lr.ncoeff] = torch.tensor(psi, dtype=dtype)
    h, ek, ep = b.locham(tp, torch.tensor(pot, dtype=dtype, device="cuda"))
    torch.cuda.synchronize()
    out = h[:lr.ncoeff].double().cpu().numpy(), float(ek[0]), float(ep[0])
    b.close()
    return out


def with_keys(lr, keyg_c, keyv_c):
    return Locreg(lr.n, lr.periodic, lr.hgrid, keyg_c, keyv_c, lr.keyg_f, lr.keyv_f)


def test_malformed_keys_are_refused_and_context_stays_usable(oracle, torch_cuda, wctx):
    torch = torch_cuda
    lr, rng = region((9, 8, 10), (1, 1, 1), 0.4, 1)
    bad = []
    kg = lr.keyg_c.copy()
    kg[[0, 1]] = kg[[1, 0]]                      # segments out of order
    bad.append(with_keys(lr, kg, lr.keyv_c))
    kg = lr.keyg_c.copy()
    kg[0, 1] = kg[0, 0] + lr.n[0]                # a segment running past its x-line
    bad.append(with_keys(lr, kg, lr.keyv_c))
    kv = lr.keyv_c.copy()
    kv[1] += 1                                   # keyv not the running offset
    bad.append(with_keys(lr, lr.keyg_c, kv))
    kg = lr.keyg_c.copy()
    kg[-1, 1] = int(np.prod(lr.n)) + 1           # past the box
    bad.append(with_keys(lr, kg, lr.keyv_c))
    for b in bad:
        with pytest.raises(WvlhError, match="code 3"):
            Batch(wctx, [b], [0])
    # periodic boxes below 8 cells are refused (argument error)
    small, _ = region((7, 9, 9), (1, 1, 1), 0.5, 2)
    with pytest.raises(WvlhError, match="code 2"):
        Batch(wctx, [small], [0])
    # the context still runs a valid batch
    psi, pot = rng.uniform(-1, 1, lr.ncoeff), rng.uniform(-1, 0, lr.nisf)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    got, gek, gep = gpu_locham(torch, wctx, lr, psi, pot, torch.float64)
    assert rel(got, ref) < 1e-13 and abs(gek - ek) <= 1e-12 * abs(ek) and abs(gep - ep) <= 1e-12 * abs(ep)


@pytest.mark.parametrize("N,per", [((1, 1, 1), (0, 0, 0)), ((1, 2, 3), (0, 0, 0)), ((8, 8, 8), (1, 1, 1)),
                                   ((8, 1, 8), (1, 0, 1))])
@pytest.mark.parametrize("dtype_name,tol,etol", [("float64", 1e-13, 1e-12), ("float32", 1e-5, None)])
def test_smallest_boxes_match_oracle(oracle, torch_cuda, wctx, N, per, dtype_name, tol, etol):
    torch = torch_cuda
    lr, rng = region(N, per, 0.6, 3)
    psi = rng.uniform(-1, 1, lr.ncoeff)
    psi /= np.linalg.norm(psi)
    pot = rng.uniform(-1, 0, lr.nisf)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    got, gek, gep = gpu_locham(torch, wctx, lr, psi, pot, getattr(torch, dtype_name))
    assert rel(got, ref) < tol
    if etol is None:
        # FP32: on a box of a few cells the energy is a sum of few terms, so
        # its rounding does not average out: 2e-7 relative (the 1e-6 Ha bar
        # holds for orbitals spread over many cells)
        assert abs(gek - ek) < max(1e-6, 2e-7 * abs(ek)) and abs(gep - ep) < max(1e-6, 2e-7 * abs(ep))
    else:
        assert abs(gek - ek) <= etol * abs(ek) and abs(gep - ep) <= etol * abs(ep)


def test_zero_orbital_and_no_fine_cells(oracle, torch_cuda, wctx):
    """A zero orbital gives zero Hpsi and energies exactly; a region without
    fine cells (keyg_f empty) runs with the others in one batch."""
    torch = torch_cuda
    lr_a, rng = region((10, 9, 8), (1, 1, 1), 0.5, 4)
    mc = np.ones((8, 9, 10), bool)
    lr_b = Locreg.from_masks(mc, np.zeros_like(mc), (0, 0, 0), (0.45, 0.4, 0.5))
    assert lr_b.nvctr_f == 0
    pot_off = [0, lr_a.nisf, 0]
    b = Batch(wctx, [lr_a, lr_b], [0, 1, 0], pot_off)
    psi_b = rng.uniform(-1, 1, lr_b.ncoeff)
    psi_a = rng.uniform(-1, 1, lr_a.ncoeff)
    pot = np.concatenate([rng.uniform(-1, 0, lr_a.nisf), rng.uniform(-1, 0, lr_b.nisf)])
    psi = np.zeros(b.psi_size)
    psi[b.psi_offset(1):b.psi_offset(1) + lr_b.ncoeff] = psi_b
    psi[b.psi_offset(2):b.psi_offset(2) + lr_a.ncoeff] = psi_a      # orbital 0 stays zero
    h, ek, ep = b.locham(torch.tensor(psi, device="cuda"), torch.tensor(pot, device="cuda"))
    torch.cuda.synchronize()
    h, ek, ep = h.cpu().numpy(), ek.cpu().numpy(), ep.cpu().numpy()
    assert not h[b.psi_offset(0):b.psi_offset(0) + lr_a.ncoeff].any() and ek[0] == 0.0 and ep[0] == 0.0
    for o, lr, p, v in ((1, lr_b, psi_b, pot[lr_a.nisf:]), (2, lr_a, psi_a, pot[:lr_a.nisf])):
        ref, e1, e2 = oracle_locham(oracle, lr, p, v)
        assert rel(h[b.psi_offset(o):b.psi_offset(o) + lr.ncoeff], ref) < 1e-13
        assert abs(ek[o] - e1) <= 1e-12 * abs(e1) and abs(ep[o] - e2) <= 1e-12 * abs(e2)
    b.close()


def test_mixed_boundary_conditions_in_one_batch(oracle, torch_cuda, wctx):
    """Periodic, free (with and without fine cells) and surface regions in one
    batch: each orbital gives its own region's oracle result."""
    torch = torch_cuda
    lrs = [region((10, 9, 8), (1, 1, 1), 0.5, 5)[0], region((10, 9, 8), (0, 0, 0), 0.0, 6)[0],
           region((9, 11, 7), (0, 0, 0), 0.5, 7)[0], region((8, 7, 9), (1, 0, 1), 0.4, 8)[0]]
    orb_lr = [2, 0, 3, 1, 0, 2]
    offs = np.cumsum([0] + [lr.nisf for lr in lrs])[:-1]
    b = Batch(wctx, lrs, orb_lr, [int(offs[r]) for r in orb_lr])
    rng = np.random.default_rng(9)
    psis = [rng.uniform(-1, 1, lrs[r].ncoeff) for r in orb_lr]
    pots = [rng.uniform(-1, 0, lr.nisf) for lr in lrs]
    psi = np.zeros(b.psi_size)
    for o, p in enumerate(psis):
        psi[b.psi_offset(o):b.psi_offset(o) + len(p)] = p
    h, ek, ep = b.locham(torch.tensor(psi, device="cuda"), torch.tensor(np.concatenate(pots), device="cuda"))
    torch.cuda.synchronize()
    h, ek, ep = h.cpu().numpy(), ek.cpu().numpy(), ep.cpu().numpy()
    for o, r in enumerate(orb_lr):
        ref, e1, e2 = oracle_locham(oracle, lrs[r], psis[o], pots[r])
        assert rel(h[b.psi_offset(o):b.psi_offset(o) + lrs[r].ncoeff], ref) < 1e-13
        assert abs(ek[o] - e1) <= 1e-12 * abs(e1) and abs(ep[o] - e2) <= 1e-12 * abs(e2)
    b.close()
